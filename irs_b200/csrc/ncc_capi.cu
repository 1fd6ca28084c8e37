// extern "C" entry points of lib_ncc.so (double), the symbol set of the
// reference's src/lib_ncc.cu (lines 15-44) with the same signatures, so its
// ctypes wrapper (microlensing/NCC/lib_ncc.py) binds them unchanged.
// Declarations and the extensions are in include/lib_ncc.h.
#include "ncc_host.cuh"

#include <limits>

using dtype = double;
using Obj = irsb::NCC<dtype>;

extern "C" {

Obj* init() { return new Obj(); }

void set_infile_prefix(Obj* self, const char* val) { self->infile_prefix = val ? val : ""; }
void set_center_y1(Obj* self, dtype val) { self->center_y.re = val; }
void set_center_y2(Obj* self, dtype val) { self->center_y.im = val; }
void set_half_length_y1(Obj* self, dtype val) { self->half_length_y.re = val; }
void set_half_length_y2(Obj* self, dtype val) { self->half_length_y.im = val; }
void set_num_pixels_y1(Obj* self, int val) { self->num_pixels_y.re = val; }
void set_num_pixels_y2(Obj* self, int val) { self->num_pixels_y.im = val; }
void set_over_sample(Obj* self, int val) { self->over_sample = val; }
void set_write_maps(Obj* self, int val) { self->write_maps = val; }
void set_write_histograms(Obj* self, int val) { self->write_histograms = val; }
void set_outfile_prefix(Obj* self, const char* val) { self->outfile_prefix = val ? val : ""; }

const char* get_infile_prefix(Obj* self) { return self->infile_prefix.c_str(); }
dtype get_center_y1(Obj* self) { return self->center_y.re; }
dtype get_center_y2(Obj* self) { return self->center_y.im; }
dtype get_half_length_y1(Obj* self) { return self->half_length_y.re; }
dtype get_half_length_y2(Obj* self) { return self->half_length_y.im; }
int get_num_pixels_y1(Obj* self) { return self->num_pixels_y.re; }
int get_num_pixels_y2(Obj* self) { return self->num_pixels_y.im; }
int get_over_sample(Obj* self) { return self->over_sample; }
int get_write_maps(Obj* self) { return self->write_maps; }
int get_write_histograms(Obj* self) { return self->write_histograms; }
const char* get_outfile_prefix(Obj* self) { return self->outfile_prefix.c_str(); }

int* get_num_crossings(Obj* self) { return self->num_crossings(); }

bool run(Obj* self, int verbose) { return self->run(verbose); }
bool save(Obj* self, int verbose) { return self->save(verbose); }

// ---- extensions
void destroy(Obj* self) { delete self; }
// Caustics from host memory, nrows x ncols complex values (re, im
// interleaved), used instead of <infile_prefix>ccf_caustics.bin; nrows = 0
// returns to the file.
void set_caustics(Obj* self, const double* vals, int nrows, int ncols) {
  self->host_rows = vals && nrows > 0 && ncols > 0 ? nrows : 0;
  self->host_cols = self->host_rows ? ncols : 0;
  self->host_caustics.assign(size_t(self->host_rows) * self->host_cols, make_double2(0, 0));
  for (size_t k = 0; k < self->host_caustics.size(); k++)
    self->host_caustics[k] = make_double2(vals[2 * k], vals[2 * k + 1]);
}
double get_value(Obj* self, const char* name) {
  const std::string n = name ? name : "";
  if (n == "t_ncc") return self->t_ncc;
  if (n == "t_reduce") return self->t_reduce;
  if (n == "num_rows") return self->num_rows;
  if (n == "num_cols") return self->num_cols;
  if (n == "min_num") return self->min_num;
  if (n == "max_num") return self->max_num;
  if (n == "errors") return self->errors;
  return std::numeric_limits<double>::quiet_NaN();
}

}  // extern "C"
