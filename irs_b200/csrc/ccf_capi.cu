// extern "C" entry points of lib_ccf.so (double), the symbol set of the
// reference's src/lib_ccf.cu (lines 15-81) with the same signatures, so its
// ctypes wrapper (microlensing/CCF/lib_ccf.py) binds them unchanged.
// Declarations and the extensions are in include/lib_ccf.h.
#include "ccf_host.cuh"

#include <cstring>
#include <limits>

using dtype = double;
using Obj = irsb::CCF<dtype>;

#define SETTER(name, field) \
  void set_##name(Obj* self, dtype val) { self->field = val; } \
  dtype get_##name(Obj* self) { return self->field; }
#define ISETTER(name, field) \
  void set_##name(Obj* self, int val) { self->field = val; } \
  int get_##name(Obj* self) { return self->field; }
#define SSETTER(name, field) \
  void set_##name(Obj* self, const char* val) { self->field = val ? val : ""; } \
  const char* get_##name(Obj* self) { return self->field.c_str(); }

extern "C" {

Obj* init() { return new Obj(); }

SETTER(kappa_tot, kappa_tot)
SETTER(shear, shear)
SETTER(kappa_star, kappa_star)
SETTER(theta_star, theta_star)
SSETTER(mass_function, mass_function_str)
SETTER(m_solar, m_solar)
SETTER(m_lower, m_lower)
SETTER(m_upper, m_upper)
ISETTER(rectangular, rectangular)
ISETTER(approx, approx)
SETTER(safety_scale, safety_scale)
ISETTER(num_stars, num_stars)
SSETTER(starfile, starfile)
ISETTER(num_phi, num_phi)
ISETTER(num_branches, num_branches)
ISETTER(random_seed, random_seed)
ISETTER(write_stars, write_stars)
ISETTER(write_critical_curves, write_critical_curves)
ISETTER(write_caustics, write_caustics)
ISETTER(write_mu_length_scales, write_mu_length_scales)
SSETTER(outfile_prefix, outfile_prefix)

int get_num_roots(Obj* self) { return self->get_num_roots(); }
dtype get_corner_x1(Obj* self) { return self->get_corner().re; }
dtype get_corner_x2(Obj* self) { return self->get_corner().im; }
dtype* get_stars(Obj* self) { return self->stars_ptr(); }
dtype* get_critical_curves(Obj* self) { return self->ccs_ptr(); }
dtype* get_caustics(Obj* self) { return self->caustics_ptr(); }
dtype* get_mu_length_scales(Obj* self) { return self->mu_ptr(); }
double get_t_ccs(Obj* self) { return self->t_ccs; }

bool run(Obj* self, int verbose) { return self->run(verbose); }
bool save(Obj* self, int verbose) { return self->save(verbose); }

// ---- extensions
void destroy(Obj* self) { delete self; }
void set_num_iters(Obj* self, int init_iters, int step_iters) {
  self->num_iters_init = init_iters;
  self->num_iters_step = step_iters;
}
// Derived values and timings by name (NaN for an unknown name).
double get_value(Obj* self, const char* name) {
  const std::string n = name ? name : "";
  if (n == "max_error") return double(self->max_error);
  if (n == "t_init_roots") return self->t_init_roots;
  if (n == "t_ccs") return self->t_ccs;
  if (n == "t_caustics") return self->t_caustics;
  if (n == "num_roots") return self->num_roots;
  if (n == "expansion_order") return self->expansion_order;
  if (n == "tree_levels") return self->tree_levels;
  if (n == "taylor_smooth") return self->taylor_smooth;
  if (n == "root_half_length") return double(self->root_half_length);
  if (n == "mu_ave") return double(self->mu_ave);
  if (n == "kappa_star_actual") return double(self->kappa_star_actual);
  if (n == "mean_mass_actual") return double(self->mean_mass_actual);
  return std::numeric_limits<double>::quiet_NaN();
}

}  // extern "C"
