// extern "C" entry points. One translation unit, compiled four times:
//   -DIRSB_DOUBLE=0 -DIRSB_IRS=0  -> lib_ipm.so         (IPM, float)
//   -DIRSB_DOUBLE=1 -DIRSB_IRS=0  -> lib_ipm_double.so  (IPM, double)
//   -DIRSB_DOUBLE=0 -DIRSB_IRS=1  -> lib_irs.so         (IRS, float)
//   -DIRSB_DOUBLE=1 -DIRSB_IRS=1  -> lib_irs_double.so  (IRS, double)
// The IPM libraries export the symbol set of the reference's src/lib_ipm.cu
// (lines 15-81) with the same signatures, so its ctypes wrapper
// (microlensing/IPM/lib_ipm.py) binds them unchanged. The IRS libraries use
// the same conventions (the reference has no IRS library). Declarations and
// the list of extensions are in include/lib_ipm.h and include/lib_irs.h.
#include "adaptive_host.cuh"
#include "batch.cuh"
#include "engine.cuh"

#include <cstring>
#include <limits>
#include <mutex>

#ifndef IRSB_DOUBLE
#define IRSB_DOUBLE 0
#endif
#ifndef IRSB_IRS
#define IRSB_IRS 0
#endif

#if IRSB_DOUBLE
using dtype = double;
#else
using dtype = float;
#endif
using Obj = irsb::MapMaker<dtype, bool(IRSB_IRS)>;
using Pix = Obj::Pix;

#define SETTER(name, field) \
  void set_##name(Obj* self, dtype val) { self->prm.field = val; } \
  dtype get_##name(Obj* self) { return self->prm.field; }
#define ISETTER(name, field) \
  void set_##name(Obj* self, int val) { self->prm.field = val; } \
  int get_##name(Obj* self) { return self->prm.field; }
#define SSETTER(name, field) \
  void set_##name(Obj* self, const char* val) { self->prm.field = val ? val : ""; } \
  const char* get_##name(Obj* self) { return self->prm.field.c_str(); }

extern "C" {

Obj* init() { return new Obj(); }

SETTER(kappa_tot, kappa_tot)
SETTER(shear, shear)
SETTER(kappa_star, kappa_star)
SETTER(theta_star, theta_star)
SSETTER(mass_function, mass_function)
SETTER(m_solar, m_solar)
SETTER(m_lower, m_lower)
SETTER(m_upper, m_upper)
SETTER(light_loss, light_loss)
ISETTER(rectangular, rectangular)
ISETTER(approx, approx)
SETTER(safety_scale, safety_scale)
SSETTER(starfile, starfile)
SETTER(center_y1, center_y.re)
SETTER(center_y2, center_y.im)
SETTER(half_length_y1, half_length_y.re)
SETTER(half_length_y2, half_length_y.im)
ISETTER(num_pixels_y1, num_pixels_y.re)
ISETTER(num_pixels_y2, num_pixels_y.im)
ISETTER(num_rays_y, num_rays_y)
ISETTER(random_seed, random_seed)
ISETTER(write_stars, write_stars)
ISETTER(write_maps, write_maps)
ISETTER(write_parities, write_parities)
ISETTER(write_histograms, write_histograms)
SSETTER(outfile_prefix, outfile_prefix)

int get_num_stars(Obj* self) { return self->prm.num_stars; }
dtype get_corner_x1(Obj* self) { return self->corner_out().re; }
dtype get_corner_x2(Obj* self) { return self->corner_out().im; }
dtype* get_stars(Obj* self) { return self->stars_ptr(); }
Pix* get_pixels(Obj* self) { return self->pixels(); }
Pix* get_pixels_minima(Obj* self) { return self->pixels_minima(); }
Pix* get_pixels_saddles(Obj* self) { return self->pixels_saddles(); }
bool copy_pixels(Obj* self, int which, Pix* dst) { return self->copy_pixels(which, dst); }
void set_pixels_out(Obj* self, Pix* dst) { self->set_pixels_out(dst); }
#if IRSB_IRS
double get_t_shoot_rays(Obj* self) { return self->t_shoot; }
unsigned long long get_num_rays_shot(Obj* self) { return self->num_rays_shot; }
unsigned long long get_num_rays_received(Obj* self) { return self->num_rays_received; }
#else
double get_t_shoot_cells(Obj* self) { return self->t_shoot; }
#endif

bool run(Obj* self, int verbose) { return self->run(verbose); }
bool save(Obj* self, int verbose) { return self->save(verbose); }

// ---------------------------------------------------------------- extensions
void destroy(Obj* self) { delete self; }

// 0: expansion order from the reference formula (default); 3..31: fixed order
void set_expansion_order(Obj* self, int order) { self->prm.expansion_order_override = order; }
int get_expansion_order(Obj* self) { return self->prm.expansion_order; }

// 0: default form (FP32 for float libraries, FP64 for double ones), 1: FP64, 2: FP32
void set_precision(Obj* self, int mode) { self->precision = mode; }
void set_shoot_launch(Obj* self, int threads, int ctas_per_sm) {
  // anything else than 128, 256 or 512 threads, or CTAs per SM <= 0: the default
  self->shoot_threads = (threads == 128 || threads == 256 || threads == 512) ? threads : 128;
  self->shoot_ctas_per_sm = ctas_per_sm > 0 ? ctas_per_sm : 64;
}
int get_shoot_threads(Obj* self) { return self->shoot_threads; }
int get_shoot_ctas_per_sm(Obj* self) { return self->shoot_ctas_per_sm; }
int get_precision(Obj* self) { return self->precision; }

// Star field from host memory: n records of (x1, x2, mass), with the field
// shape, corner and theta_star of a star file. Used instead of generating
// stars; the array is copied.
void set_stars(Obj* self, const dtype* xym, int n, int rectangular, dtype corner_x1, dtype corner_x2, dtype theta) {
  if (!xym || n <= 0) {
    self->use_host_stars = false;
    self->host_stars.clear();
    return;
  }
  self->host_stars.resize(n);
  std::memcpy(self->host_stars.data(), xym, size_t(n) * 3 * sizeof(dtype));
  self->host_rect = rectangular;
  self->host_corner = irsb::mk<dtype>(corner_x1, corner_x2);
  self->host_theta = theta;
  self->use_host_stars = true;
}

double get_t_pipeline(Obj* self) { return self->t_pipeline; }

// Re-runs tree, expansions and shoot `repeats` times on the star field of the
// last run() (device resident); *seconds receives the summed device time.
bool rerun(Obj* self, int repeats, double* seconds) { return self->rerun(repeats, seconds); }

// Checks the inputs and computes the derived parameters only (no GPU work).
bool derive(Obj* self) {
  irsb::Params<dtype> p = self->prm;
  if (!irsb::check_input_params(p)) return false;
  std::vector<irsb::StarRec<dtype>> st;
  if (!irsb::derive_params<dtype>(p, st)) return false;
  self->prm = p;
  return true;
}

// Derived or run-time quantity by name; NaN for an unknown name.
double get_value(Obj* self, const char* name) {
  const auto& p = self->prm;
  std::string n = name ? name : "";
  if (n == "mu_ave") return p.mu_ave;
  if (n == "num_rays_x") return p.num_rays_x;
  if (n == "ray_half_sep_1") return p.ray_half_sep.re;
  if (n == "ray_half_sep_2") return p.ray_half_sep.im;
  if (n == "half_length_x1") return p.half_length_x.re;
  if (n == "half_length_x2") return p.half_length_x.im;
  if (n == "center_x1") return p.center_x.re;
  if (n == "center_x2") return p.center_x.im;
  if (n == "num_ray_threads_1") return p.num_ray_threads.re;
  if (n == "num_ray_threads_2") return p.num_ray_threads.im;
  if (n == "corner_x1") return p.corner.re;
  if (n == "corner_x2") return p.corner.im;
  if (n == "rad") return irsb::cabs_(p.corner);
  if (n == "num_stars") return p.num_stars;
  if (n == "alpha_error") return p.alpha_error;
  if (n == "taylor_smooth") return p.taylor_smooth;
  if (n == "mean_mass") return p.mean_mass;
  if (n == "mean_mass2") return p.mean_mass2;
  if (n == "mean_mass2_ln_mass") return p.mean_mass2_ln_mass;
  if (n == "m_lower") return p.m_lower;
  if (n == "m_upper") return p.m_upper;
  if (n == "kappa_star_actual") return p.kappa_star_actual;
  if (n == "m_lower_actual") return p.m_lower_actual;
  if (n == "m_upper_actual") return p.m_upper_actual;
  if (n == "mean_mass_actual") return p.mean_mass_actual;
  if (n == "mean_mass2_actual") return p.mean_mass2_actual;
  if (n == "mean_mass2_ln_mass_actual") return p.mean_mass2_ln_mass_actual;
  if (n == "root_half_length") return p.root_half_length;
  if (n == "expansion_order") return p.expansion_order;
  if (n == "tree_levels") return p.tree_levels;
  if (n == "random_seed") return p.random_seed;
  if (n == "num_leaves") return self->num_leaves;
  if (n == "num_tiles") return double(self->num_tiles);
  if (n == "t_shoot") return self->t_shoot;
  if (n == "t_pipeline") return self->t_pipeline;
  if (n == "t_lattice") return self->t_lattice;
  if (n == "t_deposit") return self->t_deposit;
  if (n == "mean_near") return self->mean_near;
  if (n == "launches") return double(self->launches);
  if (n == "num_lattice_points") return double(self->num_tiles >= 0 ? 1 : 0) *
      (IRSB_IRS ? double(p.num_ray_threads.re) * p.num_ray_threads.im
                : double(p.num_ray_threads.re + 1) * (p.num_ray_threads.im + 1));
  return std::numeric_limits<double>::quiet_NaN();
}

// Row band [first, last) of the lattice computed by this object (rays for IRS,
// cells for IPM); last < 0: all rows. With the integer maps of all bands
// summed, the map equals the one-object map exactly.
void set_band(Obj* self, long long first, long long last) {
  self->band_lo = first;
  self->band_hi = last;
}
// Integer maps into caller-provided device buffers: IPM uint64 fixed point
// (2^32 per unit), IRS int32 counts; minima/saddles only with parities.
bool copy_maps_device(Obj* self, void* total, void* minima, void* saddles) {
  return self->copy_maps_device(total, minima, saddles);
}

// ---------------------------------------------------------------- diagnostics
int get_tree_num_nodes(Obj* self) { return self->tree_num_nodes(); }
bool copy_tree(Obj* self, int* ints, double* geom, int* nbr, int* sil, int* dil) {
  return self->copy_tree(ints, geom, nbr, sil, dil);
}
bool copy_coeffs(Obj* self, double* mult, double* loc) { return self->copy_coeffs(mult, loc); }
long long get_num_vertices(Obj* self) { return self->num_vertices(); }
bool copy_vertices(Obj* self, double* out) { return self->copy_vertices(out); }
bool copy_fixed_maps(Obj* self, unsigned long long* total, unsigned long long* mn, unsigned long long* sd) {
  return self->copy_fixed_maps(total, mn, sd);
}

}  // extern "C"

#if !IRSB_IRS
// ---------------------------------------------------------------- allocation-free deposition
// Some callers cannot let a library call cudaMalloc: applications whose device
// memory is owned by their own pool (a framework's caching allocator or a
// fixed memory budget), and latency-critical loops where cudaMalloc / cudaFree
// would synchronise the device. ipm_deposit_noalloc serves them: it deposits a
// cell-corner lattice the caller already holds on the device into a map the
// caller provides, and its fixed-point scratch lives in the file-scope device
// array below instead of being allocated.
//
// Limit: maps of at most kNoAllocMaxPixels = 1024 * 1024 pixels in all and at
// most kNoAllocMaxRows = 1024 rows (so 2048 x 512 is accepted, 1024 x 1025 is
// not). The array (16.8 MB) is part of the module, so every GPU that loads
// this library holds it until the process exits; with CUDA's lazy module
// loading (the default) the first call on a device may load the module,
// reserving that memory then.
namespace {
constexpr long long kNoAllocMaxPixels = 1024LL * 1024LL;
constexpr long long kNoAllocMaxRows = 1024;
constexpr long long kNoAllocWords = kNoAllocMaxPixels + kNoAllocMaxRows * (1024 + 1);
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned long long* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array for the current device; looked up once
// per device. In host code the array's name is only a host-side stand-in.
unsigned long long* noalloc_scratch_for_current_device(int* err) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    *err = 3;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      std::fprintf(stderr, "ipm_deposit_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      *err = 3;
      return nullptr;
    }
    g_noalloc_ptr[dev] = static_cast<unsigned long long*>(ptr);
  }
  return g_noalloc_ptr[dev];
}
}  // namespace

extern "C" {

// Deposits the two triangles of each of the ncx x ncy lens-plane cells whose
// (ncx+1) x (ncy+1) corner source positions (double x, y pairs in pixel units,
// row axis flipped, row-major by corner row) are at the device pointer
// `verts`, into the npx x npy magnification map at the device pointer `map`
// (overwritten). `factor` is the image-plane area of one triangle in pixel
// units. The work is queued on `stream` (a cudaStream_t; NULL for the default
// stream) and the call returns without waiting for it.
//
// Returns 0 on success, 1 for sizes beyond the limit (more than 1024 * 1024
// pixels in all or more than 1024 rows) or invalid arguments, 3 if the
// scratch address cannot be found, 4 for an error of this call's launches, 5
// if a CUDA error from earlier work is already pending on the calling thread
// (nothing is queued and the error is left for its owner to read). The call
// allocates nothing. Its first call on a device looks up the device address
// of the scratch array and may load the module: make that first call at
// start-up, before any stream capture. All calls share the one scratch array
// (cleared at the start of each call), so calls whose work overlaps on the
// GPU race: order them on one stream or synchronise between them.
int ipm_deposit_noalloc(const double* verts, long long ncx, long long ncy, dtype factor, int npx, int npy,
                        dtype* map, void* stream) {
  if (cudaPeekAtLastError() != cudaSuccess) {
    std::fprintf(stderr, "ipm_deposit_noalloc: an earlier CUDA error is pending; nothing queued\n");
    return 5;
  }
  if (!verts || !map || ncx < 1 || ncy < 1 || npx < 1 || npy < 1) {
    std::fprintf(stderr, "ipm_deposit_noalloc: invalid arguments\n");
    return 1;
  }
  const long long npix = (long long)npx * npy;
  if (npix > kNoAllocMaxPixels || npy > kNoAllocMaxRows || (long long)npy * (npx + 1) > kNoAllocWords - npix) {
    std::fprintf(stderr, "ipm_deposit_noalloc: map of %d x %d pixels exceeds the limit of %lld pixels and %lld rows\n",
                 npx, npy, kNoAllocMaxPixels, kNoAllocMaxRows);
    return 1;
  }
  int err = 0;
  unsigned long long* scratch = noalloc_scratch_for_current_device(&err);
  if (!scratch) return err;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  irsb::DepositMaps m{scratch, scratch + npix};
  const long long ndiff = (long long)npy * (npx + 1);
  if (cudaMemsetAsync(m.acc, 0, npix * sizeof(unsigned long long), s) != cudaSuccess) return 4;
  if (cudaMemsetAsync(m.diff, 0, ndiff * sizeof(unsigned long long), s) != cudaSuccess) return 4;
  const long long ncells = ncx * ncy;
  const int grid = irsb::deposit_grid((ncells + 31) / 32);
  irsb::ipm_deposit_cells<dtype><<<grid, irsb::kDepositThreads, 0, s>>>(reinterpret_cast<const double2*>(verts), ncx, ncy, factor,
                                                      npx, npy, m, m, m, 0);
  int gr = std::max(1, std::min(irsb::ceil_div((long long)npy * 32, 256), 148 * 8));
  irsb::ipm_resolve_rows<<<gr, 256, 0, s>>>(npx, npy, m);
  int g2 = int(std::max<long long>(1, std::min<long long>((npix + 255) / 256, 148LL * 16)));
  irsb::ipm_finalize<dtype><<<g2, 256, 0, s>>>(npix, m.acc, nullptr, nullptr, map, nullptr, nullptr, 0);
  if (cudaGetLastError() != cudaSuccess) return 4;
  return 0;
}

// ---------------------------------------------------------------- batches
// Many realizations through one graph-captured device pipeline (no
// counterpart in the reference). A realization is described by an object of
// this library (init + setters) and copied into the batch by batch_add.
using Batch = irsb::BatchMaker<dtype>;

void* batch_init() { return new Batch(); }
void batch_destroy(void* b) { delete static_cast<Batch*>(b); }
int batch_add(void* b, Obj* realization) {
  Batch* bt = static_cast<Batch*>(b);
  bt->in.push_back(realization->prm);
  return bt->size() - 1;
}
int batch_size(void* b) { return static_cast<Batch*>(b)->size(); }
void batch_set_expansion_order(void* b, int p) { static_cast<Batch*>(b)->expansion_order = p; }
void batch_set_corner_capacity(void* b, long long n) { static_cast<Batch*>(b)->corner_cap = n; }
bool batch_run(void* b, int verbose) { return static_cast<Batch*>(b)->run(verbose); }
bool batch_rerun(void* b, int repeats, double* seconds) { return static_cast<Batch*>(b)->rerun(repeats, seconds); }
bool batch_copy_maps(void* b, dtype* out) { return static_cast<Batch*>(b)->copy_maps(out); }
const dtype* batch_maps_device(void* b) { return static_cast<Batch*>(b)->maps_device(); }
bool batch_copy_stars(void* b, dtype* out) { return static_cast<Batch*>(b)->copy_stars(out); }
// r >= 0: a realization's derived value; r < 0: a value of the batch
double batch_get_value(void* b, int r, const char* name) {
  Batch* bt = static_cast<Batch*>(b);
  std::string n = name ? name : "";
  if (r < 0) {
    if (n == "size") return bt->size();
    if (n == "expansion_order") return bt->order;
    if (n == "passes") return bt->passes;
    if (n == "total_cells") return double(bt->total_cells);
    if (n == "total_pixels") return double(bt->total_pixels);
    if (n == "total_stars") return double(bt->total_stars);
    if (n == "t_stars") return bt->t_stars;
    if (n == "t_graph") return bt->t_graph;
    if (n == "graph_nodes") return bt->graph_nodes;
    if (n == "num_pixels_y1") return bt->npx();
    if (n == "num_pixels_y2") return bt->npy();
    return std::numeric_limits<double>::quiet_NaN();
  }
  if (r >= int(bt->prm.size())) return std::numeric_limits<double>::quiet_NaN();
  const auto& p = bt->prm[r];
  if (n == "num_stars") return p.num_stars;
  if (n == "star_offset") return double(bt->star_offset(r));
  if (n == "num_cells") return double(p.num_ray_threads.re) * p.num_ray_threads.im;
  if (n == "tree_levels") return p.tree_levels;
  if (n == "expansion_order") return p.expansion_order;
  if (n == "mu_ave") return p.mu_ave;
  if (n == "kappa_tot") return p.kappa_tot;
  if (n == "shear") return p.shear;
  if (n == "kappa_star") return p.kappa_star;
  if (n == "corner_x1") return p.corner.re;
  if (n == "corner_x2") return p.corner.im;
  if (n == "root_half_length") return p.root_half_length;
  if (n == "mean_mass_actual") return p.mean_mass_actual;
  if (n == "kappa_star_actual") return p.kappa_star_actual;
  if (n == "random_seed") return p.random_seed;
  return std::numeric_limits<double>::quiet_NaN();
}

// ---------------------------------------------------------------- adaptive IPM
// Per-tile subdivision chosen by the level network (no counterpart in the
// reference). The map inputs are set on the object returned by ada_base with
// the setters of this library.
using Ada = irsb::AdaptiveIPM<dtype>;

void* ada_init() { return new Ada(); }
void ada_destroy(void* a) { delete static_cast<Ada*>(a); }
Obj* ada_base(void* a) { return &static_cast<Ada*>(a)->base; }
void ada_set_policy(void* a, int policy, int uniform_level) {
  static_cast<Ada*>(a)->policy = policy;
  static_cast<Ada*>(a)->uniform_level = uniform_level;
}
void ada_set_levels(void* a, const int* levels, int n) {
  static_cast<Ada*>(a)->given_levels.assign(levels, levels + n);
}
void ada_set_tolerance(void* a, double eps) { static_cast<Ada*>(a)->eps = eps; }
void ada_set_quantile(void* a, float q) { static_cast<Ada*>(a)->net_quantile = q; }
void ada_set_max_level(void* a, int level) { static_cast<Ada*>(a)->max_level = level; }
void ada_set_error_mode(void* a, int mode) { static_cast<Ada*>(a)->err_mode = (mode == 1 || mode == 2) ? mode : 0; }
void ada_set_audit(void* a, double fraction, unsigned seed) {
  static_cast<Ada*>(a)->audit_fraction = fraction;
  static_cast<Ada*>(a)->audit_seed = seed;
}
void ada_set_audit_bound(void* a, double bound) { static_cast<Ada*>(a)->fail_bound = bound; }
void ada_set_refine_capacity(void* a, long long n) { static_cast<Ada*>(a)->refine_cap = n; }
void ada_set_tiled_min(void* a, int n) { static_cast<Ada*>(a)->tiled_min = n; }
void ada_set_network(void* a, const float* w, const float* mu, const float* sig) {
  Ada* ad = static_cast<Ada*>(a);
  ad->net_w.assign(w, w + irsb::kMlpParams);
  ad->net_mu.assign(mu, mu + irsb::kMlpIn);
  ad->net_sig.assign(sig, sig + irsb::kMlpIn);
}
bool ada_run(void* a, int verbose) { return static_cast<Ada*>(a)->run(verbose); }
int ada_num_tiles(void* a) { return static_cast<Ada*>(a)->num_tiles(); }
bool ada_copy_features(void* a, float* out) { return static_cast<Ada*>(a)->copy_features(out); }
bool ada_copy_levels(void* a, int* out, int predicted) {
  Ada* ad = static_cast<Ada*>(a);
  const std::vector<int>& v = predicted ? ad->predicted : ad->level;
  std::copy(v.begin(), v.end(), out);
  return true;
}
bool ada_labels(void* a, const int* tiles, int n, int* labels, float* err) {
  std::vector<int> t(tiles, tiles + n), lab;
  std::vector<float> e;
  if (!static_cast<Ada*>(a)->labels(t, lab, e)) return false;
  std::copy(lab.begin(), lab.end(), labels);
  if (err) std::copy(e.begin(), e.end(), err);
  return true;
}
bool ada_copy_map(void* a, dtype* out) { return static_cast<Ada*>(a)->copy_map(out); }
double ada_get_value(void* a, const char* name) {
  Ada* ad = static_cast<Ada*>(a);
  std::string n = name ? name : "";
  if (n == "tiles_x") return ad->ntx;
  if (n == "tiles_y") return ad->nty;
  if (n == "cells_base") return double(ad->cells_base);
  if (n == "cells_evaluated") return double(ad->cells_evaluated);
  if (n == "audit_cells") return double(ad->audit_cells);
  if (n == "audited") return ad->audited;
  if (n == "audit_failures") return ad->audit_failures;
  if (n == "fail_rate_initial") return ad->fail_rate_initial;
  if (n == "fail_rate") return ad->fail_rate;
  if (n == "fail_bound") return ad->fail_bound;
  if (n == "escalation") return ad->escalation;
  if (n == "quantile_used") return ad->quantile_used;
  if (n == "t_base") return ad->t_base;
  if (n == "t_adapt") return ad->t_adapt;
  if (n == "t_select") return ad->t_select;
  if (n == "t_audit") return ad->t_audit;
  if (n == "t_refine_deposit") return ad->t_refine_deposit;
  if (n == "tolerance") return ad->eps;
  return get_value(&ad->base, name);
}

// The level network on its own: training, gradients and prediction.
int mlp_num_params() { return irsb::kMlpParams; }
bool mlp_train(const float* feat, const int* labels, int n, int epochs, int batch, float lr, unsigned seed, float* w,
               float* mu, float* sig, float* epoch_loss) {
  return irsb::MlpTrainer::train(feat, labels, n, epochs, batch, lr, seed, w, mu, sig, epoch_loss);
}
bool mlp_gradients(const float* w, const float* mu, const float* sig, const float* feat, const int* labels, int n,
                   float* grad, float* mean_loss) {
  return irsb::MlpTrainer::gradients(w, mu, sig, feat, labels, n, grad, mean_loss);
}
bool mlp_predict(const float* w, const float* mu, const float* sig, const float* feat, int n, int* cls) {
  return irsb::MlpTrainer::predict(w, mu, sig, feat, n, cls);
}

}  // extern "C"
#endif
