/*
 * lib_ipm.so / lib_ipm_double.so -- inverse polygon mapping, C ABI.
 *
 * Drop-in for the reference's src/lib_ipm.cu (weisluke/irs): same symbol names
 * and signatures, so microlensing/IPM/lib_ipm.py and lib_ipm_double.py bind
 * them unchanged. IPM_DTYPE is float for lib_ipm.so and double for
 * lib_ipm_double.so (src/lib_ipm.cu:4-10). The object handle is opaque.
 *
 * Pointers returned by get_stars / get_pixels* are host memory owned by the
 * object, valid until the next run() or destroy() on that object (the
 * reference returns managed memory valid until the next run()).
 * run() and save() return false after printing the reason to stderr.
 */
#ifndef IRS_B200_LIB_IPM_H
#define IRS_B200_LIB_IPM_H
#include <stdbool.h>

#ifndef IPM_DTYPE
#define IPM_DTYPE float
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef void IPMHandle;

/* src/lib_ipm.cu:15 */
IPMHandle* init(void);

/* setters, src/lib_ipm.cu:17-42 */
void set_kappa_tot(IPMHandle* self, IPM_DTYPE val);
void set_shear(IPMHandle* self, IPM_DTYPE val);
void set_kappa_star(IPMHandle* self, IPM_DTYPE val);
void set_theta_star(IPMHandle* self, IPM_DTYPE val);
void set_mass_function(IPMHandle* self, const char* val);
void set_m_solar(IPMHandle* self, IPM_DTYPE val);
void set_m_lower(IPMHandle* self, IPM_DTYPE val);
void set_m_upper(IPMHandle* self, IPM_DTYPE val);
void set_light_loss(IPMHandle* self, IPM_DTYPE val);
void set_rectangular(IPMHandle* self, int val);
void set_approx(IPMHandle* self, int val);
void set_safety_scale(IPMHandle* self, IPM_DTYPE val);
void set_starfile(IPMHandle* self, const char* val);
void set_center_y1(IPMHandle* self, IPM_DTYPE val);
void set_center_y2(IPMHandle* self, IPM_DTYPE val);
void set_half_length_y1(IPMHandle* self, IPM_DTYPE val);
void set_half_length_y2(IPMHandle* self, IPM_DTYPE val);
void set_num_pixels_y1(IPMHandle* self, int val);
void set_num_pixels_y2(IPMHandle* self, int val);
void set_num_rays_y(IPMHandle* self, int val);
void set_random_seed(IPMHandle* self, int val);
void set_write_stars(IPMHandle* self, int val);
void set_write_maps(IPMHandle* self, int val);
void set_write_parities(IPMHandle* self, int val);
void set_write_histograms(IPMHandle* self, int val);
void set_outfile_prefix(IPMHandle* self, const char* val);

/* getters, src/lib_ipm.cu:44-69 */
IPM_DTYPE get_kappa_tot(IPMHandle* self);
IPM_DTYPE get_shear(IPMHandle* self);
IPM_DTYPE get_kappa_star(IPMHandle* self);
IPM_DTYPE get_theta_star(IPMHandle* self);
const char* get_mass_function(IPMHandle* self);
IPM_DTYPE get_m_solar(IPMHandle* self);
IPM_DTYPE get_m_lower(IPMHandle* self);
IPM_DTYPE get_m_upper(IPMHandle* self);
IPM_DTYPE get_light_loss(IPMHandle* self);
int get_rectangular(IPMHandle* self);
int get_approx(IPMHandle* self);
IPM_DTYPE get_safety_scale(IPMHandle* self);
const char* get_starfile(IPMHandle* self);
IPM_DTYPE get_center_y1(IPMHandle* self);
IPM_DTYPE get_center_y2(IPMHandle* self);
IPM_DTYPE get_half_length_y1(IPMHandle* self);
IPM_DTYPE get_half_length_y2(IPMHandle* self);
int get_num_pixels_y1(IPMHandle* self);
int get_num_pixels_y2(IPMHandle* self);
int get_num_rays_y(IPMHandle* self);
int get_random_seed(IPMHandle* self);
int get_write_stars(IPMHandle* self);
int get_write_maps(IPMHandle* self);
int get_write_parities(IPMHandle* self);
int get_write_histograms(IPMHandle* self);
const char* get_outfile_prefix(IPMHandle* self);

/* results, src/lib_ipm.cu:71-78 */
int get_num_stars(IPMHandle* self);
IPM_DTYPE get_corner_x1(IPMHandle* self);
IPM_DTYPE get_corner_x2(IPMHandle* self);
IPM_DTYPE* get_stars(IPMHandle* self);          /* (x1, x2, m) x num_stars, tree order */
IPM_DTYPE* get_pixels(IPMHandle* self);         /* [num_pixels_y2][num_pixels_y1] magnification */
IPM_DTYPE* get_pixels_minima(IPMHandle* self);  /* NULL unless write_parities */
IPM_DTYPE* get_pixels_saddles(IPMHandle* self); /* NULL unless write_parities */
double get_t_shoot_cells(IPMHandle* self);      /* seconds */

/* src/lib_ipm.cu:80-81 */
bool run(IPMHandle* self, int verbose);
bool save(IPMHandle* self, int verbose);

/* ---- extensions (no counterpart in the reference ABI) ---- */
void destroy(IPMHandle* self);                       /* the reference never frees its objects */
void set_expansion_order(IPMHandle* self, int order); /* 0: reference formula (ipm.cuh:848); 3..31 fixed */
int get_expansion_order(IPMHandle* self);             /* order used by the last run */
void set_precision(IPMHandle* self, int mode);        /* 0 default, 1 FP64 plain form, 2 FP32 form */
int get_precision(IPMHandle* self);
/* star field from memory: n records (x1, x2, m), with a star file's shape, corner and theta_star */
void set_stars(IPMHandle* self, const IPM_DTYPE* xym, int n, int rectangular, IPM_DTYPE corner_x1,
               IPM_DTYPE corner_x2, IPM_DTYPE theta);
double get_t_pipeline(IPMHandle* self);               /* seconds: tree + expansions + shoot */
bool rerun(IPMHandle* self, int repeats, double* seconds); /* re-run tree+expansions+shoot on the resident stars */
void set_band(IPMHandle* self, long long first, long long last); /* lattice row band [first, last); last < 0: all */
void set_shoot_launch(IPMHandle* self, int threads, int ctas_per_sm); /* FP32 lens-equation kernel: 128/256/512 threads per CTA (8/4/2 lattice points per thread), CTAs per SM of its grid; other values: 128 and 64 */
int get_shoot_threads(IPMHandle* self);
int get_shoot_ctas_per_sm(IPMHandle* self);
bool copy_maps_device(IPMHandle* self, void* total, void* minima, void* saddles); /* integer maps to device buffers */
/* the last run's map (0 total, 1 minima, 2 saddles) into dst[num_pixels_y2][num_pixels_y1], several host threads */
bool copy_pixels(IPMHandle* self, int which, IPM_DTYPE* dst);
/* host buffer [num_pixels_y2][num_pixels_y1] that the next run() also fills with its map, copied chunk by
   chunk while the transfer goes on; one run, NULL to cancel */
void set_pixels_out(IPMHandle* self, IPM_DTYPE* dst);
bool derive(IPMHandle* self);                          /* validate + derived parameters, no GPU work */
double get_value(IPMHandle* self, const char* name);   /* derived / run-time value by name, NaN if unknown */
/* diagnostics: copies of internal device state */
int get_tree_num_nodes(IPMHandle* self);
bool copy_tree(IPMHandle* self, int* ints, double* geom, int* nbr, int* sil, int* dil);
bool copy_coeffs(IPMHandle* self, double* mult, double* loc);
long long get_num_vertices(IPMHandle* self);
bool copy_vertices(IPMHandle* self, double* out);
bool copy_fixed_maps(IPMHandle* self, unsigned long long* total, unsigned long long* minima,
                     unsigned long long* saddles);

/* Allocation-free deposition. No counterpart in the reference: for callers
 * that cannot let a library call cudaMalloc (device memory owned by their own
 * pool or budget, or latency-critical loops where allocation would
 * synchronise). Deposits the two triangles of each of ncx x ncy cells from the
 * (ncx+1) x (ncy+1) corner source positions at the device pointer verts
 * (double x, y pixel units, row axis flipped) into the npx x npy map at the
 * device pointer map, on the given cudaStream_t (NULL: default stream),
 * asynchronously. Scratch is one static device array per GPU (16.8 MB): maps
 * of at most 1024 * 1024 pixels in all and at most 1024 rows; larger sizes
 * return 1. Its first call on a device looks up the array's device address
 * and may load the module (make it at start-up, before any stream capture);
 * all calls share the array, so calls that overlap on the GPU race (order
 * them on one stream). Returns 0 on success, 4 for a launch error of this
 * call, 5 when an earlier CUDA error is pending (nothing queued). */
int ipm_deposit_noalloc(const double* verts, long long ncx, long long ncy, IPM_DTYPE factor, int npx, int npy,
                        IPM_DTYPE* map, void* stream);

/* Batches of realizations (no counterpart in the reference): many star
 * fields (own seed, convergence, shear, smooth fraction, mass function; one
 * map size) through one device pipeline whose tree build, expansions,
 * shooting and deposition are captured in one CUDA graph and replayed.
 * Realizations are described by objects of this library (init + setters) and
 * copied in by batch_add. The FP32 form is used; each map equals a single
 * run of the same inputs at the same expansion order (set_precision(2) on a
 * double object). */
void* batch_init(void);
void batch_destroy(void* batch);
int batch_add(void* batch, IPMHandle* realization);   /* returns its index */
int batch_size(void* batch);
void batch_set_expansion_order(void* batch, int order);     /* 0: largest reference-formula order */
void batch_set_corner_capacity(void* batch, long long n);   /* corner positions per pass; 0: automatic */
bool batch_run(void* batch, int verbose);
bool batch_rerun(void* batch, int repeats, double* seconds); /* replay on the resident star fields */
bool batch_copy_maps(void* batch, IPM_DTYPE* out);           /* [size][npy][npx] */
const IPM_DTYPE* batch_maps_device(void* batch);             /* the same maps on the device */
bool batch_copy_stars(void* batch, IPM_DTYPE* out);          /* all star fields, tree order, (x1, x2, m) */
double batch_get_value(void* batch, int r, const char* name); /* r >= 0: realization value; r < 0: batch value */

/* Adaptive IPM (no counterpart in the reference): the cell lattice is cut into
 * 32 x 32-cell tiles, each deposited at a subdivision level 1, 2, 4, 8 or 16
 * chosen by the level network (or uniform / given levels); every run audits a
 * seeded random sample of tiles against level 16 and sends a tile that misses
 * the tolerance to level 16. Map inputs are set on the object from ada_base. */
void* ada_init(void);
void ada_destroy(void* ada);
IPMHandle* ada_base(void* ada);                                   /* the map's inputs (setters of this library) */
void ada_set_policy(void* ada, int policy, int uniform_level);    /* 0 network, 1 uniform level, 2 given levels */
void ada_set_levels(void* ada, const int* levels, int n);         /* policy 2: one level per tile, row-major */
void ada_set_tolerance(void* ada, double eps);                    /* tolerance of a tile's deposit error */
void ada_set_error_mode(void* ada, int mode);   /* error as a share of 0: the tile's flux, 1: the map's flux there, 2: the smaller */
void ada_set_quantile(void* ada, float q);                        /* network: smallest level with cumulative p >= q */
void ada_set_max_level(void* ada, int level);                     /* labels / network stop here; the audit may go to 16 */
void ada_set_audit(void* ada, double fraction, unsigned seed);
void ada_set_audit_bound(void* ada, double bound);             /* audited miss share above which the level choice escalates */
void ada_set_refine_capacity(void* ada, long long corners);       /* refinement buffer, 0: automatic */
void ada_set_tiled_min(void* ada, int tiles);  /* chunks of >= tiles use the tiled lens kernel, smaller point by point */
void ada_set_network(void* ada, const float* w, const float* mu, const float* sig); /* 5061 weights, 8 + 8 */
bool ada_run(void* ada, int verbose);
int ada_num_tiles(void* ada);
bool ada_copy_features(void* ada, float* out);                   /* [tiles][8] */
bool ada_copy_levels(void* ada, int* out, int predicted);        /* final (after audit) or predicted levels */
bool ada_labels(void* ada, const int* tiles, int n, int* labels, float* err); /* classes 0..4, errors [n][4] */
bool ada_copy_map(void* ada, IPM_DTYPE* out);
double ada_get_value(void* ada, const char* name);

/* The level network alone (8 -> 64 -> 64 -> 5, BF16 weights, FP32
 * accumulation; no counterpart in the reference): device training with Adam,
 * gradients of the mean cross-entropy, argmax prediction. */
int mlp_num_params(void);
bool mlp_train(const float* feat, const int* labels, int n, int epochs, int batch, float lr, unsigned seed, float* w,
               float* mu, float* sig, float* epoch_loss);
bool mlp_gradients(const float* w, const float* mu, const float* sig, const float* feat, const int* labels, int n,
                   float* grad, float* mean_loss);
bool mlp_predict(const float* w, const float* mu, const float* sig, const float* feat, int n, int* cls);

#ifdef __cplusplus
}
#endif
#endif
