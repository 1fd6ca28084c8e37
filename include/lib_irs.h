/*
 * lib_irs.so / lib_irs_double.so -- inverse ray shooting, C ABI.
 *
 * The reference has no IRS library (its IRS class, include/irs.cuh, is only
 * reachable through the irs_gpu CLI). This ABI follows the conventions of
 * src/lib_ipm.cu so that a ctypes wrapper written like microlensing/IPM/lib_ipm.py
 * binds it: the same init / set_* / get_* / run / save names (defaults of
 * IRS<T>: light_loss 0.01, num_rays_y 100, include/irs.cuh:51,59), integer
 * ray-count maps, and the IRS results of include/irs.cuh:930-936.
 * IRS_DTYPE is float for lib_irs.so and double for lib_irs_double.so.
 */
#ifndef IRS_B200_LIB_IRS_H
#define IRS_B200_LIB_IRS_H
#include <stdbool.h>

#ifndef IRS_DTYPE
#define IRS_DTYPE float
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef void IRSHandle;

IRSHandle* init(void);
void set_kappa_tot(IRSHandle* self, IRS_DTYPE val);
void set_shear(IRSHandle* self, IRS_DTYPE val);
void set_kappa_star(IRSHandle* self, IRS_DTYPE val);
void set_theta_star(IRSHandle* self, IRS_DTYPE val);
void set_mass_function(IRSHandle* self, const char* val);
void set_m_solar(IRSHandle* self, IRS_DTYPE val);
void set_m_lower(IRSHandle* self, IRS_DTYPE val);
void set_m_upper(IRSHandle* self, IRS_DTYPE val);
void set_light_loss(IRSHandle* self, IRS_DTYPE val);
void set_rectangular(IRSHandle* self, int val);
void set_approx(IRSHandle* self, int val);
void set_safety_scale(IRSHandle* self, IRS_DTYPE val);
void set_starfile(IRSHandle* self, const char* val);
void set_center_y1(IRSHandle* self, IRS_DTYPE val);
void set_center_y2(IRSHandle* self, IRS_DTYPE val);
void set_half_length_y1(IRSHandle* self, IRS_DTYPE val);
void set_half_length_y2(IRSHandle* self, IRS_DTYPE val);
void set_num_pixels_y1(IRSHandle* self, int val);
void set_num_pixels_y2(IRSHandle* self, int val);
void set_num_rays_y(IRSHandle* self, int val);
void set_random_seed(IRSHandle* self, int val);
void set_write_stars(IRSHandle* self, int val);
void set_write_maps(IRSHandle* self, int val);
void set_write_parities(IRSHandle* self, int val);
void set_write_histograms(IRSHandle* self, int val);
void set_outfile_prefix(IRSHandle* self, const char* val);

IRS_DTYPE get_kappa_tot(IRSHandle* self);
IRS_DTYPE get_shear(IRSHandle* self);
IRS_DTYPE get_kappa_star(IRSHandle* self);
IRS_DTYPE get_theta_star(IRSHandle* self);
const char* get_mass_function(IRSHandle* self);
IRS_DTYPE get_m_solar(IRSHandle* self);
IRS_DTYPE get_m_lower(IRSHandle* self);
IRS_DTYPE get_m_upper(IRSHandle* self);
IRS_DTYPE get_light_loss(IRSHandle* self);
int get_rectangular(IRSHandle* self);
int get_approx(IRSHandle* self);
IRS_DTYPE get_safety_scale(IRSHandle* self);
const char* get_starfile(IRSHandle* self);
IRS_DTYPE get_center_y1(IRSHandle* self);
IRS_DTYPE get_center_y2(IRSHandle* self);
IRS_DTYPE get_half_length_y1(IRSHandle* self);
IRS_DTYPE get_half_length_y2(IRSHandle* self);
int get_num_pixels_y1(IRSHandle* self);
int get_num_pixels_y2(IRSHandle* self);
int get_num_rays_y(IRSHandle* self);
int get_random_seed(IRSHandle* self);
int get_write_stars(IRSHandle* self);
int get_write_maps(IRSHandle* self);
int get_write_parities(IRSHandle* self);
int get_write_histograms(IRSHandle* self);
const char* get_outfile_prefix(IRSHandle* self);

int get_num_stars(IRSHandle* self);
IRS_DTYPE get_corner_x1(IRSHandle* self);
IRS_DTYPE get_corner_x2(IRSHandle* self);
IRS_DTYPE* get_stars(IRSHandle* self);
int* get_pixels(IRSHandle* self);          /* [num_pixels_y2][num_pixels_y1] ray counts */
int* get_pixels_minima(IRSHandle* self);   /* NULL unless write_parities */
int* get_pixels_saddles(IRSHandle* self);  /* NULL unless write_parities */
double get_t_shoot_rays(IRSHandle* self);  /* seconds (include/irs.cuh:927) */
unsigned long long get_num_rays_shot(IRSHandle* self);      /* include/irs.cuh:930-932 */
unsigned long long get_num_rays_received(IRSHandle* self);  /* include/irs.cuh:934-935 */
bool run(IRSHandle* self, int verbose);
bool save(IRSHandle* self, int verbose);

/* extensions, as in lib_ipm.h */
void destroy(IRSHandle* self);
void set_expansion_order(IRSHandle* self, int order);
int get_expansion_order(IRSHandle* self);
void set_precision(IRSHandle* self, int mode);
int get_precision(IRSHandle* self);
void set_stars(IRSHandle* self, const IRS_DTYPE* xym, int n, int rectangular, IRS_DTYPE corner_x1,
               IRS_DTYPE corner_x2, IRS_DTYPE theta);
double get_t_pipeline(IRSHandle* self);
bool rerun(IRSHandle* self, int repeats, double* seconds); /* re-run tree+expansions+shoot on the resident stars */
void set_band(IRSHandle* self, long long first, long long last); /* lattice row band [first, last); last < 0: all */
void set_shoot_launch(IRSHandle* self, int threads, int ctas_per_sm); /* FP32 lens-equation kernel: 128/256/512 threads per CTA (8/4/2 lattice points per thread), CTAs per SM of its grid; other values: 128 and 64 */
int get_shoot_threads(IRSHandle* self);
int get_shoot_ctas_per_sm(IRSHandle* self);
bool copy_maps_device(IRSHandle* self, void* total, void* minima, void* saddles); /* integer maps to device buffers */
/* the last run's map (0 total, 1 minima, 2 saddles) into dst[num_pixels_y2][num_pixels_y1], several host threads */
bool copy_pixels(IRSHandle* self, int which, int* dst);
/* host buffer [num_pixels_y2][num_pixels_y1] that the next run() also fills with its map, copied chunk by
   chunk while the transfer goes on; one run, NULL to cancel */
void set_pixels_out(IRSHandle* self, int* dst);
bool derive(IRSHandle* self);
double get_value(IRSHandle* self, const char* name);
int get_tree_num_nodes(IRSHandle* self);
bool copy_tree(IRSHandle* self, int* ints, double* geom, int* nbr, int* sil, int* dil);
bool copy_coeffs(IRSHandle* self, double* mult, double* loc);

#ifdef __cplusplus
}
#endif
#endif
