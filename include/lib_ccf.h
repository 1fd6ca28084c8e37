/*
 * lib_ccf.so -- critical curves and caustics of a star field, C ABI (double).
 *
 * Drop-in for the reference's src/lib_ccf.cu (weisluke/irs): same symbol names
 * and signatures, so microlensing/CCF/lib_ccf.py binds them unchanged. The
 * object handle is opaque.
 *
 * Pointers returned by get_stars / get_critical_curves / get_caustics /
 * get_mu_length_scales are host memory owned by the object, valid until the
 * next run() or destroy() on that object (the reference returns managed
 * memory). Critical curves and caustics are (num_roots * num_branches) rows of
 * (num_phi / num_branches + 1) complex values (re, im interleaved), row-major;
 * length scales the same shape of reals.
 * run() and save() return false after printing the reason to stderr.
 */
#ifndef IRS_B200_LIB_CCF_H
#define IRS_B200_LIB_CCF_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void CCFHandle;

/* src/lib_ccf.cu:15 */
CCFHandle* init(void);

/* setters, src/lib_ccf.cu:17-37 */
void set_kappa_tot(CCFHandle* self, double val);
void set_shear(CCFHandle* self, double val);
void set_kappa_star(CCFHandle* self, double val);
void set_theta_star(CCFHandle* self, double val);
void set_mass_function(CCFHandle* self, const char* val);
void set_m_solar(CCFHandle* self, double val);
void set_m_lower(CCFHandle* self, double val);
void set_m_upper(CCFHandle* self, double val);
void set_rectangular(CCFHandle* self, int val);
void set_approx(CCFHandle* self, int val);
void set_safety_scale(CCFHandle* self, double val);
void set_num_stars(CCFHandle* self, int val);
void set_starfile(CCFHandle* self, const char* val);
void set_num_phi(CCFHandle* self, int val);
void set_num_branches(CCFHandle* self, int val);
void set_random_seed(CCFHandle* self, int val);
void set_write_stars(CCFHandle* self, int val);
void set_write_critical_curves(CCFHandle* self, int val);
void set_write_caustics(CCFHandle* self, int val);
void set_write_mu_length_scales(CCFHandle* self, int val);
void set_outfile_prefix(CCFHandle* self, const char* val);

/* getters, src/lib_ccf.cu:39-59 */
double get_kappa_tot(CCFHandle* self);
double get_shear(CCFHandle* self);
double get_kappa_star(CCFHandle* self);
double get_theta_star(CCFHandle* self);
const char* get_mass_function(CCFHandle* self);
double get_m_solar(CCFHandle* self);
double get_m_lower(CCFHandle* self);
double get_m_upper(CCFHandle* self);
int get_rectangular(CCFHandle* self);
int get_approx(CCFHandle* self);
double get_safety_scale(CCFHandle* self);
int get_num_stars(CCFHandle* self);
const char* get_starfile(CCFHandle* self);
int get_num_phi(CCFHandle* self);
int get_num_branches(CCFHandle* self);
int get_random_seed(CCFHandle* self);
int get_write_stars(CCFHandle* self);
int get_write_critical_curves(CCFHandle* self);
int get_write_caustics(CCFHandle* self);
int get_write_mu_length_scales(CCFHandle* self);
const char* get_outfile_prefix(CCFHandle* self);

/* results, src/lib_ccf.cu:61-68 */
int get_num_roots(CCFHandle* self);
double get_corner_x1(CCFHandle* self);
double get_corner_x2(CCFHandle* self);
double* get_stars(CCFHandle* self);
double* get_critical_curves(CCFHandle* self);
double* get_caustics(CCFHandle* self);
double* get_mu_length_scales(CCFHandle* self);
double get_t_ccs(CCFHandle* self);

/* src/lib_ccf.cu:70-71 */
bool run(CCFHandle* self, int verbose);
bool save(CCFHandle* self, int verbose);

/* ---- extensions (no counterpart in the reference) ---- */
void destroy(CCFHandle* self);                                   /* the reference never frees its objects */
void set_num_iters(CCFHandle* self, int init_iters, int step_iters); /* default 30 and 20 (ccf.cuh:913, :985) */
double get_value(CCFHandle* self, const char* name);            /* derived / run-time value by name, NaN if unknown */

#ifdef __cplusplus
}
#endif
#endif
