/*
 * lib_ncc.so -- number-of-caustic-crossings maps, C ABI (double).
 *
 * Drop-in for the reference's src/lib_ncc.cu (weisluke/irs): same symbol names
 * and signatures, so microlensing/NCC/lib_ncc.py binds them unchanged. The
 * object handle is opaque. run() reads <infile_prefix>ccf_caustics.bin (the
 * caustics written by a CCF run, float or double) unless set_caustics gave
 * them. get_num_crossings returns host memory owned by the object
 * (num_pixels_y2 rows of num_pixels_y1 int32, row 0 at the top), valid until
 * the next run() or destroy(). run() and save() return false after printing
 * the reason to stderr.
 */
#ifndef IRS_B200_LIB_NCC_H
#define IRS_B200_LIB_NCC_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void NCCHandle;

/* src/lib_ncc.cu:15 */
NCCHandle* init(void);

/* setters, src/lib_ncc.cu:17-27 */
void set_infile_prefix(NCCHandle* self, const char* val);
void set_center_y1(NCCHandle* self, double val);
void set_center_y2(NCCHandle* self, double val);
void set_half_length_y1(NCCHandle* self, double val);
void set_half_length_y2(NCCHandle* self, double val);
void set_num_pixels_y1(NCCHandle* self, int val);
void set_num_pixels_y2(NCCHandle* self, int val);
void set_over_sample(NCCHandle* self, int val);
void set_write_maps(NCCHandle* self, int val);
void set_write_histograms(NCCHandle* self, int val);
void set_outfile_prefix(NCCHandle* self, const char* val);

/* getters, src/lib_ncc.cu:29-39 */
const char* get_infile_prefix(NCCHandle* self);
double get_center_y1(NCCHandle* self);
double get_center_y2(NCCHandle* self);
double get_half_length_y1(NCCHandle* self);
double get_half_length_y2(NCCHandle* self);
int get_num_pixels_y1(NCCHandle* self);
int get_num_pixels_y2(NCCHandle* self);
int get_over_sample(NCCHandle* self);
int get_write_maps(NCCHandle* self);
int get_write_histograms(NCCHandle* self);
const char* get_outfile_prefix(NCCHandle* self);

/* src/lib_ncc.cu:41-44 */
int* get_num_crossings(NCCHandle* self);
bool run(NCCHandle* self, int verbose);
bool save(NCCHandle* self, int verbose);

/* ---- extensions (no counterpart in the reference) ---- */
void destroy(NCCHandle* self);                                               /* the reference never frees its objects */
void set_caustics(NCCHandle* self, const double* vals, int nrows, int ncols); /* caustics from memory (re, im pairs) */
double get_value(NCCHandle* self, const char* name);                         /* t_ncc, t_reduce, min_num, max_num, ... */

#ifdef __cplusplus
}
#endif
#endif
