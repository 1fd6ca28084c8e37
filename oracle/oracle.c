/*
 * CPU oracle for the irs_b200 map engine -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is a plain-C, FP64 restatement of the reference's IRS/IPM
 * algorithm (weisluke/irs). Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark load it; the product never calls it.
 *
 * Restated pieces (reference file:line):
 *   complex arithmetic (Smith division)     include/complex.cuh:218-280
 *   derived parameters (double)             include/ipm.cuh:434-559
 *   quadtree build, neighbour rules         include/tree_node.cuh:151-267, 321-519
 *   nearest node descent                    include/tree_node.cuh:529-561
 *   FMM coefficients P2M/M2M/L2L/M2L/P2L     include/fmm.cuh:21-413, schedule ipm.cuh:874-901
 *   alpha_star / alpha_local / alpha_smooth include/alpha_star.cuh:18-41, alpha_local.cuh:18-36,
 *                                           alpha_smooth.cuh:62-127 (+ derivatives :141-236)
 *   lens equation and magnification         include/irs_functions.cuh:33-81
 *   IRS binning (clamp, row flip)           include/irs_functions.cuh:147-198
 *   IPM triangles and polygon deposition    include/ipm_functions.cuh:123-216, polygon.cuh:116-467
 * Additionally:
 *   a direct FP64 sum over all stars (no expansion), OpenMP-parallel: the
 *   accuracy oracle;
 *   the fixed-point deposition of the GPU kernels (linear-interpolation edge
 *   intersections, explicitly rounded float/double operations, 2^32 fixed
 *   point), for the bit-exactness check. Compile with -ffp-contract=off.
 *
 * Tree construction order: the reference places children and partitions
 * stars with atomics (nondeterministic order); here node slots follow the
 * level order and the quadrant partition is stable, which gives the same tree
 * structure in a reproducible order.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAX_DIRECT 32
#define MAX_ORDER 31
#define NBR_CAP 8
#define SIL_CAP 27
#define DIL_CAP 5

typedef struct {
  double re, im;
} cx;

static inline cx C(double a, double b) {
  cx c;
  c.re = a;
  c.im = b;
  return c;
}
static inline cx cadd(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
static inline cx cmul(cx a, cx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx cscal(cx a, double s) { return C(a.re * s, a.im * s); }
static inline cx cdivr(cx a, double s) { return C(a.re / s, a.im / s); }
static inline cx cconj(cx a) { return C(a.re, -a.im); }
static inline cx cneg(cx a) { return C(-a.re, -a.im); }
/* complex.cuh:247-262 */
static inline cx cdiv(cx a, cx b) {
  if (fabs(b.im) < fabs(b.re)) {
    double f = b.im / b.re, d = b.re + b.im * f;
    return C((a.re + a.im * f) / d, (a.im - a.re * f) / d);
  } else {
    double f = b.re / b.im, d = b.re * f + b.im;
    return C((a.re * f + a.im) / d, (a.im * f - a.re) / d);
  }
}
/* complex.cuh:267-280: real / complex */
static inline cx rdiv(double num, cx b) {
  if (fabs(b.im) < fabs(b.re)) {
    double f = b.im / b.re, d = b.re + b.im * f;
    return C(num / d, (-num * f) / d);
  } else {
    double f = b.re / b.im, d = b.re * f + b.im;
    return C((num * f) / d, -num / d);
  }
}
static inline double cabsv(cx a) { return hypot(a.re, a.im); }
static inline cx clogc(cx a) { return C(log(cabsv(a)), atan2(a.im, a.re)); }
static inline cx cexpc(cx a) { return C(exp(a.re) * cos(a.im), exp(a.re) * sin(a.im)); }
static inline cx cpowi(cx a, int n) {
  cx r = C(1, 0);
  for (int i = 0; i < n; i++) r = cmul(r, a);
  return r;
}

/* ------------------------------------------------------------ lens model */
typedef struct {
  double kappa, gamma, kstar, theta;
  int rect, approx, taylor_smooth;
  double corner_re, corner_im;
} OrcLens;

/* alpha_smooth.cuh:62-127 */
static cx alpha_smooth(cx z, const OrcLens* L) {
  const double ks = L->kstar, ip = 1.0 / M_PI;
  cx c = C(L->corner_re, L->corner_im);
  cx a;
  if (L->rect) {
    cx zb = cconj(z);
    if (L->approx) {
      cx s1 = C(0, 0), s2 = s1, s3 = s1, s4 = s1;
      for (int i = L->taylor_smooth; i >= 1; i--) {
        s1.re += 1.0 / i;
        s2.re += 1.0 / i;
        s3.re += 1.0 / i;
        s4.re += 1.0 / i;
        s1 = cmul(s1, cdiv(zb, c));
        s2 = cmul(s2, cdiv(zb, cconj(c)));
        s3 = cmul(s3, cdiv(zb, cneg(c)));
        s4 = cmul(s4, cdiv(zb, cneg(cconj(c))));
      }
      a = csub(cmul(csub(c, zb), csub(clogc(c), s1)), cmul(csub(cconj(c), zb), csub(clogc(cconj(c)), s2)));
      a = cadd(a, cmul(csub(cneg(c), zb), csub(clogc(cneg(c)), s3)));
      a = csub(a, cmul(csub(cneg(cconj(c)), zb), csub(clogc(cconj(cneg(c))), s4)));
      a = cmul(a, C(0, -ks * ip));
      a.re -= ks * 2 * (c.re + z.re);
    } else {
      cx c1 = csub(c, zb), c2 = csub(cconj(c), zb), c3 = csub(cneg(c), zb), c4 = csub(cneg(cconj(c)), zb);
      a = csub(cadd(csub(cmul(c1, clogc(c1)), cmul(c2, clogc(c2))), cmul(c3, clogc(c3))), cmul(c4, clogc(c4)));
      a = cmul(a, C(0, -ks * ip));
      double box = (-c.re <= z.re && z.re <= c.re && -c.im <= z.im && z.im <= c.im) ? 1.0 : 0.0;
      a.re -= ks * 2 * (c.re + z.re) * box;
      double h = ((c.im + z.im) >= 0 ? 1.0 : 0.0) * ((c.im - z.im) >= 0 ? 1.0 : 0.0) * ((z.re - c.re) >= 0 ? 1.0 : 0.0);
      a.re -= ks * 4 * c.re * h;
    }
  } else {
    if (L->approx) {
      a = cscal(z, -ks);
    } else {
      double ca = cabsv(c);
      if (cabsv(z) <= ca)
        a = cscal(z, -ks);
      else
        a = rdiv(-ks * ca * ca, cconj(z));
    }
  }
  return a;
}
/* alpha_smooth.cuh:141-170 */
static double d_alpha_smooth_dz(cx z, const OrcLens* L) {
  cx c = C(L->corner_re, L->corner_im);
  if (L->approx) return -L->kstar;
  if (L->rect) {
    double box = (-c.re <= z.re && z.re <= c.re && -c.im <= z.im && z.im <= c.im) ? 1.0 : 0.0;
    return -L->kstar * box;
  }
  return -L->kstar * ((cabsv(c) - cabsv(z)) >= 0 ? 1.0 : 0.0);
}
/* alpha_smooth.cuh:185-236 */
static cx d_alpha_smooth_dzbar(cx z, const OrcLens* L) {
  const double ks = L->kstar, ip = 1.0 / M_PI;
  cx c = C(L->corner_re, L->corner_im);
  cx d = C(0, 0);
  if (L->rect) {
    if (L->approx) {
      cx r = cdiv(cconj(z), c);
      double ph = atan2(c.im, c.re);
      for (int i = L->taylor_smooth - 1; i >= 2; i -= 2) {
        cx e = cexpc(C(0, 2 * ph * i));
        d = cadd(d, cdivr(C(1 - e.re, -e.im), (double)i));
        d = cmul(d, cmul(r, r));
      }
      d = cscal(d, 2.0);
      d = cmul(d, C(0, -ks * ip));
      d.re += ks - 4 * ks * ph * ip;
    } else {
      cx c1 = csub(cconj(c), cconj(z)), c2 = csub(c, cconj(z)), c3 = csub(cneg(c), cconj(z)),
         c4 = csub(cneg(cconj(c)), cconj(z));
      d = cadd(csub(csub(clogc(c1), clogc(c2)), clogc(c3)), clogc(c4));
      d = cmul(d, C(0, -ks * ip));
      double box = (-c.re <= z.re && z.re <= c.re && -c.im <= z.im && z.im <= c.im) ? 1.0 : 0.0;
      d.re -= ks * box;
    }
  } else if (!L->approx) {
    double ca = cabsv(c);
    cx zb = cconj(z);
    d = rdiv(ks * ca * ca, cmul(zb, zb));
  }
  return d;
}

/* ------------------------------------------------------------ quadtree */
typedef struct {
  int n, cap, levels, nlevels_alloc;
  int* level_off;
  double *cx, *cy, *hl;
  int *level, *parent, *child0, *sbeg, *scnt;
  int *nbr, *n_nbr, *sil, *n_sil, *dil, *n_dil;
  int p;
  cx *mult, *loc;
  int nstars;
  double *sx, *sy, *sm;
  int overflow;
} OrcTree;

static void tree_grow(OrcTree* t, int want) {
  if (want <= t->cap) return;
  int nc = t->cap ? t->cap : 1024;
  while (nc < want) nc *= 2;
#define GROW(f, ty, k) t->f = (ty*)realloc(t->f, (size_t)nc * (k) * sizeof(ty))
  GROW(cx, double, 1);
  GROW(cy, double, 1);
  GROW(hl, double, 1);
  GROW(level, int, 1);
  GROW(parent, int, 1);
  GROW(child0, int, 1);
  GROW(sbeg, int, 1);
  GROW(scnt, int, 1);
  GROW(nbr, int, NBR_CAP);
  GROW(n_nbr, int, 1);
  GROW(sil, int, SIL_CAP);
  GROW(n_sil, int, 1);
  GROW(dil, int, DIL_CAP);
  GROW(n_dil, int, 1);
#undef GROW
  t->cap = nc;
}

static int quadrant(double x, double y, double cxv, double cyv) {
  if (x >= cxv && y >= cyv) return 0;
  if (x < cxv && y >= cyv) return 1;
  if (x < cxv && y < cyv) return 2;
  return 3;
}

/* tree_node.cuh:183-267 */
static void set_neighbors(OrcTree* t, int k) {
  int p = t->parent[k];
  double h = t->hl[k], x = t->cx[k], y = t->cy[k];
  int nn = 0, ns = 0, nd = 0;
  for (int i = 0; i < 4; i++) {
    int c = t->child0[p] + i;
    if (t->scnt[c] == 0) continue;
    if (c != k) {
      if (nn < NBR_CAP) t->nbr[k * NBR_CAP + nn] = c;
      else t->overflow |= 1;
      nn++;
    }
  }
  for (int i = 0; i < t->n_nbr[p]; i++) {
    int nb = t->nbr[p * NBR_CAP + i];
    if (t->scnt[nb] == 0) continue;
    if (t->child0[nb] < 0) {
      if (fabs(t->cx[nb] - x) < 3.5 * h && fabs(t->cy[nb] - y) < 3.5 * h) {
        if (nn < NBR_CAP) t->nbr[k * NBR_CAP + nn] = nb;
        else t->overflow |= 1;
        nn++;
      } else {
        if (nd < DIL_CAP) t->dil[k * DIL_CAP + nd] = nb;
        else t->overflow |= 4;
        nd++;
      }
    } else {
      for (int j = 0; j < 4; j++) {
        int c = t->child0[nb] + j;
        if (t->scnt[c] == 0) continue;
        if (fabs(t->cx[c] - x) < 3 * h && fabs(t->cy[c] - y) < 3 * h) {
          if (nn < NBR_CAP) t->nbr[k * NBR_CAP + nn] = c;
          else t->overflow |= 1;
          nn++;
        } else {
          if (ns < SIL_CAP) t->sil[k * SIL_CAP + ns] = c;
          else t->overflow |= 2;
          ns++;
        }
      }
    }
  }
  t->n_nbr[k] = nn < NBR_CAP ? nn : NBR_CAP;
  t->n_sil[k] = ns < SIL_CAP ? ns : SIL_CAP;
  t->n_dil[k] = nd < DIL_CAP ? nd : DIL_CAP;
}

static double binom_tab[(2 * MAX_ORDER + 1) * (2 * MAX_ORDER + 2) / 2];
static void binom_init(void) {
  static int done = 0;
  if (done) return;
  long long t[(2 * MAX_ORDER + 1) * (2 * MAX_ORDER + 2) / 2];
  for (int n = 0; n <= 2 * MAX_ORDER; n++) {
    int r = n * (n + 1) / 2, pr = (n - 1) * n / 2;
    for (int i = 0; i <= n; i++) t[r + i] = (i == 0 || i == n) ? 1 : t[pr + i - 1] + t[pr + i];
  }
  for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); i++) binom_tab[i] = (double)t[i];
  done = 1;
}
static inline double binom(int n, int k) {
  if (n < k || k < 0) return 0.0;
  return binom_tab[n * (n + 1) / 2 + k];
}

/* fmm.cuh:21-49 */
static void p2m(OrcTree* t, int k) {
  int P = t->p;
  cx* a = t->mult + (size_t)k * (P + 1);
  for (int l = 0; l <= P; l++) {
    cx r = C(0, 0);
    for (int i = 0; i < t->scnt[k]; i++) {
      int s = t->sbeg[k] + i;
      if (l == 0) {
        r.re += t->sm[s];
      } else {
        cx d = C((t->sx[s] - t->cx[k]) / t->hl[k], (t->sy[s] - t->cy[k]) / t->hl[k]);
        r = csub(r, cscal(cpowi(d, l), t->sm[s]));
      }
    }
    if (l > 0) r = cdivr(r, (double)l);
    a[l] = r;
  }
}
/* fmm.cuh:109-139 and the child sum of :183-189 */
static void m2m(OrcTree* t, int k) {
  int P = t->p;
  cx* b = t->mult + (size_t)k * (P + 1);
  for (int j = 0; j < 4; j++) {
    int c = t->child0[k] + j;
    cx* a = t->mult + (size_t)c * (P + 1);
    cx dz = C((t->cx[c] - t->cx[k]) / t->hl[c], (t->cy[c] - t->cy[k]) / t->hl[c]);
    for (int l = 0; l <= P; l++) {
      cx r;
      if (l == 0) {
        r = a[0];
      } else {
        r = C(0, 0);
        for (int i = P; i >= 1; i--) {
          r = cadd(r, cscal(a[i], binom(l - 1, i - 1)));
          r = cdiv(r, dz);
        }
        r = csub(r, cdivr(a[0], (double)l));
        r = cmul(r, cpowi(dz, l));
        r = cdivr(r, (double)(1u << l));
      }
      b[l] = cadd(b[l], r);
    }
  }
}
/* fmm.cuh:204-223 */
static void l2l(OrcTree* t, int k, cx* out) {
  int P = t->p, pa = t->parent[k];
  cx* cpar = t->loc + (size_t)pa * (P + 1);
  cx dz = C((t->cx[k] - t->cx[pa]) / t->hl[pa], (t->cy[k] - t->cy[pa]) / t->hl[pa]);
  for (int l = 0; l <= P; l++) {
    cx r = C(0, 0);
    for (int i = P; i >= 1; i--) {
      r = cadd(r, cscal(cpar[i], binom(i, l)));
      r = cmul(r, dz);
    }
    r = cdiv(r, cpowi(dz, l));
    r = cdivr(r, (double)(1u << l));
    out[l] = r;
  }
}
/* fmm.cuh:281-322 */
static void m2l(OrcTree* t, int f, int k, cx* acc) {
  int P = t->p;
  cx* b = t->mult + (size_t)f * (P + 1);
  cx dz = C((t->cx[f] - t->cx[k]) / t->hl[f], (t->cy[f] - t->cy[k]) / t->hl[f]);
  for (int l = 0; l <= P; l++) {
    cx r = C(0, 0);
    if (l == 0) {
      for (int i = P; i >= 1; i--) {
        r = cadd(r, b[i]);
        r = cdiv(r, cneg(dz));
      }
      r = cadd(r, cmul(b[0], clogc(cneg(dz))));
      r = cadd(r, cscal(b[0], log(t->hl[f])));
    } else {
      for (int i = P; i >= 1; i--) {
        r = cadd(r, cscal(b[i], binom(l + i - 1, i - 1)));
        r = cdiv(r, cneg(dz));
      }
      r = csub(r, cdivr(b[0], (double)l));
      r = cdiv(r, cpowi(dz, l));
    }
    acc[l] = cadd(acc[l], r);
  }
}
/* fmm.cuh:387-413 */
static void p2l(OrcTree* t, int f, int k, cx* acc) {
  int P = t->p;
  for (int l = 0; l <= P; l++) {
    cx r = C(0, 0);
    for (int i = 0; i < t->scnt[f]; i++) {
      int s = t->sbeg[f] + i;
      cx d = C((t->sx[s] - t->cx[k]) / t->hl[k], (t->sy[s] - t->cy[k]) / t->hl[k]);
      double m = t->sm[s];
      if (l == 0) {
        r = cadd(r, cscal(clogc(cneg(d)), m));
        r.re += m * log(t->hl[k]);
      } else {
        r = csub(r, rdiv(m, cscal(cpowi(d, l), (double)l)));
      }
    }
    acc[l] = cadd(acc[l], r);
  }
}

void orc_tree_free(OrcTree* t) {
  if (!t) return;
  free(t->level_off);
  free(t->cx);
  free(t->cy);
  free(t->hl);
  free(t->level);
  free(t->parent);
  free(t->child0);
  free(t->sbeg);
  free(t->scnt);
  free(t->nbr);
  free(t->n_nbr);
  free(t->sil);
  free(t->n_sil);
  free(t->dil);
  free(t->n_dil);
  free(t->mult);
  free(t->loc);
  free(t->sx);
  free(t->sy);
  free(t->sm);
  free(t);
}

/* Builds the tree (include/ipm.cuh:740-842) and the expansions (:848-901).
 * xym: n records (x, y, m). p: expansion order, or 0 for the reference
 * formula with theta and alpha_error. */
OrcTree* orc_tree_build(int n, const double* xym, double root_hl, int p, double theta, double alpha_error) {
  binom_init();
  OrcTree* t = (OrcTree*)calloc(1, sizeof(OrcTree));
  t->nstars = n;
  t->sx = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  t->sy = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  t->sm = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    t->sx[i] = xym[3 * i];
    t->sy[i] = xym[3 * i + 1];
    t->sm[i] = xym[3 * i + 2];
  }
  tree_grow(t, 1024);
  t->nlevels_alloc = 64;
  t->level_off = (int*)malloc(sizeof(int) * t->nlevels_alloc);
  t->cx[0] = 0;
  t->cy[0] = 0;
  t->hl[0] = root_hl;
  t->level[0] = 0;
  t->parent[0] = -1;
  t->child0[0] = -1;
  t->sbeg[0] = 0;
  t->scnt[0] = n;
  t->n_nbr[0] = t->n_sil[0] = t->n_dil[0] = 0;
  t->level_off[0] = 0;
  t->level_off[1] = 1;
  t->levels = 0;
  double *tx = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *ty = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *tm = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int l = 0; l < 40; l++) {
    int beg = t->level_off[l], end = t->level_off[l + 1];
    int maxc = 0, nsplit = 0;
    int* split = (int*)malloc(sizeof(int) * (size_t)(end - beg + 1));
    for (int k = beg; k < end; k++) {
      int c = t->scnt[k];
      for (int j = 0; j < t->n_nbr[k]; j++) c += t->scnt[t->nbr[k * NBR_CAP + j]];
      split[k - beg] = c > MAX_DIRECT;
      nsplit += split[k - beg];
      if (c > maxc) maxc = c;
    }
    if (maxc <= MAX_DIRECT) {
      free(split);
      break;
    }
    tree_grow(t, end + 4 * nsplit);
    int next = end;
    static const double ox[4] = {1, -1, -1, 1}, oy[4] = {1, 1, -1, -1};
    for (int k = beg; k < end; k++) {
      if (!split[k - beg]) {
        t->child0[k] = -1;
        continue;
      }
      t->child0[k] = next;
      double h = t->hl[k] / 2;
      for (int q = 0; q < 4; q++) {
        int c = next + q;
        t->cx[c] = t->cx[k] + h * ox[q];
        t->cy[c] = t->cy[k] + h * oy[q];
        t->hl[c] = h;
        t->level[c] = l + 1;
        t->parent[c] = k;
        t->child0[c] = -1;
        t->sbeg[c] = t->sbeg[k];
        t->scnt[c] = 0;
        t->n_nbr[c] = t->n_sil[c] = t->n_dil[c] = 0;
      }
      /* stable quadrant partition (sort_stars_kernel, tree_node.cuh:392-501) */
      int b = t->sbeg[k], m = t->scnt[k], cnt[4] = {0, 0, 0, 0};
      for (int i = 0; i < m; i++) cnt[quadrant(t->sx[b + i], t->sy[b + i], t->cx[k], t->cy[k])]++;
      int off[4];
      off[0] = b;
      for (int q = 1; q < 4; q++) off[q] = off[q - 1] + cnt[q - 1];
      for (int q = 0; q < 4; q++) {
        t->sbeg[next + q] = off[q];
        t->scnt[next + q] = cnt[q];
      }
      for (int i = 0; i < m; i++) {
        int q = quadrant(t->sx[b + i], t->sy[b + i], t->cx[k], t->cy[k]);
        int d = off[q]++;
        tx[d] = t->sx[b + i];
        ty[d] = t->sy[b + i];
        tm[d] = t->sm[b + i];
      }
      for (int i = 0; i < m; i++) {
        t->sx[b + i] = tx[b + i];
        t->sy[b + i] = ty[b + i];
        t->sm[b + i] = tm[b + i];
      }
      next += 4;
    }
    free(split);
    for (int c = end; c < next; c++) set_neighbors(t, c);
    t->levels++;
    t->level_off[l + 2] = next;
  }
  free(tx);
  free(ty);
  free(tm);
  t->n = t->level_off[t->levels + 1];
  if (p <= 0) p = (int)ceil(2 * log2(theta) + t->levels - log2(root_hl) - log2(alpha_error));
  if (p < 1) p = 1;
  if (p > MAX_ORDER) p = MAX_ORDER;
  t->p = p;
  t->mult = (cx*)calloc((size_t)t->n * (p + 1), sizeof(cx));
  t->loc = (cx*)calloc((size_t)t->n * (p + 1), sizeof(cx));
  for (int l = t->levels; l >= 0; l--) {
    for (int k = t->level_off[l]; k < t->level_off[l + 1]; k++) {
      if (t->child0[k] < 0 && t->scnt[k] > 0) p2m(t, k);
      if (t->child0[k] >= 0) m2m(t, k);
    }
  }
  for (int l = 2; l <= t->levels; l++) {
    for (int k = t->level_off[l]; k < t->level_off[l + 1]; k++) {
      cx* acc = t->loc + (size_t)k * (p + 1);
      l2l(t, k, acc);
      for (int j = 0; j < t->n_sil[k]; j++) m2l(t, t->sil[k * SIL_CAP + j], k, acc);
      for (int j = 0; j < t->n_dil[k]; j++) p2l(t, t->dil[k * DIL_CAP + j], k, acc);
    }
  }
  return t;
}

int orc_tree_num_nodes(const OrcTree* t) { return t->n; }
int orc_tree_levels(const OrcTree* t) { return t->levels; }
int orc_tree_order(const OrcTree* t) { return t->p; }
int orc_tree_overflow(const OrcTree* t) { return t->overflow; }
void orc_tree_stars(const OrcTree* t, double* xym) {
  for (int i = 0; i < t->nstars; i++) {
    xym[3 * i] = t->sx[i];
    xym[3 * i + 1] = t->sy[i];
    xym[3 * i + 2] = t->sm[i];
  }
}
/* ints[k*8 + .] = level, parent, child0, sbeg, scnt, n_nbr, n_sil, n_dil; geom[k*3+.] = cx, cy, hl */
void orc_tree_nodes(const OrcTree* t, int* ints, double* geom, int* nbr, int* sil, int* dil) {
  for (int k = 0; k < t->n; k++) {
    int* o = ints + 8 * (size_t)k;
    o[0] = t->level[k];
    o[1] = t->parent[k];
    o[2] = t->child0[k];
    o[3] = t->sbeg[k];
    o[4] = t->scnt[k];
    o[5] = t->n_nbr[k];
    o[6] = t->n_sil[k];
    o[7] = t->n_dil[k];
    geom[3 * (size_t)k] = t->cx[k];
    geom[3 * (size_t)k + 1] = t->cy[k];
    geom[3 * (size_t)k + 2] = t->hl[k];
    if (nbr) memcpy(nbr + (size_t)k * NBR_CAP, t->nbr + (size_t)k * NBR_CAP, sizeof(int) * NBR_CAP);
    if (sil) memcpy(sil + (size_t)k * SIL_CAP, t->sil + (size_t)k * SIL_CAP, sizeof(int) * SIL_CAP);
    if (dil) memcpy(dil + (size_t)k * DIL_CAP, t->dil + (size_t)k * DIL_CAP, sizeof(int) * DIL_CAP);
  }
}
void orc_tree_coeffs(const OrcTree* t, double* mult, double* loc) {
  size_t m = (size_t)t->n * (t->p + 1);
  for (size_t i = 0; i < m; i++) {
    mult[2 * i] = t->mult[i].re;
    mult[2 * i + 1] = t->mult[i].im;
    loc[2 * i] = t->loc[i].re;
    loc[2 * i + 1] = t->loc[i].im;
  }
}

/* tree_node.cuh:529-561 */
static int nearest_node(const OrcTree* t, cx z) {
  int k = 0;
  while (t->child0[k] >= 0) {
    if (fabs(z.re - t->cx[k]) > t->hl[k] || fabs(z.im - t->cy[k]) > t->hl[k]) return k;
    int q;
    if (z.re >= t->cx[k] && z.im >= t->cy[k]) q = 0;
    else if (z.re < t->cx[k] && z.im >= t->cy[k]) q = 1;
    else if (z.re < t->cx[k] && z.im < t->cy[k]) q = 2;
    else q = 3;
    k = t->child0[k] + q;
  }
  return k;
}

/* alpha_star.cuh:18-41 */
static cx alpha_star_node(const OrcTree* t, cx z, int k, double theta) {
  cx a = C(0, 0);
  for (int j = 0; j < t->n_nbr[k]; j++) {
    int nb = t->nbr[k * NBR_CAP + j];
    for (int i = 0; i < t->scnt[nb]; i++) {
      int s = t->sbeg[nb] + i;
      a = cadd(a, rdiv(t->sm[s], csub(z, C(t->sx[s], t->sy[s]))));
    }
  }
  for (int i = 0; i < t->scnt[k]; i++) {
    int s = t->sbeg[k] + i;
    a = cadd(a, rdiv(t->sm[s], csub(z, C(t->sx[s], t->sy[s]))));
  }
  a = cscal(a, theta * theta);
  return cconj(a);
}
static cx d_alpha_star_node(const OrcTree* t, cx z, int k, double theta) {
  cx a = C(0, 0);
  for (int j = 0; j <= t->n_nbr[k]; j++) {
    int nb = j < t->n_nbr[k] ? t->nbr[k * NBR_CAP + j] : k;
    for (int i = 0; i < t->scnt[nb]; i++) {
      int s = t->sbeg[nb] + i;
      cx d = csub(z, C(t->sx[s], t->sy[s]));
      a = cadd(a, rdiv(t->sm[s], cmul(d, d)));
    }
  }
  a = cscal(a, -theta * theta);
  return cconj(a);
}
/* alpha_local.cuh:18-36 */
static cx alpha_local_node(const OrcTree* t, cx z, int k, double theta) {
  int P = t->p;
  const cx* c = t->loc + (size_t)k * (P + 1);
  cx dz = cdivr(csub(z, C(t->cx[k], t->cy[k])), t->hl[k]);
  cx a = C(0, 0);
  for (int i = P; i >= 1; i--) {
    a = cmul(a, dz);
    a = cadd(a, cscal(c[i], (double)i));
  }
  a = cscal(a, theta * theta);
  a = cdivr(a, t->hl[k]);
  return cconj(a);
}
static cx d_alpha_local_node(const OrcTree* t, cx z, int k, double theta) {
  int P = t->p;
  const cx* c = t->loc + (size_t)k * (P + 1);
  cx dz = cdivr(csub(z, C(t->cx[k], t->cy[k])), t->hl[k]);
  cx a = C(0, 0);
  for (int i = P; i >= 2; i--) {
    a = cmul(a, dz);
    a = cadd(a, cscal(c[i], (double)(i * (i - 1))));
  }
  a = cscal(a, theta * theta);
  a = cdivr(a, t->hl[k] * t->hl[k]);
  return cconj(a);
}

/* Source positions of npts image-plane points, FMM form (complex_image_to_source).
 * mu (optional) receives the magnification (irs_functions.cuh:66-81). */
void orc_shoot_fmm(const OrcTree* t, const OrcLens* L, long long npts, const double* zx, const double* zy, double* wx,
                   double* wy, double* mu) {
#pragma omp parallel for schedule(dynamic, 4096)
  for (long long i = 0; i < npts; i++) {
    cx z = C(zx[i], zy[i]);
    int k = nearest_node(t, z);
    cx as = alpha_star_node(t, z, k, L->theta);
    cx al = alpha_local_node(t, z, k, L->theta);
    cx sm = alpha_smooth(z, L);
    cx w = cadd(cscal(z, 1 - L->kappa), cscal(cconj(z), L->gamma));
    w = csub(csub(csub(w, as), al), sm);
    wx[i] = w.re;
    wy[i] = w.im;
    if (mu) {
      cx das = d_alpha_star_node(t, z, k, L->theta);
      cx dal = d_alpha_local_node(t, z, k, L->theta);
      double dsz = d_alpha_smooth_dz(z, L);
      cx dszb = d_alpha_smooth_dzbar(z, L);
      double dwdz = (1 - L->kappa) - dsz;
      cx dwdzb = csub(csub(csub(C(L->gamma, 0), das), dal), dszb);
      double a = cabsv(dwdzb);
      mu[i] = 1 / (dwdz * dwdz - a * a);
    }
  }
}

/* Direct FP64 sum over all n stars: w = (1-k) z + g conj(z) - theta^2 conj(sum m/(z - z_i)) - alpha_smooth. */
void orc_shoot_direct(int n, const double* xym, const OrcLens* L, long long npts, const double* zx, const double* zy,
                      double* wx, double* wy, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const double th2 = L->theta * L->theta;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < npts; i++) {
    double x = zx[i], y = zy[i];
    double sr = 0, si = 0;
    for (int s = 0; s < n; s++) {
      double dx = x - xym[3 * s], dy = y - xym[3 * s + 1];
      double q = xym[3 * s + 2] / (dx * dx + dy * dy);
      sr += q * dx;
      si += q * dy;
    }
    cx z = C(x, y);
    cx sm = alpha_smooth(z, L);
    cx w = cadd(cscal(z, 1 - L->kappa), cscal(cconj(z), L->gamma));
    w = csub(w, C(sr * th2, si * th2));
    w = csub(w, sm);
    wx[i] = w.re;
    wy[i] = w.im;
  }
}

/* Same as orc_shoot_direct for a regular lattice x_i = bx + 2 (rx i), y_j = by + 2 (ry j),
 * i in [i0, i0+ni), j in [j0, j0+nj); output row-major [nj][ni]. */
void orc_shoot_direct_lattice(int n, const double* xym, const OrcLens* L, double bx, double by, double rx, double ry,
                              long long i0, long long ni, long long j0, long long nj, double* wx, double* wy,
                              int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const double th2 = L->theta * L->theta;
#pragma omp parallel for schedule(static)
  for (long long jj = 0; jj < nj; jj++) {
    double y = by + 2.0 * (ry * (double)(j0 + jj));
    for (long long ii = 0; ii < ni; ii++) {
      double x = bx + 2.0 * (rx * (double)(i0 + ii));
      double sr = 0, si = 0;
      for (int s = 0; s < n; s++) {
        double dx = x - xym[3 * s], dy = y - xym[3 * s + 1];
        double q = xym[3 * s + 2] / (dx * dx + dy * dy);
        sr += q * dx;
        si += q * dy;
      }
      cx z = C(x, y);
      cx sm = alpha_smooth(z, L);
      cx w = cadd(cscal(z, 1 - L->kappa), cscal(cconj(z), L->gamma));
      w = csub(w, C(sr * th2, si * th2));
      w = csub(w, sm);
      wx[jj * ni + ii] = w.re;
      wy[jj * ni + ii] = w.im;
    }
  }
}

/* IRS binning of source positions (irs_functions.cuh:147-198). mu may be NULL. */
void orc_irs_bin(long long npts, const double* wx, const double* wy, const double* mu, double cy1, double cy2,
                 double hly1, double hly2, int npx, int npy, int* pix, int* pmin, int* psad) {
  for (long long i = 0; i < npts; i++) {
    double a = wx[i], b = wy[i];
    if (isnan(a) || isnan(b)) continue;
    a -= cy1;
    b -= cy2;
    if (a < -hly1 || a > hly1 || b < -hly2 || b > hly2) continue;
    int ix = (int)((a + hly1) * npx / (2 * hly1));
    int iy = (int)((b + hly2) * npy / (2 * hly2));
    if (ix == npx) ix--;
    if (iy == npy) iy--;
    iy = npy - 1 - iy;
    long long idx = (long long)iy * npx + ix;
    if (mu && pmin && psad) {
      if (mu[i] >= 0) pmin[idx]++;
      else psad[idx]++;
    }
    pix[idx]++;
  }
}

/* ------------------------------------------------------------ IPM, reference algorithm */
typedef struct {
  double x[7], y[7];
  int n;
} RPoly;

static void rp_add(RPoly* p, double x, double y) {
  if (p->n >= 7) {
    p->n = 0;
    return;
  }
  p->x[p->n] = x;
  p->y[p->n] = y;
  p->n++;
}
/* polygon.cuh:116-144 */
static double rp_area(const RPoly* p) {
  if (p->n < 3) return 0;
  double r = 0;
  for (int i = 0; i < p->n; i++) {
    int j = (i + 1) % p->n;
    double dx = p->x[j] - p->x[i], dy = p->y[j] - p->y[i];
    r += dy * p->x[i] - dx * p->y[i];
  }
  return r / 2;
}
static double sgn(double v) { return v < 0 ? -1 : (v > 0 ? 1 : 0); }
/* polygon.cuh:150-197: intersections through log / exp */
static double rp_x_at(double y, double x1, double y1, double x2, double y2) {
  double dx = x2 - x1;
  if (dx == 0) return x1;
  double ldx = log(fabs(dx)), dy = y2 - y1, ldy = log(fabs(dy));
  double lt = log(fabs(y - y1)) - ldy;
  return x1 + sgn(y - y1) * sgn(dy) * sgn(dx) * exp(lt + ldx);
}
static double rp_y_at(double x, double x1, double y1, double x2, double y2) {
  double dy = y2 - y1;
  if (dy == 0) return y1;
  double ldy = log(fabs(dy)), dx = x2 - x1, ldx = log(fabs(dx));
  double lt = log(fabs(x - x1)) - ldx;
  return y1 + sgn(x - x1) * sgn(dx) * sgn(dy) * exp(lt + ldy);
}
static double rp_minx(const RPoly* p) {
  double m = p->x[0];
  for (int i = 1; i < p->n; i++) if (p->x[i] < m) m = p->x[i];
  return m;
}
static double rp_maxx(const RPoly* p) {
  double m = p->x[0];
  for (int i = 1; i < p->n; i++) if (p->x[i] > m) m = p->x[i];
  return m;
}
static double rp_miny(const RPoly* p) {
  double m = p->y[0];
  for (int i = 1; i < p->n; i++) if (p->y[i] < m) m = p->y[i];
  return m;
}
static double rp_maxy(const RPoly* p) {
  double m = p->y[0];
  for (int i = 1; i < p->n; i++) if (p->y[i] > m) m = p->y[i];
  return m;
}
/* polygon.cuh:254-347: *self keeps the side that is not returned */
static RPoly rp_clip_x(RPoly* self, double X, int clip_left) {
  RPoly L = {{0}, {0}, 0}, R = {{0}, {0}, 0};
  for (int i = 0; i < self->n; i++) {
    int j = (i + 1) % self->n;
    if (self->x[i] < X) {
      rp_add(&L, self->x[i], self->y[i]);
      if (self->x[j] > X) {
        double y = rp_y_at(X, self->x[i], self->y[i], self->x[j], self->y[j]);
        rp_add(&L, X, y);
        rp_add(&R, X, y);
      }
    } else if (self->x[i] > X) {
      rp_add(&R, self->x[i], self->y[i]);
      if (self->x[j] < X) {
        double y = rp_y_at(X, self->x[i], self->y[i], self->x[j], self->y[j]);
        rp_add(&L, X, y);
        rp_add(&R, X, y);
      }
    } else {
      rp_add(&L, self->x[i], self->y[i]);
      rp_add(&R, self->x[i], self->y[i]);
    }
  }
  if (clip_left) {
    *self = R;
    return L;
  }
  *self = L;
  return R;
}
static RPoly rp_clip_y(RPoly* self, double Y, int clip_bottom) {
  RPoly B = {{0}, {0}, 0}, T = {{0}, {0}, 0};
  for (int i = 0; i < self->n; i++) {
    int j = (i + 1) % self->n;
    if (self->y[i] < Y) {
      rp_add(&B, self->x[i], self->y[i]);
      if (self->y[j] > Y) {
        double x = rp_x_at(Y, self->x[i], self->y[i], self->x[j], self->y[j]);
        rp_add(&B, x, Y);
        rp_add(&T, x, Y);
      }
    } else if (self->y[i] > Y) {
      rp_add(&T, self->x[i], self->y[i]);
      if (self->y[j] < Y) {
        double x = rp_x_at(Y, self->x[i], self->y[i], self->x[j], self->y[j]);
        rp_add(&B, x, Y);
        rp_add(&T, x, Y);
      }
    } else {
      rp_add(&B, self->x[i], self->y[i]);
      rp_add(&T, self->x[i], self->y[i]);
    }
  }
  if (clip_bottom) {
    *self = T;
    return B;
  }
  *self = B;
  return T;
}
/* polygon.cuh:349-467 */
static void rp_allocate(RPoly* P, double factor, double* pix, int npx, int npy) {
  if (P->n < 3) return;
  if (rp_minx(P) >= npx || rp_maxx(P) <= 0 || rp_miny(P) >= npy || rp_maxy(P) <= 0) return;
  double whole = fabs(rp_area(P));
  if (whole == 0) return;
  if (rp_minx(P) < 0) rp_clip_x(P, 0, 1);
  if (rp_maxx(P) > npx) rp_clip_x(P, npx, 0);
  if (rp_miny(P) < 0) rp_clip_y(P, 0, 1);
  if (rp_maxy(P) > npy) rp_clip_y(P, npy, 0);
  if (P->n < 3) return;
  int xmin = (int)rp_minx(P), xmax = (int)rp_maxx(P);
  if (xmax == npx) xmax--;
  for (int x = xmin; x < xmax; x++) {
    RPoly top = rp_clip_x(P, x + 1, 1);
    if (top.n < 3) continue;
    int ymin = (int)rp_miny(&top), ymax = (int)rp_maxy(&top);
    if (ymax == npy) ymax--;
    for (int y = ymin; y < ymax; y++) {
      RPoly bot = rp_clip_y(&top, y + 1, 1);
      if (bot.n < 3) continue;
      pix[(long long)npx * y + x] += factor * fabs(rp_area(&bot)) / whole;
    }
    pix[(long long)npx * ymax + x] += factor * fabs(rp_area(&top)) / whole;
  }
  if (P->n < 3) return;
  int ymin = (int)rp_miny(P), ymax = (int)rp_maxy(P);
  if (ymax == npy) ymax--;
  for (int y = ymin; y < ymax; y++) {
    RPoly bot = rp_clip_y(P, y + 1, 1);
    if (bot.n < 3) continue;
    pix[(long long)npx * y + xmax] += factor * fabs(rp_area(&bot)) / whole;
  }
  pix[(long long)npx * ymax + xmax] += factor * fabs(rp_area(P)) / whole;
}

/* IPM deposition of an ncx x ncy cell lattice from its (ncx+1) x (ncy+1) vertex
 * positions (pixel units, row axis flipped), reference algorithm in FP64. */
void orc_ipm_deposit_ref(long long ncx, long long ncy, const double* vx, const double* vy, double factor, int npx,
                         int npy, double* pix, double* pmin, double* psad, int parities) {
  long long W = ncx + 1;
  for (long long j = 0; j < ncy; j++) {
    for (long long i = 0; i < ncx; i++) {
      double y0x = vx[(j + 1) * W + i + 1], y0y = vy[(j + 1) * W + i + 1];
      double y1x = vx[(j + 1) * W + i], y1y = vy[(j + 1) * W + i];
      double y2x = vx[j * W + i], y2y = vy[j * W + i];
      double y3x = vx[j * W + i + 1], y3y = vy[j * W + i + 1];
      for (int tri = 0; tri < 2; tri++) {
        RPoly P;
        P.n = 3;
        if (tri == 0) {
          P.x[0] = y0x; P.y[0] = y0y; P.x[1] = y1x; P.y[1] = y1y; P.x[2] = y2x; P.y[2] = y2y;
        } else {
          P.x[0] = y2x; P.y[0] = y2y; P.x[1] = y3x; P.y[1] = y3y; P.x[2] = y0x; P.y[2] = y0y;
        }
        double A = rp_area(&P);
        if (!(fabs(A) < 10000 * factor)) continue;
        if (parities)
          rp_allocate(&P, factor, A < 0 ? pmin : psad, npx, npy);
        else
          rp_allocate(&P, factor, pix, npx, npy);
      }
    }
  }
  if (parities) {
    long long n = (long long)npx * npy;
    for (long long k = 0; k < n; k++) pix[k] = pmin[k] + psad[k];
  }
}

/* ------------------------------------------------------------ IPM, fixed-point variant */
#define FIXSCALE 4294967296.0
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)
#define TRI(suf) CAT(Tri, suf)
#define STRIP(suf) CAT(Strip, suf)

#define D float
#define SUF f32
#define RINT llrintf
#define FMA fmaf
#define DMAX FLT_MAX
#include "fixdep.inc"
#undef D
#undef SUF
#undef RINT
#undef FMA
#undef DMAX

#define D double
#define SUF f64
#define RINT llrint
#define FMA fma
#define DMAX DBL_MAX
#include "fixdep.inc"
#undef D
#undef SUF
#undef RINT
#undef FMA
#undef DMAX

/* ------------------------------------------------------------ derived parameters (double) */
/* calculate_derived_params, include/ipm.cuh:434-506 for a generated circular or
 * rectangular field; out[] = mu_ave, num_rays_x, rhs1, rhs2, hlx1, hlx2,
 * nrt1, nrt2, center_x1, center_x2, num_stars, corner1, corner2, alpha_error */
void orc_derive(double kappa, double gamma, double kstar, double theta, double mean_mass, double mean_mass2,
                double light_loss, int rect, double safety, double cy1, double cy2, double hly1, double hly2, int npx,
                int npy, int nry, double* out) {
  double mu_ave = 1 / ((1 - kappa) * (1 - kappa) - gamma * gamma);
  double nrx = 1.0 * nry * npx * npy / (2 * hly1 * 2 * hly2);
  double r1 = sqrt(hly1 / hly2 * npy / npx), r2 = sqrt(hly2 / hly1 * npx / npy);
  double dv = 2 * sqrt(nrx);
  r1 /= dv;
  r2 /= dv;
  double t = theta * sqrt(kstar * mean_mass2 / (mean_mass * light_loss));
  double h1 = (hly1 + t) / fabs(1 - kappa + gamma), h2 = (hly2 + t) / fabs(1 - kappa - gamma);
  int n1 = (int)(h1 / (2 * r1)) + 1, n2 = (int)(h2 / (2 * r2)) + 1;
  h1 = 2 * r1 * n1;
  h2 = 2 * r2 * n2;
  double c1 = cy1 / (1 - kappa + gamma), c2 = cy2 / (1 - kappa - gamma);
  double k1 = fabs(c1) + h1, k2 = fabs(c2) + h2;
  int ns;
  if (rect) {
    ns = (int)ceil(safety * 2 * k1 * safety * 2 * k2 * kstar / (M_PI * theta * theta * mean_mass));
    double a = sqrt(k1 / k2), b = sqrt(k2 / k1), s = sqrt(M_PI * theta * theta * ns * mean_mass / (4 * kstar));
    k1 = a * s;
    k2 = b * s;
  } else {
    double ca = hypot(k1, k2);
    ns = (int)ceil(safety * ca * safety * ca * kstar / (theta * theta * mean_mass));
    double s = sqrt(theta * theta * ns * mean_mass / kstar);
    k1 = k1 / ca * s;
    k2 = k2 / ca * s;
  }
  double ae = fmin(hly1 / (10 * npx), hly2 / (10 * npy));
  double v[14] = {mu_ave, nrx, r1, r2, h1, h2, 2.0 * n1, 2.0 * n2, c1, c2, (double)ns, k1, k2, ae};
  memcpy(out, v, sizeof(v));
}

/* ---------------------------------------------------------------- NCC
 * Number of caustic crossings (include/ncc_functions.cuh:149-367 and
 * include/ncc.cuh:208-327), restated: the same clipping of every caustic
 * segment into the region y1 > -hl1, |y2| < hl2, the same pixel-centre row
 * crossings adding -1 (segment going up) or +1 (going down) to every pixel of
 * the row left of the crossing, on the 2^os times finer map, then the maximum
 * over 2^os x 2^os blocks. The intersection of a segment with a horizontal or
 * vertical line is x0 + ((y - y0) / dy) dx, each operation rounded (the
 * reference evaluates it through logarithms), as the GPU kernels
 * (irs_b200/csrc/ncc.cuh) compute it. out: npy x npx int32, row 0 at the top. */
static double ncc_sgn(double v) { return v < 0 ? -1.0 : (v > 0 ? 1.0 : 0.0); }
static double ncc_x_at(double y, double x0, double y0, double x1, double y1) {
  double dx = x1 - x0;
  if (dx == 0.0) return x0;
  double dy = y1 - y0, t = y - y0;
  t = t / dy;
  t = t * dx;
  return x0 + t;
}
static double ncc_y_at(double x, double x0, double y0, double x1, double y1) {
  double dy = y1 - y0;
  if (dy == 0.0) return y0;
  double dx = x1 - x0, t = x - x0;
  t = t / dx;
  t = t * dy;
  return y0 + t;
}
static void ncc_correct(double* x, double* y, double xo, double yo, double hl1, double hl2, int fx, int fy) {
  double x0 = *x, y0 = *y;
  if (*x <= -hl1) {
    double d = 0.01 * 2;
    d = d * hl1;
    d = d / (double)fx;
    *x = -hl1 + d;
    *y = ncc_y_at(*x, x0, y0, xo, yo);
  }
  if (fabs(*y) >= hl2) {
    double d = 0.01 * 2;
    d = d * hl2;
    d = d / (double)fy;
    d = hl2 - d;
    *y = ncc_sgn(*y) * d;
    *x = ncc_x_at(*y, x0, y0, xo, yo);
  }
}

int orc_ncc(const double* caus, int nrows, int ncols, double cy1, double cy2, double hl1, double hl2, int npx, int npy,
            int os, int* out) {
  int B = 1 << os, fx = npx * B, fy = npy * B, errors = 0;
  int* fine = (int*)calloc((size_t)fx * fy, sizeof(int));
  for (long long i = 0; i < nrows; i++)
    for (long long j = 0; j + 1 < ncols; j++) {
      const double* a = caus + 2 * (i * ncols + j);
      const double* b = a + 2;
      double x0 = a[0] - cy1, y0 = a[1] - cy2, x1 = b[0] - cy1, y1 = b[1] - cy2;
      int use = (x0 > -hl1 && fabs(y0) < hl2) || (x1 > -hl1 && fabs(y1) < hl2);
      if (!use)
        use = ncc_x_at(hl2, x0, y0, x1, y1) >= -hl1 || ncc_x_at(-hl2, x0, y0, x1, y1) >= -hl1 ||
              fabs(ncc_y_at(-hl1, x0, y0, x1, y1)) <= hl2;
      if (!use) continue;
      ncc_correct(&x0, &y0, x1, y1, hl1, hl2, fx, fy);
      ncc_correct(&x1, &y1, x0, y0, hl1, hl2, fx, fy);
      double s1 = 2 * hl1, s2 = 2 * hl2, t;
      t = x0 + hl1; t = t * (double)fx; double px0 = t / s1;
      t = y0 + hl2; t = t * (double)fy; double py0 = t / s2;
      t = x1 + hl1; t = t * (double)fx; double px1 = t / s1;
      t = y1 + hl2; t = t * (double)fy; double py1 = t / s2;
      if (py0 == py1) continue;
      int up = py0 < py1, k0 = (int)(py0 + 0.5), k1 = (int)(py1 + 0.5), v = up ? -1 : 1;
      for (int k = k0; up ? k < k1 : k > k1; k += up ? 1 : -1) {
        double yc = up ? (double)k + 0.5 : (double)k - 0.5;
        double xc = ncc_x_at(yc, px0, py0, px1, py1);
        int col = (int)(xc + 0.5) - 1, row = fy - 1 - (up ? k : k - 1);
        if (col > fx - 1) col = fx - 1;
        if (col < 0) continue;
        if (row < 0 || row >= fy) { /* the reference reports it and adds nothing */
          errors++;
          continue;
        }
        for (int l = 0; l <= col; l++) fine[(long long)row * fx + l] += v;
      }
    }
  for (int r = 0; r < npy; r++)
    for (int c = 0; c < npx; c++) {
      int m = fine[(long long)r * B * fx + (long long)c * B];
      for (int dy = 0; dy < B; dy++)
        for (int dx = 0; dx < B; dx++) {
          int q = fine[((long long)r * B + dy) * fx + (long long)c * B + dx];
          m = q > m ? q : m;
        }
      out[(long long)r * npx + c] = m;
    }
  free(fine);
  return errors;
}
