// IPM deposition: each lens-plane cell maps to two source-plane triangles whose
// image-plane area is spread over the pixels they overlap, in proportion to the
// overlap area.
//
// Semantics of the reference (ipm_functions.cuh:168-216 and
// Polygon::allocate_area_among_pixels, polygon.cuh:349-467): triangles
// (y0,y1,y2) and (y2,y3,y0) from the cell corners; skip |A| >= 1e4 * cell
// area; route by the sign of A to the minima (A < 0) or saddle map when
// parities are kept; every pixel of the map receives
// factor * |A ∩ pixel| / |A|.
//
// How, differently by design:
//   * the overlap of a triangle with a pixel is computed directly from
//     Green's theorem instead of by successive polygon clips: the edges are
//     clipped once per row strip (row_geometry), and each pixel of the row
//     then only clamps those segments to its column (pixel_coverage):
//     register-only arithmetic, no polygon arrays;
//   * rows of a triangle are independent work items; a warp expands the rows
//     of its 64 triangles and shares them out 32 at a time;
//   * pixels inside both the bottom and the top chord of a row strip are fully
//     covered (area exactly 1) and are added as a run through a per-row
//     difference array;
//   * coordinates are relative to an integer origin at the triangle's
//     lower-left pixel; the map accumulates unsigned 64-bit fixed point (2^32
//     per unit) with integer atomics, so the result does not depend on thread
//     order: given the same corner positions the map is bit-exact.
// Every floating-point operation is an explicitly rounded intrinsic (fused
// multiply-adds only where written, no contraction by the compiler), so a host
// implementation with the same operation sequence reproduces the map bit for
// bit.
#pragma once
#include "common.cuh"

#include <limits>

namespace irsb {

template <typename D>
struct RN;
template <>
struct RN<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float rcp(float a) { return __frcp_rn(a); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ unsigned long long to_fix(float a) {
    return (unsigned long long)__float2ll_rn(a);
  }
};
template <>
struct RN<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ unsigned long long to_fix(double a) {
    return (unsigned long long)__double2ll_rn(a);
  }
};

// Fire-and-forget add to a map word in global memory (PTX red): the adding
// thread never reads the word back, so no old value has to travel back to it
// (a plain atomicAdd on these generic pointers compiles to a returning atom).
__device__ __forceinline__ void red_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}

template <typename D>
__device__ __forceinline__ D dabs(D a) {
  return a < D(0) ? -a : a;
}

// Output of the deposition: per-pixel fixed-point pieces plus a per-row
// difference array for runs of fully covered pixels (row stride npx + 1).
struct DepositMaps {
  unsigned long long* acc;   // [npy][npx] boundary pieces
  unsigned long long* diff;  // [npy][npx + 1] span starts (+q) and ends (-q), modulo 2^64
};

// A triangle prepared for deposition: CCW vertices relative to the integer
// origin (ox, oy), per-edge reciprocals, fixed-point scale and target map.
template <typename D>
struct Tri {
  D x[3], y[3];     // CCW, relative to (ox, oy)
  D idy[3];         // 1 / (y[k+1] - y[k]) (0 for a zero difference)
  D sl[3];          // slope (y[k+1] - y[k]) * (1 / (x[k+1] - x[k])); 0 for a vertical edge or an overflow
  D scale;          // factor * 2^32 / |area|
  int ox, oy;
  int rlo, nrows;   // first row (relative) and number of rows to visit
  int map;          // 0 total, 1 minima, 2 saddles
  int single;       // 1: the triangle lies inside one map pixel, (ox, oy)
};

template <typename D>
__device__ __forceinline__ D rcp_or_zero(D v) {
  return v != D(0) ? RN<D>::rcp(v) : D(0);  // correctly rounded 1 / v
}

// Triangle (a, b, c) in absolute pixel coordinates (row axis flipped) ->
// Tri without its reciprocals and scale (setup_tail), or nrows = 0 when it
// deposits nothing; scale holds the triangle's area. Tests of the reference
// (ipm_functions.cuh:170-193, polygon.cuh:351-372): NaN corner, |A| >= 1e4
// * factor, entirely outside the map, zero area.
template <typename D>
__device__ __forceinline__ Tri<D> setup_head(double ax, double ay, double bx, double by, double cx, double cy,
                                             D factor, int npx, int npy, bool parities) {
  Tri<D> t;
  t.nrows = 0;
  t.rlo = 0;
  t.ox = t.oy = 0;
  t.map = 0;
  t.single = 0;
  t.scale = D(0);
  for (int k = 0; k < 3; k++) t.x[k] = t.y[k] = t.sl[k] = t.idy[k] = D(0);
  if (isnan(ax) || isnan(ay) || isnan(bx) || isnan(by) || isnan(cx) || isnan(cy)) return t;
  double fx = floor(fmin(ax, fmin(bx, cx)));
  double fy = floor(fmin(ay, fmin(by, cy)));
  if (!(fx > -1.0e9 && fx < 1.0e9 && fy > -1.0e9 && fy < 1.0e9)) return t;
  D x0 = D(ax - fx), y0 = D(ay - fy), x1 = D(bx - fx), y1 = D(by - fy), x2 = D(cx - fx), y2 = D(cy - fy);
  // shoelace, as Poly::area
  D s = D(0);
  s = RN<D>::add(s, RN<D>::fma(RN<D>::sub(y1, y0), x0, -RN<D>::mul(RN<D>::sub(x1, x0), y0)));
  s = RN<D>::add(s, RN<D>::fma(RN<D>::sub(y2, y1), x1, -RN<D>::mul(RN<D>::sub(x2, x1), y1)));
  s = RN<D>::add(s, RN<D>::fma(RN<D>::sub(y0, y2), x2, -RN<D>::mul(RN<D>::sub(x0, x2), y2)));
  D A = RN<D>::mul(s, D(0.5));  // the correctly rounded s / 2, as a division gives
  if (!(dabs(A) < RN<D>::mul(D(10000), factor))) return t;
  D whole = dabs(A);
  if (whole == D(0)) return t;
  const int ox = int(fx), oy = int(fy);
  const D X0 = D(-ox), X1 = D(npx - ox), Y0 = D(-oy), Y1 = D(npy - oy);
  D mnx = x0 < x1 ? x0 : x1, mxx = x0 > x1 ? x0 : x1, mny = y0 < y1 ? y0 : y1, mxy = y0 > y1 ? y0 : y1;
  mnx = x2 < mnx ? x2 : mnx;
  mxx = x2 > mxx ? x2 : mxx;
  mny = y2 < mny ? y2 : mny;
  mxy = y2 > mxy ? y2 : mxy;
  if (mnx >= X1 || mxx <= X0 || mny >= Y1 || mxy <= Y0) return t;
  t.map = parities ? (A < D(0) ? 1 : 2) : 0;
  if (A < D(0)) {  // make counter-clockwise
    D tx = x1, ty = y1;
    x1 = x2;
    y1 = y2;
    x2 = tx;
    y2 = ty;
  }
  t.x[0] = x0;
  t.y[0] = y0;
  t.x[1] = x1;
  t.y[1] = y1;
  t.x[2] = x2;
  t.y[2] = y2;
  t.scale = whole;  // setup_tail turns it into the fixed-point scale
  t.ox = ox;
  t.oy = oy;
  int rlo = 0 > -oy ? 0 : -oy;
  int rhi = mxy < D(npy - oy) ? int(floor(mxy)) : npy - 1 - oy;
  t.rlo = rlo;
  t.nrows = rhi >= rlo ? rhi - rlo + 1 : 0;
  // inside one pixel of the map: all its area goes there
  t.single = (t.nrows == 1 && mxx < D(1) && mxy < D(1) && ox >= 0 && ox < npx) ? 1 : 0;
  return t;
}

// Edge reciprocals, slopes and the fixed-point scale of a triangle that
// deposits row by row (nrows > 0, not single).
template <typename D>
__device__ __forceinline__ void setup_tail(Tri<D>& t, D factor) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int j = k == 2 ? 0 : k + 1;
    const D dx = RN<D>::sub(t.x[j], t.x[k]), dy = RN<D>::sub(t.y[j], t.y[k]);
    t.idy[k] = rcp_or_zero(dy);
    const D g = RN<D>::mul(dy, rcp_or_zero(dx));
    t.sl[k] = dabs(g) <= std::numeric_limits<D>::max() ? g : D(0);
  }
  t.scale = RN<D>::div(RN<D>::mul(factor, D(kFixScale)), t.scale);
}

// Shared-memory staging of the 64 triangles of a warp's 32 cells that go row
// by row (one array per field: lane k touches word k, no bank conflicts).
template <typename D>
struct TriSlots {
  D x[3][64], y[3][64], area[64];
  int ox[64], oy[64], rlo[64], nrows[64], map[64];
  __device__ __forceinline__ void put(int k, const Tri<D>& t) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      x[q][k] = t.x[q];
      y[q][k] = t.y[q];
    }
    area[k] = t.scale;
    ox[k] = t.ox;
    oy[k] = t.oy;
    rlo[k] = t.rlo;
    nrows[k] = t.nrows;
    map[k] = t.map;
  }
  __device__ __forceinline__ void get(int k, Tri<D>& t) const {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      t.x[q] = x[q][k];
      t.y[q] = y[q][k];
    }
    t.scale = area[k];
    t.ox = ox[k];
    t.oy = oy[k];
    t.rlo = rlo[k];
    t.nrows = nrows[k];
    t.map = map[k];
    t.single = 0;
  }
};
constexpr int kDepositWarps = 2;  // warps per CTA of the deposition kernels
constexpr int kDepositThreads = kDepositWarps * 32;
// Grid of the deposition kernels over nchunks 32-cell chunks: one warp per
// chunk, at most 256 CTAs per SM (148 SMs), the warps striding over the rest.
// Small CTAs retire as soon as their two warps are done, so the SMs stay full
// to the end: 6.25 ms against 6.72 ms with 8-warp CTAs at 16 per SM on the
// 2000-pixel bench workload, maps bit-identical.
inline int deposit_grid(long long nchunks) {
  const long long ctas = (nchunks + kDepositWarps - 1) / kDepositWarps, cap = 148LL * 256;
  return int(ctas < 1 ? 1 : (ctas > cap ? cap : ctas));
}

// Geometry of one row strip [rb, rt = rb + 1] of a triangle.
//   Strip segments: each edge clipped to the strip, endpoints (xa, ya) ->
//   (xb, yb) with y relative to rb, a zero segment where the edge misses the
//   strip. A horizontal edge belongs to the strip only on [rb, rt), so an edge
//   lying on the line between two rows is counted once (by the top chord of
//   the row below).
//   Chords: x-extent of the triangle on the lines y = rb and y = rt (an edge
//   reaching the line contributes its crossing, x1 + ((y - y1) / dy) dx, or
//   both ends when it lies on the line).
template <typename D>
struct Strip {
  D xa[3], ya[3], xb[3], yb[3];
};

template <typename D>
__device__ __forceinline__ void extend(bool& any, D& lo, D& hi, D a, D b) {
  const D mn = a < b ? a : b, mx = a > b ? a : b;
  lo = any ? (mn < lo ? mn : lo) : mn;
  hi = any ? (mx > hi ? mx : hi) : mx;
  any = true;
}

// Fills the strip segments and both chords; returns false when the triangle
// does not enter the strip, else sets its x-extent [xlo, xhi] there.
template <typename D>
__device__ __forceinline__ bool row_geometry(const Tri<D>& t, D rb, D rt, Strip<D>& g, D& xlo, D& xhi, bool& hb,
                                             D& cb0, D& cb1, bool& ht, D& ct0, D& ct1) {
  bool any = false;
  xlo = xhi = cb0 = cb1 = ct0 = ct1 = D(0);
  hb = ht = false;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int j = k == 2 ? 0 : k + 1;
    const D x1 = t.x[k], y1 = t.y[k], x2 = t.x[j], y2 = t.y[j];
    const D dx = RN<D>::sub(x2, x1), dy = RN<D>::sub(y2, y1);
    const bool on_b = (y1 <= rb && rb <= y2) || (y2 <= rb && rb <= y1);
    const bool on_t = (y1 <= rt && rt <= y2) || (y2 <= rt && rt <= y1);
    D t0 = D(0), t1 = D(1);
    bool ok;
    if (dy != D(0)) {
      const D ta = RN<D>::mul(RN<D>::sub(rb, y1), t.idy[k]), tb = RN<D>::mul(RN<D>::sub(rt, y1), t.idy[k]);
      if (on_b) {
        const D p = RN<D>::fma(ta, dx, x1);
        extend(hb, cb0, cb1, p, p);
      }
      if (on_t) {
        const D p = RN<D>::fma(tb, dx, x1);
        extend(ht, ct0, ct1, p, p);
      }
      const D lo = ta < tb ? ta : tb, hi = ta > tb ? ta : tb;
      t0 = lo > t0 ? lo : t0;
      t1 = hi < t1 ? hi : t1;
      ok = t0 < t1;
    } else {
      if (on_b) extend(hb, cb0, cb1, x1, x2);
      if (on_t) extend(ht, ct0, ct1, x1, x2);
      ok = y1 >= rb && y1 < rt;
    }
    D xa = D(0), ya = D(0), xb = D(0), yb = D(0);
    if (ok) {
      xa = RN<D>::fma(t0, dx, x1);
      xb = RN<D>::fma(t1, dx, x1);
      ya = RN<D>::sub(RN<D>::fma(t0, dy, y1), rb);
      yb = RN<D>::sub(RN<D>::fma(t1, dy, y1), rb);
      extend(any, xlo, xhi, xa, xb);
    }
    g.xa[k] = xa;
    g.ya[k] = ya;
    g.xb[k] = xb;
    g.yb[k] = yb;
  }
  return any;
}

// Area of the triangle inside the pixel [c, c+1] x [rb, rb+1] from Green's
// theorem, area = -(sum over the boundary of the integral of (y - rb) dx):
// each strip segment restricted to the column (both ends clamped to
// [c, c+1], an edge being monotone in x) is a trapezoid; the pixel's top side
// adds the top chord's length inside the column; the vertical sides and the
// bottom side add nothing.
template <typename D>
__device__ __forceinline__ D pixel_coverage(const Tri<D>& t, const Strip<D>& g, D c, bool has_top, D ct0, D ct1) {
  const D c1 = RN<D>::add(c, D(1));
  D s = D(0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    D xs = g.xa[k], xe = g.xb[k];
    xs = xs > c ? xs : c;
    xs = xs < c1 ? xs : c1;
    xe = xe > c ? xe : c;
    xe = xe < c1 ? xe : c1;
    const D w = RN<D>::sub(xe, xs);
    if (w != D(0)) {
      const D ys = RN<D>::fma(RN<D>::sub(xs, g.xa[k]), t.sl[k], g.ya[k]);
      const D ye = RN<D>::fma(RN<D>::sub(xe, g.xa[k]), t.sl[k], g.ya[k]);
      s = RN<D>::fma(RN<D>::mul(w, D(-0.5)), RN<D>::add(ys, ye), s);
    }
  }
  if (has_top) {
    D lo = ct0 > c ? ct0 : c, hi = ct1 < c1 ? ct1 : c1;
    if (hi > lo) s = RN<D>::add(s, RN<D>::sub(hi, lo));
  }
  return s;
}

// One row of a triangle: the run of fully covered pixels goes to the
// difference array, the other overlapped pixels get their coverage.
template <typename D>
__device__ __forceinline__ void deposit_row(const Tri<D>& t, int r, int npx, DepositMaps M) {
  const D rb = D(r), rt = D(r + 1);
  Strip<D> g;
  D xlo, xhi, cb0, cb1, ct0, ct1;
  bool hb, ht;
  if (!row_geometry(t, rb, rt, g, xlo, xhi, hb, cb0, cb1, ht, ct0, ct1)) return;
  const int cmap_lo = -t.ox, cmap_hi = npx - 1 - t.ox;  // columns inside the map (relative)
  int cmin = int(floor(xlo)), cmax = int(floor(xhi));
  if (cmin < cmap_lo) cmin = cmap_lo;
  if (cmax > cmap_hi) cmax = cmap_hi;
  if (cmin > cmax) return;
  int xa = 1, xb = 0;  // full run [xa, xb)
  if (hb && ht) {
    D l = cb0 > ct0 ? cb0 : ct0, h = cb1 < ct1 ? cb1 : ct1;
    xa = int(ceil(l));
    xb = int(floor(h));
    if (xa < cmap_lo) xa = cmap_lo;
    if (xb > cmap_hi + 1) xb = cmap_hi + 1;
  }
  const long long row = (long long)t.oy + r;
  const long long rbase = row * npx + t.ox;
  if (xa < xb) {
    const unsigned long long q = RN<D>::to_fix(t.scale);
    const long long dbase = row * ((long long)npx + 1) + t.ox;
    red_add(M.diff + dbase + xa, q);
    red_add(M.diff + dbase + xb, (unsigned long long)(0ULL - q));
  }
  for (int c = cmin; c <= cmax; c++) {
    if (xa < xb && c == xa) {
      c = xb - 1;
      continue;
    }
    D a = pixel_coverage(t, g, D(c), ht, ct0, ct1);
    if (a > D(0)) {
      unsigned long long q = RN<D>::to_fix(RN<D>::mul(a, t.scale));
      if (q) red_add(M.acc + rbase + c, q);
    }
  }
}

// The rows of the triangles of a warp, one triangle per lane (nrows = 0: none):
// each lane deposits its own triangle's first row; the warp then scans the
// counts of the remaining rows and works through those (triangle, row) items
// 32 at a time, each lane finding its item's owner lane by a binary search
// over the scan and reading the triangle through shuffles, so a triangle with
// many rows is spread over the warp instead of holding one lane.
template <typename D>
__device__ __forceinline__ void deposit_rows_warp(const Tri<D>& mine, int npx, const DepositMaps& m_total,
                                                  const DepositMaps& m_min, const DepositMaps& m_sad) {
  const int lane = threadIdx.x & 31;
  if (mine.nrows > 0) {
    const DepositMaps& M = mine.map == 0 ? m_total : (mine.map == 1 ? m_min : m_sad);
    deposit_row<D>(mine, mine.rlo, npx, M);
  }
  const int extra = mine.nrows > 1 ? mine.nrows - 1 : 0;
  int incl = extra;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  for (int it0 = 0; it0 < total; it0 += 32) {
    const int item = it0 + lane;
    int lo = 0, hi = 31;  // owner: first lane whose inclusive count exceeds item
#pragma unroll
    for (int step = 0; step < 5; step++) {
      int mid = (lo + hi) >> 1;
      int v = __shfl_sync(0xffffffffu, incl, mid);
      if (v > item) hi = mid;
      else lo = mid + 1;
    }
    const int owner = lo;
    const int before = __shfl_sync(0xffffffffu, incl - extra, owner);
    Tri<D> t;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      t.x[q] = __shfl_sync(0xffffffffu, mine.x[q], owner);
      t.y[q] = __shfl_sync(0xffffffffu, mine.y[q], owner);
      t.sl[q] = __shfl_sync(0xffffffffu, mine.sl[q], owner);
      t.idy[q] = __shfl_sync(0xffffffffu, mine.idy[q], owner);
    }
    t.scale = __shfl_sync(0xffffffffu, mine.scale, owner);
    t.ox = __shfl_sync(0xffffffffu, mine.ox, owner);
    t.oy = __shfl_sync(0xffffffffu, mine.oy, owner);
    t.rlo = __shfl_sync(0xffffffffu, mine.rlo, owner);
    t.map = __shfl_sync(0xffffffffu, mine.map, owner);
    if (item < total) {
      const DepositMaps& M = t.map == 0 ? m_total : (t.map == 1 ? m_min : m_sad);
      deposit_row<D>(t, t.rlo + 1 + (item - before), npx, M);
    }
  }
}

// The 32 cells [base, base + 32) of an ncx-wide lattice whose corner rows are
// vx apart (whole warp; lanes past ncells idle).
template <typename D>
__device__ __forceinline__ void deposit_warp_cells(const double2* __restrict__ verts, long long ncx, long long vx,
                                                   long long ncells, long long base, D factor, int npx, int npy,
                                                   const DepositMaps& m_total, const DepositMaps& m_min,
                                                   const DepositMaps& m_sad, int parities, TriSlots<D>& stage,
                                                   long long vstep = 1, double ox = 0.0, double oy = 0.0,
                                                   double inv_scale = 1.0) {
  const int lane = threadIdx.x & 31;
  const long long c = base + lane;
  double2 y0 = make_double2(0, 0), y1 = y0, y2 = y0, y3 = y0;
  if (c < ncells) {
    long long j, i;
    if (((c | ncx) >> 31) == 0) {  // 32-bit division where it suffices
      const unsigned jj = unsigned(c) / unsigned(ncx);
      j = jj;
      i = unsigned(c) - jj * unsigned(ncx);
    } else {
      j = c / ncx;
      i = c - j * ncx;
    }
    y0 = verts[((j + 1) * vx + (i + 1)) * vstep];  // z + rhs
    y1 = verts[((j + 1) * vx + i) * vstep];        // z - conj(rhs)
    y2 = verts[(j * vx + i) * vstep];              // z - rhs
    y3 = verts[(j * vx + (i + 1)) * vstep];        // z + conj(rhs)
    if (ox != 0.0 || oy != 0.0) {  // origin of the piece's map in the positions' pixel frame
      y0.x -= ox, y1.x -= ox, y2.x -= ox, y3.x -= ox;
      y0.y -= oy, y1.y -= oy, y2.y -= oy, y3.y -= oy;
    }
    if (inv_scale != 1.0) {  // the piece's map has pixels 1 / inv_scale wide
      y0.x *= inv_scale, y1.x *= inv_scale, y2.x *= inv_scale, y3.x *= inv_scale;
      y0.y *= inv_scale, y1.y *= inv_scale, y2.y *= inv_scale, y3.y *= inv_scale;
    }
  }
  // each half's head: a triangle inside one pixel deposits at once, the
  // others are staged in the warp's slots, compacted in lane order
  // a cell whose four corners all lie beyond one edge of the map deposits
  // nothing (setup_head would reject both its triangles)
  const bool live =
      c < ncells &&
      !((y0.x >= npx && y1.x >= npx && y2.x >= npx && y3.x >= npx) || (y0.x <= 0 && y1.x <= 0 && y2.x <= 0 && y3.x <= 0) ||
        (y0.y >= npy && y1.y >= npy && y2.y >= npy && y3.y >= npy) || (y0.y <= 0 && y1.y <= 0 && y2.y <= 0 && y3.y <= 0));
  if (__ballot_sync(0xffffffffu, live) == 0u) return;
  const unsigned lt = (1u << lane) - 1u;
  int n = 0;
#pragma unroll 1
  for (int half = 0; half < 2; half++) {
    Tri<D> h;
    h.nrows = 0;  // idle lanes (past the last cell) deposit nothing
    h.single = 0;
    if (live) {
      h = half == 0 ? setup_head<D>(y0.x, y0.y, y1.x, y1.y, y2.x, y2.y, factor, npx, npy, parities != 0)
                    : setup_head<D>(y2.x, y2.y, y3.x, y3.y, y0.x, y0.y, factor, npx, npy, parities != 0);
    }
    {
      // lanes in a row whose triangles fall in the same pixel add once for
      // all of them (adjacent cells of a fine lattice share pixels)
      unsigned long long* a = nullptr;
      if (h.single) a = (h.map == 0 ? m_total : (h.map == 1 ? m_min : m_sad)).acc + (long long)h.oy * npx + h.ox;
      const unsigned long long key = (unsigned long long)a;
      const unsigned long long prev = __shfl_up_sync(0xffffffffu, key, 1);
      const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
      if (h.single && (starts >> lane & 1u)) {
        const unsigned later = starts & ~((2u << lane) - 1u);  // lane 31: mask of all bits, none later
        const int end = later ? __ffs(later) - 1 : 32;
        red_add(a, (unsigned long long)(end - lane) * RN<D>::to_fix(RN<D>::mul(factor, D(kFixScale))));
      }
    }
    const bool cx = h.nrows > 0 && !h.single;
    const unsigned b = __ballot_sync(0xffffffffu, cx);
    if (cx) stage.put(n + __popc(b & lt), h);
    n += __popc(b);
  }
  __syncwarp();
  // the staged ones go row by row, one per lane: one round when at most 32
  // of the warp's 64 triangles need it (fine lattices), else two
  for (int r0 = 0; r0 < n; r0 += 32) {
    Tri<D> mine;
    mine.nrows = 0;
    if (r0 + lane < n) {
      stage.get(r0 + lane, mine);
      setup_tail(mine, factor);
    }
    deposit_rows_warp<D>(mine, npx, m_total, m_min, m_sad);
  }
  __syncwarp();  // slots free for the warp's next cells
}

// Cells of an ncx x ncy lattice whose (ncx+1) x (ncy+1) corner positions are in
// `verts`. A warp takes 32 consecutive cells; each lane classifies the two
// triangles of its cell (setup_head); a triangle inside one pixel is
// deposited at once; the others are staged in shared memory, compacted, and
// then get their reciprocals and scale (setup_tail) and go row by row
// (deposit_rows_warp), one per lane: one round when at most 32 of the warp's
// 64 triangles need it (fine lattices), else two.
template <typename D>
__global__ void __launch_bounds__(kDepositThreads, sizeof(D) == 4 ? 16 : 8)
    ipm_deposit_cells(const double2* __restrict__ verts, long long ncx, long long ncy, D factor, int npx, int npy,
                      DepositMaps m_total, DepositMaps m_min, DepositMaps m_sad, int parities) {
  const long long ncells = ncx * ncy;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  __shared__ TriSlots<D> slots[kDepositWarps];
  TriSlots<D>& stage = slots[threadIdx.x >> 5];
  for (long long base = warp0 * 32; base < ncells; base += nwarps * 32)
    deposit_warp_cells<D>(verts, ncx, ncx + 1, ncells, base, factor, npx, npy, m_total, m_min, m_sad, parities, stage);
}

// A block of cells inside a pass of the batched (or adaptive) deposition: its
// corner rows start at `voff` in the pass's corner buffer, vstride apart.
template <typename D>
struct DepositPiece {
  long long voff;
  long long vstride;   // corner row stride (ncx + 1 for a whole lattice row)
  long long vstep;     // corner (i, j) is at (j * vstride + i) * vstep (a coarser view of a finer grid)
  double ox, oy;       // origin of the piece's map in the positions' pixel frame
  double inv_scale;    // 1 / width of the piece's map pixels in the positions' pixels
  long long ncx, ncy;  // cells
  long long chunk0;    // first 32-cell chunk of the piece in the pass
  D factor;
  int r;               // realization (map index)
};

// Batched deposition: the warps stride over blocks of 8 consecutive 32-cell
// chunks of all pieces of the pass; a block's first piece is found by a
// binary search over chunk0 and the next chunks advance from it (one search
// per 8 chunks: 1.79 against 1.88 s for the 4096-pixel adaptive map).
// Realization r accumulates into the maps at r * map_stride / r * diff_stride.
template <typename D>
__global__ void __launch_bounds__(kDepositThreads, sizeof(D) == 4 ? 16 : 8)
    ipm_deposit_batch(const double2* __restrict__ verts, const DepositPiece<D>* __restrict__ pieces, int npieces,
                      long long nchunks, int npx, int npy, DepositMaps maps, long long map_stride,
                      long long diff_stride) {
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  __shared__ TriSlots<D> slots[kDepositWarps];
  TriSlots<D>& stage = slots[threadIdx.x >> 5];
  constexpr int K = 8;  // consecutive chunks per visit: one piece search per K chunks
  for (long long g0 = warp0 * K; g0 < nchunks; g0 += nwarps * K) {
    int lo = 0, hi = npieces - 1;  // last piece with chunk0 <= g0
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (pieces[mid].chunk0 <= g0) lo = mid;
      else hi = mid - 1;
    }
    const long long gend = g0 + K < nchunks ? g0 + K : nchunks;
    for (long long g = g0; g < gend; g++) {
      while (lo + 1 < npieces && pieces[lo + 1].chunk0 <= g) lo++;
      const DepositPiece<D> pc = pieces[lo];
      const DepositMaps M{maps.acc + pc.r * map_stride, maps.diff + pc.r * diff_stride};
      deposit_warp_cells<D>(verts + pc.voff, pc.ncx, pc.vstride, pc.ncx * pc.ncy, (g - pc.chunk0) * 32, pc.factor,
                            npx, npy, M, M, M, 0, stage, pc.vstep, pc.ox, pc.oy, pc.inv_scale);
    }
  }
}

// Row prefix sum of the difference array added to the pieces: one warp per
// row, 32 columns per step with a carried running sum (integer, exact).
__global__ void ipm_resolve_rows(int npx, int npy, DepositMaps m) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; y < npy; y += warps) {
    unsigned long long carry = 0;
    const long long rs = (long long)npx + 1;
    for (int x0 = 0; x0 < npx; x0 += 32) {
      int x = x0 + lane;
      unsigned long long v = x < npx ? m.diff[y * rs + x] : 0ULL;
      for (int o = 1; o < 32; o <<= 1) {
        unsigned long long u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      v += carry;
      if (x < npx) m.acc[(long long)y * npx + x] += v;
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// The row resolve and the conversion to T in one pass, for a run without
// parity maps: one warp per row, each lane 4 consecutive pixels (a
// 2000-pixel row in 16 dependent steps). The fixed-point map is still written
// (the resolved accumulators); integer sums, so both maps are those of
// ipm_resolve_rows followed by ipm_finalize.
template <typename T>
__global__ void ipm_resolve_rows_out(int npx, int npy, DepositMaps m, T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const long long rs = (long long)npx + 1;
  for (int y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; y < npy; y += warps) {
    unsigned long long carry = 0;
    for (int x0 = 0; x0 < npx; x0 += 128) {
      const int x = x0 + 4 * lane;
      unsigned long long d[4];
#pragma unroll
      for (int i = 0; i < 4; i++) d[i] = x + i < npx ? m.diff[y * rs + x + i] : 0ULL;
      d[1] += d[0];
      d[2] += d[1];
      d[3] += d[2];
      unsigned long long incl = d[3];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
      }
      const unsigned long long base = carry + (incl - d[3]);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        if (x + i < npx) {
          const long long k = (long long)y * npx + x + i;
          const unsigned long long v = m.acc[k] + (base + d[i]);
          m.acc[k] = v;
          out[k] = T(double(v) * kFixInv);
        }
      }
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
}

// map (fixed point) -> magnification in T; with parities total = min + sad.
template <typename T>
__global__ void ipm_finalize(long long n, const unsigned long long* __restrict__ acc_total,
                             const unsigned long long* __restrict__ acc_min,
                             const unsigned long long* __restrict__ acc_sad, T* __restrict__ out_total,
                             T* __restrict__ out_min, T* __restrict__ out_sad, int parities) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    if (parities) {
      unsigned long long a = acc_min[k], b = acc_sad[k];
      out_min[k] = T(double(a) * kFixInv);
      out_sad[k] = T(double(b) * kFixInv);
      out_total[k] = T(double(a + b) * kFixInv);
    } else {
      out_total[k] = T(double(acc_total[k]) * kFixInv);
    }
  }
}

}  // namespace irsb
