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
//   * no polygon clipping: each triangle's area is spread over the pixels by
//     accumulating its edges into a per-row difference array (a coverage
//     accumulation rasterizer). An edge piece lying inside pixel column c of
//     row strip r, running from height ya to yb, contributes the cover
//     K = F(ya) - F(yb) to every pixel right of c and the share
//     K (1 - f) to pixel c itself, f being the piece's mean x inside the
//     column; in the difference array that is K - a1 at c and a1 = round(K f)
//     at c + 1, so that the row's prefix sum gives each pixel's covered area.
//     F(y) = round(y * scale) is evaluated once per break point (a vertex, a
//     crossing of a row line or of a column line) and shared by the two pieces
//     meeting there, so the covers of every row of a triangle sum to exactly
//     zero: nothing leaks right of a triangle, whatever the rounding;
//   * rows of a triangle are independent work items; a warp expands the rows
//     of its 64 triangles and shares them out 32 at a time;
//   * pieces left of the map are merged into one cover at the map's first
//     column; pieces right of it are dropped;
//   * coordinates are relative to an integer origin at the triangle's
//     lower-left pixel; the map accumulates 64-bit fixed point (2^32 per unit,
//     modulo 2^64, read as signed) with integer atomics, so the result does not
//     depend on thread order: given the same corner positions the map is
//     bit-exact.
// Every floating-point operation is an explicitly rounded intrinsic (no FMA
// contraction), so a host implementation with the same operation sequence
// reproduces the map bit for bit.
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
  static __device__ __forceinline__ unsigned long long to_fix(double a) {
    return (unsigned long long)__double2ll_rn(a);
  }
};

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
// origin (ox, oy), per-edge slopes, the vertices' heights times the
// fixed-point scale, and the target map.
template <typename D>
struct Tri {
  D x[3], y[3];     // CCW, relative to (ox, oy)
  D pv[3];          // y[k] * scale (unrounded): F(y[k]) = round(pv[k])
  D gxy[3];         // dx * (1 / dy) of edge k -> k+1 (0 for a horizontal edge)
  D gyx[3];         // dy * (1 / dx) of edge k -> k+1 (0 for a vertical edge or an overflow)
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
  for (int k = 0; k < 3; k++) t.x[k] = t.y[k] = t.pv[k] = t.gxy[k] = t.gyx[k] = D(0);
  if (isnan(ax) || isnan(ay) || isnan(bx) || isnan(by) || isnan(cx) || isnan(cy)) return t;
  double fx = floor(fmin(ax, fmin(bx, cx)));
  double fy = floor(fmin(ay, fmin(by, cy)));
  if (!(fx > -1.0e9 && fx < 1.0e9 && fy > -1.0e9 && fy < 1.0e9)) return t;
  D x0 = D(ax - fx), y0 = D(ay - fy), x1 = D(bx - fx), y1 = D(by - fy), x2 = D(cx - fx), y2 = D(cy - fy);
  // shoelace, as Poly::area
  D s = D(0);
  s = RN<D>::add(s, RN<D>::sub(RN<D>::mul(RN<D>::sub(y1, y0), x0), RN<D>::mul(RN<D>::sub(x1, x0), y0)));
  s = RN<D>::add(s, RN<D>::sub(RN<D>::mul(RN<D>::sub(y2, y1), x1), RN<D>::mul(RN<D>::sub(x2, x1), y1)));
  s = RN<D>::add(s, RN<D>::sub(RN<D>::mul(RN<D>::sub(y0, y2), x2), RN<D>::mul(RN<D>::sub(x0, x2), y2)));
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
  // a sliver too thin for the fixed point (its heights times the scale
  // factor * 2^32 / area would pass 2^61): its whole flux at the pixel of its
  // centroid, if that is on the map
  const D ylim = mxy > D(1) ? mxy : D(1);
  if (whole < RN<D>::mul(RN<D>::mul(factor, ylim), D(1.0 / 536870912.0))) {
    const D third = D(1.0 / 3.0);
    D gx = RN<D>::mul(RN<D>::add(RN<D>::add(x0, x1), x2), third);
    D gy = RN<D>::mul(RN<D>::add(RN<D>::add(y0, y1), y2), third);
    gx = gx < X1 ? gx : X1;  // only whether it is on the map matters beyond the map's edge
    gy = gy < Y1 ? gy : Y1;
    const int px = ox + int(floor(gx)), py = oy + int(floor(gy));
    if (px >= 0 && px < npx && py >= 0 && py < npy) {
      t.ox = px;
      t.oy = py;
      t.nrows = 1;
      t.single = 1;
    }
    return t;
  }
  int rlo = 0 > -oy ? 0 : -oy;
  int rhi = mxy < D(npy - oy) ? int(floor(mxy)) : npy - 1 - oy;
  t.rlo = rlo;
  t.nrows = rhi >= rlo ? rhi - rlo + 1 : 0;
  // inside one pixel of the map: all its area goes there
  t.single = (t.nrows == 1 && mxx < D(1) && mxy < D(1) && ox >= 0 && ox < npx) ? 1 : 0;
  return t;
}

// Slopes, scaled vertex heights and the fixed-point scale of a triangle that
// deposits row by row (nrows > 0, not single).
template <typename D>
__device__ __forceinline__ void setup_tail(Tri<D>& t, D factor) {
  t.scale = RN<D>::div(RN<D>::mul(factor, D(kFixScale)), t.scale);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int j = k == 2 ? 0 : k + 1;
    const D dx = RN<D>::sub(t.x[j], t.x[k]), dy = RN<D>::sub(t.y[j], t.y[k]);
    t.gxy[k] = RN<D>::mul(dx, rcp_or_zero(dy));
    const D g = RN<D>::mul(dy, rcp_or_zero(dx));
    t.gyx[k] = dabs(g) <= std::numeric_limits<D>::max() ? g : D(0);
    t.pv[k] = RN<D>::mul(t.y[k], t.scale);
  }
}

// Shared-memory staging of the (at most 32) prepared triangles of one half of
// a warp's 32 cells that go row by row: one array per field, slot s of field
// f at f[s] (lanes reading distinct slots hit distinct banks; lanes reading
// one slot get a broadcast).
template <typename D>
struct TriStage {
  D x[3][32], y[3][32], pv[3][32], gxy[3][32], gyx[3][32], scale[32];
  int ox[32], oy[32], rlo[32], nrows[32], map[32];
  __device__ __forceinline__ void put(int s, const Tri<D>& t) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      x[q][s] = t.x[q];
      y[q][s] = t.y[q];
      pv[q][s] = t.pv[q];
      gxy[q][s] = t.gxy[q];
      gyx[q][s] = t.gyx[q];
    }
    scale[s] = t.scale;
    ox[s] = t.ox;
    oy[s] = t.oy;
    rlo[s] = t.rlo;
    nrows[s] = t.nrows;
    map[s] = t.map;
  }
};
constexpr int kDepositWarps = 8;  // warps per CTA of the deposition kernels (256 threads)

// Fire-and-forget 64-bit add to global memory (the map's difference array).
__device__ __forceinline__ void red_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}

// Edge k of staged triangle s inside row strip [rb, rt = rb + 1] (relative):
// the pieces between its entry and exit points, split at the column lines,
// into the row's difference array drow (relative column c at drow[c]). Each
// piece in column c adds a0 = K - a1 at c and a1 at c + 1; the add shared by
// two neighbouring pieces is made once. pb, pt: rb and rt times the scale.
// Columns left of the map (relative column clo) are merged into one cover at
// clo; the part right of column chi is dropped.
template <typename D>
__device__ __forceinline__ void deposit_edge_row(const TriStage<D>& st, int s, int k, D scale, D rb, D rt, D pb, D pt,
                                                 int clo, int chi, unsigned long long* drow) {
  const int j = k == 2 ? 0 : k + 1;
  const D yk = st.y[k][s], yj = st.y[j][s];
  if (yk == yj) return;  // a horizontal edge has no cover
  const D ylo = yk < yj ? yk : yj, yhi = yk > yj ? yk : yj;
  if (!(ylo < rt && yhi > rb)) return;
  const D xk = st.x[k][s], xj = st.x[j][s];
  const D xlo = xk < xj ? xk : xj, xhi = xk > xj ? xk : xj;
  // entry (a) and exit (b) of the edge in the strip, in the edge's direction:
  // a vertex, or the crossing with a row line (x from the edge, y exact)
  D xa, ya, qa, xb, yb, qb;
  const bool up = yj > yk;
  const D ea = up ? rb : rt, eb = up ? rt : rb;  // row lines where the edge enters / leaves
  if (up ? (yk >= rb) : (yk <= rt)) {
    xa = xk, ya = yk, qa = st.pv[k][s];
  } else {
    const D x = RN<D>::add(xk, RN<D>::mul(RN<D>::sub(ea, yk), st.gxy[k][s]));
    xa = x < xlo ? xlo : (x > xhi ? xhi : x), ya = ea, qa = up ? pb : pt;
  }
  if (up ? (yj <= rt) : (yj >= rb)) {
    xb = xj, yb = yj, qb = st.pv[j][s];
  } else {
    const D x = RN<D>::add(xk, RN<D>::mul(RN<D>::sub(eb, yk), st.gxy[k][s]));
    xb = x < xlo ? xlo : (x > xhi ? xhi : x), yb = eb, qb = up ? pt : pb;
  }
  const D h = st.gyx[k][s];
  const D plo = ya < yb ? ya : yb, phi = ya > yb ? ya : yb;
  // height (times scale) where the edge crosses the column line X, kept inside the piece's range
  auto cross = [&](D X) {
    D y = RN<D>::add(yk, RN<D>::mul(RN<D>::sub(X, xk), h));
    y = y < plo ? plo : (y > phi ? phi : y);
    return RN<D>::mul(y, scale);
  };
  // columns visited: right- or leftward from the entry's column to the exit's
  // (positions beyond the map are clamped first: only their side matters)
  const D cl = D(clo - 1), ch = D(chi + 1);
  const D ua = xa < cl ? cl : (xa > ch ? ch : xa), ub = xb < cl ? cl : (xb > ch ? ch : xb);
  int dir, c, ce;
  if (xb > xa) {
    dir = 1, c = int(floor(ua)), ce = int(ceil(ub)) - 1;
  } else if (xb < xa) {
    dir = -1, c = int(ceil(ua)) - 1, ce = int(floor(ub));
  } else {
    dir = 0, c = ce = int(floor(ua));
  }
  long long fa = (long long)RN<D>::to_fix(qa);
  long long fb = (long long)RN<D>::to_fix(qb);
  unsigned long long carry = 0;  // pending add at the column shared with the next piece
  if (dir >= 0) {
    if (ce < clo) {  // all of it left of the map
      red_add(drow + clo, (unsigned long long)(fa - fb));
      return;
    }
    if (c >= chi) return;
    if (c < clo) {  // the part left of the map: one cover at its first column
      const D X = D(clo);
      const D q = cross(X);
      const long long f = (long long)RN<D>::to_fix(q);
      carry = (unsigned long long)(fa - f);
      xa = X, qa = q, fa = f, c = clo;
    }
    if (ce >= chi) {  // stop at the map's right edge
      const D X = D(chi);
      xb = X, qb = cross(X), fb = (long long)RN<D>::to_fix(qb), ce = chi - 1;
    }
  } else {
    if (c < clo) {
      red_add(drow + clo, (unsigned long long)(fa - fb));
      return;
    }
    if (ce >= chi) return;
    if (c >= chi) {  // start at the map's right edge
      const D X = D(chi);
      xa = X, qa = cross(X), fa = (long long)RN<D>::to_fix(qa), c = chi - 1;
    }
  }
  const bool left_tail = dir < 0 && ce < clo;  // leftward past the map's first column
  const int cstop = left_tail ? clo : ce;
  const bool rightward = dir >= 0;
  for (;;) {
    const bool last = c == cstop;
    D xq, qq;
    long long fq;
    if (!last || left_tail) {
      xq = D(rightward ? c + 1 : c);  // the column line where the piece leaves column c
      qq = cross(xq);
      fq = (long long)RN<D>::to_fix(qq);
    } else {
      xq = xb, qq = qb, fq = fb;
    }
    const long long K = fa - fq;
    D fm = RN<D>::sub(RN<D>::mul(RN<D>::add(xa, xq), D(0.5)), D(c));
    fm = fm < D(0) ? D(0) : (fm > D(1) ? D(1) : fm);
    const long long a1 = (long long)RN<D>::to_fix(RN<D>::mul(RN<D>::sub(qa, qq), fm));
    const long long a0 = K - a1;
    // rightward: column c gets the carry and a0, a1 is carried to c + 1;
    // leftward: column c + 1 gets the carry and a1, a0 is carried to c
    const int near = rightward ? c : c + 1;
    const unsigned long long v = carry + (unsigned long long)(rightward ? a0 : a1);
    carry = (unsigned long long)(rightward ? a1 : a0);
    if (near < chi && v) red_add(drow + near, v);
    xa = xq, qa = qq, fa = fq;
    if (last) break;
    c += dir;
  }
  if (left_tail) carry += (unsigned long long)(fa - fb);
  const int far = rightward ? c + 1 : c;
  if (far < chi && carry) red_add(drow + far, carry);
}

// Row r (relative) of staged triangle s: its three edges into the row's
// difference array.
template <typename D>
__device__ __forceinline__ void deposit_row(const TriStage<D>& st, int s, int r, int npx, const DepositMaps& m_total,
                                            const DepositMaps& m_min, const DepositMaps& m_sad) {
  const D scale = st.scale[s];
  const int ox = st.ox[s], oy = st.oy[s], map = st.map[s];
  const D rb = D(r), rt = D(r + 1);
  const D pb = RN<D>::mul(rb, scale), pt = RN<D>::mul(rt, scale);
  const DepositMaps& M = map == 0 ? m_total : (map == 1 ? m_min : m_sad);
  unsigned long long* drow = M.diff + ((long long)oy + r) * ((long long)npx + 1) + ox;
  const int clo = -ox, chi = npx - ox;
#pragma unroll 1
  for (int k = 0; k < 3; k++) deposit_edge_row<D>(st, s, k, scale, rb, rt, pb, pt, clo, chi, drow);
}

// The 32 cells [base, base + 32) of an ncx-wide lattice whose corner rows are
// vx apart (whole warp; lanes past ncells idle). For each half of the cells
// (the triangles (y0, y1, y2), then (y2, y3, y0)): each lane classifies its
// triangle (setup_head); a triangle inside one pixel deposits at once, lanes
// in a row whose triangles fall in the same pixel adding once for all of
// them; the others are prepared (setup_tail) and staged in shared memory,
// compacted in lane order; the warp then scans their row counts and works
// through the (triangle, row) items 32 at a time, each lane finding its
// item's triangle by a binary search over the scan.
template <typename D>
__device__ __forceinline__ void deposit_warp_cells(const double2* __restrict__ verts, long long ncx, long long vx,
                                                   long long ncells, long long base, D factor, int npx, int npy,
                                                   const DepositMaps& m_total, const DepositMaps& m_min,
                                                   const DepositMaps& m_sad, int parities, TriStage<D>& stage,
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
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll 1
  for (int half = 0; half < 2; half++) {
    Tri<D> h;
    h.nrows = 0;  // idle lanes (past the last cell) deposit nothing
    h.single = 0;
    if (c < ncells) {
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
    const bool rows = h.nrows > 0 && !h.single;
    const unsigned b = __ballot_sync(0xffffffffu, rows);
    if (b == 0u) continue;
    const int slot = __popc(b & lt);
    if (rows) {
      setup_tail(h, factor);
      stage.put(slot, h);
    }
    __syncwarp();
    // inclusive scan of the staged triangles' row counts, lane s holding slot s
    const int mycnt = lane < __popc(b) ? stage.nrows[lane] : 0;
    int incl = mycnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int it0 = 0; it0 < total; it0 += 32) {
      const int item = it0 + lane;
      int lo = 0, hi = 31;  // slot: first lane whose inclusive count exceeds item
#pragma unroll
      for (int step = 0; step < 5; step++) {
        const int mid = (lo + hi) >> 1;
        const int v = __shfl_sync(0xffffffffu, incl, mid);
        if (v > item) hi = mid;
        else lo = mid + 1;
      }
      const int before = __shfl_sync(0xffffffffu, incl - mycnt, lo);
      if (item < total) deposit_row<D>(stage, lo, stage.rlo[lo] + (item - before), npx, m_total, m_min, m_sad);
    }
    __syncwarp();  // slots free for the next half
  }
}

// Cells of an ncx x ncy lattice whose (ncx+1) x (ncy+1) corner positions are in
// `verts`, 32 consecutive cells per warp (deposit_warp_cells).
template <typename D>
__global__ void __launch_bounds__(kDepositWarps * 32, sizeof(D) == 4 ? 4 : 2)
    ipm_deposit_cells(const double2* __restrict__ verts, long long ncx, long long ncy, D factor, int npx, int npy,
                      DepositMaps m_total, DepositMaps m_min, DepositMaps m_sad, int parities) {
  const long long ncells = ncx * ncy;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  __shared__ TriStage<D> stages[kDepositWarps];
  TriStage<D>& stage = stages[threadIdx.x >> 5];
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

// Batched deposition: the warps stride over the 32-cell chunks of all pieces
// of the pass; a chunk's piece is found by a binary search over chunk0.
// Realization r accumulates into the maps at r * map_stride / r * diff_stride.
template <typename D>
__global__ void __launch_bounds__(kDepositWarps * 32, sizeof(D) == 4 ? 4 : 2)
    ipm_deposit_batch(const double2* __restrict__ verts, const DepositPiece<D>* __restrict__ pieces, int npieces,
                      long long nchunks, int npx, int npy, DepositMaps maps, long long map_stride,
                      long long diff_stride) {
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  __shared__ TriStage<D> stages[kDepositWarps];
  TriStage<D>& stage = stages[threadIdx.x >> 5];
  for (long long g = warp0; g < nchunks; g += nwarps) {
    int lo = 0, hi = npieces - 1;  // last piece with chunk0 <= g
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (pieces[mid].chunk0 <= g) lo = mid;
      else hi = mid - 1;
    }
    const DepositPiece<D> pc = pieces[lo];
    const DepositMaps M{maps.acc + pc.r * map_stride, maps.diff + pc.r * diff_stride};
    deposit_warp_cells<D>(verts + pc.voff, pc.ncx, pc.vstride, pc.ncx * pc.ncy, (g - pc.chunk0) * 32, pc.factor,
                          npx, npy, M, M, M, 0, stage, pc.vstep, pc.ox, pc.oy, pc.inv_scale);
  }
}

// Fixed point (modulo 2^64, read as signed) -> magnification: the rounding of
// the pieces of a pixel's coverage can leave a few units below zero where its
// true coverage is zero or nearly so; those read as 0.
__device__ __forceinline__ double fix_to_double(unsigned long long v) {
  const long long s = (long long)v;
  return s > 0 ? double(s) * kFixInv : 0.0;
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
          out[k] = T(fix_to_double(v));
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
      out_min[k] = T(fix_to_double(a));
      out_sad[k] = T(fix_to_double(b));
      out_total[k] = T(fix_to_double(a + b));
    } else {
      out_total[k] = T(fix_to_double(acc_total[k]));
    }
  }
}

}  // namespace irsb
