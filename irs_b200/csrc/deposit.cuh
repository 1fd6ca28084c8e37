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
//     Green's theorem (pixel_coverage) instead of by successive polygon
//     clips: register-only arithmetic, no polygon arrays;
//   * rows of a triangle are independent work items; a warp expands the rows
//     of its 64 triangles and shares them out 32 at a time;
//   * pixels inside both the bottom and the top chord of a row strip are fully
//     covered (area exactly 1) and are added as a run through a per-row
//     difference array;
//   * coordinates are relative to an integer origin at the triangle's
//     lower-left pixel; the map accumulates unsigned 64-bit fixed point (2^32
//     per unit) with integer atomics, so the result does not depend on thread
//     order: given the same corner positions the map is bit-exact.
// Every floating-point operation is an explicitly rounded intrinsic (no FMA
// contraction), so a host implementation with the same operation sequence
// reproduces the map bit for bit.
#pragma once
#include "common.cuh"

namespace irsb {

template <typename D>
struct RN;
template <>
struct RN<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
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
// origin (ox, oy), per-edge reciprocals, fixed-point scale and target map.
template <typename D>
struct Tri {
  D x[3], y[3];     // CCW, relative to (ox, oy)
  D idx[3], idy[3]; // 1 / (x[k+1] - x[k]), 1 / (y[k+1] - y[k]) (0 for a zero difference)
  D scale;          // factor * 2^32 / |area|
  int ox, oy;
  int rlo, nrows;   // first row (relative) and number of rows to visit
  int map;          // 0 total, 1 minima, 2 saddles
};

template <typename D>
__device__ __forceinline__ D rcp_or_zero(D v) {
  return v != D(0) ? RN<D>::div(D(1), v) : D(0);
}

// Triangle (a, b, c) in absolute pixel coordinates (row axis flipped) ->
// Tri, or nrows = 0 when it deposits nothing. Tests of the reference
// (ipm_functions.cuh:170-193, polygon.cuh:351-372): NaN corner, |A| >= 1e4
// * factor, entirely outside the map, zero area.
template <typename D>
__device__ __forceinline__ Tri<D> setup_triangle(double ax, double ay, double bx, double by, double cx, double cy,
                                                 D factor, int npx, int npy, bool parities) {
  Tri<D> t;
  t.nrows = 0;
  t.rlo = 0;
  t.ox = t.oy = 0;
  t.map = 0;
  t.scale = D(0);
  for (int k = 0; k < 3; k++) t.x[k] = t.y[k] = t.idx[k] = t.idy[k] = D(0);
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
  D A = RN<D>::div(s, D(2));
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
  for (int k = 0; k < 3; k++) {
    int j = k == 2 ? 0 : k + 1;
    t.idx[k] = rcp_or_zero(RN<D>::sub(t.x[j], t.x[k]));
    t.idy[k] = rcp_or_zero(RN<D>::sub(t.y[j], t.y[k]));
  }
  t.scale = RN<D>::div(RN<D>::mul(factor, D(kFixScale)), whole);
  t.ox = ox;
  t.oy = oy;
  int rlo = 0 > -oy ? 0 : -oy;
  int rhi = int(floor(mxy));
  if (rhi > npy - 1 - oy) rhi = npy - 1 - oy;
  t.rlo = rlo;
  t.nrows = rhi >= rlo ? rhi - rlo + 1 : 0;
  return t;
}

// x-extent [lo, hi] of the triangle on the horizontal line y = yk; false if it
// does not reach that line.
template <typename D>
__device__ __forceinline__ bool chord(const Tri<D>& t, D yk, D& lo, D& hi) {
  bool any = false;
  lo = D(0);
  hi = D(0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int j = k == 2 ? 0 : k + 1;
    const D y1 = t.y[k], y2 = t.y[j], x1 = t.x[k], x2 = t.x[j];
    if ((y1 <= yk && yk <= y2) || (y2 <= yk && yk <= y1)) {
      D xa, xb;
      if (y1 != y2) {
        xa = RN<D>::add(x1, RN<D>::mul(RN<D>::mul(RN<D>::sub(yk, y1), t.idy[k]), RN<D>::sub(x2, x1)));
        xb = xa;
      } else {
        xa = x1;
        xb = x2;
      }
      D mn = xa < xb ? xa : xb, mx = xa > xb ? xa : xb;
      lo = any ? (mn < lo ? mn : lo) : mn;
      hi = any ? (mx > hi ? mx : hi) : mx;
      any = true;
    }
  }
  return any;
}

// Area of the triangle inside the pixel [c, c+1] x [r, r+1] (relative
// coordinates) from Green's theorem, area = -sum over the boundary of
// integral (y - r) dx: each edge contributes its segment clipped to the pixel
// (a trapezoid), the pixel's top side contributes the chord length at y = r+1
// inside [c, c+1], the vertical sides and the bottom side contribute nothing.
template <typename D>
__device__ __forceinline__ D pixel_coverage(const Tri<D>& t, D c, D r, bool has_top, D ct0, D ct1) {
  const D c1 = RN<D>::add(c, D(1)), r1 = RN<D>::add(r, D(1));
  D s = D(0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int j = k == 2 ? 0 : k + 1;
    const D x1 = t.x[k], y1 = t.y[k];
    const D dx = RN<D>::sub(t.x[j], x1), dy = RN<D>::sub(t.y[j], y1);
    D t0 = D(0), t1 = D(1);
    bool ok = true;
    if (dx != D(0)) {
      D ta = RN<D>::mul(RN<D>::sub(c, x1), t.idx[k]), tb = RN<D>::mul(RN<D>::sub(c1, x1), t.idx[k]);
      D lo = ta < tb ? ta : tb, hi = ta > tb ? ta : tb;
      t0 = lo > t0 ? lo : t0;
      t1 = hi < t1 ? hi : t1;
    } else {
      ok = !(x1 < c || x1 > c1);
    }
    if (dy != D(0)) {
      D ta = RN<D>::mul(RN<D>::sub(r, y1), t.idy[k]), tb = RN<D>::mul(RN<D>::sub(r1, y1), t.idy[k]);
      D lo = ta < tb ? ta : tb, hi = ta > tb ? ta : tb;
      t0 = lo > t0 ? lo : t0;
      t1 = hi < t1 ? hi : t1;
    } else {
      ok = ok && !(y1 < r || y1 > r1);
    }
    if (ok && t0 < t1) {
      const D xa = RN<D>::add(x1, RN<D>::mul(t0, dx)), xb = RN<D>::add(x1, RN<D>::mul(t1, dx));
      const D ya = RN<D>::sub(RN<D>::add(y1, RN<D>::mul(t0, dy)), r);
      const D yb = RN<D>::sub(RN<D>::add(y1, RN<D>::mul(t1, dy)), r);
      s = RN<D>::sub(s, RN<D>::mul(RN<D>::mul(RN<D>::sub(xb, xa), RN<D>::add(ya, yb)), D(0.5)));
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
  D cb0, cb1, ct0, ct1;
  const bool hb = chord(t, rb, cb0, cb1);
  const bool ht = chord(t, rt, ct0, ct1);
  // x-extent of the triangle within the row
  bool any = false;
  D xlo = D(0), xhi = D(0);
  if (hb) {
    xlo = cb0;
    xhi = cb1;
    any = true;
  }
  if (ht) {
    xlo = any ? (ct0 < xlo ? ct0 : xlo) : ct0;
    xhi = any ? (ct1 > xhi ? ct1 : xhi) : ct1;
    any = true;
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (t.y[k] > rb && t.y[k] < rt) {
      xlo = any ? (t.x[k] < xlo ? t.x[k] : xlo) : t.x[k];
      xhi = any ? (t.x[k] > xhi ? t.x[k] : xhi) : t.x[k];
      any = true;
    }
  }
  if (!any) return;
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
    atomicAdd(M.diff + dbase + xa, q);
    atomicAdd(M.diff + dbase + xb, (unsigned long long)(0ULL - q));
  }
  for (int c = cmin; c <= cmax; c++) {
    if (xa < xb && c == xa) {
      c = xb - 1;
      continue;
    }
    D a = pixel_coverage(t, D(c), rb, ht, ct0, ct1);
    if (a > D(0)) {
      unsigned long long q = RN<D>::to_fix(RN<D>::mul(a, t.scale));
      if (q) atomicAdd(M.acc + rbase + c, q);
    }
  }
}

// Cells of an ncx x ncy lattice whose (ncx+1) x (ncy+1) corner positions are in
// `verts`. A warp takes 32 consecutive cells (64 triangles), scans their row
// counts and then works through all (triangle, row) items 32 at a time: each
// lane finds its item's owner lane by a binary search over the scan and reads
// the triangle through shuffles, so a triangle with many rows is spread over
// the warp instead of holding one lane.
template <typename D>
__global__ void __launch_bounds__(256) ipm_deposit_cells(const double2* __restrict__ verts, long long ncx,
                                                         long long ncy, D factor, int npx, int npy,
                                                         DepositMaps m_total, DepositMaps m_min, DepositMaps m_sad,
                                                         int parities) {
  const long long ncells = ncx * ncy;
  const long long vx = ncx + 1;
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long base = warp0 * 32; base < ncells; base += nwarps * 32) {
    const long long c = base + lane;
    Tri<D> ta, tb;
    ta.nrows = tb.nrows = 0;
    if (c < ncells) {
      long long j = c / ncx, i = c - j * ncx;
      double2 y0 = verts[(j + 1) * vx + (i + 1)];  // z + rhs
      double2 y1 = verts[(j + 1) * vx + i];        // z - conj(rhs)
      double2 y2 = verts[j * vx + i];              // z - rhs
      double2 y3 = verts[j * vx + (i + 1)];        // z + conj(rhs)
      ta = setup_triangle<D>(y0.x, y0.y, y1.x, y1.y, y2.x, y2.y, factor, npx, npy, parities != 0);
      tb = setup_triangle<D>(y2.x, y2.y, y3.x, y3.y, y0.x, y0.y, factor, npx, npy, parities != 0);
    }
    // inclusive scan of this lane's row count over the warp
    const int mine = ta.nrows + tb.nrows;
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int it0 = 0; it0 < total; it0 += 32) {
      const int item = it0 + lane;
      // owner: first lane whose inclusive count exceeds item
      int lo = 0, hi = 31;
#pragma unroll
      for (int step = 0; step < 5; step++) {
        int mid = (lo + hi) >> 1;
        int v = __shfl_sync(0xffffffffu, incl, mid);
        if (v > item) hi = mid;
        else lo = mid + 1;
      }
      const int owner = lo;
      const int before = __shfl_sync(0xffffffffu, incl - mine, owner);
      const int na = __shfl_sync(0xffffffffu, ta.nrows, owner);
      const int k = item - before;
      const bool first = k < na;
      // fetch the owner's triangle (both candidates, then select)
      Tri<D> t;
#pragma unroll
      for (int q = 0; q < 3; q++) {
        D xa_ = __shfl_sync(0xffffffffu, ta.x[q], owner), xb_ = __shfl_sync(0xffffffffu, tb.x[q], owner);
        D ya_ = __shfl_sync(0xffffffffu, ta.y[q], owner), yb_ = __shfl_sync(0xffffffffu, tb.y[q], owner);
        D ia_ = __shfl_sync(0xffffffffu, ta.idx[q], owner), ib_ = __shfl_sync(0xffffffffu, tb.idx[q], owner);
        D ja_ = __shfl_sync(0xffffffffu, ta.idy[q], owner), jb_ = __shfl_sync(0xffffffffu, tb.idy[q], owner);
        t.x[q] = first ? xa_ : xb_;
        t.y[q] = first ? ya_ : yb_;
        t.idx[q] = first ? ia_ : ib_;
        t.idy[q] = first ? ja_ : jb_;
      }
      {
        D sa = __shfl_sync(0xffffffffu, ta.scale, owner), sb = __shfl_sync(0xffffffffu, tb.scale, owner);
        int oxa = __shfl_sync(0xffffffffu, ta.ox, owner), oxb = __shfl_sync(0xffffffffu, tb.ox, owner);
        int oya = __shfl_sync(0xffffffffu, ta.oy, owner), oyb = __shfl_sync(0xffffffffu, tb.oy, owner);
        int rla = __shfl_sync(0xffffffffu, ta.rlo, owner), rlb = __shfl_sync(0xffffffffu, tb.rlo, owner);
        int mpa = __shfl_sync(0xffffffffu, ta.map, owner), mpb = __shfl_sync(0xffffffffu, tb.map, owner);
        t.scale = first ? sa : sb;
        t.ox = first ? oxa : oxb;
        t.oy = first ? oya : oyb;
        t.rlo = first ? rla : rlb;
        t.map = first ? mpa : mpb;
      }
      if (item < total) {
        const int r = t.rlo + (first ? k : k - na);
        DepositMaps M = t.map == 0 ? m_total : (t.map == 1 ? m_min : m_sad);
        deposit_row<D>(t, r, npx, M);
      }
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
