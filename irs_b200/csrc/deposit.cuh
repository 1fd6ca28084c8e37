// IPM deposition: each lens-plane cell maps to two source-plane triangles whose
// image-plane area is spread over the pixels they overlap, in proportion to the
// overlap area.
//
// Procedure of the reference (ipm_functions.cuh:168-216 and
// Polygon::allocate_area_among_pixels, polygon.cuh:349-467): triangles
// (y0,y1,y2) and (y2,y3,y0) from the cell corners; skip |A| >= 1e4 * cell
// area; route by the sign of A to the minima (A < 0) or saddle map when
// parities are kept; clip the triangle to the map, then cut it into column
// strips at x = k+1 and each strip into rows at y = k+1 (Sutherland-Hodgman
// against one axis-parallel line at a time, at most 7 vertices), adding
// factor * |A_piece| / |A_whole| to each pixel.
//
// Differences by design:
//   * edge intersections use linear interpolation with IEEE operations
//     (the reference goes through log/exp);
//   * coordinates are taken relative to an integer origin at the triangle's
//     lower-left pixel, so clip lines stay exact in FP32;
//   * the map accumulates unsigned 64-bit fixed point (2^32 per unit) with
//     integer atomics, so the result does not depend on the order in which
//     threads arrive: given the same vertex positions the map is bit-exact.
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

constexpr int kPolyMax = 7;  // polygon.cuh:11

template <typename D>
struct Poly {
  D x[kPolyMax], y[kPolyMax];
  int n;
  __device__ __forceinline__ void add(D px, D py) {
    if (n >= kPolyMax) {  // overflow empties the polygon (polygon.cuh:95-111)
      n = 0;
      return;
    }
    x[n] = px;
    y[n] = py;
    n++;
  }
  __device__ __forceinline__ D area() const {
    if (n < 3) return D(0);
    D s = D(0);
    for (int i = 0; i < n; i++) {
      int j = (i + 1 == n) ? 0 : i + 1;
      D dx = RN<D>::sub(x[j], x[i]);
      D dy = RN<D>::sub(y[j], y[i]);
      s = RN<D>::add(s, RN<D>::sub(RN<D>::mul(dy, x[i]), RN<D>::mul(dx, y[i])));
    }
    return RN<D>::div(s, D(2));
  }
  __device__ __forceinline__ D min_x() const {
    D m = x[0];
    for (int i = 1; i < n; i++) m = x[i] < m ? x[i] : m;
    return m;
  }
  __device__ __forceinline__ D max_x() const {
    D m = x[0];
    for (int i = 1; i < n; i++) m = x[i] > m ? x[i] : m;
    return m;
  }
  __device__ __forceinline__ D min_y() const {
    D m = y[0];
    for (int i = 1; i < n; i++) m = y[i] < m ? y[i] : m;
    return m;
  }
  __device__ __forceinline__ D max_y() const {
    D m = y[0];
    for (int i = 1; i < n; i++) m = y[i] > m ? y[i] : m;
    return m;
  }
};

// point on segment (x1,y1)-(x2,y2) at abscissa X (the segment crosses X)
template <typename D>
__device__ __forceinline__ D y_at(D X, D x1, D y1, D x2, D y2) {
  return RN<D>::add(y1, RN<D>::div(RN<D>::mul(RN<D>::sub(X, x1), RN<D>::sub(y2, y1)), RN<D>::sub(x2, x1)));
}

// Split P at x = X into lo (x <= X side) and hi (x >= X side).
template <typename D>
__device__ __forceinline__ void clip_x(const Poly<D>& P, D X, Poly<D>& lo, Poly<D>& hi) {
  lo.n = hi.n = 0;
  for (int i = 0; i < P.n; i++) {
    int j = (i + 1 == P.n) ? 0 : i + 1;
    D xi = P.x[i], yi = P.y[i];
    if (xi < X) {
      lo.add(xi, yi);
      if (P.x[j] > X) {
        D yv = y_at(X, xi, yi, P.x[j], P.y[j]);
        lo.add(X, yv);
        hi.add(X, yv);
      }
    } else if (xi > X) {
      hi.add(xi, yi);
      if (P.x[j] < X) {
        D yv = y_at(X, xi, yi, P.x[j], P.y[j]);
        lo.add(X, yv);
        hi.add(X, yv);
      }
    } else {
      lo.add(xi, yi);
      hi.add(xi, yi);
    }
  }
}
// Split P at y = Y into lo (y <= Y side) and hi (y >= Y side).
template <typename D>
__device__ __forceinline__ void clip_y(const Poly<D>& P, D Y, Poly<D>& lo, Poly<D>& hi) {
  lo.n = hi.n = 0;
  for (int i = 0; i < P.n; i++) {
    int j = (i + 1 == P.n) ? 0 : i + 1;
    D xi = P.x[i], yi = P.y[i];
    if (yi < Y) {
      lo.add(xi, yi);
      if (P.y[j] > Y) {
        D xv = y_at(Y, yi, xi, P.y[j], P.x[j]);
        lo.add(xv, Y);
        hi.add(xv, Y);
      }
    } else if (yi > Y) {
      hi.add(xi, yi);
      if (P.y[j] < Y) {
        D xv = y_at(Y, yi, xi, P.y[j], P.x[j]);
        lo.add(xv, Y);
        hi.add(xv, Y);
      }
    } else {
      lo.add(xi, yi);
      hi.add(xi, yi);
    }
  }
}

template <typename D>
__device__ __forceinline__ void fix_add(unsigned long long* __restrict__ map, long long idx, D a, D scale) {
  unsigned long long q = RN<D>::to_fix(RN<D>::mul(a, scale));
  if (q) atomicAdd(map + idx, q);
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

// Deposits triangle (a, b, c) given in absolute pixel coordinates (row axis
// already flipped). factor = image-plane area of the triangle in pixel units.
//
// Sweep: the triangle is clipped to the map, then cut into row strips
// [y, y+1] (bottom to top). Within a strip, the columns between the left and
// right boundaries that lie inside both the strip's bottom edge (on y) and
// its top edge (on y+1) are fully covered: by convexity the unit pixel is
// inside, so its clipped area is exactly 1 and the run [xa, xb) is recorded
// as one +q / -q pair in the difference array. The remaining boundary columns
// are clipped one at a time (left to right) and their areas added as pieces.
template <typename D>
__device__ void deposit_triangle(double ax, double ay, double bx, double by, double cx, double cy, D factor,
                                 int npx, int npy, DepositMaps m_total, DepositMaps m_min, DepositMaps m_sad,
                                 bool parities) {
  if (isnan(ax) || isnan(ay) || isnan(bx) || isnan(by) || isnan(cx) || isnan(cy)) return;
  double fx = floor(fmin(ax, fmin(bx, cx)));
  double fy = floor(fmin(ay, fmin(by, cy)));
  if (!(fx > -2.0e9 && fx < 2.0e9 && fy > -2.0e9 && fy < 2.0e9)) return;
  const long long ox = (long long)fx, oy = (long long)fy;
  Poly<D> P;
  P.n = 3;
  P.x[0] = D(ax - fx);
  P.y[0] = D(ay - fy);
  P.x[1] = D(bx - fx);
  P.y[1] = D(by - fy);
  P.x[2] = D(cx - fx);
  P.y[2] = D(cy - fy);
  D A = P.area();
  if (!(dabs(A) < RN<D>::mul(D(10000), factor))) return;
  DepositMaps M = parities ? (A < D(0) ? m_min : m_sad) : m_total;
  // map edges in local coordinates (exact: integers)
  const D X0 = D(-ox), X1 = D(npx - ox), Y0 = D(-oy), Y1 = D(npy - oy);
  if (P.min_x() >= X1 || P.max_x() <= X0 || P.min_y() >= Y1 || P.max_y() <= Y0) return;
  D whole = dabs(A);
  if (whole == D(0)) return;
  const D scale = RN<D>::div(RN<D>::mul(factor, D(kFixScale)), whole);
  const unsigned long long qfull = RN<D>::to_fix(scale);
  Poly<D> lo, hi;
  if (P.min_x() < X0) {
    clip_x(P, X0, lo, hi);
    P = hi;
  }
  if (P.n >= 1 && P.max_x() > X1) {
    clip_x(P, X1, lo, hi);
    P = lo;
  }
  if (P.n >= 1 && P.min_y() < Y0) {
    clip_y(P, Y0, lo, hi);
    P = hi;
  }
  if (P.n >= 1 && P.max_y() > Y1) {
    clip_y(P, Y1, lo, hi);
    P = lo;
  }
  if (P.n < 3) return;
  int ymin = int(P.min_y()), ymax = int(P.max_y());
  if (ymax + oy == npy) ymax--;
  const long long rstride = (long long)npx + 1;
  for (int y = ymin; y <= ymax; y++) {
    Poly<D> S;
    if (y < ymax) {
      clip_y(P, D(y + 1), S, hi);
      P = hi;
    } else {
      S = P;
    }
    if (S.n < 3) continue;
    const long long row = oy + y;
    // full-coverage run from the strip's bottom (y) and top (y + 1) edges
    const D yb = D(y), yt = D(y + 1);
    D b0 = D(0), b1 = D(0), t0 = D(0), t1 = D(0);
    bool hb = false, ht = false;
    for (int i = 0; i < S.n; i++) {
      D vx = S.x[i], vy = S.y[i];
      if (vy == yb) {
        b0 = hb ? (vx < b0 ? vx : b0) : vx;
        b1 = hb ? (vx > b1 ? vx : b1) : vx;
        hb = true;
      }
      if (vy == yt) {
        t0 = ht ? (vx < t0 ? vx : t0) : vx;
        t1 = ht ? (vx > t1 ? vx : t1) : vx;
        ht = true;
      }
    }
    int xa = 1, xb = 0;
    if (hb && ht) {
      D l = b0 > t0 ? b0 : t0, r = b1 < t1 ? b1 : t1;
      xa = int(ceil(l));
      xb = int(floor(r));
    }
    int xmin = int(S.min_x()), xmax = int(S.max_x());
    if (xmax + ox == npx) xmax--;
    Poly<D> R = S;
    int x = xmin;
    while (x < xmax) {
      if (xa < xb && x == xa) {
        clip_x(R, D(xb), lo, hi);
        R = hi;
        atomicAdd(M.diff + row * rstride + (ox + xa), qfull);
        atomicAdd(M.diff + row * rstride + (ox + xb), (unsigned long long)(0ULL - qfull));
        x = xb;
        continue;
      }
      Poly<D> L;
      clip_x(R, D(x + 1), L, hi);
      R = hi;
      if (L.n >= 3) fix_add<D>(M.acc, row * npx + (ox + x), dabs(L.area()), scale);
      x++;
    }
    if (x == xmax) fix_add<D>(M.acc, row * npx + (ox + xmax), dabs(R.area()), scale);
  }
}

// One thread per lens-plane cell (i, j) of an ncx x ncy cell lattice whose
// (ncx+1) x (ncy+1) vertices are in `verts`.
template <typename D>
__global__ void __launch_bounds__(256) ipm_deposit_cells(const double2* __restrict__ verts, long long ncx,
                                                         long long ncy, D factor, int npx, int npy,
                                                         DepositMaps m_total, DepositMaps m_min, DepositMaps m_sad,
                                                         int parities) {
  const long long ncells = ncx * ncy;
  const long long vx = ncx + 1;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
       c += (long long)gridDim.x * blockDim.x) {
    long long j = c / ncx, i = c - j * ncx;
    double2 y0 = verts[(j + 1) * vx + (i + 1)];  // z + rhs
    double2 y1 = verts[(j + 1) * vx + i];        // z - conj(rhs)
    double2 y2 = verts[j * vx + i];              // z - rhs
    double2 y3 = verts[j * vx + (i + 1)];        // z + conj(rhs)
    deposit_triangle<D>(y0.x, y0.y, y1.x, y1.y, y2.x, y2.y, factor, npx, npy, m_total, m_min, m_sad,
                        parities != 0);
    deposit_triangle<D>(y2.x, y2.y, y3.x, y3.y, y0.x, y0.y, factor, npx, npy, m_total, m_min, m_sad,
                        parities != 0);
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
