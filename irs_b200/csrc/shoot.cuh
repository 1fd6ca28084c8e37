// Lens-equation kernels over a regular lattice, tiled by quadtree leaf.
//
// Per lattice point z the source position is (complex_image_to_source,
// irs_functions.cuh:33-45 / ipm_functions.cuh:34-46)
//     w = (1 - kappa) z + gamma conj(z) - alpha_star - alpha_local - alpha_smooth
// with alpha_star the leaf's near-field direct sum, alpha_local the Horner
// evaluation of the leaf's local expansion and alpha_smooth the smooth sheet.
//
// Two arithmetic forms:
//   * shoot_f64 -- the plain uniform FP64 form. Global coordinates and the
//     reference's operation order for the ray position, the far-field Horner
//     loop and the source-to-pixel conversion (point_to_pixel,
//     array_functions.cuh:70-75).
//   * shoot_f32 -- the FP32 form. Coordinates are taken relative to the leaf
//     centre; the near-field sum runs in FP32 with blocked two-sum
//     compensation (naive partial sums of 16 stars folded into a compensated
//     accumulator); the far field is an FP32 Horner evaluation of coefficients
//     built in FP64; the linear part of the lens equation is applied at the
//     leaf centre in FP64 and the final cell-local -> global pixel conversion
//     is FP64.
//
// Work distribution: a CTA takes one (leaf, 32x32 tile) work item at a time
// (grid-stride over the global tile list), stages the leaf's <= 32 near stars
// and <= 31 coefficients in shared memory, and every lane reads them as
// warp-wide broadcasts. Each thread evaluates R lattice points (rows ty,
// ty + 32/R, ... of the tile; R = 8, 4 or 2 at 128, 256 or 512 threads per
// CTA) against each staged star, so one shared-memory read feeds R
// evaluations. Without parities the FP32 form runs
// its near and far field on pairs of points with the paired FP32 instructions
// of sm_100 (near_far_pairs): half the issue slots, the same bits.
//
// Outputs: IRS adds one count per ray to the int32 map with the reference's
// clamp and row flip (irs_functions.cuh:147-198); the IPM vertex mode writes
// the vertex's source position in pixel units with the row axis flipped
// (ipm_functions.cuh:159-165) for the deposition pass.
#pragma once
#include "common.cuh"
#include "leaves.cuh"
#include "smooth.cuh"

namespace irsb {

constexpr int kShootThreads = 256;
constexpr int kRaysPerThread = kTileY / (kShootThreads / kTileX);  // 4

struct ShootParams {
  double kappa, gamma, kstar, theta2, inv_pi;
  int rect, approx, taylor_smooth, p;
  double corner_re, corner_im;
  double cy_re, cy_im;    // centre of the source region
  double hly_re, hly_im;  // half length of the source region
  int npx, npy;
  double base_x, base_y;  // lattice coordinate of index 0
  double rhs_x, rhs_y;    // half spacing of the lattice
  long long nx, ny;       // lattice extent
  long long jbase;        // first lattice row held in the corner buffer (row bands)
};

struct LeafPtrs {
  const double* cx;
  const double* cy;
  const double* hl;
  const int* nnear;
  const double4* near64;
  const float4* near32;
  const double2* coef64;
  const float2* coef32;
  const int4* rect;
  const long long* tile_off;
  const int4* table;  // per tile: leaf, i0, j0, (ni << 16) | nj
  int nleaves;
  // constant term, at the leaf centre, of the smooth sheet's deviation from
  // -kappa_star z where that deviation is folded into coef32 (rectangular
  // field, approximate sheet, FP32 form); nullptr: not folded
  const double2* smooth0 = nullptr;
};

struct TileInfo {
  int leaf, i0, j0, ni, nj;
};

// Corner buffers of refined tiles (adaptive IPM): a point (i, j) of the
// level-s corner lattice belongs to every tile of level s whose corner grid
// holds it (up to 4 on tile edges) and is stored in each of their buffers:
// tile t at out + slot[t] * per, row stride ncell_x(t) * s + 1.
struct TileStore {
  const int* slot;  // per tile: buffer slot, -1 when not refined in this pass
  int s;            // subdivision level
  int ntx, nty;     // tiles
  long long ncx, ncy;  // base cells
  long long per;    // corners per slot
  double2* out;
};

__device__ __forceinline__ void tile_store(const TileStore& st, long long i, long long j, double2 v) {
  // lattice indices fit 32 bits (below 32 * 16 * 2^16); side is a power of two
  const int side = 32 * st.s, sh = __ffs(side) - 1;  // lattice points per tile side
  const int ii = int(i), jj = int(j);
  const int txh = ii >> sh, tyh = jj >> sh;
  const bool on_x = (ii & (side - 1)) == 0, on_y = (jj & (side - 1)) == 0;
#pragma unroll
  for (int dy = 0; dy < 2; dy++) {
    const int ty = tyh - dy;
    if (ty < 0 || ty >= st.nty || (dy == 1 && !on_y)) continue;
#pragma unroll
    for (int dx = 0; dx < 2; dx++) {
      const int tx = txh - dx;
      if (tx < 0 || tx >= st.ntx || (dx == 1 && !on_x)) continue;
      const int k = st.slot[ty * st.ntx + tx];
      if (k < 0) continue;
      const long long cx = (st.ncx - 32LL * tx) < 32 ? (st.ncx - 32LL * tx) : 32;
      const long long a = ii - tx * side, b = jj - ty * side;
      st.out[k * st.per + b * (cx * st.s + 1) + a] = v;
    }
  }
}

// Destination of a tile's results: IRS maps, the IPM corner buffer whose
// row 0 is lattice row vrow0, or refined tile buffers (tiles != nullptr).
struct ShootOut {
  int* pix;
  int* pmin;
  int* psad;
  double2* verts;
  long long vrow0;
  const TileStore* tiles = nullptr;
};

__device__ __forceinline__ TileInfo tile_info(const LeafPtrs& lp, long long t) {
  int4 e = lp.table[t];
  TileInfo ti;
  ti.leaf = e.x;
  ti.i0 = e.y;
  ti.j0 = e.z;
  ti.ni = e.w >> 16;
  ti.nj = e.w & 0xffff;
  return ti;
}

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Two FP32 values in one 64-bit register pair. The paired (.f32x2) add, sub,
// mul and fma of sm_100 round each half exactly as the scalar instruction
// does, with one issue slot for both: the FP32 lens kernel evaluates two
// lattice points per instruction with results bit-identical to the scalar form.
struct f32x2 {
  unsigned long long v;
};
__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk2(f32x2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// A leaf's near stars and expansion coefficients staged for the paired form:
// each value twice, so that one shared-memory load gives both halves.
struct NearPairs {
  ulonglong2 xy[kMaxStarsDirect];  // (x, x), (y, y)
  unsigned long long m[kMaxStarsDirect];  // (m, m)
  ulonglong2 coef[kMaxOrder];  // (re, re), (im, im)
};

// Fire-and-forget add of a ray count in global memory (PTX red; the count is
// never read back by the adding thread).
__device__ __forceinline__ void red_add_s32(int* p, int v) {
  asm volatile("red.global.add.s32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v) : "memory");
}

// Adds one ray count with the reference's clamp and row flip; (px, py) are the
// source position in pixel units (unflipped).
__device__ __forceinline__ void irs_deposit(double px, double py, int npx, int npy, int* __restrict__ pix,
                                            int* __restrict__ pmin, int* __restrict__ psad, bool parity_min,
                                            bool parities) {
  int ix = int(px), iy = int(py);
  if (ix == npx) ix--;
  if (iy == npy) iy--;
  long long idx = (long long)(npy - 1 - iy) * npx + ix;
  if (parities) red_add_s32(parity_min ? &pmin[idx] : &psad[idx], 1);
  red_add_s32(&pix[idx], 1);
}

// ----------------------------------------------------------------- FP64 form
template <bool VERT, bool PAR>
__global__ void __launch_bounds__(kShootThreads) shoot_f64(ShootParams sp, LeafPtrs lp, long long total_tiles,
                                                           int* __restrict__ pix, int* __restrict__ pmin,
                                                           int* __restrict__ psad, double2* __restrict__ verts) {
  __shared__ double4 s_near[kMaxStarsDirect];
  __shared__ double2 s_coef[kMaxOrder];
  const int tx = threadIdx.x & (kTileX - 1), ty = threadIdx.x / kTileX;
  const cplx<double> corner = mk(sp.corner_re, sp.corner_im);
  for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    TileInfo ti = tile_info(lp, t);
    const int nn = lp.nnear[ti.leaf];
    if (threadIdx.x < kMaxStarsDirect) s_near[threadIdx.x] = lp.near64[(size_t)ti.leaf * kMaxStarsDirect + threadIdx.x];
    if (threadIdx.x >= 64 && threadIdx.x < 64 + kMaxOrder)
      s_coef[threadIdx.x - 64] = lp.coef64[(size_t)ti.leaf * kMaxOrder + threadIdx.x - 64];
    const double lcx = lp.cx[ti.leaf], lcy = lp.cy[ti.leaf], lhl = lp.hl[ti.leaf];
    __syncthreads();
    if (tx < ti.ni) {
      const long long i = ti.i0 + tx;
      const double x = sp.base_x + 2.0 * (sp.rhs_x * double(i));
#pragma unroll 1
      for (int r = 0; r < kRaysPerThread; r++) {
        int jj = ty + r * (kShootThreads / kTileX);
        if (jj >= ti.nj) break;
        const long long j = ti.j0 + jj;
        const double y = sp.base_y + 2.0 * (sp.rhs_y * double(j));
        // near field: sum m / (z - z_i)
        double ar = 0.0, ai = 0.0, dr = 0.0, di = 0.0;
        for (int s = 0; s < nn; s++) {
          double4 st = s_near[s];
          double ex = x - st.x, ey = y - st.y;
          double inv = 1.0 / (ex * ex + ey * ey);
          double q = st.z * inv;
          ar += q * ex;
          ai -= q * ey;
          if (PAR) {  // m / (z - z_i)^2 = m conj(d)^2 / |d|^4
            double t2 = q * inv;
            dr += t2 * (ex * ex - ey * ey);
            di -= t2 * (2.0 * ex * ey);
          }
        }
        cplx<double> a_star = mk(ar * sp.theta2, -(ai * sp.theta2));
        // far field: Horner in dz = (z - c) / hl
        cplx<double> dz = mk((x - lcx) / lhl, (y - lcy) / lhl);
        cplx<double> A = mk(0.0, 0.0), Ad = mk(0.0, 0.0);
        for (int k = sp.p; k >= 1; k--) {
          if (PAR && k >= 2) {
            Ad = cmul(Ad, dz);
            double2 c = s_coef[k - 1];
            Ad = cadd(Ad, mk(c.x * (k - 1), c.y * (k - 1)));
          }
          A = cmul(A, dz);
          double2 c = s_coef[k - 1];
          A = cadd(A, mk(c.x, c.y));
        }
        A = cscale(A, sp.theta2);
        A = cdivr(A, lhl);
        cplx<double> a_local = cconj(A);
        cplx<double> z = mk(x, y);
        cplx<double> a_sm = alpha_smooth_(z, sp.kstar, sp.rect, corner, sp.approx, sp.taylor_smooth, sp.inv_pi);
        cplx<double> w = cadd(cscale(z, 1.0 - sp.kappa), cscale(cconj(z), sp.gamma));
        w = csub(csub(csub(w, a_star), a_local), a_sm);
        if (VERT) {
          w.re -= sp.cy_re;
          w.im -= sp.cy_im;
          double px = (w.re + sp.hly_re) * sp.npx / (2.0 * sp.hly_re);
          double py = (w.im + sp.hly_im) * sp.npy / (2.0 * sp.hly_im);
          verts[(size_t)(j - sp.jbase) * (sp.nx) + i] = make_double2(px, double(sp.npy) - py);
        } else {
          if (isnan(w.re) || isnan(w.im)) continue;
          w.re -= sp.cy_re;
          w.im -= sp.cy_im;
          if (w.re < -sp.hly_re || w.re > sp.hly_re || w.im < -sp.hly_im || w.im > sp.hly_im) continue;
          double px = (w.re + sp.hly_re) * sp.npx / (2.0 * sp.hly_re);
          double py = (w.im + sp.hly_im) * sp.npy / (2.0 * sp.hly_im);
          bool pmin_ = false;
          if (PAR) {
            // mu = 1 / ((dw/dz)^2 - |dw/dzbar|^2)   (irs_functions.cuh:66-81)
            cplx<double> dstar = mk(-(dr * sp.theta2), (di * sp.theta2));  // -theta^2 conj(sum m/d^2)
            Ad = cscale(Ad, sp.theta2);
            Ad = cdivr(Ad, lhl * lhl);
            cplx<double> dloc = cconj(Ad);
            double dsz = d_alpha_smooth_dz_(z, sp.kstar, sp.rect, corner, sp.approx);
            cplx<double> dszb =
                d_alpha_smooth_dzbar_(z, sp.kstar, sp.rect, corner, sp.approx, sp.taylor_smooth, sp.inv_pi);
            double dwdz = (1.0 - sp.kappa) - dsz;
            cplx<double> dwdzb = csub(csub(csub(mk(sp.gamma, 0.0), dstar), dloc), dszb);
            double a = cabs_(dwdzb);
            double mu = 1.0 / (dwdz * dwdz - a * a);
            pmin_ = mu >= 0;
          }
          irs_deposit(px, py, sp.npx, sp.npy, pix, pmin, psad, pmin_, PAR);
        }
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- FP32 form
// Near-field sums and far-field Horner values of R lattice points sharing the
// column offset ux (rows uy[0..R-1], R even), on pairs of points: the same
// operations in the same order as the scalar form of shoot_f32_tile, so the
// results are the same bits. fmaf(-Ai, dzi, c) is written fma(Ai, -dzi, c),
// the same product.
template <int R>
__device__ __forceinline__ void near_far_pairs(float ux, const float* uy, float inv_hl, int nn4, int p,
                                               const NearPairs& sp2, float* sx, float* sy, float* cxr, float* cyr,
                                               float* Ar, float* Ai) {
  constexpr int P = R / 2;
  const f32x2 zero = pk2(0.f, 0.f), ux2 = pk2(ux, ux);
  f32x2 uy2[P], Sx[P], Sy[P], Cx[P], Cy[P];
#pragma unroll
  for (int q = 0; q < P; q++) {
    uy2[q] = pk2(uy[2 * q], uy[2 * q + 1]);
    Sx[q] = Sy[q] = Cx[q] = Cy[q] = zero;
  }
  auto star = [&](int s, f32x2* bx, f32x2* by) {
    const ulonglong2 xy = sp2.xy[s];
    const f32x2 xx{xy.x}, yy{xy.y}, mm{sp2.m[s]};
    const f32x2 ex = sub2(ux2, xx), ex2 = mul2(ex, ex);
#pragma unroll
    for (int q = 0; q < P; q++) {
      const f32x2 ey = sub2(uy2[q], yy);
      const f32x2 r2 = fma2(ey, ey, ex2);
      float r2a, r2b;
      upk2(r2, r2a, r2b);
      const f32x2 w = mul2(mm, pk2(rcp_approx(r2a), rcp_approx(r2b)));
      bx[q] = fma2(w, ex, bx[q]);
      by[q] = fma2(w, ey, by[q]);
    }
  };
  for (int s0 = 0; s0 < nn4; s0 += 16) {
    f32x2 bx[P], by[P];
#pragma unroll
    for (int q = 0; q < P; q++) bx[q] = by[q] = zero;
#pragma unroll
    for (int s = 0; s < 4; s++) star(s0 + s, bx, by);
#pragma unroll
    for (int g = 1; g < 4; g++) {
      if (s0 + 4 * (g + 1) <= nn4) {
#pragma unroll
        for (int s = 0; s < 4; s++) star(s0 + 4 * g + s, bx, by);
      }
    }
#pragma unroll
    for (int q = 0; q < P; q++) {  // two-sum of the block into the running sum
      f32x2 t = add2(Sx[q], bx[q]);
      f32x2 bb = sub2(t, Sx[q]);
      Cx[q] = add2(Cx[q], add2(sub2(Sx[q], sub2(t, bb)), sub2(bx[q], bb)));
      Sx[q] = t;
      t = add2(Sy[q], by[q]);
      bb = sub2(t, Sy[q]);
      Cy[q] = add2(Cy[q], add2(sub2(Sy[q], sub2(t, bb)), sub2(by[q], bb)));
      Sy[q] = t;
    }
  }
  const float dzr = ux * inv_hl;
  const f32x2 dzr2 = pk2(dzr, dzr);
  f32x2 dzi2[P], ndzi2[P], A[P], B[P];
#pragma unroll
  for (int q = 0; q < P; q++) {
    const float a = uy[2 * q] * inv_hl, b = uy[2 * q + 1] * inv_hl;
    dzi2[q] = pk2(a, b);
    ndzi2[q] = pk2(-a, -b);
    A[q] = B[q] = zero;
  }
  for (int k = p - 1; k >= 0; k--) {
    const ulonglong2 c = sp2.coef[k];
    const f32x2 cr{c.x}, ci{c.y};
#pragma unroll
    for (int q = 0; q < P; q++) {
      const f32x2 ar = fma2(A[q], dzr2, fma2(B[q], ndzi2[q], cr));
      B[q] = fma2(A[q], dzi2[q], fma2(B[q], dzr2, ci));
      A[q] = ar;
    }
  }
#pragma unroll
  for (int q = 0; q < P; q++) {
    upk2(Sx[q], sx[2 * q], sx[2 * q + 1]);
    upk2(Sy[q], sy[2 * q], sy[2 * q + 1]);
    upk2(Cx[q], cxr[2 * q], cxr[2 * q + 1]);
    upk2(Cy[q], cyr[2 * q], cyr[2 * q + 1]);
    upk2(A[q], Ar[2 * q], Ar[2 * q + 1]);
    upk2(B[q], Ai[2 * q], Ai[2 * q + 1]);
  }
}

// GENERIC_SMOOTH: the smooth sheet is not the circular approximation
// (alpha_smooth = -kappa_star z); its deviation from that linear form is then
// added per point in FP64.
template <bool VERT, bool PAR, bool GENERIC_SMOOTH, int THREADS = kShootThreads>
__device__ __forceinline__ void shoot_f32_tile(const ShootParams& sp, const LeafPtrs& lp, const TileInfo& ti,
                                               const ShootOut& o, float4* s_near, float2* s_coef,
                                               NearPairs* s_pair) {
  static_assert(THREADS >= 128 && THREADS <= 1024 && kTileY % (THREADS / kTileX) == 0, "tile shape");
  constexpr int R = kTileY / (THREADS / kTileX);  // lattice points per thread
  constexpr int RS = THREADS / kTileX;            // row stride between a thread's points
  const int tx = threadIdx.x & (kTileX - 1), ty = threadIdx.x / kTileX;
  const cplx<double> corner = mk(sp.corner_re, sp.corner_im);
  // linear part of the lens equation for the circular approximation
  const double lin_x = 1.0 - sp.kappa + sp.kstar + sp.gamma;
  const double lin_y = 1.0 - sp.kappa + sp.kstar - sp.gamma;
  const float flin_x = float(lin_x), flin_y = float(lin_y);
  const double scx = sp.npx / (2.0 * sp.hly_re), scy = sp.npy / (2.0 * sp.hly_im);
  {
    const int nn = lp.nnear[ti.leaf];
    if (threadIdx.x < kMaxStarsDirect) {
      float4 v = lp.near32[(size_t)ti.leaf * kMaxStarsDirect + threadIdx.x];
      if (threadIdx.x >= nn) v = make_float4(1e18f, 1e18f, 0.f, 0.f);  // far away, zero mass
      s_near[threadIdx.x] = v;
      s_pair->xy[threadIdx.x] = make_ulonglong2(pk2(v.x, v.x).v, pk2(v.y, v.y).v);
      s_pair->m[threadIdx.x] = pk2(v.z, v.z).v;
    }
    if (threadIdx.x >= 64 && threadIdx.x < 64 + kMaxOrder) {
      const float2 c = lp.coef32[(size_t)ti.leaf * kMaxOrder + threadIdx.x - 64];
      s_coef[threadIdx.x - 64] = c;
      s_pair->coef[threadIdx.x - 64] = make_ulonglong2(pk2(c.x, c.x).v, pk2(c.y, c.y).v);
    }
    const double lcx = lp.cx[ti.leaf], lcy = lp.cy[ti.leaf];
    const float inv_hl = float(1.0 / lp.hl[ti.leaf]);
    // leaf-centre part of the source position, in pixel units
    double pcx = ((lin_x * lcx - sp.cy_re) + sp.hly_re) * scx;
    double pcy = ((lin_y * lcy - sp.cy_im) + sp.hly_im) * scy;
    if (lp.smooth0) {  // the folded smooth sheet's value at the leaf centre
      const double2 d0 = lp.smooth0[ti.leaf];
      pcx -= d0.x * scx;
      pcy -= d0.y * scy;
    }
    __syncthreads();
    const int nn4 = (nn + 3) & ~3;
    if (tx < ti.ni) {
      const long long i = ti.i0 + tx;
      const double xg = sp.base_x + 2.0 * (sp.rhs_x * double(i));
      const float ux = float(xg - lcx);
      const long long j0 = ti.j0 + ty;
      float uy[R];
#pragma unroll
      for (int r = 0; r < R; r++)  // each row from its own index: independent of the tiling
        uy[r] = float((sp.base_y + 2.0 * (sp.rhs_y * double(j0 + r * RS))) - lcy);
      float sx[R], sy[R], cxr[R], cyr[R];
      float dxx[R], dxy[R];  // derivative sums (parity only)
      float Ar[R], Ai[R], Dr[R], Di[R];
      if constexpr (!PAR && R % 2 == 0) {
        // the same operations on pairs of points (rows r, r + 1)
        near_far_pairs<R>(ux, uy, inv_hl, nn4, sp.p, *s_pair, sx, sy, cxr, cyr, Ar, Ai);
      } else {
        // ---- near field, blocked compensated summation
#pragma unroll
        for (int r = 0; r < R; r++) sx[r] = sy[r] = cxr[r] = cyr[r] = dxx[r] = dxy[r] = 0.f;
        // blocks of 16 stars (the last one of 4, 8 or 12 when nn4 is not a
        // multiple of 16), each block's sum added to the running sum by a
        // two-sum; a thread's points share ux, so ex and ex^2 are formed once
        // per star
        auto star = [&](const float4 st, float* bx, float* by) {
          const float ex = ux - st.x, ex2 = ex * ex;
#pragma unroll
          for (int r = 0; r < R; r++) {
            float ey = uy[r] - st.y;
            float r2 = fmaf(ey, ey, ex2);
            float inv = rcp_approx(r2);
            float q = st.z * inv;
            bx[r] = fmaf(q, ex, bx[r]);
            by[r] = fmaf(q, ey, by[r]);
            if (PAR) {
              float t2 = q * inv;
              dxx[r] = fmaf(t2, (ex - ey) * (ex + ey), dxx[r]);
              dxy[r] = fmaf(t2, 2.f * ex * ey, dxy[r]);
            }
          }
        };
        for (int s0 = 0; s0 < nn4; s0 += 16) {
          float bx[R], by[R];
#pragma unroll
          for (int r = 0; r < R; r++) bx[r] = by[r] = 0.f;
#pragma unroll
          for (int s = 0; s < 4; s++) star(s_near[s0 + s], bx, by);
#pragma unroll
          for (int g = 1; g < 4; g++) {
            if (s0 + 4 * (g + 1) <= nn4) {
#pragma unroll
              for (int s = 0; s < 4; s++) star(s_near[s0 + 4 * g + s], bx, by);
            }
          }
#pragma unroll
          for (int r = 0; r < R; r++) {  // two-sum of the block into the running sum
            float s = sx[r] + bx[r];
            float bb = s - sx[r];
            cxr[r] += (sx[r] - (s - bb)) + (bx[r] - bb);
            sx[r] = s;
            s = sy[r] + by[r];
            bb = s - sy[r];
            cyr[r] += (sy[r] - (s - bb)) + (by[r] - bb);
            sy[r] = s;
          }
        }
        // ---- far field: Horner in dz = u / hl, one coefficient read per 4 points
        float dzr[R], dzi[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
          dzr[r] = ux * inv_hl;
          dzi[r] = uy[r] * inv_hl;
          Ar[r] = Ai[r] = Dr[r] = Di[r] = 0.f;
        }
        for (int k = sp.p - 1; k >= 0; k--) {
          const float2 c = s_coef[k];
#pragma unroll
          for (int r = 0; r < R; r++) {
            if (PAR && k >= 1) {  // derivative polynomial sum k e_k dz^(k-1)
              float tr = fmaf(Dr[r], dzr[r], -Di[r] * dzi[r]);
              float tt = fmaf(Dr[r], dzi[r], Di[r] * dzr[r]);
              Dr[r] = fmaf(c.x, float(k), tr);
              Di[r] = fmaf(c.y, float(k), tt);
            }
            // A <- A dz + c as two FMA chains (4 operations per order)
            const float ar = fmaf(Ar[r], dzr[r], fmaf(-Ai[r], dzi[r], c.x));
            Ai[r] = fmaf(Ar[r], dzi[r], fmaf(Ai[r], dzr[r], c.y));
            Ar[r] = ar;
          }
        }
      }
      // ---- output
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int jj = ty + r * RS;
        if (jj >= ti.nj) break;
        const long long j = ti.j0 + jj;
        const float Sx = sx[r] + cxr[r], Sy = sy[r] + cyr[r];
        // w - w(centre) = lin * u - alpha_star - conj(A)
        const float wr = fmaf(flin_x, ux, -(Sx + Ar[r]));
        const float wi = fmaf(flin_y, uy[r], -(Sy - Ai[r]));
        double px = pcx + double(wr) * scx;
        double py = pcy + double(wi) * scy;
        if (GENERIC_SMOOTH) {
          cplx<double> z = mk(lcx + double(ux), lcy + double(uy[r]));
          cplx<double> a_sm = alpha_smooth_(z, sp.kstar, sp.rect, corner, sp.approx, sp.taylor_smooth, sp.inv_pi);
          px += (-a_sm.re - sp.kstar * z.re) * scx;
          py += (-a_sm.im - sp.kstar * z.im) * scy;
        }
        if (VERT) {
          if (o.tiles)
            tile_store(*o.tiles, i, j, make_double2(px, double(sp.npy) - py));
          else
            o.verts[(size_t)(j - o.vrow0) * (sp.nx) + i] = make_double2(px, double(sp.npy) - py);
        } else {
          if (!(px >= 0.0 && px <= double(sp.npx) && py >= 0.0 && py <= double(sp.npy))) continue;
          bool pmin_ = false;
          if (PAR) {
            cplx<double> z = mk(lcx + double(ux), lcy + double(uy[r]));
            double dsz = d_alpha_smooth_dz_(z, sp.kstar, sp.rect, corner, sp.approx);
            cplx<double> dszb =
                GENERIC_SMOOTH
                    ? d_alpha_smooth_dzbar_(z, sp.kstar, sp.rect, corner, sp.approx, sp.taylor_smooth, sp.inv_pi)
                    : mk(0.0, 0.0);
            // d alpha_star / d zbar = -conj(sum m theta^2 / d^2) ; sum m/d^2 = sum q conj(d)^2/|d|^2
            double dsr = -double(dxx[r]), dsi = -double(dxy[r]);
            // d alpha_local / d zbar = conj(A'(dz)) / hl
            double dlr = double(Dr[r]) * double(inv_hl), dli = -double(Di[r]) * double(inv_hl);
            double dwdz = (1.0 - sp.kappa) - dsz;
            double gr = sp.gamma - dsr - dlr - dszb.re, gi = -dsi - dli - dszb.im;
            double mu = 1.0 / (dwdz * dwdz - (gr * gr + gi * gi));
            pmin_ = mu >= 0;
          }
          irs_deposit(px, py, sp.npx, sp.npy, o.pix, o.pmin, o.psad, pmin_, PAR);
        }
      }
    }
    __syncthreads();
  }
}

// THREADS per CTA sets the lattice points per thread, kTileY / (THREADS / 32):
// 8 at 128 threads, 4 at 256, 2 at 512 (a choice of the autotuner).
template <bool VERT, bool PAR, bool GENERIC_SMOOTH, int THREADS = kShootThreads>
__global__ void __launch_bounds__(THREADS) shoot_f32(ShootParams sp, LeafPtrs lp, long long total_tiles,
                                                     int* __restrict__ pix, int* __restrict__ pmin,
                                                     int* __restrict__ psad, double2* __restrict__ verts) {
  __shared__ float4 s_near[kMaxStarsDirect];
  __shared__ float2 s_coef[kMaxOrder];
  __shared__ NearPairs s_pair;
  const ShootOut o{pix, pmin, psad, verts, sp.jbase};
  for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x)
    shoot_f32_tile<VERT, PAR, GENERIC_SMOOTH, THREADS>(sp, lp, tile_info(lp, t), o, s_near, s_coef, &s_pair);
}

// The level-s corner lattice restricted to refined tiles: work items whose
// 32 x 32 block touches no tile with a buffer slot are skipped.
template <bool GENERIC_SMOOTH>
__global__ void __launch_bounds__(kShootThreads) shoot_f32_tiles(ShootParams sp, LeafPtrs lp, long long total_tiles,
                                                                 TileStore st) {
  __shared__ float4 s_near[kMaxStarsDirect];
  __shared__ float2 s_coef[kMaxOrder];
  __shared__ NearPairs s_pair;
  const ShootOut o{nullptr, nullptr, nullptr, nullptr, 0, &st};
  const long long side = 32LL * st.s;
  for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    const TileInfo ti = tile_info(lp, t);
    const int tx0 = int(ti.i0 / side), tx1 = int((ti.i0 + ti.ni - 1) / side);
    const int ty0 = int(ti.j0 / side), ty1 = int((ti.j0 + ti.nj - 1) / side);
    bool need = false;  // uniform over the block
    for (int ty = ty0 > 0 ? ty0 - 1 : 0; ty <= ty1 && ty < st.nty && !need; ty++)
      for (int tx = tx0 > 0 ? tx0 - 1 : 0; tx <= tx1 && tx < st.ntx && !need; tx++)
        need = st.slot[ty * st.ntx + tx] >= 0;
    if (!need) continue;
    shoot_f32_tile<true, false, GENERIC_SMOOTH>(sp, lp, ti, o, s_near, s_coef, &s_pair);
  }
}

// Many realizations in one launch: the tiles of all their leaves form one work
// list; each tile takes the lens parameters of its leaf's realization and
// writes into that realization's part of the corner buffer.
struct BatchShoot {
  const ShootParams* sps;    // per realization
  const int* leaf_rid;       // per leaf
  const long long* vrow0;    // per realization: first corner row held in the buffer
  const long long* voff;     // per realization: offset of its rows in the buffer
  const long long* total;    // number of tiles (device)
  long long table_cap;       // entries the tile table holds
  const int* err;            // error bits; a table overflow leaves the table unusable
};

// threads per CTA of the batched lens pass: 8 lattice points per thread, the
// fastest single-map shape (with a grid of 64 CTAs per SM)
constexpr int kShootBatchThreads = 128;

template <bool GENERIC_SMOOTH>
__global__ void __launch_bounds__(kShootBatchThreads) shoot_f32_batch(BatchShoot bs, LeafPtrs lp,
                                                                 double2* __restrict__ verts) {
  __shared__ float4 s_near[kMaxStarsDirect];
  __shared__ float2 s_coef[kMaxOrder];
  __shared__ NearPairs s_pair;
  if (*bs.err & kErrTableOverflow) return;
  const long long total = *bs.total < bs.table_cap ? *bs.total : bs.table_cap;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const TileInfo ti = tile_info(lp, t);
    const int r = bs.leaf_rid[ti.leaf];
    const ShootOut o{nullptr, nullptr, nullptr, verts + bs.voff[r], bs.vrow0[r]};
    shoot_f32_tile<true, false, GENERIC_SMOOTH, kShootBatchThreads>(bs.sps[r], lp, ti, o, s_near, s_coef, &s_pair);
  }
}

}  // namespace irsb
