// Adaptive IPM: per-tile subdivision of the lens-plane cell lattice.
//
// The cell lattice of a map (num_rays_y cells per unlensed pixel area) is cut
// into tiles of kAdaTile x kAdaTile cells. A tile at level s (1, 2, 4, 8, 16)
// splits each of its cells into s x s subcells: its corner lattice has
// kAdaTile * s + 1 points per side at spacing 2 * rhs / s, and each subcell
// deposits factor / s^2 through the same fixed-point deposition as the
// uniform lattice. Level 16 everywhere is the uniform-fine map; level 1
// everywhere is the plain map.
//
// Corner positions of a refined tile:
//   * points of the base lattice are taken from the base corner buffer (the
//     tiled lens-equation pass), so tiles of every level share them exactly;
//   * points on an edge shared with a coarser neighbour (level s' < s) are
//     placed on the straight segment between that neighbour's corners, so the
//     refined lattice is conforming (no gaps or overlaps between tiles);
//   * other points are evaluated one by one: descent of the quadtree to the
//     leaf that owns the point (the boxes that partition the lattice for the
//     tiled pass), then the FP32 leaf-relative lens equation of shoot_f32
//     (compensated near-field sum, FP32 Horner of FP64-built coefficients,
//     FP64 conversion to pixels). A point's position depends only on its
//     global fine index, so neighbouring tiles compute shared points
//     identically.
//
// Labels for training: a tile's label is the smallest level s whose deposit
// differs from the tile's level-16 deposit by at most eps (ada_window_errors:
// a share of the tile's own flux, or of the map's flux where it lands), 16
// when no coarser level does: the level at which the tile's deposit
// converges to the uniform-fine map.
#pragma once
#include "deposit.cuh"
#include "leaves.cuh"
#include "shoot.cuh"
#include "tree.cuh"

namespace irsb {

constexpr int kAdaTile = 32;         // cells per tile side
constexpr int kAdaMaxLevel = 16;     // finest subdivision
constexpr int kAdaLevels = 5;        // 1, 2, 4, 8, 16
constexpr int kAdaFeatures = 8;

__host__ __device__ __forceinline__ int ada_level_of(int cls) { return 1 << cls; }
__host__ __device__ __forceinline__ long long llmin_(long long a, long long b) { return a < b ? a : b; }

// A leaf's near stars and local coefficients (FP32 records), in global
// memory or staged in shared memory.
// With the constants of the lens equation at the leaf (those of shoot_f32:
// linear terms, pixel scales, the leaf centre's source position), computed
// once per view.
struct LeafView {
  const float4* near;
  const float2* coef;
  int nn;
  double cx, cy;
  float inv_hl;
  double lin_x, lin_y, scx, scy, pcx, pcy;
};

__device__ __forceinline__ LeafView make_leaf_view(const ShootParams& sp, const float4* near, const float2* coef,
                                                   int nn, double cx, double cy, double hl,
                                                   double2 smooth0 = make_double2(0.0, 0.0)) {
  LeafView L;
  L.near = near;
  L.coef = coef;
  L.nn = nn;
  L.cx = cx;
  L.cy = cy;
  L.inv_hl = float(1.0 / hl);
  L.lin_x = 1.0 - sp.kappa + sp.kstar + sp.gamma;
  L.lin_y = 1.0 - sp.kappa + sp.kstar - sp.gamma;
  L.scx = sp.npx / (2.0 * sp.hly_re);
  L.scy = sp.npy / (2.0 * sp.hly_im);
  L.pcx = ((L.lin_x * cx - sp.cy_re) + sp.hly_re) * L.scx;
  L.pcy = ((L.lin_y * cy - sp.cy_im) + sp.hly_im) * L.scy;
  L.pcx -= smooth0.x * L.scx;  // a folded smooth sheet's value at the leaf centre (else 0)
  L.pcy -= smooth0.y * L.scy;
  return L;
}

__device__ __forceinline__ LeafView leaf_view(const ShootParams& sp, const LeafPtrs& lp, int leaf) {
  return make_leaf_view(sp, lp.near32 + (size_t)leaf * kMaxStarsDirect, lp.coef32 + (size_t)leaf * kMaxOrder,
                        lp.nnear[leaf], lp.cx[leaf], lp.cy[leaf], lp.hl[leaf],
                        lp.smooth0 ? lp.smooth0[leaf] : make_double2(0.0, 0.0));
}

// Source position (pixel units, row axis flipped) of the lattice point (x, y)
// evaluated with leaf L: the arithmetic of shoot_f32 for one point, so a
// base lattice point gets the same position from either kernel.
template <bool GENERIC_SMOOTH>
__device__ __forceinline__ double2 eval_point_f32(const ShootParams& sp, const LeafView& L, double x, double y) {
  const double lcx = L.cx, lcy = L.cy;
  const float inv_hl = L.inv_hl;
  const double lin_x = L.lin_x, lin_y = L.lin_y, scx = L.scx, scy = L.scy, pcx = L.pcx, pcy = L.pcy;
  const float ux = float(x - lcx), uy = float(y - lcy);
  const int nn = L.nn;
  const float4* near = L.near;
  float sx = 0.f, sy = 0.f, cxr = 0.f, cyr = 0.f;
  for (int s0 = 0; s0 < nn; s0 += 16) {
    float bx = 0.f, by = 0.f;
    for (int s = s0; s < s0 + 16 && s < nn; s++) {
      const float4 st = near[s];
      const float ex = ux - st.x, ey = uy - st.y;
      const float r2 = fmaf(ey, ey, ex * ex);
      const float q = st.z * rcp_approx(r2);
      bx = fmaf(q, ex, bx);
      by = fmaf(q, ey, by);
    }
    float t = sx + bx, bb = t - sx;
    cxr += (sx - (t - bb)) + (bx - bb);
    sx = t;
    t = sy + by;
    bb = t - sy;
    cyr += (sy - (t - bb)) + (by - bb);
    sy = t;
  }
  const float2* coef = L.coef;
  const float dzr = ux * inv_hl, dzi = uy * inv_hl;
  float Ar = 0.f, Ai = 0.f;
  for (int k = sp.p - 1; k >= 0; k--) {
    const float2 c = coef[k];
    const float ar = fmaf(Ar, dzr, fmaf(-Ai, dzi, c.x));  // as shoot_f32
    Ai = fmaf(Ar, dzi, fmaf(Ai, dzr, c.y));
    Ar = ar;
  }
  const float Sx = sx + cxr, Sy = sy + cyr;
  const float wr = fmaf(float(lin_x), ux, -(Sx + Ar));
  const float wi = fmaf(float(lin_y), uy, -(Sy - Ai));
  double px = pcx + double(wr) * scx;
  double py = pcy + double(wi) * scy;
  if (GENERIC_SMOOTH) {
    const cplx<double> corner = mk(sp.corner_re, sp.corner_im);
    const cplx<double> z = mk(lcx + double(ux), lcy + double(uy));
    const cplx<double> a_sm = alpha_smooth_(z, sp.kstar, sp.rect, corner, sp.approx, sp.taylor_smooth, sp.inv_pi);
    px += (-a_sm.re - sp.kstar * z.re) * scx;
    py += (-a_sm.im - sp.kstar * z.im) * scy;
  }
  return make_double2(px, double(sp.npy) - py);
}

// Lattice coordinate of global fine index F (16 fine steps per base cell):
// base points (F multiple of 16) reproduce the base lattice formula exactly.
__device__ __forceinline__ double fine_coord(double base, double rhs, long long F) {
  return base + 2.0 * (rhs * (double(F) * (1.0 / kAdaMaxLevel)));
}

// Geometry of the adaptive pass of one map.
struct AdaGeom {
  double base_x, base_y, rhs_x, rhs_y;  // corner lattice (cell corners)
  long long ncx, ncy;                   // cells of the base lattice
  int ntx, nty;                         // tiles
  int npx, npy;                         // map
};

// Corner (a, b) of tile t at level s, in the tile's corner grid
// [0, ncell_x * s] x [0, ncell_y * s].
// `stage`: the records of the tile's own leaf in shared memory, when the tile
// has one (the values are those of the leaf in global memory).
template <typename T, bool GENERIC_SMOOTH>
__device__ __forceinline__ double2 tile_corner(const AdaGeom& g, const ShootParams& sp, const LeafPtrs& lp,
                                               const DescentPtrs<T>& dp, const double2* __restrict__ base_verts,
                                               int tx, int ty, int s, int a, int b,
                                               const LeafView* stage = nullptr) {
  const long long i0 = (long long)tx * kAdaTile, j0 = (long long)ty * kAdaTile;
  const int sh = __ffs(s) - 1;  // levels are powers of two
  if (((a | b) & (s - 1)) == 0) {
    const long long i = i0 + (a >> sh), j = j0 + (b >> sh);
    return base_verts[j * (g.ncx + 1) + i];
  }
  const long long F = (i0 * kAdaMaxLevel) + (long long)a * (kAdaMaxLevel >> sh);
  const long long G = (j0 * kAdaMaxLevel) + (long long)b * (kAdaMaxLevel >> sh);
  const double x = fine_coord(g.base_x, g.rhs_x, F), y = fine_coord(g.base_y, g.rhs_y, G);
  const int own = dp.tile_leaf ? dp.tile_leaf[ty * g.ntx + tx] : -1;  // the descent's answer, when uniform
  if (own >= 0 && stage) return eval_point_f32<GENERIC_SMOOTH>(sp, *stage, x, y);
  return eval_point_f32<GENERIC_SMOOTH>(sp, leaf_view(sp, lp, own >= 0 ? own : descend_leaf(dp, x, y)), x, y);
}

// Corner (a, b) of refined tile t (level s, corner grid wa x hb): points on an
// edge shared with a coarser neighbour (tile_level, per tile) are placed on
// that neighbour's edge segment; without tile_level every point is evaluated.
template <typename T, bool GENERIC_SMOOTH>
__device__ __forceinline__ double2 refine_point(const AdaGeom& g, const ShootParams& sp, const LeafPtrs& lp,
                                                const DescentPtrs<T>& dp, const double2* __restrict__ base_verts,
                                                const int* __restrict__ tile_level, int t, int tx, int ty, int s,
                                                int a, int b, int wa, int hb, const LeafView* stage) {
  // neighbour across the edge this point lies on (a point on two edges is a
  // tile corner, hence a base point)
  int nlev = s;
  bool along_b = false;  // the edge runs along b (left / right edge)
  if (!tile_level) {
    // isolated tiles (labels, audit): every point evaluated
  } else if (a == 0 && tx > 0) {
    nlev = tile_level[t - 1];
    along_b = true;
  } else if (a == wa && tx + 1 < g.ntx && wa == kAdaTile * s) {
    nlev = tile_level[t + 1];
    along_b = true;
  } else if (b == 0 && ty > 0) {
    nlev = tile_level[t - g.ntx];
  } else if (b == hb && ty + 1 < g.nty && hb == kAdaTile * s) {
    nlev = tile_level[t + g.ntx];
  }
  if (nlev < s && ((a | b) & (s - 1)) != 0) {  // levels are powers of two
    const int step = s >> (__ffs(nlev) - 1);
    const int u = along_b ? b : a;
    const int u0 = u & ~(step - 1), u1 = u0 + step;
    const double2 p0 = along_b ? tile_corner<T, GENERIC_SMOOTH>(g, sp, lp, dp, base_verts, tx, ty, s, a, u0, stage)
                               : tile_corner<T, GENERIC_SMOOTH>(g, sp, lp, dp, base_verts, tx, ty, s, u0, b, stage);
    const double2 p1 = along_b ? tile_corner<T, GENERIC_SMOOTH>(g, sp, lp, dp, base_verts, tx, ty, s, a, u1, stage)
                               : tile_corner<T, GENERIC_SMOOTH>(g, sp, lp, dp, base_verts, tx, ty, s, u1, b, stage);
    const double f = double(u - u0) / double(step);
    return make_double2(p0.x + (p1.x - p0.x) * f, p0.y + (p1.y - p0.y) * f);
  }
  return tile_corner<T, GENERIC_SMOOTH>(g, sp, lp, dp, base_verts, tx, ty, s, a, b, stage);
}

// Refined corner grids of the tiles in `list` (all at level s), written at
// out + slot * stride with row stride ncell_x * s + 1; one CTA per band of
// kAdaBandRows corner rows of a tile (refine_point for each corner). When
// every point of the tile belongs to one leaf (DescentPtrs::tile_leaf), its
// near stars and local coefficients are staged in shared memory and the
// band's corners read them as broadcasts; the other tiles take the descent
// per point.
constexpr int kAdaBandRows = 16;
__host__ __device__ __forceinline__ long long ada_band_items(long long ntiles, int s) {
  return ntiles * ((kAdaTile * s + 1 + kAdaBandRows - 1) / kAdaBandRows);
}
template <typename T, bool GENERIC_SMOOTH>
__global__ void __launch_bounds__(256) ada_refine_tiles(AdaGeom g, ShootParams sp, LeafPtrs lp, DescentPtrs<T> dp,
                                                        const double2* __restrict__ base_verts,
                                                        const int* __restrict__ tile_level,
                                                        const int* __restrict__ list, int nlist, int s,
                                                        long long stride, double2* __restrict__ out) {
  __shared__ float4 s_near[kMaxStarsDirect];
  __shared__ float2 s_coef[kMaxOrder];
  __shared__ LeafView s_view;
  const int nbands = (kAdaTile * s + 1 + kAdaBandRows - 1) / kAdaBandRows;
  for (long long item = blockIdx.x; item < (long long)nlist * nbands; item += gridDim.x) {
    const int slot = int(item / nbands), band = int(item - (long long)slot * nbands);
    const int t = list[slot];
    const int leaf = dp.tile_leaf ? dp.tile_leaf[t] : -1;  // CTA-uniform
    if (leaf >= 0) {
      if (threadIdx.x < kMaxStarsDirect) s_near[threadIdx.x] = lp.near32[(size_t)leaf * kMaxStarsDirect + threadIdx.x];
      if (threadIdx.x >= 64 && threadIdx.x < 64 + kMaxOrder)
        s_coef[threadIdx.x - 64] = lp.coef32[(size_t)leaf * kMaxOrder + threadIdx.x - 64];
      if (threadIdx.x == 0)
        s_view = make_leaf_view(sp, s_near, s_coef, lp.nnear[leaf], lp.cx[leaf], lp.cy[leaf], lp.hl[leaf],
                                lp.smooth0 ? lp.smooth0[leaf] : make_double2(0.0, 0.0));
    }
    __syncthreads();
    const LeafView* stage = leaf >= 0 ? &s_view : nullptr;
    const int tx = t % g.ntx, ty = t / g.ntx;
    const int wa = int(llmin_(kAdaTile, g.ncx - (long long)tx * kAdaTile)) * s;
    const int hb = int(llmin_(kAdaTile, g.ncy - (long long)ty * kAdaTile)) * s;
    const int w1 = wa + 1, b0 = band * kAdaBandRows, b1 = min(hb + 1, b0 + kAdaBandRows);
    double2* o = out + (long long)slot * stride;
    // corners (a, b) of the band in row-major order, thread k taking k, k + 256, ...
    int b = b0 + int(threadIdx.x) / w1, a = int(threadIdx.x) - (b - b0) * w1;
    while (b < b1) {
      o[(long long)b * w1 + a] =
          refine_point<T, GENERIC_SMOOTH>(g, sp, lp, dp, base_verts, tile_level, t, tx, ty, s, a, b, wa, hb, stage);
      a += blockDim.x;
      while (a >= w1) {
        a -= w1;
        b++;
      }
    }
    __syncthreads();  // the stage is rewritten for the next tile
  }
}

// After the tiled pass over the level-s lattice (shoot_f32_tiles): base points
// of the tiles in `list` take the base lattice's positions (so that every
// level shares them exactly), and points on an edge shared with a coarser
// neighbour move onto that neighbour's edge segment, between the tile's own
// positions at the neighbour's corners (the same lattice points the
// neighbour holds). One thread per corner; the points written (base points,
// edge points between coarse corners) and the points read (base points from
// the base lattice, coarse corners) are disjoint.
__global__ void __launch_bounds__(256) ada_fixup_corners(AdaGeom g, const double2* __restrict__ base_verts,
                                                         const int* __restrict__ tile_level,
                                                         const int* __restrict__ list, int nlist, int s,
                                                         long long stride, double2* __restrict__ out) {
  const int side = kAdaTile * s + 1;
  const long long per_tile = (long long)side * side;
  const long long total = per_tile * nlist;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int slot = int(q / per_tile);
    const int rem = int(q - (long long)slot * per_tile);
    const int b = rem / side, a = rem - b * side;
    const int t = list[slot];
    const int tx = t % g.ntx, ty = t / g.ntx;
    const int ncx_t = int(llmin_(kAdaTile, g.ncx - (long long)tx * kAdaTile));
    const int ncy_t = int(llmin_(kAdaTile, g.ncy - (long long)ty * kAdaTile));
    const int wa = ncx_t * s, hb = ncy_t * s;
    if (a > wa || b > hb) continue;
    double2* P = out + (long long)slot * stride;
    const long long W = wa + 1;
    const long long i0 = (long long)tx * kAdaTile, j0 = (long long)ty * kAdaTile;
    if (a % s == 0 && b % s == 0) {
      P[b * W + a] = base_verts[(j0 + b / s) * (g.ncx + 1) + i0 + a / s];
      continue;
    }
    int nlev = s;
    bool along_b = false;
    if (a == 0 && tx > 0) {
      nlev = tile_level[t - 1];
      along_b = true;
    } else if (a == wa && tx + 1 < g.ntx && wa == kAdaTile * s) {
      nlev = tile_level[t + 1];
      along_b = true;
    } else if (b == 0 && ty > 0) {
      nlev = tile_level[t - g.ntx];
    } else if (b == hb && ty + 1 < g.nty && hb == kAdaTile * s) {
      nlev = tile_level[t + g.ntx];
    }
    if (nlev >= s) continue;
    const int step = s / nlev;
    const int u = along_b ? b : a;
    if (u % step == 0) continue;
    const int u0 = (u / step) * step, u1 = u0 + step;
    auto at = [&](int aa, int bb) -> double2 {
      if (aa % s == 0 && bb % s == 0) return base_verts[(j0 + bb / s) * (g.ncx + 1) + i0 + aa / s];
      return P[bb * W + aa];
    };
    const double2 p0 = along_b ? at(a, u0) : at(u0, b);
    const double2 p1 = along_b ? at(a, u1) : at(u1, b);
    const double f = double(u - u0) / double(step);
    P[b * W + a] = make_double2(p0.x + (p1.x - p0.x) * f, p0.y + (p1.y - p0.y) * f);
  }
}

// slot[t] = position of tile t in list (ada_slots_set), -1 for the other
// tiles (ada_slots_clear).
__global__ void ada_slots_clear(int ntiles, int* __restrict__ slot) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) slot[t] = -1;
}
__global__ void ada_slots_set(const int* __restrict__ list, int nlist, int* __restrict__ slot) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nlist; k += gridDim.x * blockDim.x) slot[list[k]] = k;
}

// Deposit error of levels 1, 2, 4, 8 against level 16, tile by tile. Each
// tile is deposited on its own into a private pixel window at every level
// (level-s corners are every (16/s)-th level-16 corner), and
//   err[slot * 4 + c] = sum |W_c - W_16| / reference flux
// over the map pixels in the window, W_c being the tile's deposit at level 2^c
// (the reference is below).
constexpr int kAdaWindow = 256;       // pixels per side of a tile's window
constexpr int kAdaWindowLarge = 512;  // window of a chunk holding a tile whose image needs more
constexpr int kAdaWindowMargin = 2;
constexpr double kAdaMapWeight = 20.0;  // mode 2: weight of the map-relative error

// Window of each tile: the pixel bounding box of its level-16 image within the
// map, widened by kAdaWindowMargin; win[slot] = (x0, y0, w, h), w = 0 when the
// image misses the map. A box wider than the chunk's window is covered at a
// coarser pixel scale (ada_window_scale).
__global__ void __launch_bounds__(256) ada_tile_windows(AdaGeom g, const int* __restrict__ list, int nlist,
                                                        long long stride, const double2* __restrict__ fine,
                                                        int4* __restrict__ win) {
  __shared__ double red[4][8];
  for (int slot = blockIdx.x; slot < nlist; slot += gridDim.x) {
    const int t = list[slot];
    const int tx = t % g.ntx, ty = t / g.ntx;
    const int ncx_t = int(llmin_(kAdaTile, g.ncx - (long long)tx * kAdaTile));
    const int ncy_t = int(llmin_(kAdaTile, g.ncy - (long long)ty * kAdaTile));
    const int n = (ncx_t * kAdaMaxLevel + 1) * (ncy_t * kAdaMaxLevel + 1);
    const double2* P = fine + (long long)slot * stride;
    double m[4] = {1e300, 1e300, -1e300, -1e300};  // xmin, ymin, xmax, ymax
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
      const double2 v = P[q];
      if (!(fabs(v.x) < 1e12 && fabs(v.y) < 1e12)) continue;
      m[0] = fmin(m[0], v.x);
      m[1] = fmin(m[1], v.y);
      m[2] = fmax(m[2], v.x);
      m[3] = fmax(m[3], v.y);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
      double v = m[c];
      for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_down_sync(0xffffffffu, v, o);
        v = c < 2 ? fmin(v, u) : fmax(v, u);
      }
      if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double r[4] = {red[0][0], red[1][0], red[2][0], red[3][0]};
      for (int w = 1; w < int(blockDim.x >> 5); w++) {
        r[0] = fmin(r[0], red[0][w]);
        r[1] = fmin(r[1], red[1][w]);
        r[2] = fmax(r[2], red[2][w]);
        r[3] = fmax(r[3], red[3][w]);
      }
      const double x0 = fmax(floor(r[0]) - kAdaWindowMargin, 0.0), y0 = fmax(floor(r[1]) - kAdaWindowMargin, 0.0);
      const double x1 = fmin(ceil(r[2]) + kAdaWindowMargin, double(g.npx));
      const double y1 = fmin(ceil(r[3]) + kAdaWindowMargin, double(g.npy));
      int4 o = make_int4(0, 0, 0, 0);
      if (x1 > x0 && y1 > y0) o = make_int4(int(x0), int(y0), int(x1 - x0), int(y1 - y0));
      win[slot] = o;
    }
    __syncthreads();
  }
}

// Map pixels per window pixel for a tile's window (1 unless its image is
// wider than the window side ws).
__host__ __device__ __forceinline__ int ada_window_scale(int4 w, int ws) {
  const int m = w.z > w.w ? w.z : w.w;
  return m <= ws ? 1 : (m + ws - 1) / ws;
}

// Differences of the resolved windows of side ws (window of slot k, level c
// at acc + (k * 5 + c) * ws^2, placed at (win.x, win.y) on the map): the flux
// the tile puts in other map pixels at level 2^c than at level 16, as a share
// of
//   mode 0: the tile's whole flux (2 factor per cell): its own relative error,
//           which the map inherits where the errors of overlapping tiles have
//           the same sign (the bias of the triangle approximation);
//   mode 1: the flux of the plain (level 1) map `ref` in the pixels the tile
//           reaches (at least the tile's own level-16 flux): its share of the
//           map's relative error there when the errors of overlapping tiles
//           are independent;
//   mode 2: the smaller of the mode-0 error and kAdaMapWeight times the
//           mode-1 error: a tile passes when its own deposit is accurate or
//           when its error is a small part of the map where it lands (images
//           close to a star, stretched thin over pixels that other images
//           fill).
__global__ void __launch_bounds__(256) ada_window_errors(AdaGeom g, const int* __restrict__ list, int nlist, int ws,
                                                         float factor, int mode, const int4* __restrict__ win,
                                                         const unsigned long long* __restrict__ acc,
                                                         const unsigned long long* __restrict__ ref,
                                                         float* __restrict__ err) {
  __shared__ double red[5][8];
  const long long W2 = (long long)ws * ws;
  for (int slot = blockIdx.x; slot < nlist; slot += gridDim.x) {
    const int4 w = win[slot];
    if (w.z <= 0) {  // uniform over the block
      if (threadIdx.x < 4) err[(long long)slot * 4 + threadIdx.x] = 0.f;
      continue;
    }
    const int k = ada_window_scale(w, ws);
    const unsigned long long* A = acc + (long long)slot * 5 * W2;
    double d[4] = {0, 0, 0, 0}, tot = 0;
    for (long long q = threadIdx.x; q < W2; q += blockDim.x) {
      const int x = w.x + int(q % ws) * k, y = w.y + int(q / ws) * k;
      if (x >= g.npx || y >= g.npy) continue;  // the window runs past the map's edge
      const long long a16 = (long long)A[4 * W2 + q];
      bool touched = a16 != 0;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const long long ac = (long long)A[c * W2 + q];
        touched = touched || ac != 0;
        d[c] += fabs(double(ac - a16));
      }
      // where the plain map holds less than the tile's own flux, the tile's
      // flux is the reference
      if (touched && mode >= 1) tot += fmax(double((long long)ref[(long long)y * g.npx + x]), double(a16));
    }
#pragma unroll
    for (int c = 0; c < 5; c++) {
      double v = c < 4 ? d[c] : tot;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      double num = 0, den = 0;
      for (int k = 0; k < int(blockDim.x >> 5); k++) {
        num += red[threadIdx.x][k];
        den += red[4][k];
      }
      const int t = list[slot];
      const long long cells = llmin_(kAdaTile, g.ncx - (long long)(t % g.ntx) * kAdaTile) *
                              llmin_(kAdaTile, g.ncy - (long long)(t / g.ntx) * kAdaTile);
      const double own = double(cells) * 2.0 * double(factor) * kFixScale;
      const double e_map = den > 0 ? num / den : (num > 0 ? 1.0 : 0.0);
      const double e = mode == 0 ? num / own : (mode == 1 ? e_map : fmin(num / own, kAdaMapWeight * e_map));
      err[(long long)slot * 4 + threadIdx.x] = float(e);
    }
    __syncthreads();
  }
}

// Per-tile features from the base corner lattice and the tree (one thread per
// tile):
//   0  smooth convergence kappa_tot - kappa_star
//   1  local star convergence: theta^2 sum m of the near field of the leaf
//      that owns the tile centre over its area / pi (the leaf and its
//      neighbours, (6 hl)^2)
//   2  mean shear magnitude of the local Jacobian at the tile's 4 corner cells
//   3  log10 of the smallest |det J| at those cells (J = d source / d lens, in
//      pixels per unlensed pixel, from the cell's edge vectors)
//   4  log10 of the largest |det J|
//   5  1 when det J changes sign between those cells (a critical curve runs
//      through the tile), else 0
//   6  log10 of the distance from the tile centre to the nearest star of the
//      leaf that owns the centre (its near field), in cell widths
//   7  log10(1 + distance in pixels from the bounding box of the images of
//      the tile's 4 corners to the map), 0 when they overlap the map
template <typename T>
__global__ void ada_features(AdaGeom g, ShootParams sp, LeafPtrs lp, DescentPtrs<T> dp,
                             const double2* __restrict__ base_verts, float* __restrict__ feat,
                             int* __restrict__ tile_leaf) {
  const int ntiles = g.ntx * g.nty;
  const double cellpx = 2.0 * sp.rhs_x * sp.npx / (2.0 * sp.hly_re);  // unlensed cell width in pixels
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int tx = t % g.ntx, ty = t / g.ntx;
    const long long i0 = (long long)tx * kAdaTile, j0 = (long long)ty * kAdaTile;
    const long long ilast = llmin_(i0 + kAdaTile, g.ncx) - 1, jlast = llmin_(j0 + kAdaTile, g.ncy) - 1;
    const long long ci[4] = {i0, ilast, i0, ilast}, cj[4] = {j0, j0, jlast, jlast};
    double gsum = 0, dmin = 1e300, dmax = 0;
    int npos = 0, nneg = 0;
    for (int k = 0; k < 4; k++) {
      const long long i = ci[k], j = cj[k], vx = g.ncx + 1;
      const double2 p00 = base_verts[j * vx + i], p10 = base_verts[j * vx + i + 1],
                    p01 = base_verts[(j + 1) * vx + i];
      // d(source)/d(lens) per unlensed pixel; the stored row axis is flipped
      const double a = (p10.x - p00.x) / cellpx, c = -(p10.y - p00.y) / cellpx;
      const double b = (p01.x - p00.x) / cellpx, d = -(p01.y - p00.y) / cellpx;
      const double det = a * d - b * c;
      const double g1 = 0.5 * (a - d), g2 = 0.5 * (b + c);
      gsum += sqrt(g1 * g1 + g2 * g2);
      const double ad = fabs(det);
      dmin = fmin(dmin, ad);
      dmax = fmax(dmax, ad);
      if (det >= 0) npos++;
      else nneg++;
    }
    // nearest star of the near field at the tile centre
    const double xc = g.base_x + 2.0 * (g.rhs_x * (double(i0) + 0.5 * double(ilast - i0 + 1)));
    const double yc = g.base_y + 2.0 * (g.rhs_y * (double(j0) + 0.5 * double(jlast - j0 + 1)));
    const int leaf = descend_leaf(dp, xc, yc);
    {
      // The points of the tile at any level lie in the box spanned by its
      // extreme fine coordinates (fine_coord is monotone in the index). A
      // leaf's points form a box of the descent's comparisons, so when both
      // extreme corners descend to one leaf every point of the tile does.
      const double xa = fine_coord(g.base_x, g.rhs_x, i0 * kAdaMaxLevel);
      const double xb = fine_coord(g.base_x, g.rhs_x, (ilast + 1) * kAdaMaxLevel);
      const double ya = fine_coord(g.base_y, g.rhs_y, j0 * kAdaMaxLevel);
      const double yb = fine_coord(g.base_y, g.rhs_y, (jlast + 1) * kAdaMaxLevel);
      const int la = descend_leaf(dp, fmin(xa, xb), fmin(ya, yb));
      const int lb = descend_leaf(dp, fmax(xa, xb), fmax(ya, yb));
      tile_leaf[t] = la == lb ? la : -1;
    }
    const int nn = lp.nnear[leaf];
    double dn = 1e300;
    const double lcx = lp.cx[leaf], lcy = lp.cy[leaf];
    for (int s = 0; s < nn; s++) {
      const float4 st = lp.near32[(size_t)leaf * kMaxStarsDirect + s];
      dn = fmin(dn, hypot(xc - (lcx + double(st.x)), yc - (lcy + double(st.y))));
    }
    if (nn == 0) dn = 2.0 * lp.hl[leaf];
    double msum = 0;  // near32 holds m theta^2
    for (int s = 0; s < nn; s++) msum += lp.near32[(size_t)leaf * kMaxStarsDirect + s].z;
    const double hl = lp.hl[leaf];
    const double kloc = msum * 3.14159265358979323846 / (36.0 * hl * hl);
    // image of the tile's corners against the map
    double bx0 = 1e300, by0 = 1e300, bx1 = -1e300, by1 = -1e300;
    {
      const long long vx = g.ncx + 1;
      const long long qi[4] = {i0, ilast + 1, i0, ilast + 1}, qj[4] = {j0, j0, jlast + 1, jlast + 1};
      for (int k = 0; k < 4; k++) {
        const double2 q = base_verts[qj[k] * vx + qi[k]];
        bx0 = fmin(bx0, q.x);
        bx1 = fmax(bx1, q.x);
        by0 = fmin(by0, q.y);
        by1 = fmax(by1, q.y);
      }
    }
    const double ddx = fmax(0.0, fmax(bx0 - double(g.npx), -bx1)), ddy = fmax(0.0, fmax(by0 - double(g.npy), -by1));
    const double dmap = hypot(ddx, ddy);
    float* f = feat + (long long)t * kAdaFeatures;
    f[0] = float(sp.kappa - sp.kstar);
    f[1] = float(kloc);
    f[2] = float(gsum * 0.25);
    f[3] = float(log10(dmin + 1e-6));
    f[4] = float(log10(dmax + 1e-6));
    f[5] = (npos > 0 && nneg > 0) ? 1.f : 0.f;
    f[6] = float(log10(dn / (2.0 * sp.rhs_x) + 1e-6));
    f[7] = isfinite(dmap) ? float(log10(1.0 + dmap)) : 12.f;
  }
}

}  // namespace irsb
