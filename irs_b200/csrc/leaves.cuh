// Per-leaf records consumed by the shooting kernels, and the partition of a
// regular lattice (rays for IRS, cell vertices for IPM) into leaf tiles.
//
// A ray is evaluated with the leaf that get_nearest_node (tree_node.cuh:529-561)
// returns for it, i.e. its near field is the leaf's own stars plus its
// neighbours' stars (alpha_star.cuh:18-41, neighbours first) and its far field
// is the leaf's local expansion (alpha_local.cuh:18-36). Here that lookup is
// done once per leaf instead of once per ray: every leaf box [lox, hix) x
// [loy, hiy) covers a rectangle of lattice indices, found by binary search on
// the lattice coordinate formula (which is monotone in the index). The
// rectangles are cut into TX x TY tiles; a prefix sum over leaves maps a global
// tile number back to (leaf, tile).
//
// Record layout (structure of arrays over leaves, 32 slots per leaf):
//   near64[l][s] = (x, y, m, 0)            FP64 plain path, global coordinates
//   near32[l][s] = (x - cx, y - cy, m theta^2, 0)  FP32 path, leaf-relative
//   coef64[l][k] = k * c_k, k = 1..p       (slot k-1)
//   coef32[l][k] = theta^2 (k+1) c_{k+1} / hl, k = 0..p-1: conj(alpha_local) =
//                  sum_k coef32[k] dz^k with dz = (z - c) / hl
//   smooth0[l]   = D(conj(c)) when the smooth sheet is folded (below)
//
// Folding the smooth sheet (rectangular field, approximate sheet, FP32 form):
// there alpha_smooth(z) + kappa_star z is a polynomial D in conj(z) of degree
// taylor_smooth + 1 (alpha_smooth.cuh:62-127, the series in conj(z)/corner).
// Its Taylor coefficients about the leaf centre, in units of the leaf's half
// length, F_k = e_k hl^k with D = sum_k e_k (conj(z) - conj(c))^k, come from
// D at 32 points of the circle |z - c| = hl and a discrete Fourier transform
// (FP64; terms of order 32 and above, below (hl / |corner|)^32 of D, are
// dropped). F_0 goes to smooth0, conj(F_k) for k = 1..p-1 is added to
// coef32[k]; the kernels then evaluate the sheet with the far field instead of
// its series at every point.
#pragma once
#include "common.cuh"
#include "devutil.cuh"
#include "fmm.cuh"
#include "smooth.cuh"
#include "tree.cuh"

namespace irsb {

// Tree nodes needed by the descent, and the node -> leaf map. The descent is
// get_nearest_node (tree_node.cuh:529-561) for points inside the root box.
template <typename T>
struct DescentPtrs {
  const T* cx;
  const T* cy;
  const int* child0;
  const long long* leaf_of_node;  // exclusive scan of the leaf flags
  const int* tile_leaf;           // per tile: the leaf owning all its points, or -1 (nullptr: not known)
};

template <typename T>
__device__ __forceinline__ int descend_leaf(const DescentPtrs<T>& d, double x, double y) {
  int k = 0;
  for (int it = 0; it < kMaxLevels + 1; it++) {
    const int c0 = d.child0[k];
    if (c0 < 0) break;
    const double cx = double(d.cx[k]), cy = double(d.cy[k]);
    const bool right = x >= cx, top = y >= cy;
    k = c0 + (right ? (top ? 0 : 3) : (top ? 1 : 2));
  }
  return int(d.leaf_of_node[k]);
}

constexpr int kTileX = 32;
constexpr int kTileY = 32;

struct LeafSet {
  int n = 0;
  DevVec<double2> smooth0;  // folded smooth sheet at the leaf centres (when folded)
  DevVec<int> flag;
  DevVec<long long> pos;
  DevVec<int> node;
  DevVec<double> cx, cy, hl;
  DevVec<int> nnear;
  DevVec<double4> near64;
  DevVec<float4> near32;
  DevVec<double2> coef64;
  DevVec<float2> coef32;
  ScanScratch scan;
};

// Lattice partition for one lattice (rays or vertices).
struct LatticeTiles {
  DevVec<int4> rect;  // i0, i1, j0, j1
  DevVec<long long> tiles;
  DevVec<long long> tile_off;  // [n + 1]
  DevVec<int4> table;          // per tile: leaf, i0, j0, (ni << 16) | nj
  long long total = 0;
  ScanScratch scan;
};

// One thread per leaf writes the table entries of its tiles (row-major over
// the leaf's rectangle).
__global__ void leaf_tile_table(int nleaves, const int* __restrict__ dn, const int4* __restrict__ rect,
                                const long long* __restrict__ tile_off, int tx, int ty, int4* __restrict__ table,
                                long long table_cap, int* __restrict__ err) {
  if (dn) nleaves = *dn;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nleaves; l += gridDim.x * blockDim.x) {
    int4 r = rect[l];
    long long t = tile_off[l], t_end = tile_off[l + 1];
    if (t == t_end) continue;
    if (t_end > table_cap) {  // more tiles than the table holds
      atomicOr(err, kErrTableOverflow);
      continue;
    }
    int ntx = (r.y - r.x + tx - 1) / tx;
    for (long long k = 0; t + k < t_end; k++) {
      int tj = int(k / ntx), ti = int(k % ntx);
      int i0 = r.x + ti * tx, j0 = r.z + tj * ty;
      int ni = min(tx, r.y - i0), nj = min(ty, r.w - j0);
      table[t + k] = make_int4(l, i0, j0, (ni << 16) | nj);
    }
  }
}

__global__ void leaf_flags(int n, const int* __restrict__ dn, const int* __restrict__ child0, int* flag) {
  if (dn) n = *dn;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) flag[k] = child0[k] < 0;
}
__global__ void leaf_compact(int n, const int* __restrict__ dn, const int* __restrict__ flag,
                             const long long* __restrict__ pos, int* node) {
  if (dn) n = *dn;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    if (flag[k]) node[pos[k]] = k;
}

// One warp per leaf: gather the near field and the expansion coefficients.
// The smooth sheet to fold into the FP32 leaf coefficients (on = 0: none).
struct SmoothFold {
  int on;
  double kstar, corner_re, corner_im, inv_pi;
  int taylor_smooth;
  double2* smooth0;  // [nleaves] out
};

template <typename T>
__global__ void leaf_build(int nleaves, const int* __restrict__ dn, int p, double theta,
                           const double* __restrict__ theta_r, const int* __restrict__ rid,
                           const int* __restrict__ leaf_node,
                           const T* __restrict__ cx, const T* __restrict__ cy, const T* __restrict__ hl,
                           const int* __restrict__ sbeg, const int* __restrict__ scnt, const int* __restrict__ nbr,
                           const int* __restrict__ n_nbr, const StarRec<T>* __restrict__ stars,
                           const double2* __restrict__ loc, double* lcx, double* lcy, double* lhl, int* nnear,
                           double4* near64, float4* near32, double2* coef64, float2* coef32, int* leaf_rid,
                           int* dstat, SmoothFold fold = SmoothFold{0, 0, 0, 0, 0, 0, nullptr}) {
  if (dn) nleaves = *dn;
  int lane = threadIdx.x & 31;
  int warps = (gridDim.x * blockDim.x) >> 5;
  for (int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; l < nleaves; l += warps) {
    int k = leaf_node[l];
    const double th = theta_r ? theta_r[rid[k]] : theta;
    const double th2 = th * th;
    double ccx = double(cx[k]), ccy = double(cy[k]), h = double(hl[k]);
    if (lane == 0) {
      lcx[l] = ccx;
      lcy[l] = ccy;
      lhl[l] = h;
      if (leaf_rid) leaf_rid[l] = rid[k];
    }
    // near list: neighbours in order, then the leaf itself
    int nn = n_nbr[k];
    int out = 0;
    for (int j = 0; j <= nn; j++) {
      int src = j < nn ? nbr[k * kMaxNeighbors + j] : k;
      int b = sbeg[src], c = scnt[src];
      for (int i = lane; i < c; i += 32) {
        int slot = out + i;
        if (slot < kMaxStarsDirect) {
          StarRec<T> s = stars[b + i];
          if (near64)
            near64[(size_t)l * kMaxStarsDirect + slot] = make_double4(double(s.x), double(s.y), double(s.m), 0.0);
          near32[(size_t)l * kMaxStarsDirect + slot] =
              make_float4(float(double(s.x) - ccx), float(double(s.y) - ccy), float(double(s.m) * th2), 0.f);
        }
      }
      out += c;
    }
    if (out > kMaxStarsDirect) {
      if (lane == 0) atomicOr(&dstat[0], kErrNearOverflow);
      out = kMaxStarsDirect;
    }
    // zero the unused slots so that any over-read is harmless
    for (int slot = out + lane; slot < kMaxStarsDirect; slot += 32) {
      if (near64) near64[(size_t)l * kMaxStarsDirect + slot] = make_double4(0, 0, 0, 0);
      near32[(size_t)l * kMaxStarsDirect + slot] = make_float4(0, 0, 0, 0);
    }
    if (lane == 0) nnear[l] = out;
    // the folded smooth sheet: lane j samples D at the point j of the circle
    // |z - c| = hl, then lane k forms F_k = (1/32) sum_j D_j e^{2 pi i j k / 32}
    double2 fk = make_double2(0.0, 0.0);
    if (fold.on) {
      double sj, cj;
      sincospi(double(lane) / 16.0, &sj, &cj);
      const cplx<double> z = mk(ccx + h * cj, ccy + h * sj);
      const cplx<double> a = alpha_smooth_(z, fold.kstar, 1, mk(fold.corner_re, fold.corner_im), 1,
                                           fold.taylor_smooth, fold.inv_pi);
      const double dre = a.re + fold.kstar * z.re, dim = a.im + fold.kstar * z.im;
      for (int j = 0; j < 32; j++) {
        const double xr = __shfl_sync(0xffffffffu, dre, j), xi = __shfl_sync(0xffffffffu, dim, j);
        double sw, cw;
        sincospi(double((j * lane) & 31) / 16.0, &sw, &cw);
        fk.x += xr * cw - xi * sw;
        fk.y += xr * sw + xi * cw;
      }
      fk.x *= 1.0 / 32.0;
      fk.y *= 1.0 / 32.0;
      if (lane == 0) fold.smooth0[l] = fk;
    }
    // local expansion coefficients
    if (lane < p) {
      int kk = lane + 1;
      double2 c = loc[(size_t)k * (p + 1) + kk];
      if (coef64) coef64[(size_t)l * kMaxOrder + lane] = make_double2(c.x * kk, c.y * kk);
      double s = th2 * kk / h;
      double cr = c.x * s, ci = c.y * s;
      if (fold.on && lane >= 1) {  // conj(F_k) into the coefficient of dz^k
        cr += fk.x;
        ci -= fk.y;
      }
      coef32[(size_t)l * kMaxOrder + lane] = make_float2(float(cr), float(ci));
    } else if (lane < kMaxOrder) {
      if (coef64) coef64[(size_t)l * kMaxOrder + lane] = make_double2(0, 0);
      coef32[(size_t)l * kMaxOrder + lane] = make_float2(0, 0);
    }
  }
}

// Lattice coordinate of index i: base + 2 * (rhs * i), the operation order of
// the reference's ray positions (irs_functions.cuh:122).
__device__ __forceinline__ double lattice_coord(double base, double rhs, long long i) {
  return base + 2.0 * (rhs * double(i));
}
// first index in [0, n] with coordinate >= v
__device__ __forceinline__ long long lattice_lower_bound(double base, double rhs, long long n, double v) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    long long mid = (lo + hi) >> 1;
    if (lattice_coord(base, rhs, mid) >= v)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

__global__ void leaf_rects(int nleaves, const int* __restrict__ leaf_node, const double* __restrict__ lox,
                           const double* __restrict__ hix, const double* __restrict__ loy,
                           const double* __restrict__ hiy, double base_x, double base_y, double rhs_x, double rhs_y,
                           long long nx, long long ny, long long jlo, long long jhi, int tx, int ty, int4* rect,
                           long long* tiles) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nleaves; l += gridDim.x * blockDim.x) {
    int k = leaf_node[l];
    long long i0 = lattice_lower_bound(base_x, rhs_x, nx, lox[k]);
    long long i1 = lattice_lower_bound(base_x, rhs_x, nx, hix[k]);
    long long j0 = lattice_lower_bound(base_y, rhs_y, ny, loy[k]);
    long long j1 = lattice_lower_bound(base_y, rhs_y, ny, hiy[k]);
    j0 = j0 < jlo ? jlo : j0;  // restrict to the row band [jlo, jhi)
    j1 = j1 > jhi ? jhi : j1;
    if (j1 < j0) j1 = j0;
    rect[l] = make_int4(int(i0), int(i1), int(j0), int(j1));
    long long ni = i1 - i0, nj = j1 - j0;
    tiles[l] = (ni > 0 && nj > 0) ? ((ni + tx - 1) / tx) * ((nj + ty - 1) / ty) : 0;
  }
}

// Lattice of one realization and the rows of it that a pass covers.
struct LatticeGeom {
  double base_x, base_y, rhs_x, rhs_y;
  long long nx, ny;
};

// leaf_rects over the leaves of many realizations (count on the device): a
// leaf takes its realization's lattice and that realization's row band
// [jlo, jhi) of the current pass (empty when jlo >= jhi).
__global__ void leaf_rects_batch(const int* __restrict__ dn, const int* __restrict__ leaf_node,
                                 const int* __restrict__ rid, const double* __restrict__ lox,
                                 const double* __restrict__ hix, const double* __restrict__ loy,
                                 const double* __restrict__ hiy, const LatticeGeom* __restrict__ geom,
                                 const long long* __restrict__ jlo_r, const long long* __restrict__ jhi_r, int tx,
                                 int ty, int4* rect, long long* tiles) {
  const int nleaves = *dn;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nleaves; l += gridDim.x * blockDim.x) {
    const int k = leaf_node[l];
    const int r = rid[k];
    const long long jlo = jlo_r[r], jhi = jhi_r[r];
    if (jlo >= jhi) {
      rect[l] = make_int4(0, 0, 0, 0);
      tiles[l] = 0;
      continue;
    }
    const LatticeGeom g = geom[r];
    long long i0 = lattice_lower_bound(g.base_x, g.rhs_x, g.nx, lox[k]);
    long long i1 = lattice_lower_bound(g.base_x, g.rhs_x, g.nx, hix[k]);
    long long j0 = lattice_lower_bound(g.base_y, g.rhs_y, g.ny, loy[k]);
    long long j1 = lattice_lower_bound(g.base_y, g.rhs_y, g.ny, hiy[k]);
    j0 = j0 < jlo ? jlo : j0;
    j1 = j1 > jhi ? jhi : j1;
    if (j1 < j0) j1 = j0;
    rect[l] = make_int4(int(i0), int(i1), int(j0), int(j1));
    long long ni = i1 - i0, nj = j1 - j0;
    tiles[l] = (ni > 0 && nj > 0) ? ((ni + tx - 1) / tx) * ((nj + ty - 1) / ty) : 0;
  }
}

template <typename T>
bool build_leaves(LeafSet& L, TreeDev<T>& t, FmmDev& f, const StarRec<T>* stars, double theta, cudaStream_t s,
                  SmoothFold fold = SmoothFold{0, 0, 0, 0, 0, 0, nullptr}) {
  int n = t.num_nodes;
  if (!L.flag.alloc_exact(n) || !L.pos.alloc_exact(n + 1)) return false;
  int blocks = std::max(1, std::min(ceil_div(n, 256), 148 * 8));
  leaf_flags<<<blocks, 256, 0, s>>>(n, nullptr, t.child0.p, L.flag.p);
  if (!exclusive_scan<int>(L.flag.p, n, L.pos.p, L.scan, s)) return false;
  long long nl = 0;
  IRSB_CKR(cudaMemcpyAsync(&nl, L.scan.sum.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
  IRSB_CKR(cudaStreamSynchronize(s));
  L.n = int(nl);
  if (!L.node.alloc_exact(L.n) || !L.cx.alloc_exact(L.n) || !L.cy.alloc_exact(L.n) || !L.hl.alloc_exact(L.n) ||
      !L.nnear.alloc_exact(L.n) || !L.near64.alloc_exact((size_t)L.n * kMaxStarsDirect) ||
      !L.near32.alloc_exact((size_t)L.n * kMaxStarsDirect) || !L.coef64.alloc_exact((size_t)L.n * kMaxOrder) ||
      !L.coef32.alloc_exact((size_t)L.n * kMaxOrder))
    return false;
  if (fold.on) {
    if (!L.smooth0.alloc_exact(L.n)) return false;
    fold.smooth0 = L.smooth0.p;
  }
  leaf_compact<<<blocks, 256, 0, s>>>(n, nullptr, L.flag.p, L.pos.p, L.node.p);
  IRSB_LAUNCH_CK("leaf_compact");
  IRSB_CKR(cudaMemsetAsync(t.dstat.p, 0, 2 * sizeof(int), s));
  int lb = std::max(1, std::min(ceil_div(L.n, 8), 148 * 16));
  leaf_build<T><<<lb, 256, 0, s>>>(L.n, nullptr, f.p, theta, nullptr, nullptr, L.node.p, t.cx.p, t.cy.p, t.hl.p, t.sbeg.p, t.scnt.p, t.nbr.p,
                                   t.n_nbr.p, stars, f.loc.p, L.cx.p, L.cy.p, L.hl.p, L.nnear.p, L.near64.p,
                                   L.near32.p, L.coef64.p, L.coef32.p, nullptr, t.dstat.p, fold);
  IRSB_LAUNCH_CK("leaf_build");
  int st = 0;
  IRSB_CKR(cudaMemcpyAsync(&st, t.dstat.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  IRSB_CKR(cudaStreamSynchronize(s));
  if (st) {
    std::fprintf(stderr, "Error. A leaf's near field holds more than %d stars.\n", kMaxStarsDirect);
    return false;
  }
  return true;
}

template <typename T>
bool build_lattice_tiles(LatticeTiles& W, const LeafSet& L, TreeDev<T>& t, double base_x, double base_y,
                         double rhs_x, double rhs_y, long long nx, long long ny, long long jlo, long long jhi,
                         cudaStream_t s) {
  if (!W.rect.alloc_exact(L.n) || !W.tiles.alloc_exact(L.n) || !W.tile_off.alloc_exact(L.n + 1)) return false;
  int blocks = std::max(1, std::min(ceil_div(L.n, 256), 148 * 8));
  leaf_rects<<<blocks, 256, 0, s>>>(L.n, L.node.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p, base_x, base_y, rhs_x, rhs_y,
                                    nx, ny, jlo, jhi, kTileX, kTileY, W.rect.p, W.tiles.p);
  IRSB_LAUNCH_CK("leaf_rects");
  if (!exclusive_scan<long long>(W.tiles.p, L.n, W.tile_off.p, W.scan, s)) return false;
  IRSB_CKR(cudaMemcpyAsync(W.tile_off.p + L.n, W.scan.sum.p, sizeof(long long), cudaMemcpyDeviceToDevice, s));
  IRSB_CKR(cudaMemcpyAsync(&W.total, W.scan.sum.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
  IRSB_CKR(cudaStreamSynchronize(s));
  if (!W.table.alloc_exact(std::max<long long>(W.total, 1))) return false;
  leaf_tile_table<<<blocks, 256, 0, s>>>(L.n, nullptr, W.rect.p, W.tile_off.p, kTileX, kTileY, W.table.p, W.total,
                                         t.dstat.p + 1);
  IRSB_LAUNCH_CK("leaf_tile_table");
  return true;
}

}  // namespace irsb
