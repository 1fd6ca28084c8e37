// Quadtree over the star field, built level by level on the device.
//
// Semantics follow the reference tree (include/tree_node.cuh, driven from
// include/ipm.cuh:740-842):
//   * the root is centred at 0 with half length root_half_length;
//   * a node is split into 4 children when its own stars plus its neighbours'
//     stars exceed 32 (get_node_star_info_kernel / create_children_kernel,
//     tree_node.cuh:321-381), empty nodes included;
//   * child q has centre parent + hl/2 * {(1,1),(-1,1),(-1,-1),(1,-1)}[q]
//     (make_child, tree_node.cuh:151-168) and owns the stars with
//     x >= cx && y >= cy (q=0), x < cx && y >= cy (1), x < cx && y < cy (2),
//     otherwise (3); children's star ranges are contiguous in child order
//     (sort_stars_kernel, tree_node.cuh:392-501);
//   * neighbours / interaction lists as set_neighbors (tree_node.cuh:183-267).
// Differences by design: node slots are assigned by an exclusive scan over the
// split flags and stars are partitioned stably, so the tree and the star order
// are deterministic (the reference uses atomics for both). The structure
// (levels, centres, per-node star sets, neighbour sets) is the same.
//
// Layout: structure-of-arrays over a global node index; nodes of level l are
// [level_off[l], level_off[l+1]). Each node also records the half-open box
// [lox, hix) x [loy, hiy) that the descent of get_nearest_node
// (tree_node.cuh:529-561) maps to it; a ray lattice is partitioned by leaf
// with those boxes.
#pragma once
#include "common.cuh"
#include "devutil.cuh"
#include "params.hpp"

#include <vector>

namespace irsb {

// Node range of one level: [beg, end) given by the host, or read on the device
// from off[lvl], off[lvl + 1] when off is set (graph-captured builds, whose
// level sizes are not known to the host).
struct LevelRange {
  const int* off = nullptr;
  int lvl = 0;
  __device__ __forceinline__ void get(int& beg, int& end) const {
    if (off) {
      beg = off[lvl];
      end = off[lvl + 1];
    }
  }
};

template <typename T>
struct TreeDev {
  int cap = 0;
  int num_nodes = 0;
  int levels = 0;  // number of levels - 1 (the reference's tree_levels)
  std::vector<int> level_off;  // host copy, size levels + 2
  DevVec<T> cx, cy, hl;
  DevVec<int> level, parent, child0, sbeg, scnt;
  DevVec<int> rid;         // realization of the node (0 for a single star field)
  DevVec<int> nbr, n_nbr;  // [cap][kMaxNeighbors]
  DevVec<int> sil, n_sil;  // [cap][kMaxSameLevelIL]
  DevVec<int> dil, n_dil;  // [cap][kMaxDiffLevelIL]
  DevVec<double> lox, hix, loy, hiy;
  // scratch
  DevVec<int> split, cnt_near;
  DevVec<long long> rank;
  DevVec<int> dstat;  // [0] max near count, [1] error bits
  ScanScratch scan;
  DevVec<StarRec<T>> tmp_stars;
};

template <typename T>
struct NodeView {
  const T* cx;
  const T* cy;
  const T* hl;
  const int* child0;
  const int* sbeg;
  const int* scnt;
  const int* nbr;
  const int* n_nbr;
};

template <typename T>
bool tree_reserve(TreeDev<T>& t, int want, cudaStream_t s) {
  if (want <= t.cap) return true;
  int nc = t.cap ? t.cap : 1024;
  while (nc < want) nc *= 2;
  bool ok = t.cx.reserve(nc, s) && t.cy.reserve(nc, s) && t.hl.reserve(nc, s) && t.level.reserve(nc, s) &&
            t.parent.reserve(nc, s) && t.child0.reserve(nc, s) && t.sbeg.reserve(nc, s) && t.scnt.reserve(nc, s) && t.rid.reserve(nc, s) &&
            t.nbr.reserve(size_t(nc) * kMaxNeighbors, s) && t.n_nbr.reserve(nc, s) &&
            t.sil.reserve(size_t(nc) * kMaxSameLevelIL, s) && t.n_sil.reserve(nc, s) &&
            t.dil.reserve(size_t(nc) * kMaxDiffLevelIL, s) && t.n_dil.reserve(nc, s) && t.lox.reserve(nc, s) &&
            t.hix.reserve(nc, s) && t.loy.reserve(nc, s) && t.hiy.reserve(nc, s);
  if (!ok) return false;
  // keep the logical sizes in step so that growth copies every live node
  for (auto* v : {&t.cx.n, &t.cy.n, &t.hl.n}) *v = nc;
  t.level.n = t.parent.n = t.child0.n = t.sbeg.n = t.scnt.n = t.n_nbr.n = t.n_sil.n = t.n_dil.n = t.rid.n = nc;
  t.lox.n = t.hix.n = t.loy.n = t.hiy.n = nc;
  t.nbr.n = size_t(nc) * kMaxNeighbors;
  t.sil.n = size_t(nc) * kMaxSameLevelIL;
  t.dil.n = size_t(nc) * kMaxDiffLevelIL;
  t.cap = nc;
  return true;
}

template <typename T>
__global__ void tree_init_root(T* cx, T* cy, T* hl, int* level, int* parent, int* child0, int* sbeg, int* scnt,
                               int* rid, int* n_nbr, int* n_sil, int* n_dil, double* lox, double* hix, double* loy,
                               double* hiy, T root_hl, int nstars) {
  rid[0] = 0;
  cx[0] = T(0);
  cy[0] = T(0);
  hl[0] = root_hl;
  level[0] = 0;
  parent[0] = -1;
  child0[0] = -1;
  sbeg[0] = 0;
  scnt[0] = nstars;
  n_nbr[0] = n_sil[0] = n_dil[0] = 0;
  lox[0] = -INFINITY;
  hix[0] = INFINITY;
  loy[0] = -INFINITY;
  hiy[0] = INFINITY;
}

// Stars of a node and its neighbours; split flag; level maximum.
__global__ void tree_near_count(int beg, int end, LevelRange lr, const int* __restrict__ scnt,
                                const int* __restrict__ nbr, const int* __restrict__ n_nbr, int* __restrict__ split,
                                int* __restrict__ dstat) {
  lr.get(beg, end);
  int local_max = 0;
  for (int k = beg + blockIdx.x * blockDim.x + threadIdx.x; k < end; k += gridDim.x * blockDim.x) {
    int c = scnt[k];
    int nn = n_nbr[k];
    for (int j = 0; j < nn; j++) c += scnt[nbr[k * kMaxNeighbors + j]];
    split[k - beg] = c > kMaxStarsDirect ? 1 : 0;
    local_max = max(local_max, c);
  }
  for (int o = 16; o > 0; o >>= 1) local_max = max(local_max, __shfl_down_sync(0xffffffffu, local_max, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&dstat[0], local_max);
}

template <typename T>
__global__ void tree_make_children(int beg, int end, int child_base, LevelRange lr, const int* __restrict__ stop,
                                   const int* __restrict__ split, const long long* __restrict__ rank, T* cx, T* cy,
                                   T* hl, int* level, int* parent, int* child0, int* sbeg, int* scnt, int* rid,
                                   int* n_nbr, int* n_sil, int* n_dil, double* lox, double* hix, double* loy,
                                   double* hiy) {
  if (lr.off) {
    lr.get(beg, end);
    child_base = end;
  }
  const bool halt = stop && *stop;
  for (int k = beg + blockIdx.x * blockDim.x + threadIdx.x; k < end; k += gridDim.x * blockDim.x) {
    if (halt || !split[k - beg]) {
      child0[k] = -1;
      continue;
    }
    int c0 = child_base + 4 * int(rank[k - beg]);
    child0[k] = c0;
    T h = hl[k] / 2;
    T pcx = cx[k], pcy = cy[k];
    const T ox[4] = {T(1), T(-1), T(-1), T(1)};
    const T oy[4] = {T(1), T(1), T(-1), T(-1)};
    double plox = lox[k], phix = hix[k], ploy = loy[k], phiy = hiy[k];
    for (int q = 0; q < 4; q++) {
      int c = c0 + q;
      cx[c] = pcx + h * ox[q];
      cy[c] = pcy + h * oy[q];
      hl[c] = h;
      level[c] = level[k] + 1;
      parent[c] = k;
      rid[c] = rid[k];
      child0[c] = -1;
      sbeg[c] = sbeg[k];
      scnt[c] = 0;
      n_nbr[c] = n_sil[c] = n_dil[c] = 0;
      // x >= pcx for q = 0, 3; y >= pcy for q = 0, 1
      bool right = (q == 0 || q == 3), top = (q == 0 || q == 1);
      lox[c] = right ? double(pcx) : plox;
      hix[c] = right ? phix : double(pcx);
      loy[c] = top ? double(pcy) : ploy;
      hiy[c] = top ? phiy : double(pcy);
    }
  }
}

template <typename T>
__device__ __forceinline__ int star_quadrant(T x, T y, T cx, T cy) {
  if (x >= cx && y >= cy) return 0;
  if (x < cx && y >= cy) return 1;
  if (x < cx && y < cy) return 2;
  return 3;
}

// Blocks stride over the level's nodes; split nodes with stars partition their
// star range into the 4 child ranges, keeping the relative order of stars
// (stable).
template <typename T>
__global__ void __launch_bounds__(256) tree_partition_stars(int beg, int end, LevelRange lr,
                                                            const int* __restrict__ stop,
                                                            const int* __restrict__ split,
                                                            const T* __restrict__ cx, const T* __restrict__ cy,
                                                            const int* __restrict__ child0, int* sbeg, int* scnt,
                                                            StarRec<T>* __restrict__ stars,
                                                            StarRec<T>* __restrict__ tmp) {
  lr.get(beg, end);
  if (stop && *stop) return;
  __shared__ int cnt[4];
  __shared__ int warp_cnt[8][4];
  __shared__ int base[4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = beg + blockIdx.x; k < end; k += gridDim.x) {
    if (!split[k - beg]) continue;  // uniform over the block
    const int b = sbeg[k], n = scnt[k];
    const int c0 = child0[k];
    if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
    __syncthreads();
    const T pcx = cx[k], pcy = cy[k];
    int lc[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      StarRec<T> st = stars[b + i];
      lc[star_quadrant(st.x, st.y, pcx, pcy)]++;
    }
    for (int q = 0; q < 4; q++)
      if (lc[q]) atomicAdd(&cnt[q], lc[q]);
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = b;
      for (int q = 0; q < 4; q++) {
        base[q] = acc;
        sbeg[c0 + q] = acc;
        scnt[c0 + q] = cnt[q];
        acc += cnt[q];
      }
    }
    __syncthreads();
    for (int start = 0; start < n; start += blockDim.x) {
      int i = start + threadIdx.x;
      int q = -1;
      StarRec<T> st;
      if (i < n) {
        st = stars[b + i];
        q = star_quadrant(st.x, st.y, pcx, pcy);
      }
      unsigned m[4];
      for (int qq = 0; qq < 4; qq++) m[qq] = __ballot_sync(0xffffffffu, q == qq);
      if (lane < 4) warp_cnt[w][lane] = __popc(m[lane]);
      __syncthreads();
      if (q >= 0) {
        int off = base[q];
        for (int ww = 0; ww < w; ww++) off += warp_cnt[ww][q];
        off += __popc(m[q] & ((1u << lane) - 1u));
        tmp[off] = st;
      }
      __syncthreads();
      if (threadIdx.x < 4) {
        int add = 0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) add += warp_cnt[ww][threadIdx.x];
        base[threadIdx.x] += add;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) stars[b + i] = tmp[b + i];
    __syncthreads();
  }
}

// set_neighbors (tree_node.cuh:183-267) for the nodes of one level (>= 1).
template <typename T>
__global__ void tree_set_neighbors(int beg, int end, LevelRange lr, const T* __restrict__ cx,
                                   const T* __restrict__ cy, const T* __restrict__ hl, const int* __restrict__ parent,
                                   const int* __restrict__ child0, const int* __restrict__ scnt, int* nbr,
                                   int* n_nbr, int* sil, int* n_sil, int* dil, int* n_dil, int* dstat) {
  lr.get(beg, end);
  for (int k = beg + blockIdx.x * blockDim.x + threadIdx.x; k < end; k += gridDim.x * blockDim.x) {
    int p = parent[k];
    T h = hl[k];
    T x = cx[k], y = cy[k];
    int nn = 0, ns = 0, nd = 0, err = 0;
    int pc0 = child0[p];
    for (int i = 0; i < 4; i++) {
      int c = pc0 + i;
      if (scnt[c] == 0) continue;
      if (c != k) {
        if (nn < kMaxNeighbors) nbr[k * kMaxNeighbors + nn] = c;
        else err |= kErrNeighborOverflow;
        nn++;
      }
    }
    int pn = n_nbr[p];
    for (int i = 0; i < pn; i++) {
      int nb = nbr[p * kMaxNeighbors + i];
      if (scnt[nb] == 0) continue;
      int nc0 = child0[nb];
      if (nc0 < 0) {
        if (double(xfabs(T(cx[nb] - x))) < 3.5 * double(h) && double(xfabs(T(cy[nb] - y))) < 3.5 * double(h)) {
          if (nn < kMaxNeighbors) nbr[k * kMaxNeighbors + nn] = nb;
          else err |= kErrNeighborOverflow;
          nn++;
        } else {
          if (nd < kMaxDiffLevelIL) dil[k * kMaxDiffLevelIL + nd] = nb;
          else err |= kErrDiffLevelOverflow;
          nd++;
        }
      } else {
        for (int j = 0; j < 4; j++) {
          int c = nc0 + j;
          if (scnt[c] == 0) continue;
          if (xfabs(T(cx[c] - x)) < 3 * h && xfabs(T(cy[c] - y)) < 3 * h) {
            if (nn < kMaxNeighbors) nbr[k * kMaxNeighbors + nn] = c;
            else err |= kErrNeighborOverflow;
            nn++;
          } else {
            if (ns < kMaxSameLevelIL) sil[k * kMaxSameLevelIL + ns] = c;
            else err |= kErrSameLevelOverflow;
            ns++;
          }
        }
      }
    }
    n_nbr[k] = min(nn, kMaxNeighbors);
    n_sil[k] = min(ns, kMaxSameLevelIL);
    n_dil[k] = min(nd, kMaxDiffLevelIL);
    if (err) atomicOr(&dstat[1], err);
  }
}

// Builds the tree over `stars` (device, permuted in place into tree order).
// Returns false on a CUDA error or a list overflow.
template <typename T>
bool build_tree(TreeDev<T>& t, StarRec<T>* stars, int nstars, T root_hl, cudaStream_t s) {
  if (!tree_reserve(t, 1024, s)) return false;
  if (!t.tmp_stars.reserve(nstars, s)) return false;
  if (!t.dstat.reserve(2, s)) return false;
  tree_init_root<T><<<1, 1, 0, s>>>(t.cx.p, t.cy.p, t.hl.p, t.level.p, t.parent.p, t.child0.p, t.sbeg.p, t.scnt.p,
                                    t.rid.p, t.n_nbr.p, t.n_sil.p, t.n_dil.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p, root_hl,
                                    nstars);
  IRSB_LAUNCH_CK("tree_init_root");
  t.level_off.assign({0, 1});
  t.levels = 0;
  IRSB_CKR(cudaMemsetAsync(t.dstat.p, 0, 2 * sizeof(int), s));
  int hstat[2];
  for (int l = 0; l < kMaxLevels; l++) {
    int beg = t.level_off[l], end = t.level_off[l + 1];
    int nl = end - beg;
    if (!t.split.reserve(nl, s) || !t.rank.reserve(nl + 1, s)) return false;
    IRSB_CKR(cudaMemsetAsync(t.dstat.p, 0, sizeof(int), s));
    int blocks = std::min(ceil_div(nl, 256), 148 * 8);
    tree_near_count<<<blocks, 256, 0, s>>>(beg, end, LevelRange{}, t.scnt.p, t.nbr.p, t.n_nbr.p, t.split.p, t.dstat.p);
    IRSB_LAUNCH_CK("tree_near_count");
    if (!exclusive_scan<int>(t.split.p, nl, t.rank.p, t.scan, s)) return false;
    long long nsplit = 0;
    IRSB_CKR(cudaMemcpyAsync(hstat, t.dstat.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaMemcpyAsync(&nsplit, t.scan.sum.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    if (hstat[1]) {
      std::fprintf(stderr, "Error. Tree neighbour/interaction list overflow (code %d).\n", hstat[1]);
      return false;
    }
    if (hstat[0] <= kMaxStarsDirect) {
      // leaves of the final level
      fill_kernel<int><<<std::max(1, ceil_div(nl, 256)), 256, 0, s>>>(t.child0.p + beg, nl, -1);
      IRSB_LAUNCH_CK("fill child0");
      break;
    }
    if (l + 1 >= kMaxLevels) {
      std::fprintf(stderr, "Error. Tree exceeded %d levels.\n", kMaxLevels);
      return false;
    }
    int child_base = end;
    int nnew = int(4 * nsplit);
    if (!tree_reserve(t, end + nnew, s)) return false;
    tree_make_children<T><<<blocks, 256, 0, s>>>(beg, end, child_base, LevelRange{}, nullptr, t.split.p, t.rank.p,
                                                 t.cx.p, t.cy.p, t.hl.p, t.level.p, t.parent.p, t.child0.p, t.sbeg.p,
                                                 t.scnt.p, t.rid.p, t.n_nbr.p,
                                                 t.n_sil.p, t.n_dil.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p);
    IRSB_LAUNCH_CK("tree_make_children");
    tree_partition_stars<T><<<nl, 256, 0, s>>>(beg, end, LevelRange{}, nullptr, t.split.p, t.cx.p, t.cy.p, t.child0.p, t.sbeg.p, t.scnt.p,
                                               stars, t.tmp_stars.p);
    IRSB_LAUNCH_CK("tree_partition_stars");
    int nb2 = std::min(ceil_div(nnew, 256), 148 * 8);
    tree_set_neighbors<T><<<std::max(nb2, 1), 256, 0, s>>>(child_base, child_base + nnew, LevelRange{}, t.cx.p, t.cy.p, t.hl.p,
                                                           t.parent.p, t.child0.p, t.scnt.p, t.nbr.p, t.n_nbr.p,
                                                           t.sil.p, t.n_sil.p, t.dil.p, t.n_dil.p, t.dstat.p);
    IRSB_LAUNCH_CK("tree_set_neighbors");
    t.level_off.push_back(child_base + nnew);
    t.levels++;
  }
  t.num_nodes = t.level_off.back();
  IRSB_CKR(cudaMemcpyAsync(hstat, t.dstat.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  IRSB_CKR(cudaStreamSynchronize(s));
  if (hstat[1]) {
    std::fprintf(stderr, "Error. Tree neighbour/interaction list overflow (code %d).\n", hstat[1]);
    return false;
  }
  return true;
}

}  // namespace irsb
