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

#include <algorithm>
#include <cstdio>
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
  DevVec<StarRec<T>> tmp_stars, star_backup;
  DevVec<int> d_off, d_lvl_n, d_stop;  // level offsets and sizes on the device
  DevVec<int> chunk_cnt;               // per-chunk key counts of the wide partition
  long long launches = 0;              // kernels the last build launched
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

// Blocks of NT threads stride over the level's nodes; split nodes with stars
// partition their star range into the 4 child ranges, keeping the relative
// order of stars (stable). The top levels, a few nodes holding many stars each,
// take NT = 1024 (a quarter of the block-synchronised chunks), the rest 256.
template <typename T, int NT = 256>
__global__ void __launch_bounds__(NT) tree_partition_stars(int beg, int end, LevelRange lr,
                                                            const int* __restrict__ stop,
                                                            const int* __restrict__ split,
                                                            const T* __restrict__ cx, const T* __restrict__ cy,
                                                            const int* __restrict__ child0, int* sbeg, int* scnt,
                                                            StarRec<T>* __restrict__ stars,
                                                            StarRec<T>* __restrict__ tmp) {
  lr.get(beg, end);
  if (stop && *stop) return;
  __shared__ int cnt[4];
  __shared__ int warp_cnt[NT / 32][4];
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
        for (int ww = 0; ww < NT / 32; ww++) add += warp_cnt[ww][threadIdx.x];
        base[threadIdx.x] += add;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) stars[b + i] = tmp[b + i];
    __syncthreads();
  }
}

// The same stable partition for the first two levels, whose NN nodes (1 or 4)
// hold every star between them, on many blocks: the stars are cut into chunks
// of kPartChunk; a star's key is its node's index in the level times 4 plus its
// quadrant (0 in a node that does not split). Count per chunk and key, scan
// each key over the chunks (stable), scatter, copy back. A level that is
// absent (the root did not split) is left alone.
constexpr int kPartChunk = 1024;

template <typename T, int NN>
__device__ __forceinline__ int wide_key(int i, int beg, const int* __restrict__ split, const T* __restrict__ cx,
                                        const T* __restrict__ cy, const int* __restrict__ sbeg,
                                        const int* __restrict__ scnt, const StarRec<T>& st) {
  int j = 0;
#pragma unroll
  for (int jj = 1; jj < NN; jj++)
    if (i >= sbeg[beg + jj]) j = jj;  // the level's nodes are consecutive star ranges in node order
  const int k = beg + j;
  return 4 * j + (split[j] ? star_quadrant(st.x, st.y, cx[k], cy[k]) : 0);
}

template <int NN>
__device__ __forceinline__ bool wide_level(LevelRange lr, const int* stop, int& beg) {
  int b = 0, e = 0;
  lr.get(b, e);
  beg = b;
  return !(stop && *stop) && e - b == NN;
}

template <typename T, int NN>
__global__ void __launch_bounds__(256) tree_wide_count(LevelRange lr, const int* __restrict__ stop,
                                                       const int* __restrict__ split, const T* __restrict__ cx,
                                                       const T* __restrict__ cy, const int* __restrict__ sbeg,
                                                       const int* __restrict__ scnt,
                                                       const StarRec<T>* __restrict__ stars, int nstars, int* cnt) {
  int beg;
  if (!wide_level<NN>(lr, stop, beg)) return;
  __shared__ int c[4 * NN];
  if (threadIdx.x < 4 * NN) c[threadIdx.x] = 0;
  __syncthreads();
  const int i0 = blockIdx.x * kPartChunk, i1 = min(i0 + kPartChunk, nstars);
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    atomicAdd(&c[wide_key<T, NN>(i, beg, split, cx, cy, sbeg, scnt, stars[i])], 1);
  __syncthreads();
  if (threadIdx.x < 4 * NN) cnt[blockIdx.x * 4 * NN + threadIdx.x] = c[threadIdx.x];
}

// One block: per key, the exclusive scan over the chunks plus the key's base
// (its node's first star plus the counts of the node's lower quadrants); the
// children's star ranges.
template <int NN>
__global__ void tree_wide_offsets(LevelRange lr, const int* __restrict__ stop, const int* __restrict__ split,
                                  const int* __restrict__ child0, int* sbeg, int* scnt, int nchunks, int* cnt) {
  int beg;
  if (!wide_level<NN>(lr, stop, beg)) return;
  constexpr int K = 4 * NN;
  __shared__ int tot[K], base[K];
  if (threadIdx.x < K) {
    int run = 0;
    for (int c = 0; c < nchunks; c++) {
      const int v = cnt[c * K + threadIdx.x];
      cnt[c * K + threadIdx.x] = run;
      run += v;
    }
    tot[threadIdx.x] = run;
  }
  __syncthreads();
  if (threadIdx.x < NN) {
    const int j = threadIdx.x, k = beg + j;
    int acc = sbeg[k];
    for (int q = 0; q < 4; q++) {
      base[4 * j + q] = acc;
      if (split[j]) {
        sbeg[child0[k] + q] = acc;
        scnt[child0[k] + q] = tot[4 * j + q];
      }
      acc += tot[4 * j + q];
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nchunks * K; idx += blockDim.x) cnt[idx] += base[idx % K];
}

template <typename T, int NN>
__global__ void __launch_bounds__(256) tree_wide_scatter(LevelRange lr, const int* __restrict__ stop,
                                                         const int* __restrict__ split, const T* __restrict__ cx,
                                                         const T* __restrict__ cy, const int* __restrict__ sbeg,
                                                         const int* __restrict__ scnt,
                                                         const StarRec<T>* __restrict__ stars, int nstars,
                                                         const int* __restrict__ off, StarRec<T>* __restrict__ tmp) {
  int beg;
  if (!wide_level<NN>(lr, stop, beg)) return;
  constexpr int K = 4 * NN;
  __shared__ int run[K];
  __shared__ int wc[8][K];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x < K) run[threadIdx.x] = off[blockIdx.x * K + threadIdx.x];
  __syncthreads();
  const int i0 = blockIdx.x * kPartChunk, i1 = min(i0 + kPartChunk, nstars);
  for (int r = i0; r < i1; r += 256) {  // rounds in star order
    const int i = r + threadIdx.x;
    int key = -1;
    StarRec<T> st;
    if (i < i1) {
      st = stars[i];
      key = wide_key<T, NN>(i, beg, split, cx, cy, sbeg, scnt, st);
    }
    unsigned mine = 0;
#pragma unroll
    for (int kk = 0; kk < K; kk++) {
      const unsigned m = __ballot_sync(0xffffffffu, key == kk);
      if (lane == 0) wc[w][kk] = __popc(m);
      if (key == kk) mine = m;
    }
    __syncthreads();
    if (key >= 0) {
      int pos = run[key];
      for (int ww = 0; ww < w; ww++) pos += wc[ww][key];
      tmp[pos + __popc(mine & ((1u << lane) - 1u))] = st;
    }
    __syncthreads();
    if (threadIdx.x < K) {
      int add = 0;
      for (int ww = 0; ww < 8; ww++) add += wc[ww][threadIdx.x];
      run[threadIdx.x] += add;
    }
    __syncthreads();
  }
}

template <typename T, int NN>
__global__ void tree_wide_copy(LevelRange lr, const int* __restrict__ stop, int nstars,
                               const StarRec<T>* __restrict__ tmp, StarRec<T>* __restrict__ stars) {
  int beg;
  if (!wide_level<NN>(lr, stop, beg)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nstars; i += gridDim.x * blockDim.x) stars[i] = tmp[i];
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

// The same lists with one warp per node: lane q examines candidate q in the
// order of the loops above (the 4 siblings, then for each of the parent's
// neighbours either the neighbour itself, a leaf, or its 4 children), and
// each list takes its candidates in that order through a ballot prefix, so
// the lists are identical to the one-thread form.
template <typename T>
__global__ void tree_set_neighbors_warp(LevelRange lr, const T* __restrict__ cx, const T* __restrict__ cy,
                                        const T* __restrict__ hl, const int* __restrict__ parent,
                                        const int* __restrict__ child0, const int* __restrict__ scnt, int* nbr,
                                        int* n_nbr, int* sil, int* n_sil, int* dil, int* n_dil, int* dstat) {
  int beg = 0, end = 0;
  lr.get(beg, end);
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int k = beg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < end; k += warps) {
    const int p = parent[k];
    const T h = hl[k], x = cx[k], y = cy[k];
    const int pc0 = child0[p];
    const int nq = 4 + 4 * n_nbr[p];
    int nn = 0, ns = 0, nd = 0, err = 0;
    for (int q0 = 0; q0 < nq; q0 += 32) {
      const int q = q0 + lane;
      int cat = 0, c = -1;  // 1 neighbour, 2 same-level interaction, 3 different-level interaction
      if (q < 4) {
        c = pc0 + q;
        if (scnt[c] != 0 && c != k) cat = 1;
      } else if (q < nq) {
        const int i = (q - 4) >> 2, j = (q - 4) & 3;
        const int nb = nbr[p * kMaxNeighbors + i];
        if (scnt[nb] != 0) {
          const int nc0 = child0[nb];
          if (nc0 < 0) {
            if (j == 0) {
              c = nb;
              cat = (double(xfabs(T(cx[nb] - x))) < 3.5 * double(h) && double(xfabs(T(cy[nb] - y))) < 3.5 * double(h))
                        ? 1
                        : 3;
            }
          } else {
            c = nc0 + j;
            if (scnt[c] != 0) cat = (xfabs(T(cx[c] - x)) < 3 * h && xfabs(T(cy[c] - y)) < 3 * h) ? 1 : 2;
          }
        }
      }
      const unsigned m1 = __ballot_sync(0xffffffffu, cat == 1);
      const unsigned m2 = __ballot_sync(0xffffffffu, cat == 2);
      const unsigned m3 = __ballot_sync(0xffffffffu, cat == 3);
      if (cat == 1) {
        const int pos = nn + __popc(m1 & below);
        if (pos < kMaxNeighbors) nbr[k * kMaxNeighbors + pos] = c;
        else err |= kErrNeighborOverflow;
      } else if (cat == 2) {
        const int pos = ns + __popc(m2 & below);
        if (pos < kMaxSameLevelIL) sil[k * kMaxSameLevelIL + pos] = c;
        else err |= kErrSameLevelOverflow;
      } else if (cat == 3) {
        const int pos = nd + __popc(m3 & below);
        if (pos < kMaxDiffLevelIL) dil[k * kMaxDiffLevelIL + pos] = c;
        else err |= kErrDiffLevelOverflow;
      }
      nn += __popc(m1);
      ns += __popc(m2);
      nd += __popc(m3);
    }
    err = __reduce_or_sync(0xffffffffu, unsigned(err));
    if (lane == 0) {
      n_nbr[k] = min(nn, kMaxNeighbors);
      n_sil[k] = min(ns, kMaxSameLevelIL);
      n_dil[k] = min(nd, kMaxDiffLevelIL);
      if (err) atomicOr(&dstat[1], err);
    }
  }
}

// Level bookkeeping of a build driven on the device: level l's nodes are
// off[l] .. off[l + 1]; lvl_n[l] is their count.
__global__ void tree_levels_init(int* off, int* lvl_n, int nlev, int roots, int* stop, int* dstat) {
  off[0] = 0;
  for (int l = 1; l <= nlev + 1; l++) off[l] = roots;
  lvl_n[0] = roots;
  for (int l = 1; l <= nlev; l++) lvl_n[l] = 0;
  *stop = 0;
  dstat[0] = dstat[1] = 0;
}

// After level l's split flags are scanned: the next level holds 4 children per
// split node. Running out of levels or of node capacity stops the build (the
// remaining level kernels see an empty range) and raises an error bit.
__global__ void tree_advance_level(int l, int nlev, int* off, int* lvl_n, const long long* __restrict__ nsplit_p,
                                   int node_cap, int* stop, int* dstat) {
  const int end = off[l + 1];
  long long nsplit = *stop ? 0 : *nsplit_p;
  if (nsplit > 0 && l == nlev - 1) {
    atomicOr(&dstat[1], kErrLevelOverflow);
    *stop = 1;
    nsplit = 0;
  }
  if (end + 4 * nsplit > node_cap) {
    atomicOr(&dstat[1], kErrNodeOverflow);
    *stop = 1;
    nsplit = 0;
  }
  off[l + 2] = end + int(4 * nsplit);
  lvl_n[l + 1] = int(4 * nsplit);
}

template <typename T, int NN>
bool wide_partition(TreeDev<T>& t, LevelRange lr, StarRec<T>* stars, int nstars, int nchunks, cudaStream_t s) {
  tree_wide_count<T, NN><<<nchunks, 256, 0, s>>>(lr, t.d_stop.p, t.split.p, t.cx.p, t.cy.p, t.sbeg.p, t.scnt.p, stars,
                                                nstars, t.chunk_cnt.p);
  tree_wide_offsets<NN><<<1, 256, 0, s>>>(lr, t.d_stop.p, t.split.p, t.child0.p, t.sbeg.p, t.scnt.p, nchunks,
                                          t.chunk_cnt.p);
  tree_wide_scatter<T, NN><<<nchunks, 256, 0, s>>>(lr, t.d_stop.p, t.split.p, t.cx.p, t.cy.p, t.sbeg.p, t.scnt.p,
                                                  stars, nstars, t.chunk_cnt.p, t.tmp_stars.p);
  tree_wide_copy<T, NN><<<std::min(nchunks * 4, 148 * 8), 256, 0, s>>>(lr, t.d_stop.p, nstars, t.tmp_stars.p, stars);
  return IRSB_CK(cudaGetLastError());
}

// Builds the tree over `stars` (device, permuted in place into tree order).
// Returns false on a CUDA error or a list overflow.
//
// The level loop runs on the device: every level kernel reads its node range
// from the device offsets (LevelRange) on a grid sized by the most nodes the
// level can hold (4^l), and the host reads the offsets back once per block of
// levels (the first block covers the depth a uniform field of this size
// reaches) instead of synchronising on every level. Node storage is reserved
// up front; a field that needs more restores its star order and builds again
// with twice the capacity.
template <typename T>
bool build_tree(TreeDev<T>& t, StarRec<T>* stars, int nstars, T root_hl, cudaStream_t s) {
  if (!t.tmp_stars.reserve(nstars, s) || !t.star_backup.reserve(nstars, s) || !t.dstat.reserve(2, s) ||
      !t.d_off.reserve(kMaxLevels + 2, s) || !t.d_lvl_n.reserve(kMaxLevels + 1, s) || !t.d_stop.reserve(1, s))
    return false;
  const int nchunks = std::max(1, ceil_div(nstars, kPartChunk));
  if (!t.chunk_cnt.reserve(size_t(nchunks) * 16, s)) return false;
  IRSB_CKR(cudaMemcpyAsync(t.star_backup.p, stars, size_t(nstars) * sizeof(StarRec<T>), cudaMemcpyDeviceToDevice, s));
  long long cap = std::max<long long>(t.cap, nstars + nstars / 2 + 1024);
  int depth = 1;  // levels of a uniform field: 4^depth >= nstars
  while (depth < kMaxLevels && (1LL << (2 * depth)) < nstars) depth++;
  const int G = 148 * 8;
  auto grid = [&](int l, int per_block) {
    const long long most = l >= 15 ? (1LL << 30) : (1LL << (2 * l));
    return int(std::max<long long>(1, std::min<long long>(ceil_div(most, (long long)per_block), G)));
  };
  std::vector<int> hoff(kMaxLevels + 2);
  t.launches = 0;
  for (int attempt = 0;; attempt++) {
    if (cap > (1LL << 28)) {
      std::fprintf(stderr, "Error. Tree needs more than %lld nodes.\n", 1LL << 28);
      return false;
    }
    if (!tree_reserve(t, int(cap), s) || !t.split.reserve(cap, s) || !t.rank.reserve(cap + 1, s) ||
        !scan_reserve(t.scan, cap, s))
      return false;
    if (attempt > 0)
      IRSB_CKR(cudaMemcpyAsync(stars, t.star_backup.p, size_t(nstars) * sizeof(StarRec<T>), cudaMemcpyDeviceToDevice,
                               s));
    tree_init_root<T><<<1, 1, 0, s>>>(t.cx.p, t.cy.p, t.hl.p, t.level.p, t.parent.p, t.child0.p, t.sbeg.p, t.scnt.p,
                                      t.rid.p, t.n_nbr.p, t.n_sil.p, t.n_dil.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p,
                                      root_hl, nstars);
    tree_levels_init<<<1, 1, 0, s>>>(t.d_off.p, t.d_lvl_n.p, kMaxLevels, 1, t.d_stop.p, t.dstat.p);
    IRSB_LAUNCH_CK("tree_init_root");
    t.launches += 2;
    int l = 0, levels = -1, err = 0, block = depth + 1;
    while (levels < 0 && l < kMaxLevels) {
      const int lend = std::min(kMaxLevels, l + block);
      for (; l < lend; l++) {
        const LevelRange lr{t.d_off.p, l}, next{t.d_off.p, l + 1};
        const int g1 = grid(l, 256);
        tree_near_count<<<g1, 256, 0, s>>>(0, 0, lr, t.scnt.p, t.nbr.p, t.n_nbr.p, t.split.p, t.dstat.p);
        if (!exclusive_scan_dev<int>(t.split.p, t.d_lvl_n.p + l, cap, t.rank.p, t.scan, s)) return false;
        tree_advance_level<<<1, 1, 0, s>>>(l, kMaxLevels, t.d_off.p, t.d_lvl_n.p, t.scan.sum.p, int(cap), t.d_stop.p,
                                           t.dstat.p);
        tree_make_children<T><<<g1, 256, 0, s>>>(0, 0, 0, lr, t.d_stop.p, t.split.p, t.rank.p, t.cx.p, t.cy.p, t.hl.p,
                                                 t.level.p, t.parent.p, t.child0.p, t.sbeg.p, t.scnt.p, t.rid.p,
                                                 t.n_nbr.p, t.n_sil.p, t.n_dil.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p);
        if (l == 0) {  // the root: every star, on many blocks
          if (!wide_partition<T, 1>(t, lr, stars, nstars, nchunks, s)) return false;
          t.launches += 3;
        } else if (l == 1) {  // the root's 4 children: every star
          if (!wide_partition<T, 4>(t, lr, stars, nstars, nchunks, s)) return false;
          t.launches += 3;
        } else if (l <= 3)  // a few nodes holding many stars each
          tree_partition_stars<T, 1024><<<grid(l, 1), 1024, 0, s>>>(0, 0, lr, t.d_stop.p, t.split.p, t.cx.p, t.cy.p,
                                                                      t.child0.p, t.sbeg.p, t.scnt.p, stars,
                                                                      t.tmp_stars.p);
        else
          tree_partition_stars<T><<<grid(l, 1), 256, 0, s>>>(0, 0, lr, t.d_stop.p, t.split.p, t.cx.p, t.cy.p,
                                                              t.child0.p, t.sbeg.p, t.scnt.p, stars, t.tmp_stars.p);
        tree_set_neighbors_warp<T><<<grid(l + 1, 8), 256, 0, s>>>(next, t.cx.p, t.cy.p, t.hl.p, t.parent.p,
                                                                  t.child0.p, t.scnt.p, t.nbr.p, t.n_nbr.p, t.sil.p,
                                                                  t.n_sil.p, t.dil.p, t.n_dil.p, t.dstat.p);
        IRSB_LAUNCH_CK("tree level");
        t.launches += 9;
      }
      int hst[2];
      IRSB_CKR(cudaMemcpyAsync(hoff.data(), t.d_off.p, hoff.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
      IRSB_CKR(cudaMemcpyAsync(hst, t.dstat.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      IRSB_CKR(cudaStreamSynchronize(s));
      err = hst[1];
      if (err) break;
      for (int k = 0; k < l; k++)
        if (hoff[k + 2] == hoff[k + 1]) {  // level k split nothing: its nodes are the last leaves
          levels = k;
          break;
        }
      block = 4;
    }
    if (err & kErrNodeOverflow) {
      cap *= 2;
      continue;
    }
    if (err & kErrLevelOverflow) {
      std::fprintf(stderr, "Error. Tree exceeded %d levels.\n", kMaxLevels);
      return false;
    }
    if (err) {
      std::fprintf(stderr, "Error. Tree neighbour/interaction list overflow (code %d).\n", err);
      return false;
    }
    if (levels < 0) {
      std::fprintf(stderr, "Error. Tree exceeded %d levels.\n", kMaxLevels);
      return false;
    }
    t.levels = levels;
    t.level_off.assign(hoff.begin(), hoff.begin() + levels + 2);
    t.num_nodes = t.level_off.back();
    return true;
  }
}

}  // namespace irsb
