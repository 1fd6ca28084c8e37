// Device memory helpers and a deterministic exclusive scan.
#pragma once
#include "common.cuh"

#include <vector>

namespace irsb {

// Owning device array with amortised growth (contents preserved on growth).
template <typename T>
struct DevVec {
  T* p = nullptr;
  size_t n = 0;    // logical size
  size_t cap = 0;  // allocated elements
  DevVec() = default;
  DevVec(const DevVec&) = delete;
  DevVec& operator=(const DevVec&) = delete;
  ~DevVec() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = cap = 0;
  }
  bool reserve(size_t want, cudaStream_t s) {
    if (want <= cap) return true;
    size_t nc = cap ? cap : 1;
    while (nc < want) nc *= 2;
    T* q = nullptr;
    if (!IRSB_CK(cudaMalloc(&q, nc * sizeof(T)))) return false;
    if (p && n) {
      if (!IRSB_CK(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, s))) {
        cudaFree(q);
        return false;
      }
      if (!IRSB_CK(cudaStreamSynchronize(s))) return false;
    }
    if (p) cudaFree(p);
    p = q;
    cap = nc;
    return true;
  }
  bool resize(size_t want, cudaStream_t s) {
    if (!reserve(want, s)) return false;
    n = want;
    return true;
  }
  // exact-size allocation without preserving contents
  bool alloc_exact(size_t want) {
    if (want <= cap) {
      n = want;
      return true;
    }
    release();
    if (want == 0) return true;
    if (!IRSB_CK(cudaMalloc(&p, want * sizeof(T)))) return false;
    cap = want;
    n = want;
    return true;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Pinned host buffer.
template <typename T>
struct HostVec {
  T* p = nullptr;
  size_t n = 0;
  HostVec() = default;
  HostVec(const HostVec&) = delete;
  HostVec& operator=(const HostVec&) = delete;
  ~HostVec() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  bool alloc(size_t want) {
    if (want == n && p) return true;
    release();
    if (want == 0) return true;
    if (!IRSB_CK(cudaMallocHost(&p, want * sizeof(T)))) return false;
    n = want;
    return true;
  }
};

// ---------------------------------------------------------------- scan
// Exclusive prefix sum of n values (int or long long input), written as long
// long. Three passes: per-block totals, a single-block scan of the totals, and
// a per-block local scan plus offset. Deterministic (integer arithmetic).
constexpr int kScanBlock = 512;
constexpr int kScanItems = 4;  // per thread
constexpr int kScanTile = kScanBlock * kScanItems;

template <typename In>
__global__ void scan_block_totals(const In* __restrict__ in, long long n, const int* __restrict__ dn,
                                  long long* __restrict__ totals) {
  __shared__ long long red[kScanBlock / 32];
  if (dn) n = *dn;
  long long base = (long long)blockIdx.x * kScanTile;
  long long s = 0;
  for (int k = 0; k < kScanItems; k++) {
    long long i = base + (long long)k * kScanBlock + threadIdx.x;
    if (i < n) s += (long long)in[i];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    long long v = threadIdx.x < kScanBlock / 32 ? red[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) totals[blockIdx.x] = v;
  }
}

// Single block: in-place exclusive scan of `totals` (m entries), grand total to *sum.
__global__ void scan_totals_single(long long* __restrict__ totals, long long m, long long* __restrict__ sum) {
  __shared__ long long warp_sums[kScanBlock / 32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long start = 0; start < m; start += kScanBlock) {
    long long i = start + threadIdx.x;
    long long v = i < m ? totals[i] : 0;
    long long x = v;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
      long long ws = lane < kScanBlock / 32 ? warp_sums[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o) ws += y;
      }
      if (lane < kScanBlock / 32) warp_sums[lane] = ws;
    }
    __syncthreads();
    long long incl = x + (w > 0 ? warp_sums[w - 1] : 0) + carry;
    if (i < m) totals[i] = incl - v;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry = incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *sum = carry;
}

template <typename In>
__global__ void scan_block_apply(const In* __restrict__ in, long long n, const int* __restrict__ dn,
                                 const long long* __restrict__ offsets, long long* __restrict__ out) {
  __shared__ long long warp_sums[kScanBlock / 32];
  if (dn) n = *dn;
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = offsets[blockIdx.x];
  __syncthreads();
  long long base = (long long)blockIdx.x * kScanTile;
  for (int k = 0; k < kScanItems; k++) {
    long long i = base + (long long)k * kScanBlock + threadIdx.x;
    long long v = i < n ? (long long)in[i] : 0;
    long long x = v;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
      long long ws = lane < kScanBlock / 32 ? warp_sums[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o) ws += y;
      }
      if (lane < kScanBlock / 32) warp_sums[lane] = ws;
    }
    __syncthreads();
    long long incl = x + (w > 0 ? warp_sums[w - 1] : 0) + carry;
    if (i < n) out[i] = incl - v;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry = incl;
    __syncthreads();
  }
}

struct ScanScratch {
  DevVec<long long> totals;
  DevVec<long long> sum;
};

// out[i] = sum_{j<i} in[j]; *d_sum (device) receives the grand total.
template <typename In>
bool exclusive_scan(const In* in, long long n, long long* out, ScanScratch& sc, cudaStream_t s) {
  long long nb = (n + kScanTile - 1) / kScanTile;
  if (nb < 1) nb = 1;
  if (!sc.totals.reserve(size_t(nb), s)) return false;
  if (!sc.sum.reserve(1, s)) return false;
  scan_block_totals<In><<<unsigned(nb), kScanBlock, 0, s>>>(in, n, nullptr, sc.totals.p);
  scan_totals_single<<<1, kScanBlock, 0, s>>>(sc.totals.p, nb, sc.sum.p);
  scan_block_apply<In><<<unsigned(nb), kScanBlock, 0, s>>>(in, n, nullptr, sc.totals.p, out);
  return IRSB_CK(cudaGetLastError());
}

// The same with the element count read on the device from *dn (at most
// n_cap), for work whose size the host does not know (graph-captured
// pipelines). The scratch must already hold the blocks for n_cap.
template <typename In>
bool exclusive_scan_dev(const In* in, const int* dn, long long n_cap, long long* out, ScanScratch& sc,
                        cudaStream_t s) {
  long long nb = (n_cap + kScanTile - 1) / kScanTile;
  if (nb < 1) nb = 1;
  scan_block_totals<In><<<unsigned(nb), kScanBlock, 0, s>>>(in, n_cap, dn, sc.totals.p);
  scan_totals_single<<<1, kScanBlock, 0, s>>>(sc.totals.p, nb, sc.sum.p);
  scan_block_apply<In><<<unsigned(nb), kScanBlock, 0, s>>>(in, n_cap, dn, sc.totals.p, out);
  return IRSB_CK(cudaGetLastError());
}

inline bool scan_reserve(ScanScratch& sc, long long n_cap, cudaStream_t s) {
  long long nb = (n_cap + kScanTile - 1) / kScanTile;
  return sc.totals.reserve(size_t(nb < 1 ? 1 : nb), s) && sc.sum.reserve(1, s);
}

template <typename T>
__global__ void fill_kernel(T* p, long long n, T v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace irsb
