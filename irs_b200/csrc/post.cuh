// Post-pass over the finished maps: ray totals, value ranges and histograms.
//
// Reference behaviour (include/ipm.cuh:950-1120, include/irs.cuh:930-1028,
// include/array_functions.cuh:114-160): IRS histograms count pixels per ray
// count; IPM histograms bin round(mu * 1000) and round(log10(mu) * 1000),
// offset by the minimum bin. Ranges come from a min/max over the map; sums and
// ranges here are integer reductions, so they are deterministic.
#pragma once
#include "common.cuh"
#include "devutil.cuh"

#include <type_traits>

namespace irsb {

// Total of an int map (num_rays_received, include/irs.cuh:934-935).
__global__ void sum_int_map(const int* __restrict__ v, long long n, unsigned long long* out) {
  unsigned long long s = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    s += (unsigned long long)v[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// min / max of non-negative values through their ordered integer encodings.
template <typename V>
struct OrderedKey;
template <>
struct OrderedKey<int> {
  using K = int;
  static __device__ __forceinline__ K enc(int v) { return v; }
};
template <>
struct OrderedKey<float> {
  using K = int;
  static __device__ __forceinline__ K enc(float v) { return __float_as_int(v); }
};
template <>
struct OrderedKey<double> {
  using K = long long;
  static __device__ __forceinline__ K enc(double v) { return __double_as_longlong(v); }
};

template <typename V>
__global__ void minmax_nonneg(const V* __restrict__ v, long long n, typename OrderedKey<V>::K* out) {
  using K = typename OrderedKey<V>::K;
  K lo = OrderedKey<V>::enc(v[0]), hi = lo;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    K e = OrderedKey<V>::enc(v[k]);
    lo = e < lo ? e : lo;
    hi = e > hi ? e : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    K a = __shfl_down_sync(0xffffffffu, lo, o), b = __shfl_down_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], lo);
    atomicMax(&out[1], hi);
  }
}

// histogram[round(v * factor - hmin)]++ ; log form uses log10(v). Values whose
// bin falls outside [0, len) (log10 of an empty pixel) are not counted.
template <typename V>
__device__ __forceinline__ long long hist_bin(V v, int hmin, int len, int factor, int use_log) {
  double x;
  if constexpr (std::is_floating_point<V>::value) {
    if (use_log) {
      V lv = log10(v);
      x = round(double(V(lv * factor - hmin)));
    } else {
      x = round(1.0 * v * factor - hmin);
    }
  } else {
    x = round(1.0 * v * factor - hmin);
  }
  return (x >= 0 && x < len) ? (long long)x : -1;
}

// One warp-uniform pass over the map: lanes that fall in the same bin are
// matched (neighbouring pixels mostly do) and their leader adds their count
// with one atomic.
template <typename V, typename Add>
__device__ __forceinline__ void hist_pass(const V* __restrict__ v, long long n, int hmin, int len, int factor,
                                          int use_log, Add add) {
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (blockIdx.x * (long long)blockDim.x + threadIdx.x) - lane; base < n; base += stride) {
    const long long k = base + lane;
    const long long b = k < n ? hist_bin<V>(v[k], hmin, len, factor, use_log) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    if (b >= 0 && lane == __ffs(peers) - 1) add(b, __popc(peers));
  }
}

template <typename V>
__global__ void histogram_map(const V* __restrict__ v, long long n, int hmin, int len, int factor, int use_log,
                              int* __restrict__ hist) {
  hist_pass<V>(v, n, hmin, len, factor, use_log, [&](long long b, int c) { atomicAdd(&hist[b], c); });
}

// The same for histograms of at most kHistSmemBins bins: each block counts in
// shared memory, then adds its non-zero bins to the global histogram.
constexpr int kHistSmemBins = 12288;
template <typename V>
__global__ void histogram_map_smem(const V* __restrict__ v, long long n, int hmin, int len, int factor,
                                   int use_log, int* __restrict__ hist) {
  extern __shared__ int sh[];
  for (int i = threadIdx.x; i < len; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  hist_pass<V>(v, n, hmin, len, factor, use_log, [&](long long b, int c) { atomicAdd(&sh[b], c); });
  __syncthreads();
  for (int i = threadIdx.x; i < len; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

}  // namespace irsb
