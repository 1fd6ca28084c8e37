// Host shim that lets the reference's CUDA headers compile as ordinary C++ so
// that its own device functions and kernel bodies run on the CPU (test
// infrastructure only). Kernels become plain functions; a launch is emulated
// by setting the thread-local grid coordinates below and calling the function,
// so each grid-stride loop in a kernel visits its share of the iterations.
#pragma once
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

// CUDA device code calls the unqualified math names
using std::isnan;
using std::isinf;

#define __host__
#define __device__
#define __global__
#define __shared__
#define __forceinline__ inline

struct dim3 {
  unsigned x, y, z;
  dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct shim_uint3 {
  unsigned x = 0, y = 0, z = 0;
};
extern thread_local shim_uint3 threadIdx, blockIdx;
extern thread_local dim3 blockDim, gridDim;
inline void __syncthreads() {}

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline const char* cudaGetErrorString(cudaError_t) { return "host shim"; }
struct cudaDeviceProp {
  char name[256];
  int major, minor, clockRate, memoryClockRate, memoryBusWidth, singleToDoublePrecisionPerfRatio;
  size_t totalGlobalMem, sharedMemPerMultiprocessor, sharedMemPerBlock;
  int multiProcessorCount, maxBlocksPerMultiProcessor, maxThreadsPerMultiProcessor, maxThreadsPerBlock, warpSize;
  int maxThreadsDim[3], maxGridSize[3];
};
inline cudaError_t cudaGetDevice(int* d) {
  *d = 0;
  return cudaSuccess;
}
inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int) {
  std::memset(p, 0, sizeof(*p));
  p->maxThreadsPerBlock = 1024;
  p->multiProcessorCount = 1;
  return cudaSuccess;
}
template <typename T>
inline cudaError_t cudaMallocManaged(T** p, size_t n) {
  *p = static_cast<T*>(std::calloc(1, n ? n : 1));
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}

// integer min / max of the device math library
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }

// atomics (real atomics: emulated launches may run on several host threads)
template <typename T, typename U>
inline T atomicAdd(T* a, U v) {
  return std::atomic_ref<T>(*a).fetch_add(static_cast<T>(v));
}
template <typename T, typename U>
inline T atomicSub(T* a, U v) {
  return std::atomic_ref<T>(*a).fetch_sub(static_cast<T>(v));
}
template <typename T, typename U>
inline T atomicMin(T* a, U v) {
  std::atomic_ref<T> r(*a);
  T old = r.load();
  while (static_cast<T>(v) < old && !r.compare_exchange_weak(old, static_cast<T>(v))) {
  }
  return old;
}
template <typename T, typename U>
inline T atomicExch(T* a, U v) {
  return std::atomic_ref<T>(*a).exchange(static_cast<T>(v));
}
template <typename T, typename U>
inline T atomicMax(T* a, U v) {
  std::atomic_ref<T> r(*a);
  T old = r.load();
  while (static_cast<T>(v) > old && !r.compare_exchange_weak(old, static_cast<T>(v))) {
  }
  return old;
}
