// Shared definitions for the irs_b200 microlensing map engine (sm_100a).
//
// Complex arithmetic, CUDA error plumbing and the tree constants that fix the
// behaviour of the reference quadtree (include/tree_node.cuh:14-25 of
// weisluke/irs): a node is refined while it and its neighbours hold more than
// 32 stars, expansions carry at most 31 terms, and a node has 4 children.
#pragma once

#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>

namespace irsb {

constexpr int kMaxStarsDirect = 32;     // tree_node.cuh:14
constexpr int kMaxOrder = 31;           // tree_node.cuh:20
constexpr int kChildren = 4;            // tree_node.cuh:22
constexpr int kMaxNeighbors = 8;        // tree_node.cuh:23
constexpr int kMaxSameLevelIL = 27;     // tree_node.cuh:24
constexpr int kMaxDiffLevelIL = 5;      // tree_node.cuh:25
constexpr int kMaxLevels = 40;          // guard on the refinement loop

// Fixed point used by the IPM deposit: one unit of pixel area is 2^32.
constexpr double kFixScale = 4294967296.0;
constexpr double kFixInv = 1.0 / 4294967296.0;

// Error codes written by device code into a status word.
enum DeviceError : int {
  kErrNone = 0,
  kErrNeighborOverflow = 1,
  kErrSameLevelOverflow = 2,
  kErrDiffLevelOverflow = 4,
  kErrNearOverflow = 8,
  kErrTableOverflow = 16,   // lattice tile table capacity (graph-captured pipelines)
  kErrNodeOverflow = 32,    // node capacity (graph-captured pipelines)
  kErrLevelOverflow = 64,   // more tree levels than the captured build holds
};

#define IRSB_HD __host__ __device__ __forceinline__

// Math wrappers: std:: overloads in host code, CUDA overloads in device code,
// so that float arguments use the float functions on both sides.
#ifdef __CUDA_ARCH__
#define IRSB_MATH1(name) \
  template <typename T> IRSB_HD T x##name(T a) { return ::name(a); }
#define IRSB_MATH2(name) \
  template <typename T> IRSB_HD T x##name(T a, T b) { return ::name(a, b); }
#else
#define IRSB_MATH1(name) \
  template <typename T> IRSB_HD T x##name(T a) { return std::name(a); }
#define IRSB_MATH2(name) \
  template <typename T> IRSB_HD T x##name(T a, T b) { return std::name(a, b); }
#endif
IRSB_MATH1(log)
IRSB_MATH1(exp)
IRSB_MATH1(cos)
IRSB_MATH1(sin)
IRSB_MATH1(sqrt)
IRSB_MATH1(fabs)
IRSB_MATH2(pow)
IRSB_MATH2(hypot)
IRSB_MATH2(atan2)

template <typename T>
struct cplx {
  T re, im;
};

template <typename T>
IRSB_HD cplx<T> mk(T re, T im) {
  cplx<T> c;
  c.re = re;
  c.im = im;
  return c;
}
template <typename T>
IRSB_HD cplx<T> cadd(cplx<T> a, cplx<T> b) { return mk<T>(a.re + b.re, a.im + b.im); }
template <typename T>
IRSB_HD cplx<T> csub(cplx<T> a, cplx<T> b) { return mk<T>(a.re - b.re, a.im - b.im); }
template <typename T>
IRSB_HD cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mk<T>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
IRSB_HD cplx<T> cscale(cplx<T> a, T s) { return mk<T>(a.re * s, a.im * s); }
template <typename T>
IRSB_HD cplx<T> cconj(cplx<T> a) { return mk<T>(a.re, -a.im); }
template <typename T>
IRSB_HD cplx<T> cneg(cplx<T> a) { return mk<T>(-a.re, -a.im); }

// Complex quotient a / b by Smith's algorithm (R. L. Smith, CACM 5, 1962),
// which avoids overflow in |b|^2.
template <typename T>
IRSB_HD cplx<T> cdiv(cplx<T> a, cplx<T> b) {
  if (xfabs(b.im) < xfabs(b.re)) {
    T f = b.im / b.re;
    T d = b.re + b.im * f;
    return mk<T>((a.re + a.im * f) / d, (a.im - a.re * f) / d);
  } else {
    T f = b.re / b.im;
    T d = b.re * f + b.im;
    return mk<T>((a.re * f + a.im) / d, (a.im * f - a.re) / d);
  }
}
template <typename T>
IRSB_HD cplx<T> cdivr(cplx<T> a, T s) { return mk<T>(a.re / s, a.im / s); }

template <typename T>
IRSB_HD T cabs_(cplx<T> a) { return xhypot(a.re, a.im); }
template <typename T>
IRSB_HD T carg(cplx<T> a) { return xatan2(a.im, a.re); }
template <typename T>
IRSB_HD cplx<T> clog_(cplx<T> a) { return mk<T>(xlog(cabs_(a)), carg(a)); }
template <typename T>
IRSB_HD cplx<T> cexp_(cplx<T> a) {
  T e = xexp(a.re);
  return mk<T>(e * xcos(a.im), e * xsin(a.im));
}
// Integer power by repeated multiplication starting from 1.
template <typename T>
IRSB_HD cplx<T> cpowi(cplx<T> a, int n) {
  cplx<T> r = mk<T>(T(1), T(0));
  for (int i = 0; i < n; i++) r = cmul(r, a);
  return r;
}

inline bool cuda_ok(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "CUDA error in %s at %s:%d: %s (%d)\n", what, file, line,
                 cudaGetErrorString(e), int(e));
    return false;
  }
  return true;
}
#define IRSB_CK(call) cuda_ok((call), #call, __FILE__, __LINE__)
#define IRSB_CKR(call)                          \
  do {                                          \
    if (!IRSB_CK(call)) return false;           \
  } while (0)
#define IRSB_LAUNCH_CK(name)                                          \
  do {                                                                \
    if (!cuda_ok(cudaGetLastError(), name, __FILE__, __LINE__)) return false; \
  } while (0)

inline int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }

}  // namespace irsb
