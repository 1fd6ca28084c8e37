// Star-field generation on the device.
//
// Same draw protocol as the reference (include/star.cuh:40-107): star i owns
// the curand XORWOW sequence (seed, subsequence i, offset 0); a rectangular
// field takes two uniform doubles for x1 and x2 in [-corner, corner]; a
// circular field takes an angle U*2pi and a radius sqrt(U)*|corner|; the mass
// is then drawn from the mass function with one more uniform double. The curand
// state lives in registers only (the reference keeps one state per star in
// global memory; the draws are the same).
#pragma once
#include "common.cuh"
#include "massfn.cuh"
#include "params.hpp"

#include <curand_kernel.h>

namespace irsb {

template <typename T>
__global__ void __launch_bounds__(256) generate_stars_kernel(StarRec<T>* __restrict__ stars, int n, int seed,
                                                             int rectangular, cplx<T> corner, int mf_kind,
                                                             T m_lower, T m_upper, T m_solar) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    curandState st;
    curand_init((unsigned long long)seed, (unsigned long long)i, 0ULL, &st);
    T x1, x2;
    if (rectangular) {
      x1 = T(curand_uniform_double(&st) * 2 * corner.re - corner.re);
      x2 = T(curand_uniform_double(&st) * 2 * corner.im - corner.im);
    } else {
      T a = T(curand_uniform_double(&st) * 2 * kPi<T>);
      T r = T(sqrt(curand_uniform_double(&st)) * cabs_(corner));
      x1 = r * xcos(a);
      x2 = r * xsin(a);
    }
    T p = T(curand_uniform_double(&st));
    StarRec<T> s;
    s.x = x1;
    s.y = x2;
    s.m = mf_mass<T>(mf_kind, p, m_lower, m_upper, m_solar);
    stars[i] = s;
  }
}

}  // namespace irsb
