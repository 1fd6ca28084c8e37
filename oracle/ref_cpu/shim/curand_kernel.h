// Declarations only: the host build of the reference headers never draws
// random numbers (star fields are passed in).
#pragma once
struct curandState {
  int unused;
};
inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState*) {}
inline double curand_uniform_double(curandState*) { return 0.0; }
