// Critical curves and caustics of a star field (CCF).
//
// Semantics of the reference (include/ccf_functions.cuh, include/ccf.cuh):
// the critical curves are the roots z(phi) of the parametric equation
//   f0(z, phi) = gamma - conj(d alpha_star / d zbar) - conj(d alpha_local / d zbar)
//                - conj(d alpha_smooth / d zbar) - (1 - kappa - d alpha_smooth / dz) e^{-i phi}
// (ccf_functions.cuh:69-85), followed in phi from the centre of each branch
// outwards in both directions (ccf.cuh:979-1037). Every root moves by the
// simultaneous Newton step with pole and root repulsion terms
//   z <- z - f0 / (f1 + f0 (2 sum_stars 1/(z - z_i) - sum_{k != j} 1/(z - z_k)))
// with f1 = d f0 / dz (ccf_functions.cuh:196-253); a root is final once a step
// moves it by less than 1e-9 theta_star (ccf_functions.cuh:367-372), or when
// the 1/mu bound at it is already below 1e-9 (:205-210). Caustics are the lens
// equation at the roots (:499-513); magnification length scales follow
// mu_length_scale (:145-166).
//
// How, differently by design:
//   * one warp per (chain, root), a chain being one side of one branch: the
//     lanes split the near-field stars and the O(N) sums over all stars and
//     over the chain's roots, then reduce them in a fixed order; FP64
//     throughout;
//   * the update is a Jacobi step (all roots read the previous iterate from
//     one buffer and write the next to another) instead of the reference's
//     in-place update, whose result depends on thread timing; the roots, their
//     order and every output are deterministic;
//   * the near field and the local expansion come from the leaf records of
//     the lens-equation kernels (near64, coef64 = k c_k); a point outside the
//     root box takes the direct sum over all stars, as get_nearest_node
//     returns the root there (tree_node.cuh:535-539);
//   * a final root costs its warp one load and one store.
#pragma once
#include "leaves.cuh"
#include "shoot.cuh"  // LeafPtrs
#include "smooth.cuh"

namespace irsb {

constexpr int kCcfThreads = 256;

struct CcfParams {
  double kappa, gamma, kstar, theta2, inv_pi;
  int rect, approx, taylor_smooth, p;
  double corner_re, corner_im;
  double root_hl;  // half length of the tree's root box (centre 0)
  int nstars, nroots, nphi, nbranches;
};

// Row of the root array holding phi step j (signed) of branch c: the centre
// of branch c is row nphi / (2 nb) + c (nphi / nb + 1) (ccf_functions.cuh:355).
__host__ __device__ __forceinline__ int ccf_row(const CcfParams& P, int c, int j) {
  return P.nphi / (2 * P.nbranches) + c * (P.nphi / P.nbranches) + c + j;
}
__host__ __device__ __forceinline__ double ccf_phi(const CcfParams& P, int c, int j) {
  const double pi = 3.14159265358979323846;
  return pi / P.nbranches + c * 2 * pi / P.nbranches + 2 * pi / P.nphi * j;
}

// Near-field sums and local-expansion Horner values at z:
//   s1 = sum m / (z - z_i), s2 = sum m / (z - z_i)^2, s3 = sum m / (z - z_i)^3
//   a0 = sum_k k c_k dz^(k-1), a1 = sum_k k (k-1) c_k dz^(k-2),
//   a2 = sum_k k (k-1) (k-2) c_k dz^(k-3), dz = (z - centre) / hl
struct CcfField {
  cplx<double> s1, s2, s3, a0, a1, a2;
  double hl;
};

__device__ __forceinline__ void ccf_add_star(CcfField& f, cplx<double> z, double sx, double sy, double m) {
  const cplx<double> d = mk(z.re - sx, z.im - sy);
  const double inv = 1.0 / (d.re * d.re + d.im * d.im);
  const cplx<double> r = mk(d.re * inv, -d.im * inv);  // 1 / d
  const cplx<double> r2 = cmul(r, r), r3 = cmul(r2, r);
  f.s1 = cadd(f.s1, cscale(r, m));
  f.s2 = cadd(f.s2, cscale(r2, m));
  f.s3 = cadd(f.s3, cscale(r3, m));
}

template <typename T>
__device__ __forceinline__ CcfField ccf_field(const CcfParams& P, const LeafPtrs& lp, const DescentPtrs<T>& dp,
                                              const StarRec<T>* __restrict__ stars, cplx<double> z) {
  CcfField f;
  f.s1 = f.s2 = f.s3 = f.a0 = f.a1 = f.a2 = mk(0.0, 0.0);
  f.hl = 1.0;
  if (fabs(z.re) > P.root_hl || fabs(z.im) > P.root_hl) {
    // outside the root box: the root node, i.e. every star and no expansion
    for (int i = 0; i < P.nstars; i++) ccf_add_star(f, z, double(stars[i].x), double(stars[i].y), double(stars[i].m));
    return f;
  }
  const int leaf = descend_leaf(dp, z.re, z.im);
  const int nn = lp.nnear[leaf];
  const double4* near = lp.near64 + (size_t)leaf * kMaxStarsDirect;
  for (int s = 0; s < nn; s++) {
    const double4 st = near[s];
    ccf_add_star(f, z, st.x, st.y, st.z);
  }
  f.hl = lp.hl[leaf];
  const cplx<double> dz = mk((z.re - lp.cx[leaf]) / f.hl, (z.im - lp.cy[leaf]) / f.hl);
  const double2* coef = lp.coef64 + (size_t)leaf * kMaxOrder;
  for (int k = P.p; k >= 1; k--) {
    const double2 c = coef[k - 1];  // k c_k
    f.a0 = cadd(cmul(f.a0, dz), mk(c.x, c.y));
    if (k >= 2) f.a1 = cadd(cmul(f.a1, dz), mk(c.x * (k - 1), c.y * (k - 1)));
    if (k >= 3) f.a2 = cadd(cmul(f.a2, dz), mk(c.x * ((k - 1) * (k - 2)), c.y * ((k - 1) * (k - 2))));
  }
  return f;
}

// Derivatives of the lens mapping at z: dw/dz (real) and dw/dzbar, and
// d2w/dzbar2 (ccf_functions.cuh:145-166 names).
struct CcfDerivs {
  double dwdz;
  cplx<double> dwdzb, d2wdzb2;
};

__device__ __forceinline__ CcfDerivs ccf_derivs(const CcfParams& P, const CcfField& f, cplx<double> z) {
  const cplx<double> corner = mk(P.corner_re, P.corner_im);
  const double t2 = P.theta2;
  // d alpha_star / d zbar = conj(-theta^2 s2); d2 alpha_star / d zbar2 = conj(2 theta^2 s3)
  const cplx<double> das = cconj(cscale(f.s2, -t2)), d2as = cconj(cscale(f.s3, 2.0 * t2));
  const cplx<double> dal = cconj(cscale(f.a1, t2 / (f.hl * f.hl)));
  const cplx<double> d2al = cconj(cscale(f.a2, t2 / (f.hl * f.hl * f.hl)));
  const double dsz = d_alpha_smooth_dz_(z, P.kstar, P.rect, corner, P.approx);
  const cplx<double> dszb = d_alpha_smooth_dzbar_(z, P.kstar, P.rect, corner, P.approx, P.taylor_smooth, P.inv_pi);
  const cplx<double> d2szb = d2_alpha_smooth_dzbar2_(z, P.kstar, P.rect, corner, P.approx, P.taylor_smooth, P.inv_pi);
  CcfDerivs d;
  d.dwdz = 1.0 - P.kappa - dsz;
  d.dwdzb = csub(csub(csub(mk(P.gamma, 0.0), das), dal), dszb);
  d.d2wdzb2 = cneg(cadd(cadd(d2as, d2al), d2szb));
  return d;
}

// f0 = conj(dw/dzbar) - dw/dz e^{-i phi} (the reference's parametric form:
// gamma is real, so gamma - conj(...) = conj(dw/dzbar)).
__device__ __forceinline__ cplx<double> ccf_f0(const CcfDerivs& d, double phi) {
  return csub(cconj(d.dwdzb), mk(d.dwdz * cos(phi), -d.dwdz * sin(phi)));
}

// Largest possible error in 1/mu at a point where f0 has modulus |f0|
// (ccf_functions.cuh:205-210, :455-461).
__device__ __forceinline__ double ccf_inv_mu_bound(double af0, double dwdz) {
  return fmax(fabs(af0 * (af0 + 2 * dwdz)), fabs(af0 * (af0 - 2 * dwdz)));
}

__device__ __forceinline__ cplx<double> recip(cplx<double> d) {
  const double inv = 1.0 / (d.re * d.re + d.im * d.im);
  return mk(d.re * inv, -d.im * inv);
}

// sum over k = lane, lane + 32, ... < n, k != skip, of 1 / (z - p[k]): four
// independent accumulators (four reciprocals in flight per lane), added in a
// fixed order.
__device__ __forceinline__ cplx<double> lane_recip_sum(const double2* __restrict__ p, int n, cplx<double> z,
                                                       int skip, int lane) {
  cplx<double> acc[4];
#pragma unroll
  for (int u = 0; u < 4; u++) acc[u] = mk(0.0, 0.0);
  int i = lane;
  for (; i + 96 < n; i += 128) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = i + 32 * u;
      const double2 w = p[k];
      const cplx<double> r = recip(mk(z.re - w.x, z.im - w.y));
      if (k != skip) acc[u] = cadd(acc[u], r);
    }
  }
  for (; i < n; i += 32) {
    const double2 w = p[i];
    const cplx<double> r = recip(mk(z.re - w.x, z.im - w.y));
    if (i != skip) acc[0] = cadd(acc[0], r);
  }
  return cadd(cadd(acc[0], acc[1]), cadd(acc[2], acc[3]));
}

__device__ __forceinline__ cplx<double> warp_sum(cplx<double> v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.re += __shfl_xor_sync(0xffffffffu, v.re, o);
    v.im += __shfl_xor_sync(0xffffffffu, v.im, o);
  }
  return v;
}

// ccf_field with the work of one root spread over a warp: lane l takes the
// near-field stars l, l + 32, ... (one each for a leaf's <= 32) and the
// partial sums meet in a butterfly reduction (fixed order: deterministic);
// every lane then evaluates the local expansion (the same dz) itself.
template <typename T>
__device__ __forceinline__ CcfField ccf_field_warp(const CcfParams& P, const LeafPtrs& lp, const DescentPtrs<T>& dp,
                                                   const StarRec<T>* __restrict__ stars, cplx<double> z, int lane) {
  CcfField f;
  f.s1 = f.s2 = f.s3 = f.a0 = f.a1 = f.a2 = mk(0.0, 0.0);
  f.hl = 1.0;
  const bool outside = fabs(z.re) > P.root_hl || fabs(z.im) > P.root_hl;
  int leaf = 0;
  if (outside) {  // the root node: every star, no expansion
    for (int i = lane; i < P.nstars; i += 32) ccf_add_star(f, z, double(stars[i].x), double(stars[i].y), double(stars[i].m));
  } else {
    leaf = descend_leaf(dp, z.re, z.im);
    const int nn = lp.nnear[leaf];
    if (lane < nn) {
      const double4 st = lp.near64[(size_t)leaf * kMaxStarsDirect + lane];
      ccf_add_star(f, z, st.x, st.y, st.z);
    }
  }
  f.s1 = warp_sum(f.s1);
  f.s2 = warp_sum(f.s2);
  f.s3 = warp_sum(f.s3);
  if (outside) return f;
  f.hl = lp.hl[leaf];
  const cplx<double> dz = mk((z.re - lp.cx[leaf]) / f.hl, (z.im - lp.cy[leaf]) / f.hl);
  const double2* coef = lp.coef64 + (size_t)leaf * kMaxOrder;
  for (int k = P.p; k >= 1; k--) {
    const double2 c = coef[k - 1];  // k c_k
    f.a0 = cadd(cmul(f.a0, dz), mk(c.x, c.y));
    if (k >= 2) f.a1 = cadd(cmul(f.a1, dz), mk(c.x * (k - 1), c.y * (k - 1)));
    if (k >= 3) f.a2 = cadd(cmul(f.a2, dz), mk(c.x * ((k - 1) * (k - 2)), c.y * ((k - 1) * (k - 2))));
  }
  return f;
}

// One Jacobi step for chains [0, nchains): chain ch is branch ch / sides,
// side (ch % sides) (0: phi decreasing, 1: increasing; sides = 1 at j = 0,
// where both sides start from the branch centre). Positions are read from
// `src` (rows of the root array, or the chain's scratch row) and written to
// `dst`; fin[ch][a] marks final roots, which are copied. One warp per root:
// the lanes split the sums over all stars (their positions `spos`, in tree
// order) and over the chain's other roots (strided, so a warp reads 32
// consecutive positions at a time; both arrays stay in L1) and reduce them in
// a fixed order.
template <typename T>
__global__ void __launch_bounds__(kCcfThreads) ccf_iterate(CcfParams P, LeafPtrs lp, DescentPtrs<T> dp,
                                                           const StarRec<T>* __restrict__ stars,
                                                           const double2* __restrict__ spos, int j, int sides,
                                                           int from_scratch, double2* __restrict__ roots,
                                                           double2* __restrict__ scratch,
                                                           unsigned char* __restrict__ fin) {
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.y;
  const int c = ch / sides, side = ch % sides;
  const int sj = side == 0 ? -j : j;
  const int a = blockIdx.x * (kCcfThreads / 32) + (threadIdx.x >> 5);  // root of this warp
  if (a >= P.nroots) return;                                           // whole warps only
  const double2* src = from_scratch ? scratch + (size_t)ch * P.nroots : roots + (size_t)ccf_row(P, c, sj) * P.nroots;
  double2* dst = from_scratch ? roots + (size_t)ccf_row(P, c, sj) * P.nroots : scratch + (size_t)ch * P.nroots;
  unsigned char* fn = fin + (size_t)ch * P.nroots;
  const double2 z2 = src[a];
  const cplx<double> z = mk(z2.x, z2.y);
  if (fn[a]) {
    if (lane == 0) dst[a] = z2;
    return;
  }
  const CcfField f = ccf_field_warp(P, lp, dp, stars, z, lane);
  const CcfDerivs d = ccf_derivs(P, f, z);
  const cplx<double> f0 = ccf_f0(d, ccf_phi(P, c, sj));
  if (ccf_inv_mu_bound(cabs_(f0), d.dwdz) < 1e-9) {  // already a root to the precision sought: final
    __syncwarp();
    if (lane == 0) {
      fn[a] = 1;
      dst[a] = z2;
    }
    return;
  }
  const cplx<double> f1 = cconj(d.d2wdzb2);  // d f0 / dz
  cplx<double> ps = warp_sum(lane_recip_sum(spos, P.nstars, z, -1, lane));
  cplx<double> rs = warp_sum(lane_recip_sum(src, P.nroots, z, a, lane));
  if (lane != 0) return;
  if (!P.rect && !P.approx) ps = cadd(ps, recip(z));
  ps = cscale(ps, 2.0);
  const cplx<double> den = cadd(f1, cmul(f0, csub(ps, rs)));
  const cplx<double> zn = csub(z, cdiv(f0, den));
  if (cabs_(csub(zn, z)) / sqrt(P.theta2) < 1e-9) fn[a] = 1;
  dst[a] = make_double2(zn.re, zn.im);
}

// Step j of every chain starts from step j - 1 (ccf_functions.cuh:268-301);
// the final flags are reset.
__global__ void ccf_prepare(CcfParams P, int j, double2* __restrict__ roots, unsigned char* __restrict__ fin) {
  const int nch = 2 * P.nbranches;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)nch * P.nroots;
       q += (long long)gridDim.x * blockDim.x) {
    const int ch = int(q / P.nroots), a = int(q - (long long)ch * P.nroots);
    const int c = ch / 2, sgn = (ch % 2) ? 1 : -1;
    roots[(size_t)ccf_row(P, c, sgn * j) * P.nroots + a] = roots[(size_t)ccf_row(P, c, sgn * (j - 1)) * P.nroots + a];
    fin[q] = 0;
  }
}

// Per root of every row: the error bound in 1/mu (ccf_functions.cuh:420-463),
// its maximum (as the bits of a non-negative double) and a non-finite flag.
template <typename T>
__global__ void ccf_errors(CcfParams P, LeafPtrs lp, DescentPtrs<T> dp, const StarRec<T>* __restrict__ stars,
                           const double2* __restrict__ roots, unsigned long long* __restrict__ max_bits,
                           int* __restrict__ nonfinite) {
  const int rows = P.nphi + P.nbranches, half = P.nphi / (2 * P.nbranches);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)rows * P.nroots;
       q += (long long)gridDim.x * blockDim.x) {
    const int row = int(q / P.nroots);
    const int c = row / (P.nphi / P.nbranches + 1), sj = row - c * (P.nphi / P.nbranches + 1) - half;
    const cplx<double> z = mk(roots[q].x, roots[q].y);
    const CcfField f = ccf_field(P, lp, dp, stars, z);
    const CcfDerivs d = ccf_derivs(P, f, z);
    const double e = ccf_inv_mu_bound(cabs_(ccf_f0(d, ccf_phi(P, c, sj))), d.dwdz);
    if (!isfinite(e))
      atomicExch(nonfinite, 1);
    else
      atomicMax(max_bits, __double_as_longlong(e));
  }
}

// Critical curves in the output layout [root][row] (the reference transposes
// its [row][root] array, ccf.cuh:1073-1077), the caustics w(z)
// (complex_image_to_source, ccf_functions.cuh:33-46) and the magnification
// length scales 1 / (2 |caustic tangent|) (ccf_functions.cuh:145-166).
template <typename T>
__global__ void ccf_outputs(CcfParams P, LeafPtrs lp, DescentPtrs<T> dp, const StarRec<T>* __restrict__ stars,
                            const double2* __restrict__ roots, double2* __restrict__ ccs, double2* __restrict__ caustics,
                            double* __restrict__ mu_len) {
  const int rows = P.nphi + P.nbranches;
  const cplx<double> corner = mk(P.corner_re, P.corner_im);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)rows * P.nroots;
       q += (long long)gridDim.x * blockDim.x) {
    const int a = int(q / rows), row = int(q - (long long)a * rows);
    const double2 zz = roots[(size_t)row * P.nroots + a];
    ccs[q] = zz;
    if (!caustics && !mu_len) continue;
    const cplx<double> z = mk(zz.x, zz.y);
    const CcfField f = ccf_field(P, lp, dp, stars, z);
    if (caustics) {
      const cplx<double> as = cconj(cscale(f.s1, P.theta2));
      const cplx<double> al = cconj(cscale(f.a0, P.theta2 / f.hl));
      const cplx<double> asm_ = alpha_smooth_(z, P.kstar, P.rect, corner, P.approx, P.taylor_smooth, P.inv_pi);
      cplx<double> w = cadd(cscale(z, 1.0 - P.kappa), cscale(cconj(z), P.gamma));
      w = csub(csub(csub(w, as), al), asm_);
      caustics[q] = make_double2(w.re, w.im);
    }
    if (mu_len) {
      const CcfDerivs d = ccf_derivs(P, f, z);
      const cplx<double> cct = cmul(mk(0.0, -2.0), cmul(cconj(d.dwdzb), d.d2wdzb2));
      const cplx<double> ct = cadd(cscale(cct, d.dwdz), cmul(d.dwdzb, cconj(cct)));
      mu_len[q] = 1.0 / (2.0 * cabs_(ct));
    }
  }
}

}  // namespace irsb
