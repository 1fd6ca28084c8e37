// Multipole / local expansion coefficients of the quadtree, in FP64.
//
// Formulas of the reference's fmm.cuh (coefficients in units of the node half
// length):
//   P2M  a_0 = sum m_i, a_k = -sum m_i ((z_i - c)/hl)^k / k          fmm.cuh:21-49
//   M2M  dz = (c_child - c_parent)/hl_child,
//        b_l = (sum_k a_k C(l-1,k-1) / dz^k - a_0/l) * (dz/2)^l       fmm.cuh:109-139
//   L2L  dz = (c - c_parent)/hl_parent,
//        d_l = sum_{k>=1} c_k C(k,l) dz^k / (2 dz)^l                 fmm.cuh:204-223
//   M2L  dz = (c_from - c_to)/hl_from,
//        c_0 = sum_k b_k/(-dz)^k + b_0 log(-dz) + b_0 log(hl_from),
//        c_l = (sum_k b_k C(l+k-1,k-1)/(-dz)^k - b_0/l) / dz^l       fmm.cuh:281-322
//   P2L  dz = (z_i - c_to)/hl_to,
//        c_0 = sum m_i (log(-dz) + log(hl_to)), c_l = -sum m_i/(l dz^l) fmm.cuh:387-413
// evaluated in FP64 as binomial-weighted sums of scaled coefficients (each
// power z^k from a product scan over a group of lanes, each division by l,
// dz^l or 2^l as a product): the reference's quantities, summed in another
// order than its Horner form (the coefficients agree to rounding). Level
// schedule as
// include/ipm.cuh:874-901: P2M+M2M bottom-up, then L2L, M2L, P2L top-down from
// level 2. The reference builds an int binomial table, which overflows beyond
// order ~17 (binomial_coefficients.cuh:11-44); this table is int64, exact up to
// row 62, and is used as double.
//
// Layout: coefficients of node k, order l at [k * (p + 1) + l] as double2.
// Kernel shape: one warp (or, for levels of few nodes, one block) per node, in
// groups of p + 1 lanes, lane l of a group computing order l (p <= 31).
#pragma once
#include "common.cuh"
#include "devutil.cuh"
#include "tree.cuh"

#include <vector>

namespace irsb {

__device__ __forceinline__ cplx<double> ld2(const double2* p) {
  double2 v = *p;
  return mk<double>(v.x, v.y);
}
__device__ __forceinline__ void st2(double2* p, cplx<double> c) { *p = make_double2(c.re, c.im); }

inline std::vector<double> binomial_table(int nmax) {
  // row n starts at n(n+1)/2
  std::vector<long long> t((nmax + 1) * (nmax + 2) / 2);
  for (int n = 0; n <= nmax; n++) {
    int r = n * (n + 1) / 2, pr = (n - 1) * n / 2;
    for (int i = 0; i <= n; i++) t[r + i] = (i == 0 || i == n) ? 1 : t[pr + i - 1] + t[pr + i];
  }
  return std::vector<double>(t.begin(), t.end());
}
__device__ __forceinline__ double binom(const double* tab, int n, int k) {
  if (n < k || k < 0) return 0.0;
  return tab[n * (n + 1) / 2 + k];
}

// Powers of z within each group of P1 lanes: lane l of a group returns z^l
// (z^0 = 1), by a product scan over the group (log2(P1) steps).
__device__ __forceinline__ cplx<double> group_powers(cplx<double> z, int l, int P1) {
  cplx<double> v = l == 0 ? mk(1.0, 0.0) : z;
  for (int o = 1; o < P1; o <<= 1) {
    const cplx<double> u = mk(__shfl_up_sync(0xffffffffu, v.re, o), __shfl_up_sync(0xffffffffu, v.im, o));
    if (l >= o) v = cmul(u, v);
  }
  return v;
}

// Multipoles of the leaves of one level from their stars. One warp per leaf in
// groups of p + 1 lanes (lane l of a group computes order l); group g takes
// stars g, g + G, ... with the star's powers ((z - c) / hl)^l from a product
// scan over the group, and the groups' sums are added in group order.
template <typename T>
__global__ void fmm_p2m(int beg, int end, LevelRange lr, int p, const T* __restrict__ cx, const T* __restrict__ cy,
                        const T* __restrict__ hl, const int* __restrict__ child0, const int* __restrict__ sbeg,
                        const int* __restrict__ scnt, const StarRec<T>* __restrict__ stars, double2* mult) {
  lr.get(beg, end);
  const int lane = threadIdx.x & 31;
  const int P1 = p + 1;
  const int G = 32 / P1;
  const int g = lane / P1, l = lane - g * P1;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int k = beg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < end; k += warps) {
    if (child0[k] >= 0 || scnt[k] == 0) continue;  // uniform over the warp
    const double ccx = cx[k], ccy = cy[k], h = hl[k];
    const int b = sbeg[k], n = scnt[k];
    cplx<double> r = mk(0.0, 0.0);
    for (int i0 = 0; i0 < n; i0 += G) {
      const int i = i0 + g;
      const bool valid = g < G && i < n;
      const StarRec<T> st = stars[b + (valid ? i : 0)];
      const cplx<double> d = mk((double(st.x) - ccx) / h, (double(st.y) - ccy) / h);
      const cplx<double> pw = group_powers(d, l, P1);
      if (!valid) continue;
      if (l == 0) r.re += double(st.m);
      else r = csub(r, cscale(pw, double(st.m)));
    }
    for (int gg = 1; gg < G; gg++) {
      const int src = min(l + gg * P1, 31);
      const cplx<double> o = mk(__shfl_sync(0xffffffffu, r.re, src), __shfl_sync(0xffffffffu, r.im, src));
      if (g == 0) r = cadd(r, o);
    }
    if (g == 0) st2(&mult[(size_t)k * P1 + l], l > 0 ? cdivr(r, double(l)) : r);
  }
}

// Parent multipoles from its 4 children (internal nodes of one level). One
// warp per node in groups of p + 1 lanes (lane l of a group computes order l);
// group g shifts children g, g + G, ... and the groups' sums are added into
// group 0 in group order. Each shift is a binomial-weighted sum: with
// u_i = a_i (1 / dz)^i (lane i, its power from a product scan over the group),
//   b_0 = a_0,  b_l = (sum_i C(l - 1, i - 1) u_i - a_0 / l) dz^l 2^-l,
// the reference's quantity (fmm.cuh:109-139) with real weights, staged per
// block in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) fmm_m2m(int beg, int end, LevelRange lr, int p, const T* __restrict__ cx,
                                               const T* __restrict__ cy, const T* __restrict__ hl,
                                               const int* __restrict__ child0, const double* __restrict__ btab,
                                               double2* mult) {
  lr.get(beg, end);
  const int lane = threadIdx.x & 31, ws = threadIdx.x >> 5;
  const int P1 = p + 1;
  const int G = 32 / P1;
  const int g = lane / P1, l = lane - g * P1, gb = g * P1;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const double inv_l = l > 0 ? 1.0 / double(l) : 0.0;
  const double inv_2l = 1.0 / double(1u << (l & 31));  // exact
  __shared__ double2 s_u[8][32];
  __shared__ double s_w[32][32];  // [i][lane]: C(l - 1, i - 1)
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int i = idx >> 5, ln = idx & 31, ll = ln - (ln / P1) * P1;
    s_w[i][ln] = i >= 1 && i <= p ? binom(btab, ll - 1, i - 1) : 0.0;
  }
  __syncthreads();
  const cplx<double> zero = mk(0.0, 0.0);
  for (int k = beg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < end; k += warps) {
    const int c0 = child0[k];
    if (c0 < 0) continue;  // uniform over the warp
    cplx<double> acc = zero;
    for (int j0 = 0; j0 < 4; j0 += G) {
      const int j = j0 + g;
      const bool valid = g < G && j < 4;
      const int c = c0 + (valid ? j : 0);
      const double hc = hl[c];
      const cplx<double> dz = mk((double(cx[c]) - double(cx[k])) / hc, (double(cy[c]) - double(cy[k])) / hc);
      const cplx<double> pz = group_powers(dz, l, P1);
      const cplx<double> pi = group_powers(cdiv(mk(1.0, 0.0), dz), l, P1);
      const cplx<double> al = ld2(mult + (size_t)c * P1 + l);
      const cplx<double> u = l == 0 ? al : cmul(al, pi);
      __syncwarp();
      s_u[ws][lane] = make_double2(u.re, u.im);
      __syncwarp();
      if (!valid) continue;
      cplx<double> r;
      if (l == 0) {
        r = al;
      } else {
        r = zero;
#pragma unroll 4
        for (int i = p; i >= 1; i--) {
          const double C = s_w[i][lane];
          const double2 ui = s_u[ws][gb + i];
          r.re = fma(C, ui.x, r.re);
          r.im = fma(C, ui.y, r.im);
        }
        const double2 a0 = s_u[ws][gb];
        r = cscale(cmul(csub(r, cscale(mk(a0.x, a0.y), inv_l)), pz), inv_2l);
      }
      acc = cadd(acc, r);
    }
    for (int gg = 1; gg < G; gg++) {
      const int src = min(l + gg * P1, 31);
      const cplx<double> o = mk(__shfl_sync(0xffffffffu, acc.re, src), __shfl_sync(0xffffffffu, acc.im, src));
      if (g == 0) acc = cadd(acc, o);
    }
    if (g == 0) st2(&mult[(size_t)k * P1 + l], acc);
  }
}

// Local coefficients of the nodes of one level (>= 2): L2L from the parent,
// then M2L over the same-level interaction list, then P2L over the
// different-level list.
//
// W warps per node (W = 1: one warp per node; W = 8: a block per node, for
// levels with few nodes), each split into G = 32 / (p + 1) groups of p + 1
// lanes (lane l of a group computes order l). The per-interaction quantities
// every order needs (the source's reciprocal distance and the logarithms of
// the order-0 term) are computed once per warp, interaction j (or star j) on
// lane j, and read by the groups through shuffles; group gid of the node's
// GW = W G groups takes interactions gid, gid + GW, ... and the groups' sums
// are added in group order (deterministic).
//
// Each translation is a binomial-weighted sum over scaled coefficients, with
// the powers from a product scan over the group (lane k holds z^k) and the
// binomial weights of lane l staged once per block in shared memory:
//   M2L, w = 1 / (-dz), u_k = b_k w^k (fmm.cuh:281-322):
//     c_0 = sum_k u_k + b_0 log(-dz) + b_0 log(hl_from),
//     c_l = (sum_k C(l + k - 1, k - 1) u_k - b_0 / l) (-w)^l;
//   L2L, v_i = c_i dz^i (fmm.cuh:204-223):
//     d_l = sum_{i >= 1} C(i, l) v_i (1 / dz)^l 2^-l;
//   P2L: -m / (l d^l) with (1 / d)^l from the scan.
// The same quantities as the reference's Horner forms, with real weights (two
// FMAs per term) and the divisions by l, dz^l and 2^l as products.
static_assert(kMaxSameLevelIL <= 32, "one lane per same-level interaction");
template <typename T, int W = 1>
__global__ void __launch_bounds__(256) fmm_local(int beg, int end, LevelRange lr, int p, const T* __restrict__ cx,
                                                 const T* __restrict__ cy, const T* __restrict__ hl,
                                                 const int* __restrict__ parent, const int* __restrict__ sbeg,
                                                 const int* __restrict__ scnt, const int* __restrict__ sil,
                                                 const int* __restrict__ n_sil, const int* __restrict__ dil,
                                                 const int* __restrict__ n_dil, const StarRec<T>* __restrict__ stars,
                                                 const double* __restrict__ btab, const double2* __restrict__ mult,
                                                 double2* loc) {
  lr.get(beg, end);
  const int lane = threadIdx.x & 31, ws = threadIdx.x >> 5, w = W > 1 ? ws : 0;
  const int P1 = p + 1;
  const int G = 32 / P1;
  const int g = lane / P1, l = lane - g * P1, gb = g * P1;
  const bool grp = g < G;
  const int GW = G * W, gid = w * G + g;
  const double inv_l = l > 0 ? 1.0 / double(l) : 0.0;
  const double inv_2l = 1.0 / double(1u << (l & 31));  // exact
  __shared__ double2 s_acc[W][32];
  __shared__ double2 s_u[8][32];   // per warp: the scaled coefficients of each group's term
  __shared__ double s_wm[32][32];  // [k][lane]: C(l + k - 1, k - 1) (M2L)
  __shared__ double s_wl[32][32];  // [i][lane]: C(i, l) (L2L)
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int kk = idx >> 5, ln = idx & 31, ll = ln - (ln / P1) * P1;
    s_wm[kk][ln] = kk >= 1 && kk <= p ? binom(btab, ll + kk - 1, kk - 1) : 0.0;
    s_wl[kk][ln] = kk >= 1 && kk <= p ? binom(btab, kk, ll) : 0.0;
  }
  __syncthreads();
  const cplx<double> zero = mk(0.0, 0.0);
  const int k0 = W > 1 ? beg + int(blockIdx.x) : beg + int((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int kstep = W > 1 ? int(gridDim.x) : int((gridDim.x * blockDim.x) >> 5);
  for (int k = k0; k < end; k += kstep) {
    const double ccx = cx[k], ccy = cy[k], h = hl[k];
    cplx<double> acc = zero;
    // L2L (every group of warp 0 forms it; group 0 keeps it)
    if (w == 0) {
      const int pa = parent[k];
      const double hp = hl[pa];
      const cplx<double> dz = mk((ccx - double(cx[pa])) / hp, (ccy - double(cy[pa])) / hp);
      const cplx<double> pz = group_powers(dz, l, P1);
      const cplx<double> pi = group_powers(cdiv(mk(1.0, 0.0), dz), l, P1);
      const cplx<double> v = cmul(ld2(loc + (size_t)pa * P1 + l), pz);
      __syncwarp();
      s_u[ws][lane] = make_double2(v.re, v.im);
      __syncwarp();
      cplx<double> r = zero;
#pragma unroll 4
      for (int i = p; i >= 1; i--) {
        const double C = s_wl[i][lane];
        const double2 vi = s_u[ws][gb + i];
        r.re = fma(C, vi.x, r.re);
        r.im = fma(C, vi.y, r.im);
      }
      if (g == 0) acc = cscale(cmul(r, pi), inv_2l);
    }
    // M2L: interaction j's source, 1 / (-dz), log(-dz) and log(hl_from) on lane j
    const int ns = n_sil[k];
    int fj = 0;
    cplx<double> imdj = zero, lgj = zero;
    double lhj = 0.0;
    if (lane < ns) {
      fj = sil[k * kMaxSameLevelIL + lane];
      const double hf = hl[fj];
      const cplx<double> md = cneg(mk((double(cx[fj]) - ccx) / hf, (double(cy[fj]) - ccy) / hf));
      imdj = cdiv(mk(1.0, 0.0), md);
      lgj = clog_(md);
      lhj = log(hf);
    }
    for (int j0 = 0; j0 < ns; j0 += GW) {
      const int j = j0 + gid;
      const int src = j < 32 ? j : 31;
      const int f = __shfl_sync(0xffffffffu, fj, src);
      const cplx<double> imd = mk(__shfl_sync(0xffffffffu, imdj.re, src), __shfl_sync(0xffffffffu, imdj.im, src));
      const cplx<double> lg = mk(__shfl_sync(0xffffffffu, lgj.re, src), __shfl_sync(0xffffffffu, lgj.im, src));
      const double lh = __shfl_sync(0xffffffffu, lhj, src);
      const bool valid = grp && j < ns;
      const cplx<double> pw = group_powers(imd, l, P1);  // w^l
      const cplx<double> bl = valid ? ld2(mult + (size_t)f * P1 + l) : zero;
      const cplx<double> u = l == 0 ? bl : cmul(bl, pw);
      __syncwarp();
      s_u[ws][lane] = make_double2(u.re, u.im);
      __syncwarp();
      if (valid) {
        cplx<double> t = zero;
#pragma unroll 4
        for (int kk = p; kk >= 1; kk--) {  // C(l + k - 1, k - 1) is 1 for l = 0
          const double C = s_wm[kk][lane];
          const double2 uk = s_u[ws][gb + kk];
          t.re = fma(C, uk.x, t.re);
          t.im = fma(C, uk.y, t.im);
        }
        const double2 b0v = s_u[ws][gb];
        const cplx<double> b0 = mk(b0v.x, b0v.y);
        if (l == 0) {
          t = cadd(t, cmul(b0, lg));
          t = cadd(t, cscale(b0, lh));
        } else {
          t = csub(t, cscale(b0, inv_l));
          t = cmul(t, (l & 1) ? cneg(pw) : pw);  // 1 / dz^l = (-w)^l
        }
        acc = cadd(acc, t);
      }
    }
    // P2L: star u of each list's chunk of 32: 1 / dz and log(-dz) on lane u
    const int nd = n_dil[k];
    const double lhk = nd > 0 ? log(h) : 0.0;
    for (int q = 0; q < nd; q++) {
      const int f = dil[k * kMaxDiffLevelIL + q];
      const int sb0 = sbeg[f], sn = scnt[f];
      cplx<double> t = zero;
      for (int i0 = 0; i0 < sn; i0 += 32) {
        cplx<double> idu = zero, lgu = zero;
        double mu = 0.0;
        if (i0 + lane < sn) {
          const StarRec<T> st = stars[sb0 + i0 + lane];
          const cplx<double> d = mk((double(st.x) - ccx) / h, (double(st.y) - ccy) / h);
          mu = double(st.m);
          idu = cdiv(mk(1.0, 0.0), d);
          lgu = clog_(cneg(d));
        }
        const int cnt = min(32, sn - i0);
        for (int u0 = 0; u0 < cnt; u0 += GW) {
          const int u = u0 + gid;
          const int src = u < 32 ? u : 31;
          const cplx<double> id = mk(__shfl_sync(0xffffffffu, idu.re, src), __shfl_sync(0xffffffffu, idu.im, src));
          const cplx<double> lg = mk(__shfl_sync(0xffffffffu, lgu.re, src), __shfl_sync(0xffffffffu, lgu.im, src));
          const double m = __shfl_sync(0xffffffffu, mu, src);
          const cplx<double> pw = group_powers(id, l, P1);  // (1 / d)^l
          if (!grp || u >= cnt) continue;
          if (l == 0) {
            t = cadd(t, cscale(lg, m));
            t.re += m * lhk;
          } else {
            t = csub(t, cscale(pw, m * inv_l));  // m / (l d^l)
          }
        }
      }
      acc = cadd(acc, t);
    }
    // the groups' sums into group 0 of the warp, then the warps' into warp 0
    for (int gg = 1; gg < G; gg++) {
      const int src = min(l + gg * P1, 31);
      const cplx<double> o = mk(__shfl_sync(0xffffffffu, acc.re, src), __shfl_sync(0xffffffffu, acc.im, src));
      if (g == 0) acc = cadd(acc, o);
    }
    if (W > 1) {
      if (g == 0) s_acc[w][l] = make_double2(acc.re, acc.im);
      __syncthreads();
      if (w == 0 && g == 0) {
        for (int ww = 1; ww < W; ww++) acc = cadd(acc, ld2(&s_acc[ww][l]));
        st2(&loc[(size_t)k * P1 + l], acc);
      }
      __syncthreads();
    } else if (g == 0) {
      st2(&loc[(size_t)k * P1 + l], acc);
    }
  }
}

struct FmmDev {
  int p = 0;
  DevVec<double2> mult, loc;
  DevVec<double> btab;
};

template <typename T>
bool compute_fmm(FmmDev& f, TreeDev<T>& t, const StarRec<T>* stars, int p, cudaStream_t s) {
  f.p = p;
  size_t ncoef = size_t(t.num_nodes) * (p + 1);
  if (!f.mult.alloc_exact(ncoef) || !f.loc.alloc_exact(ncoef)) return false;
  IRSB_CKR(cudaMemsetAsync(f.mult.p, 0, ncoef * sizeof(double2), s));
  IRSB_CKR(cudaMemsetAsync(f.loc.p, 0, ncoef * sizeof(double2), s));
  std::vector<double> bt = binomial_table(2 * kMaxOrder);
  if (!f.btab.alloc_exact(bt.size())) return false;
  IRSB_CKR(cudaMemcpyAsync(f.btab.p, bt.data(), bt.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  for (int l = t.levels; l >= 0; l--) {
    int beg = t.level_off[l], end = t.level_off[l + 1];
    int nw = end - beg;
    int blocks = std::max(1, std::min(ceil_div(nw, 8), 148 * 16));
    fmm_p2m<T><<<blocks, 256, 0, s>>>(beg, end, LevelRange{}, p, t.cx.p, t.cy.p, t.hl.p, t.child0.p, t.sbeg.p, t.scnt.p, stars,
                                      f.mult.p);
    IRSB_LAUNCH_CK("fmm_p2m");
    fmm_m2m<T><<<blocks, 256, 0, s>>>(beg, end, LevelRange{}, p, t.cx.p, t.cy.p, t.hl.p, t.child0.p, f.btab.p, f.mult.p);
    IRSB_LAUNCH_CK("fmm_m2m");
  }
  for (int l = 2; l <= t.levels; l++) {
    int beg = t.level_off[l], end = t.level_off[l + 1];
    int nw = end - beg;
    int blocks = std::max(1, std::min(ceil_div(nw, 8), 148 * 16));
    if (nw <= 512)  // few nodes: a block of 8 warps per node
      fmm_local<T, 8><<<std::max(1, std::min(nw, 148 * 16)), 256, 0, s>>>(
          beg, end, LevelRange{}, p, t.cx.p, t.cy.p, t.hl.p, t.parent.p, t.sbeg.p, t.scnt.p, t.sil.p, t.n_sil.p,
          t.dil.p, t.n_dil.p, stars, f.btab.p, f.mult.p, f.loc.p);
    else
      fmm_local<T><<<blocks, 256, 0, s>>>(beg, end, LevelRange{}, p, t.cx.p, t.cy.p, t.hl.p, t.parent.p, t.sbeg.p,
                                          t.scnt.p, t.sil.p, t.n_sil.p, t.dil.p, t.n_dil.p, stars, f.btab.p, f.mult.p,
                                          f.loc.p);
    IRSB_LAUNCH_CK("fmm_local");
  }
  return true;
}

}  // namespace irsb
