// The reference's own IPM/IRS code, compiled for the host (test infrastructure
// and CPU baseline only).
//
// Built by oracle/Makefile from the reference sources where they lie
// (include/*.cuh of weisluke/irs) together with shim/cuda_host_shim.hpp; the
// outputs go to oracle/_ref/. Two libraries are built from this file:
//   -DREF_IPM -> libref_ipm.so  (ipm_functions.cuh: shoot_cells_kernel)
//   -DREF_IRS -> libref_irs.so  (irs_functions.cuh: shoot_rays_kernel)
//   -DREF_CCF -> libref_ccf.so  (ccf_functions.cuh: the critical-curve kernels)
//   -DREF_NCC -> libref_ncc.so  (ncc_functions.cuh: the caustic-crossing kernels)
// (the two headers define the same lens-equation templates, so they cannot
// share a translation unit).
//
// What is restated here is only the host orchestration of include/ipm.cuh:
// the tree-build loop (:789-837), the expansion schedule (:874-901) and the
// shoot launch (:930-932). Every kernel body and device function that runs is
// the reference's: the tree kernels of tree_node.cuh, the FMM kernels of
// fmm.cuh, get_nearest_node, complex_image_to_source, and shoot_cells_kernel /
// shoot_rays_kernel with Polygon::allocate_area_among_pixels. A launch is
// emulated by calling the kernel function with the grid coordinates of the
// host thread set, so its grid-stride loops partition the work between
// OpenMP threads exactly as between CUDA blocks.
#include <omp.h>

#include <unordered_map>
#include <vector>

#include "binomial_coefficients.cuh"
#include "fmm.cuh"
#include "tree_node.cuh"
#if defined(REF_IPM)
#include "ipm_functions.cuh"
#elif defined(REF_IRS)
#include "irs_functions.cuh"
#elif defined(REF_CCF)
#include "array_functions.cuh"
#include "ccf_functions.cuh"
#elif defined(REF_NCC)
#include "ncc_functions.cuh"
#else
#error "define REF_IPM, REF_IRS, REF_CCF or REF_NCC"
#endif

thread_local shim_uint3 threadIdx, blockIdx;
thread_local dim3 blockDim, gridDim;
namespace treenode {
int shared_memory[64];
}
namespace fmm {
Complex<double> coeffs[32 * 32];
}

namespace {
using T = double;

void serial_grid() {
  threadIdx = shim_uint3();
  blockIdx = shim_uint3();
  blockDim = dim3(1, 1, 1);
  gridDim = dim3(1, 1, 1);
}

struct RefTree {
  std::vector<TreeNode<T>*> tree;
  std::vector<int> num_nodes;
  star<T>* stars = nullptr;
  star<T>* temp_stars = nullptr;
  int* binom = nullptr;
  int levels = 0;
  int p = 0;
  int nstars = 0;
};

struct RefLens {
  double kappa, gamma, kstar, theta;
  int rect, approx, taylor_smooth;
  double corner_re, corner_im;
};
}  // namespace

extern "C" {

// include/ipm.cuh:746-901 with the given star field; p = 0 takes the
// reference's expansion-order formula (ipm.cuh:848).
RefTree* ref_tree_build(int n, const double* xym, double root_half_length, int p, double theta, double alpha_error) {
  serial_grid();
  RefTree* r = new RefTree();
  r->nstars = n;
  cudaMallocManaged(&r->stars, n * sizeof(star<T>));
  cudaMallocManaged(&r->temp_stars, n * sizeof(star<T>));
  for (int i = 0; i < n; i++) {
    r->stars[i].position = Complex<T>(xym[3 * i], xym[3 * i + 1]);
    r->stars[i].mass = xym[3 * i + 2];
  }
  r->tree.push_back(nullptr);
  r->num_nodes.push_back(1);
  cudaMallocManaged(&r->tree.back(), sizeof(TreeNode<T>));
  r->tree[0][0] = TreeNode<T>(Complex<T>(0, 0), root_half_length, 0);
  r->tree[0][0].numstars = n;
  int maxs, mins, nonempty;
  int lvl = 0;
  do {
    maxs = 0;
    mins = n;
    nonempty = 0;
    treenode::get_node_star_info_kernel<T>(r->tree[lvl], r->num_nodes[lvl], &nonempty, &mins, &maxs);
    if (maxs > treenode::MAX_NUM_STARS_DIRECT) {
      r->tree.push_back(nullptr);
      r->num_nodes.push_back(nonempty * treenode::MAX_NUM_CHILDREN);
      cudaMallocManaged(&r->tree.back(), r->num_nodes.back() * sizeof(TreeNode<T>));
      nonempty--;
      treenode::create_children_kernel<T>(r->tree[lvl], r->num_nodes[lvl], &nonempty, r->tree[lvl + 1]);
      treenode::sort_stars_kernel<T>(r->tree[lvl], r->num_nodes[lvl], r->stars, r->temp_stars);
      lvl++;
      treenode::set_neighbors_kernel<T>(r->tree[lvl], r->num_nodes[lvl]);
    }
  } while (maxs > treenode::MAX_NUM_STARS_DIRECT);
  r->levels = lvl;
  if (p <= 0) p = int(std::ceil(2 * std::log2(theta) + lvl - std::log2(root_half_length) - std::log2(alpha_error)));
  r->p = p;
  cudaMallocManaged(&r->binom, (2 * treenode::MAX_EXPANSION_ORDER * (2 * treenode::MAX_EXPANSION_ORDER + 3) / 2 + 1) *
                                   sizeof(int));
  calculate_binomial_coeffs(r->binom, 2 * p);
  for (int i = lvl; i >= 0; i--) {
    fmm::calculate_multipole_coeffs_kernel<T>(r->tree[i], r->num_nodes[i], p, r->stars);
    fmm::calculate_M2M_coeffs_kernel<T>(r->tree[i], r->num_nodes[i], p, r->binom);
  }
  for (int i = 2; i <= lvl; i++) {
    fmm::calculate_L2L_coeffs_kernel<T>(r->tree[i], r->num_nodes[i], p, r->binom);
    fmm::calculate_M2L_coeffs_kernel<T>(r->tree[i], r->num_nodes[i], p, r->binom);
    fmm::calculate_P2L_coeffs_kernel<T>(r->tree[i], r->num_nodes[i], p, r->binom, r->stars);
  }
  return r;
}

void ref_tree_free(RefTree* r) {
  if (!r) return;
  for (auto* t : r->tree) cudaFree(t);
  cudaFree(r->stars);
  cudaFree(r->temp_stars);
  cudaFree(r->binom);
  delete r;
}

int ref_tree_levels(RefTree* r) { return r->levels; }
int ref_tree_order(RefTree* r) { return r->p; }
int ref_tree_num_nodes(RefTree* r) {
  int s = 0;
  for (int v : r->num_nodes) s += v;
  return s;
}

// Nodes in level order. ints[k*8+.] = level, numstars, num_children, n_nbr,
// n_sil, n_dil, expansion_order, 0; geom[k*3+.] = cx, cy, hl; neighbour and
// interaction lists as node indices in this enumeration; coefficients
// (p+1 complex per node, interleaved).
void ref_tree_nodes(RefTree* r, int* ints, double* geom, int* nbr, int* sil, int* dil, double* mult, double* loc) {
  std::unordered_map<const TreeNode<T>*, int> idx;
  int k = 0;
  for (size_t l = 0; l < r->tree.size(); l++)
    for (int i = 0; i < r->num_nodes[l]; i++) idx[&r->tree[l][i]] = k++;
  k = 0;
  const int P = r->p;
  for (size_t l = 0; l < r->tree.size(); l++)
    for (int i = 0; i < r->num_nodes[l]; i++, k++) {
      const TreeNode<T>& nd = r->tree[l][i];
      int* o = ints + 8 * (size_t)k;
      o[0] = nd.level;
      o[1] = nd.numstars;
      o[2] = nd.num_children;
      o[3] = nd.num_neighbors;
      o[4] = nd.num_same_level_interaction_list;
      o[5] = nd.num_different_level_interaction_list;
      o[6] = nd.expansion_order;
      o[7] = 0;
      geom[3 * (size_t)k] = nd.center.re;
      geom[3 * (size_t)k + 1] = nd.center.im;
      geom[3 * (size_t)k + 2] = nd.half_length;
      for (int j = 0; j < 8; j++) nbr[8 * (size_t)k + j] = j < nd.num_neighbors ? idx[nd.neighbors[j]] : -1;
      for (int j = 0; j < 27; j++)
        sil[27 * (size_t)k + j] = j < nd.num_same_level_interaction_list ? idx[nd.same_level_interaction_list[j]] : -1;
      for (int j = 0; j < 5; j++)
        dil[5 * (size_t)k + j] =
            j < nd.num_different_level_interaction_list ? idx[nd.different_level_interaction_list[j]] : -1;
      for (int j = 0; j <= P; j++) {
        mult[2 * ((size_t)k * (P + 1) + j)] = nd.multipole_coeffs[j].re;
        mult[2 * ((size_t)k * (P + 1) + j) + 1] = nd.multipole_coeffs[j].im;
        loc[2 * ((size_t)k * (P + 1) + j)] = nd.local_coeffs[j].re;
        loc[2 * ((size_t)k * (P + 1) + j) + 1] = nd.local_coeffs[j].im;
      }
    }
}

#if !defined(REF_NCC)
// complex_image_to_source at arbitrary points (nearest node per point).
void ref_points(RefTree* r, const RefLens* L, long long n, const double* zx, const double* zy, double* wx, double* wy,
                int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4096)
  for (long long i = 0; i < n; i++) {
    Complex<T> z(zx[i], zy[i]);
    TreeNode<T>* node = treenode::get_nearest_node(z, r->tree[0]);
    Complex<T> w = complex_image_to_source<T>(z, L->kappa, L->gamma, L->theta, r->stars, L->kstar, node, L->rect,
                                              Complex<T>(L->corner_re, L->corner_im), L->approx, L->taylor_smooth);
    wx[i] = w.re;
    wy[i] = w.im;
  }
}

#endif

#if defined(REF_IPM)
// shoot_cells_kernel (ipm_functions.cuh:112-230) over the whole cell lattice,
// the grid emulated by nthreads host threads along y.
void ref_shoot_cells(RefTree* r, const RefLens* L, double rhs1, double rhs2, int nrt1, int nrt2, double cx1,
                     double cx2, double hlx1, double hlx2, double cy1, double cy2, double hly1, double hly2, int npx,
                     int npy, double* pixels, double* pmin, double* psad, int nthreads) {
  unsigned long long percentage = 1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    int t = omp_get_thread_num(), nt = omp_get_num_threads();
    threadIdx = shim_uint3();
    blockIdx = shim_uint3();
    blockIdx.y = t;
    blockDim = dim3(1, 1, 1);
    gridDim = dim3(1, nt, 1);
    shoot_cells_kernel<T>(L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0], L->rect,
                          Complex<T>(L->corner_re, L->corner_im), L->approx, L->taylor_smooth, Complex<T>(rhs1, rhs2),
                          Complex<int>(nrt1, nrt2), Complex<T>(cx1, cx2), Complex<T>(hlx1, hlx2), Complex<T>(cy1, cy2),
                          Complex<T>(hly1, hly2), pmin, psad, pixels, Complex<int>(npx, npy), &percentage, 0);
  }
  serial_grid();
}

// The deposition of shoot_cells_kernel (ipm_functions.cuh:168-216) for given
// cell-corner source positions (pixel units, row axis flipped), through
// Polygon::allocate_area_among_pixels.
void ref_deposit_cells(long long ncx, long long ncy, const double* vxy, double factor, int npx, int npy, double* pixels,
                       double* pmin, double* psad, int parities) {
  const long long W = ncx + 1;
  for (long long j = 0; j < ncy; j++)
    for (long long i = 0; i < ncx; i++) {
      const double* a = vxy + 2 * ((j + 1) * W + i + 1);
      const double* b = vxy + 2 * ((j + 1) * W + i);
      const double* c = vxy + 2 * (j * W + i);
      const double* d = vxy + 2 * (j * W + i + 1);
      Complex<T> y[4] = {Complex<T>(a[0], a[1]), Complex<T>(b[0], b[1]), Complex<T>(c[0], c[1]), Complex<T>(d[0], d[1])};
      const int tri[2][3] = {{0, 1, 2}, {2, 3, 0}};
      for (int t = 0; t < 2; t++) {
        Polygon<T> poly;
        poly.points[0] = y[tri[t][0]];
        poly.points[1] = y[tri[t][1]];
        poly.points[2] = y[tri[t][2]];
        poly.numsides = 3;
        if (fabs(poly.area()) < 10000 * factor) {
          if (parities)
            poly.allocate_area_among_pixels(factor, poly.area() < 0 ? pmin : psad, Complex<int>(npx, npy));
          else
            poly.allocate_area_among_pixels(factor, pixels, Complex<int>(npx, npy));
        }
      }
    }
}
#endif

#if defined(REF_IRS)
// shoot_rays_kernel (irs_functions.cuh:111-212) over the whole ray lattice.
void ref_shoot_rays(RefTree* r, const RefLens* L, double rhs1, double rhs2, int nrt1, int nrt2, double cx1, double cx2,
                    double hlx1, double hlx2, double cy1, double cy2, double hly1, double hly2, int npx, int npy,
                    int* pixels, int* pmin, int* psad, int nthreads) {
  unsigned long long percentage = 1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    int t = omp_get_thread_num(), nt = omp_get_num_threads();
    threadIdx = shim_uint3();
    blockIdx = shim_uint3();
    blockIdx.y = t;
    blockDim = dim3(1, 1, 1);
    gridDim = dim3(1, nt, 1);
    shoot_rays_kernel<T>(L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0], L->rect,
                         Complex<T>(L->corner_re, L->corner_im), L->approx, L->taylor_smooth, Complex<T>(rhs1, rhs2),
                         Complex<int>(nrt1, nrt2), Complex<T>(cx1, cx2), Complex<T>(hlx1, hlx2), Complex<T>(cy1, cy2),
                         Complex<T>(hly1, hly2), pmin, psad, pixels, Complex<int>(npx, npy), &percentage, 0);
  }
  serial_grid();
}
#endif

#if defined(REF_CCF)
// The root finding of include/ccf.cuh (find_initial_roots :906-977 and
// find_ccs :979-1083) with the reference's own kernels, the grid emulated by
// one host thread (its loops visit branch, side, root in order), followed by
// find_caustics_kernel and find_mu_length_scales_kernel (:1085-1121).
// roots: (nphi + nb) x nroots complex values, the branch centre rows holding
// the initial roots; on return every row holds its roots. ccs / caustics /
// mu_len: outputs in the [root][row] layout; *max_error: the largest error in
// 1/mu (negative when one is not finite).
void ref_ccf_run(RefTree* r, const RefLens* L, int nroots, int nphi, int nb, double* roots, int iters_init,
                 int iters_step, double* ccs, double* caustics, double* mu_len, double* max_error) {
  serial_grid();
  const int rows = nphi + nb;
  Complex<T>* z = reinterpret_cast<Complex<T>*>(roots);
  bool* fin = new bool[(size_t)nb * 2 * nroots]();
  T* errs = new T[(size_t)rows * nroots];
  const Complex<T> corner(L->corner_re, L->corner_im);
  for (int i = 0; i < iters_init; i++)
    find_critical_curve_roots_kernel<T>(L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0], L->rect, corner,
                                        L->approx, L->taylor_smooth, z, nroots, 0, nphi, nb, fin);
  for (int j = 1; j <= nphi / (2 * nb); j++) {
    prepare_roots_kernel<T>(z, nroots, j, nphi, nb, fin);
    for (int i = 0; i < iters_step; i++)
      find_critical_curve_roots_kernel<T>(L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0], L->rect,
                                          corner, L->approx, L->taylor_smooth, z, nroots, j, nphi, nb, fin);
  }
  for (long long q = 0; q < (long long)rows * nroots; q++) errs[q] = 1;
  for (int j = 0; j <= nphi / (2 * nb); j++)
    find_errors_kernel<T>(z, nroots, L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0], L->rect, corner,
                          L->approx, L->taylor_smooth, j, nphi, nb, errs);
  double me = 0;
  for (long long q = 0; q < (long long)rows * nroots; q++) {
    if (!std::isfinite(errs[q])) {
      me = -1;
      break;
    }
    me = std::max(me, double(errs[q]));
  }
  *max_error = me;
  Complex<T>* out = reinterpret_cast<Complex<T>*>(ccs);
  transpose_array_kernel<Complex<T>>(z, rows, nroots, out);
  find_caustics_kernel<T>(out, rows * nroots, L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0], L->rect,
                          corner, L->approx, L->taylor_smooth, reinterpret_cast<Complex<T>*>(caustics));
  find_mu_length_scales_kernel<T>(out, rows * nroots, L->kappa, L->gamma, L->theta, r->stars, L->kstar, r->tree[0],
                                  L->rect, corner, L->approx, L->taylor_smooth, mu_len);
  delete[] fin;
  delete[] errs;
}
#endif

#if defined(REF_NCC)
// The map of include/ncc.cuh (calculate_num_caustic_crossings, :235-327) with
// the reference's own kernels on one host thread: the crossings on the
// 2^os times finer map, then os rounds of the 2 x 2 maximum and the row /
// column shifts. caus: nrows x ncols complex values; out: npy x npx.
void ref_ncc_run(const double* caus, int nrows, int ncols, double cy1, double cy2, double hl1, double hl2, int npx,
                 int npy, int os, int* out) {
  serial_grid();
  Complex<int> np(npx << os, npy << os);
  int* num = new int[(size_t)np.re * np.im]();
  unsigned long long percentage = 1;
  Complex<T>* c = const_cast<Complex<T>*>(reinterpret_cast<const Complex<T>*>(caus));
  find_num_caustic_crossings_kernel<T>(c, nrows, ncols, Complex<T>(cy1, cy2), Complex<T>(hl1, hl2), num, np,
                                       &percentage, 0);
  for (int i = 0; i < os; i++) {
    np.re >>= 1;
    np.im >>= 1;
    reduce_pix_array_kernel<T>(num, np);
    for (int j = 1; j < np.re; j++) shift_pix_column_kernel<T>(num, np, j);
    for (int j = 1; j < np.im; j++) shift_pix_row_kernel<T>(num, np, j);
  }
  for (long long q = 0; q < (long long)npx * npy; q++) out[q] = num[q];
  delete[] num;
}
#endif

}  // extern "C"
