// Host pipeline driver for IPM and IRS magnification maps.
//
// Mirrors the reference's IPM<T>::run / IRS<T>::run stage order
// (include/ipm.cuh:1327-1340, include/irs.cuh:1224-1237): check inputs ->
// derive parameters -> allocate -> star field -> tree + expansions -> shoot ->
// histograms, and save() (include/ipm.cuh:1122-1322, irs.cuh:1122-1221) for
// the output files. Differences by design: everything runs on one private
// CUDA stream of the current device (no cudaDeviceReset, so several objects
// can coexist); device buffers are owned by the object and reused across
// runs; maps are returned through pinned host copies owned by the object and
// valid until the next run() or destroy; the shoot phase is timed with CUDA
// events.
#pragma once
#include "common.cuh"
#include "deposit.cuh"
#include "devutil.cuh"
#include "fmm.cuh"
#include "leaves.cuh"
#include "params.hpp"
#include "post.cuh"
#include "shoot.cuh"
#include "stars.cuh"
#include "tree.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

namespace irsb {

enum Precision : int {
  kPrecisionDefault = 0,  // FP32 form for float objects, FP64 plain form for double objects
  kPrecisionFP64 = 1,
  kPrecisionFP32 = 2,
};

// Kernel parameters of the lens-equation pass over the ray lattice (IRS) or
// the cell-corner lattice (IPM, vertices), the latter held from row jbase on.
template <typename T>
ShootParams make_shoot_params(const Params<T>& p, bool vertices, long long jbase) {
  ShootParams sp;
  sp.kappa = double(p.kappa_tot);
  sp.gamma = double(p.shear);
  sp.kstar = double(p.kappa_star);
  sp.theta2 = double(p.theta_star) * double(p.theta_star);
  sp.inv_pi = 0.318309886183790671537767526745028724;
  sp.rect = p.rectangular;
  sp.approx = p.approx;
  sp.taylor_smooth = p.taylor_smooth;
  sp.p = p.expansion_order;
  sp.corner_re = double(p.corner.re);
  sp.corner_im = double(p.corner.im);
  sp.cy_re = double(p.center_y.re);
  sp.cy_im = double(p.center_y.im);
  sp.hly_re = double(p.half_length_y.re);
  sp.hly_im = double(p.half_length_y.im);
  sp.npx = p.num_pixels_y.re;
  sp.npy = p.num_pixels_y.im;
  sp.rhs_x = double(p.ray_half_sep.re);
  sp.rhs_y = double(p.ray_half_sep.im);
  const double ox = double(p.center_x.re) - double(p.half_length_x.re);
  const double oy = double(p.center_x.im) - double(p.half_length_x.im);
  sp.jbase = 0;
  if (vertices) {
    sp.base_x = ox;
    sp.base_y = oy;
    sp.nx = (long long)p.num_ray_threads.re + 1;
    sp.ny = (long long)p.num_ray_threads.im + 1;
    sp.jbase = jbase;
  } else {
    sp.base_x = ox + sp.rhs_x;
    sp.base_y = oy + sp.rhs_y;
    sp.nx = p.num_ray_threads.re;
    sp.ny = p.num_ray_threads.im;
  }
  return sp;
}

// Image-plane area of one IPM triangle in pixel units (include/ipm.cuh, the
// factor of ipm_functions.cuh:170), in the arithmetic type of the deposition.
template <typename T, typename D>
D ipm_triangle_factor(const Params<T>& p) {
  return D(2 * p.ray_half_sep.re * p.ray_half_sep.im * p.num_pixels_y.re * p.num_pixels_y.im /
           (2 * p.half_length_y.re * 2 * p.half_length_y.im));
}

template <typename T>
class AdaptiveIPM;

template <typename T, bool IS_IRS>
class MapMaker {
  friend class AdaptiveIPM<T>;

 public:
  using Pix = typename std::conditional<IS_IRS, int, T>::type;
  Params<T> prm;
  int precision = kPrecisionDefault;
  // lattice row band [band_lo, band_hi) of this object (rays for IRS, cells for
  // IPM); band_hi < 0 means all rows. Used to split one map over several GPUs.
  long long band_lo = 0, band_hi = -1;
  // host-provided star field (extension): used instead of generation / star file
  std::vector<StarRec<T>> host_stars;
  bool use_host_stars = false;
  cplx<T> host_corner = mk<T>(0, 0);
  int host_rect = 0;
  T host_theta = T(1);

  // results
  double t_shoot = 0;     // seconds, shoot phase (lattice evaluation + deposition)
  double t_pipeline = 0;  // seconds, tree + expansions + leaf records + shoot
  unsigned long long num_rays_shot = 0, num_rays_received = 0;
  std::vector<StarRec<T>> stars_out;
  HostVec<Pix> h_pix, h_pmin, h_psad;
  bool have_parities = false;
  // histograms
  int hist_min = 0, hist_len = 0, log_hist_min = 0, log_hist_len = 0;
  std::vector<int> hist, hist_minima, hist_saddles, log_hist, log_hist_minima, log_hist_saddles;
  int num_leaves = 0;
  long long num_tiles = 0;
  double mean_near = 0;      // mean near-field star count per lattice point
  double t_lattice = 0;      // seconds, lens-equation kernel of the last shoot
  double t_deposit = 0;      // seconds, IPM deposition kernel of the last shoot
  long long launches = 0;    // kernels launched by the last run / pipeline call
  // IPM: stop after the corner lattice (no deposition, no maps); used by the
  // adaptive deposition, which deposits the lattice itself
  bool verts_only = false;
  // launch shape of the FP32 lens-equation kernel (set by the autotuner):
  // threads per CTA (128, 256 or 512: 8, 4 or 2 lattice points per thread)
  // and CTAs per SM of its grid-stride grid (more CTAs than fit at once:
  // the tiles are dealt out in smaller shares, which evens out the tail);
  // default the fastest measured on the 2000-pixel IPM workload and the
  // 500-pixel ray-shooting case
  int shoot_threads = 128;
  int shoot_ctas_per_sm = 64;

  MapMaker() {
    if (IS_IRS) {
      prm.light_loss = T(0.01);  // include/irs.cuh:51
      prm.num_rays_y = 100;      // include/irs.cuh:59
    }
  }
  ~MapMaker() {
    if (stream_) cudaStreamDestroy(stream_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (ev2_) cudaEventDestroy(ev2_);
    if (ev_lat0_) cudaEventDestroy(ev_lat0_);
    if (ev_lat1_) cudaEventDestroy(ev_lat1_);
    if (ev_dep1_) cudaEventDestroy(ev_dep1_);
    for (cudaEvent_t e : out_ev_)
      if (e) cudaEventDestroy(e);
    if (ev_map_) cudaEventDestroy(ev_map_);
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
  }

  bool use_fp32() const {
    if (precision == kPrecisionFP64) return false;
    if (precision == kPrecisionFP32) return true;
    return sizeof(T) == 4;
  }
  // The FP32 form folds an approximate rectangular smooth sheet into the
  // leaves' expansions (leaves.cuh) instead of summing its series per point.
  bool smooth_folded() const { return use_fp32() && prm.rectangular && prm.approx; }

  Pix* pixels() { return h_pix.p; }
  // host buffer of num_pixels_y2 x num_pixels_y1 values that the next run()
  // also fills with its total map (chunk by chunk, overlapped with the
  // transfer); applies to one run
  void set_pixels_out(Pix* dst) { out_user_ = dst; }
  // The map of the last run (0 total, 1 minima, 2 saddles) copied into dst
  // (npix values) by the OpenMP threads (a persistent pool: no thread start
  // per call); false if that map does not exist.
  bool copy_pixels(int which, Pix* dst) const {
    const Pix* src = which == 0 ? h_pix.p : (have_parities ? (which == 1 ? h_pmin.p : h_psad.p) : nullptr);
    if (!src || !dst || which < 0 || which > 2) return false;
    const long long n = (long long)prm.num_pixels_y.re * prm.num_pixels_y.im;
    const long long chunk = 1 << 18;
    const long long nchunk = (n + chunk - 1) / chunk;
#pragma omp parallel for schedule(static) num_threads(8) if (nchunk > 1)
    for (long long c = 0; c < nchunk; c++) {
      const long long a = c * chunk, b = std::min(n, a + chunk);
      std::memcpy(dst + a, src + a, size_t(b - a) * sizeof(Pix));
    }
    return true;
  }
  Pix* pixels_minima() { return have_parities ? h_pmin.p : nullptr; }
  Pix* pixels_saddles() { return have_parities ? h_psad.p : nullptr; }
  T* stars_ptr() { return stars_out.empty() ? nullptr : &stars_out[0].x; }
  cplx<T> corner_out() const {
    return prm.rectangular ? prm.corner : mk<T>(cabs_(prm.corner), T(0));
  }

  bool run(int verbose) {
    if (!init_stream()) return false;
    Params<T> p = prm;  // inputs of this run; prm keeps derived values afterwards
    if (use_host_stars) p.starfile = "<memory>";  // star-file rules for a field passed in memory
    if (!check_input_params(p)) return false;
    std::vector<StarRec<T>> file_stars;
    if (use_host_stars) {
      if (host_stars.empty()) {
        std::cerr << "Error. No stars were provided.\n";
        return false;
      }
      file_stars = host_stars;
      p.num_stars = int(host_stars.size());
      p.rectangular = host_rect;
      p.corner = host_corner;
      p.theta_star = host_theta;
    }
    if (!derive_params<T>(p, file_stars, use_host_stars)) return false;
    const bool from_stars = !p.starfile.empty();
    const int n = p.num_stars;
    if (!d_stars_.alloc_exact(n)) return false;
    // ---- star field
    if (from_stars) {
      // the host copy is the field itself: no read-back before the moments
      stars_out.swap(file_stars);
      IRSB_CKR(cudaMemcpyAsync(d_stars_.p, stars_out.data(), size_t(n) * sizeof(StarRec<T>), cudaMemcpyHostToDevice,
                               stream_));
      p.random_seed = 0;
    } else {
      while (p.random_seed == 0)
        p.random_seed = int(std::chrono::system_clock::now().time_since_epoch().count());
      int blocks = std::max(1, std::min(ceil_div(n, 256), 148 * 16));
      generate_stars_kernel<T><<<blocks, 256, 0, stream_>>>(d_stars_.p, n, p.random_seed, p.rectangular, p.corner,
                                                            p.mf_kind, p.m_lower, p.m_upper, p.m_solar);
      IRSB_LAUNCH_CK("generate_stars_kernel");
      stars_out.resize(n);
      IRSB_CKR(cudaMemcpyAsync(stars_out.data(), d_stars_.p, size_t(n) * sizeof(StarRec<T>), cudaMemcpyDeviceToHost,
                               stream_));
      IRSB_CKR(cudaStreamSynchronize(stream_));
    }
    star_field_moments<T>(n, p.rectangular, p.corner, p.theta_star, stars_out.data(), p.kappa_star_actual,
                          p.m_lower_actual, p.m_upper_actual, p.mean_mass_actual, p.mean_mass2_actual,
                          p.mean_mass2_ln_mass_actual);
    if (!from_stars) recompute_corner(p);
    p.root_half_length = root_half_length_of(p);
    if (use_host_stars) p.starfile = "";
    prm = p;

    launches = from_stars ? 0 : 1;  // star generation
    if (!device_pipeline()) return false;
    // stars in tree order, as the reference leaves them
    IRSB_CKR(cudaMemcpyAsync(stars_out.data(), d_stars_.p, size_t(n) * sizeof(StarRec<T>), cudaMemcpyDeviceToHost,
                             stream_));
    n_hist_ = 0;
    if (!verts_only && !post(verbose)) return false;
    IRSB_CKR(cudaStreamSynchronize(stream_));
    if (verbose >= 1) {
      std::cout << (IS_IRS ? "irs" : "ipm") << ": stars " << n << ", tree levels " << prm.tree_levels
                << ", expansion order " << prm.expansion_order << ", leaves " << num_leaves << ", shoot "
                << t_shoot << " s\n";
    }
    return true;
  }

  // Tree -> expansions -> leaf records -> shoot on the resident star field,
  // timed with CUDA events (t_pipeline, t_shoot, t_lattice, t_deposit).
  bool device_pipeline() {
    const int n = prm.num_stars;
    IRSB_CKR(cudaEventRecord(ev0_, stream_));
    if (!build_tree<T>(tree_, d_stars_.p, n, prm.root_half_length, stream_)) return false;
    launches += tree_.launches;
    prm.tree_levels = tree_.levels;
    prm.expansion_order =
        prm.expansion_order_override > 0 ? prm.expansion_order_override : expansion_order_of(prm);
    if (prm.expansion_order < 3) {
      std::cerr << "Error. Expansion order needs to be >= 3\n";
      return false;
    }
    if (prm.expansion_order > kMaxOrder) {
      std::cerr << "Error. Maximum allowed expansion order is " << kMaxOrder << "\n";
      return false;
    }
    if (!compute_fmm<T>(fmm_, tree_, d_stars_.p, prm.expansion_order, stream_)) return false;
    launches += 2LL * (tree_.levels + 1) + std::max(0, tree_.levels - 1);
    const SmoothFold fold{smooth_folded() ? 1 : 0, double(prm.kappa_star), double(prm.corner.re),
                          double(prm.corner.im), 0.318309886183790671537767526745028724, prm.taylor_smooth, nullptr};
    if (!build_leaves<T>(leaves_, tree_, fmm_, d_stars_.p, double(prm.theta_star), stream_, fold)) return false;
    launches += 6;
    num_leaves = leaves_.n;
    if (!shoot()) return false;
    IRSB_CKR(cudaEventRecord(ev2_, stream_));
    IRSB_CKR(cudaEventSynchronize(ev2_));
    float ms_shoot = 0, ms_all = 0, ms_lat = 0, ms_dep = 0;
    IRSB_CKR(cudaEventElapsedTime(&ms_shoot, ev1_, ev2_));
    IRSB_CKR(cudaEventElapsedTime(&ms_all, ev0_, ev2_));
    IRSB_CKR(cudaEventElapsedTime(&ms_lat, ev_lat0_, ev_lat1_));
    t_shoot = ms_shoot * 1e-3;
    t_pipeline = ms_all * 1e-3;
    t_lattice = ms_lat * 1e-3;
    if (!IS_IRS) {
      IRSB_CKR(cudaEventElapsedTime(&ms_dep, ev_lat1_, ev_dep1_));
      t_deposit = ms_dep * 1e-3;
    }
    return true;
  }

  // Re-runs the device pipeline `repeats` times on the star field of the last
  // run(); returns the summed device time of the repeats in *seconds.
  bool rerun(int repeats, double* seconds) {
    if (!stream_ || d_stars_.n == 0) {
      std::cerr << "Error. rerun() needs a completed run().\n";
      return false;
    }
    double tot = 0;
    launches = 0;
    for (int r = 0; r < repeats; r++) {
      if (!device_pipeline()) return false;
      tot += t_pipeline;
    }
    if (seconds) *seconds = tot;
    return true;
  }

  // Writes the reference's output files (include/ipm.cuh:1122-1322).
  bool save(int verbose) {
    if (!fetch_hists()) return false;
    const Params<T>& p = prm;
    const std::string pre = p.outfile_prefix + (IS_IRS ? "irs_" : "ipm_");
    {
      std::ofstream f(pre + "parameter_info.txt");
      if (!f) {
        std::cerr << "Error. Failed to open file " << pre << "parameter_info.txt\n";
        return false;
      }
      f.precision(9);
      f << "kappa_tot " << p.kappa_tot << "\n";
      f << "shear " << p.shear << "\n";
      f << "mu_ave " << p.mu_ave << "\n";
      f << "smooth_fraction " << (1 - p.kappa_star / p.kappa_tot) << "\n";
      f << "kappa_star " << p.kappa_star << "\n";
      if (p.starfile.empty() && !use_host_stars) f << "kappa_star_actual " << p.kappa_star_actual << "\n";
      f << "theta_star " << p.theta_star << "\n";
      f << "random_seed " << p.random_seed << "\n";
      if (p.starfile.empty() && !use_host_stars) {
        f << "mass_function " << p.mass_function << "\n";
        if (p.mass_function == "salpeter" || p.mass_function == "kroupa") f << "m_solar " << p.m_solar << "\n";
        f << "m_lower " << p.m_lower << "\n";
        f << "m_upper " << p.m_upper << "\n";
        f << "mean_mass " << p.mean_mass << "\n";
        f << "mean_mass2 " << p.mean_mass2 << "\n";
        f << "mean_mass2_ln_mass " << p.mean_mass2_ln_mass << "\n";
      }
      f << "m_lower_actual " << p.m_lower_actual << "\n";
      f << "m_upper_actual " << p.m_upper_actual << "\n";
      f << "mean_mass_actual " << p.mean_mass_actual << "\n";
      f << "mean_mass2_actual " << p.mean_mass2_actual << "\n";
      f << "mean_mass2_ln_mass_actual " << p.mean_mass2_ln_mass_actual << "\n";
      f << "light_loss " << p.light_loss << "\n";
      f << "num_stars " << p.num_stars << "\n";
      if (p.rectangular) {
        f << "corner_x1 " << p.corner.re << "\n";
        f << "corner_x2 " << p.corner.im << "\n";
        if (p.approx) f << "taylor_smooth " << p.taylor_smooth << "\n";
      } else {
        f << "rad " << cabs_(p.corner) << "\n";
      }
      f << "safety_scale " << p.safety_scale << "\n";
      f << "center_y1 " << p.center_y.re << "\n";
      f << "center_y2 " << p.center_y.im << "\n";
      f << "half_length_y1 " << p.half_length_y.re << "\n";
      f << "half_length_y2 " << p.half_length_y.im << "\n";
      f << "num_pixels_y1 " << p.num_pixels_y.re << "\n";
      f << "num_pixels_y2 " << p.num_pixels_y.im << "\n";
      f << "center_x1 " << p.center_x.re << "\n";
      f << "center_x2 " << p.center_x.im << "\n";
      f << "half_length_x1 " << p.half_length_x.re << "\n";
      f << "half_length_x2 " << p.half_length_x.im << "\n";
      f << "num_rays_y " << p.num_rays_y << "\n";
      f << "num_rays_x " << p.num_rays_x << "\n";
      f << "ray_half_sep_1 " << p.ray_half_sep.re << "\n";
      f << "ray_half_sep_2 " << p.ray_half_sep.im << "\n";
      f << "alpha_error " << p.alpha_error << "\n";
      f << "expansion_order " << p.expansion_order << "\n";
      f << "root_half_length " << p.root_half_length << "\n";
      f << "num_ray_threads_1 " << p.num_ray_threads.re << "\n";
      f << "num_ray_threads_2 " << p.num_ray_threads.im << "\n";
      f << "tree_levels " << p.tree_levels << "\n";
      if (IS_IRS) {
        f << "num_rays_shot " << num_rays_shot << "\n";
        f << "num_rays_received " << num_rays_received << "\n";
        f << "mean_num_rays_y " << (1.0 * num_rays_received / (1.0 * p.num_pixels_y.re * p.num_pixels_y.im)) << "\n";
        f << "t_shoot_rays " << t_shoot << "\n";
      } else {
        f << "t_shoot_cells " << t_shoot << "\n";
      }
      if (verbose >= 1) std::cout << "Done writing parameter info to file " << pre << "parameter_info.txt\n";
    }
    if (p.write_stars) {
      if (!write_star_file_bin<T>(pre + "stars.bin", p.num_stars, p.rectangular, p.corner, p.theta_star,
                                  stars_out.data())) {
        std::cerr << "Error. Unable to write star info to file " << pre << "stars.bin\n";
        return false;
      }
    }
    if (p.write_histograms) {
      const char* hname = IS_IRS ? "numrays_numpixels" : "mags_numpixels";
      if (!write_hist(pre + hname + ".txt", hist, hist_min)) return false;
      if (!IS_IRS && !write_hist(pre + "log_mags_numpixels.txt", log_hist, log_hist_min)) return false;
      if (p.write_parities) {
        if (!write_hist(pre + hname + "_minima.txt", hist_minima, hist_min)) return false;
        if (!IS_IRS && !write_hist(pre + "log_mags_numpixels_minima.txt", log_hist_minima, log_hist_min)) return false;
        if (!write_hist(pre + hname + "_saddles.txt", hist_saddles, hist_min)) return false;
        if (!IS_IRS && !write_hist(pre + "log_mags_numpixels_saddles.txt", log_hist_saddles, log_hist_min))
          return false;
      }
    }
    if (p.write_maps) {
      if (!write_map(pre + "magnifications.bin", h_pix.p)) return false;
      if (p.write_parities) {
        if (!write_map(pre + "magnifications_minima.bin", h_pmin.p)) return false;
        if (!write_map(pre + "magnifications_saddles.bin", h_psad.p)) return false;
      }
    }
    return true;
  }

  // ---- diagnostics: copies of internal device state (tests and tools)
  int tree_num_nodes() const { return tree_.num_nodes; }
  int tree_levels() const { return tree_.levels; }
  // ints[k*8+.] = level, parent, child0, sbeg, scnt, n_nbr, n_sil, n_dil; geom[k*3+.] = cx, cy, hl
  bool copy_tree(int* ints, double* geom, int* nbr, int* sil, int* dil) {
    const int n = tree_.num_nodes;
    std::vector<int> a(n);
    std::vector<T> g(n);
    auto get_i = [&](const DevVec<int>& v, int col) -> bool {
      if (!IRSB_CK(cudaMemcpy(a.data(), v.p, n * sizeof(int), cudaMemcpyDeviceToHost))) return false;
      for (int k = 0; k < n; k++) ints[8 * (size_t)k + col] = a[k];
      return true;
    };
    auto get_g = [&](const DevVec<T>& v, int col) -> bool {
      if (!IRSB_CK(cudaMemcpy(g.data(), v.p, n * sizeof(T), cudaMemcpyDeviceToHost))) return false;
      for (int k = 0; k < n; k++) geom[3 * (size_t)k + col] = double(g[k]);
      return true;
    };
    if (!get_i(tree_.level, 0) || !get_i(tree_.parent, 1) || !get_i(tree_.child0, 2) || !get_i(tree_.sbeg, 3) ||
        !get_i(tree_.scnt, 4) || !get_i(tree_.n_nbr, 5) || !get_i(tree_.n_sil, 6) || !get_i(tree_.n_dil, 7))
      return false;
    if (!get_g(tree_.cx, 0) || !get_g(tree_.cy, 1) || !get_g(tree_.hl, 2)) return false;
    if (nbr && !IRSB_CK(cudaMemcpy(nbr, tree_.nbr.p, size_t(n) * kMaxNeighbors * sizeof(int), cudaMemcpyDeviceToHost)))
      return false;
    if (sil && !IRSB_CK(cudaMemcpy(sil, tree_.sil.p, size_t(n) * kMaxSameLevelIL * sizeof(int), cudaMemcpyDeviceToHost)))
      return false;
    if (dil && !IRSB_CK(cudaMemcpy(dil, tree_.dil.p, size_t(n) * kMaxDiffLevelIL * sizeof(int), cudaMemcpyDeviceToHost)))
      return false;
    return true;
  }
  // (p+1) complex coefficients per node, interleaved re/im
  bool copy_coeffs(double* mult, double* loc) {
    size_t m = size_t(tree_.num_nodes) * (fmm_.p + 1) * sizeof(double2);
    return IRSB_CK(cudaMemcpy(mult, fmm_.mult.p, m, cudaMemcpyDeviceToHost)) &&
           IRSB_CK(cudaMemcpy(loc, fmm_.loc.p, m, cudaMemcpyDeviceToHost));
  }
  long long num_vertices() const { return (long long)d_verts_.n; }
  // IPM vertex source positions, (x, y) pixel units with the row axis flipped
  bool copy_vertices(double* out) {
    return IRSB_CK(cudaMemcpy(out, d_verts_.p, d_verts_.n * sizeof(double2), cudaMemcpyDeviceToHost));
  }
  // Integer maps copied to caller-provided device buffers (row band reduction):
  // IPM fixed point (uint64), IRS counts (int32). min/sad only with parities.
  bool copy_maps_device(void* total, void* mn, void* sd) {
    const size_t n = size_t(prm.num_pixels_y.re) * prm.num_pixels_y.im;
    const size_t es = IS_IRS ? sizeof(int) : sizeof(unsigned long long);
    const void* a = IS_IRS ? (const void*)d_pix_.p : (const void*)d_acc_.p;
    const void* b = IS_IRS ? (const void*)d_pmin_.p : (const void*)d_acc_min_.p;
    const void* c = IS_IRS ? (const void*)d_psad_.p : (const void*)d_acc_sad_.p;
    if (total && (IS_IRS || !have_parities) && !IRSB_CK(cudaMemcpyAsync(total, a, n * es, cudaMemcpyDeviceToDevice, stream_)))
      return false;
    if (have_parities && mn && !IRSB_CK(cudaMemcpyAsync(mn, b, n * es, cudaMemcpyDeviceToDevice, stream_))) return false;
    if (have_parities && sd && !IRSB_CK(cudaMemcpyAsync(sd, c, n * es, cudaMemcpyDeviceToDevice, stream_))) return false;
    return IRSB_CK(cudaStreamSynchronize(stream_));
  }

  // IPM fixed-point accumulators (2^32 per unit); min/sad only with parities
  bool copy_fixed_maps(unsigned long long* total, unsigned long long* mn, unsigned long long* sd) {
    const size_t n = size_t(prm.num_pixels_y.re) * prm.num_pixels_y.im;
    if (have_parities) {
      return IRSB_CK(cudaMemcpy(mn, d_acc_min_.p, n * 8, cudaMemcpyDeviceToHost)) &&
             IRSB_CK(cudaMemcpy(sd, d_acc_sad_.p, n * 8, cudaMemcpyDeviceToHost));
    }
    return IRSB_CK(cudaMemcpy(total, d_acc_.p, n * 8, cudaMemcpyDeviceToHost));
  }

  // Pointers for in-process callers that keep working on the device maps.
  const Pix* device_pixels() const { return IS_IRS ? (const Pix*)d_pix_.p : (const Pix*)d_map_.p; }
  cudaStream_t stream() const { return stream_; }

 private:
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, ev2_ = nullptr;
  struct HistSlot {
    DevVec<int> dev;
    std::vector<int>* out = nullptr;
    int len = 0;
  };
  static constexpr int kMaxHists = 6;  // linear and log10, of the total, minima and saddle maps
  HistSlot hist_slots_[kMaxHists];
  int n_hist_ = 0;
  cudaEvent_t ev_lat0_ = nullptr, ev_lat1_ = nullptr, ev_dep1_ = nullptr;
  static constexpr int kOutChunks = 16;
  cudaEvent_t out_ev_[kOutChunks] = {};
  Pix* out_user_ = nullptr;  // the next run's map is also copied here (host memory)
  long long out_chunk_ = 0;
  int out_nch_ = 0;
  cudaStream_t copy_stream_ = nullptr;  // the map's transfer beside the histograms
  cudaEvent_t ev_map_ = nullptr;
  DevVec<StarRec<T>> d_stars_;
  TreeDev<T> tree_;
  FmmDev fmm_;
  LeafSet leaves_;
  LatticeTiles tiles_;
  DevVec<int> d_pix_, d_pmin_, d_psad_;
  DevVec<unsigned long long> d_acc_, d_acc_min_, d_acc_sad_;
  DevVec<unsigned long long> d_diff_, d_diff_min_, d_diff_sad_;
  DevVec<T> d_map_, d_map_min_, d_map_sad_;
  DevVec<double2> d_verts_;
  DevVec<unsigned long long> d_red_;
  DevVec<long long> d_mm_;

  bool init_stream() {
    if (stream_) return true;
    IRSB_CKR(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    IRSB_CKR(cudaEventCreate(&ev0_));
    IRSB_CKR(cudaEventCreate(&ev1_));
    IRSB_CKR(cudaEventCreate(&ev2_));
    IRSB_CKR(cudaEventCreate(&ev_lat0_));
    IRSB_CKR(cudaEventCreate(&ev_lat1_));
    IRSB_CKR(cudaEventCreate(&ev_dep1_));
    for (cudaEvent_t& e : out_ev_) IRSB_CKR(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    IRSB_CKR(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    IRSB_CKR(cudaEventCreateWithFlags(&ev_map_, cudaEventDisableTiming));
    return true;
  }

  ShootParams shoot_params(bool vertices) const {
    return make_shoot_params(prm, vertices, vertices ? band_rows().first : 0);
  }

  // [first, last) lattice rows of this object's band (rays or cells).
  std::pair<long long, long long> band_rows() const {
    long long n = prm.num_ray_threads.im;
    long long lo = std::max(0LL, std::min(band_lo, n));
    long long hi = band_hi < 0 ? n : std::max(lo, std::min(band_hi, n));
    return {lo, hi};
  }

  LeafPtrs leaf_ptrs() const {
    LeafPtrs lp;
    lp.cx = leaves_.cx.p;
    lp.cy = leaves_.cy.p;
    lp.hl = leaves_.hl.p;
    lp.nnear = leaves_.nnear.p;
    lp.near64 = leaves_.near64.p;
    lp.near32 = leaves_.near32.p;
    lp.coef64 = leaves_.coef64.p;
    lp.coef32 = leaves_.coef32.p;
    lp.rect = tiles_.rect.p;
    lp.tile_off = tiles_.tile_off.p;
    lp.table = tiles_.table.p;
    lp.smooth0 = smooth_folded() ? leaves_.smooth0.p : nullptr;
    lp.nleaves = leaves_.n;
    return lp;
  }

  int shoot_grid(long long tiles) const {
    long long g = std::min<long long>(tiles, 148LL * std::max(1, shoot_ctas_per_sm));
    return int(std::max<long long>(g, 1));
  }

  template <bool VERT, bool PAR, bool GEN>
  void launch_f32(int grid, const ShootParams& sp, const LeafPtrs& lp, int* pix, int* pmin, int* psad,
                  double2* verts) {
    switch (shoot_threads) {
      case 128:
        shoot_f32<VERT, PAR, GEN, 128><<<grid, 128, 0, stream_>>>(sp, lp, tiles_.total, pix, pmin, psad, verts);
        break;
      case 512:
        shoot_f32<VERT, PAR, GEN, 512><<<grid, 512, 0, stream_>>>(sp, lp, tiles_.total, pix, pmin, psad, verts);
        break;
      default:
        shoot_f32<VERT, PAR, GEN, 256><<<grid, 256, 0, stream_>>>(sp, lp, tiles_.total, pix, pmin, psad, verts);
    }
  }

  template <bool VERT>
  bool launch_shoot(const ShootParams& sp, int* pix, int* pmin, int* psad, double2* verts) {
    LeafPtrs lp = leaf_ptrs();
    int grid = shoot_grid(tiles_.total);
    const bool par = !VERT && prm.write_parities;
    const bool generic = !(prm.approx && !prm.rectangular) && !smooth_folded();
    IRSB_CKR(cudaEventRecord(ev_lat0_, stream_));
    launches++;
    if (tiles_.total == 0) {
      IRSB_CKR(cudaEventRecord(ev_lat1_, stream_));
      return true;
    }
    if (use_fp32()) {
      if (par) {
        if (generic)
          launch_f32<VERT, true, true>(grid, sp, lp, pix, pmin, psad, verts);
        else
          launch_f32<VERT, true, false>(grid, sp, lp, pix, pmin, psad, verts);
      } else {
        if (generic)
          launch_f32<VERT, false, true>(grid, sp, lp, pix, pmin, psad, verts);
        else
          launch_f32<VERT, false, false>(grid, sp, lp, pix, pmin, psad, verts);
      }
    } else {
      if (par)
        shoot_f64<VERT, true><<<grid, kShootThreads, 0, stream_>>>(sp, lp, tiles_.total, pix, pmin, psad, verts);
      else
        shoot_f64<VERT, false><<<grid, kShootThreads, 0, stream_>>>(sp, lp, tiles_.total, pix, pmin, psad, verts);
    }
    IRSB_LAUNCH_CK("shoot");
    IRSB_CKR(cudaEventRecord(ev_lat1_, stream_));
    return true;
  }

  bool shoot() {
    const Params<T>& p = prm;
    const long long npix = (long long)p.num_pixels_y.re * p.num_pixels_y.im;
    const bool par = p.write_parities != 0;
    have_parities = par;
    ShootParams sp = shoot_params(!IS_IRS);
    const auto band = band_rows();
    // rays: rows [lo, hi); cells: rows [lo, hi) need corner rows [lo, hi]
    const long long jlo = band.first, jhi = IS_IRS ? band.second : band.second + 1;
    if (!build_lattice_tiles<T>(tiles_, leaves_, tree_, sp.base_x, sp.base_y, sp.rhs_x, sp.rhs_y, sp.nx, sp.ny, jlo,
                                jhi, stream_))
      return false;
    num_tiles = tiles_.total;
    launches += 4;
    if (!mean_near_count()) return false;
    if (IS_IRS) {
      if (!d_pix_.alloc_exact(npix)) return false;
      if (par && (!d_pmin_.alloc_exact(npix) || !d_psad_.alloc_exact(npix))) return false;
      IRSB_CKR(cudaMemsetAsync(d_pix_.p, 0, npix * sizeof(int), stream_));
      if (par) {
        IRSB_CKR(cudaMemsetAsync(d_pmin_.p, 0, npix * sizeof(int), stream_));
        IRSB_CKR(cudaMemsetAsync(d_psad_.p, 0, npix * sizeof(int), stream_));
      }
      IRSB_CKR(cudaEventRecord(ev1_, stream_));
      if (!launch_shoot<false>(sp, d_pix_.p, d_pmin_.p, d_psad_.p, nullptr)) return false;
      num_rays_shot = (unsigned long long)p.num_ray_threads.re * (unsigned long long)(band.second - band.first);
    } else {
      const long long nverts = sp.nx * (band.second - band.first + 1);
      if (!d_verts_.alloc_exact(nverts)) return false;
      const long long ndiff = (long long)p.num_pixels_y.im * (p.num_pixels_y.re + 1);
      if (!d_acc_.alloc_exact(npix) || !d_map_.alloc_exact(npix) || !d_diff_.alloc_exact(ndiff)) return false;
      if (par && (!d_acc_min_.alloc_exact(npix) || !d_acc_sad_.alloc_exact(npix) || !d_map_min_.alloc_exact(npix) ||
                  !d_map_sad_.alloc_exact(npix) || !d_diff_min_.alloc_exact(ndiff) || !d_diff_sad_.alloc_exact(ndiff)))
        return false;
      IRSB_CKR(cudaEventRecord(ev1_, stream_));
      IRSB_CKR(cudaMemsetAsync(d_acc_.p, 0, npix * sizeof(unsigned long long), stream_));
      IRSB_CKR(cudaMemsetAsync(d_diff_.p, 0, ndiff * sizeof(unsigned long long), stream_));
      if (par) {
        IRSB_CKR(cudaMemsetAsync(d_acc_min_.p, 0, npix * sizeof(unsigned long long), stream_));
        IRSB_CKR(cudaMemsetAsync(d_acc_sad_.p, 0, npix * sizeof(unsigned long long), stream_));
        IRSB_CKR(cudaMemsetAsync(d_diff_min_.p, 0, ndiff * sizeof(unsigned long long), stream_));
        IRSB_CKR(cudaMemsetAsync(d_diff_sad_.p, 0, ndiff * sizeof(unsigned long long), stream_));
      }
      DepositMaps mt{d_acc_.p, d_diff_.p}, mmin{d_acc_min_.p, d_diff_min_.p}, msad{d_acc_sad_.p, d_diff_sad_.p};
      if (!launch_shoot<true>(sp, nullptr, nullptr, nullptr, d_verts_.p)) return false;
      if (verts_only) {  // the corner lattice is the product (adaptive deposition)
        IRSB_CKR(cudaEventRecord(ev_dep1_, stream_));
        return true;
      }
      const long long ncx = p.num_ray_threads.re, ncy = band.second - band.first;
      long long ncells = ncx * ncy;
      const int grid = deposit_grid((ncells + 31) / 32);
      if (use_fp32()) {
        const float factor = ipm_triangle_factor<T, float>(p);
        ipm_deposit_cells<float><<<grid, kDepositThreads, 0, stream_>>>(d_verts_.p, ncx, ncy, factor, p.num_pixels_y.re,
                                                            p.num_pixels_y.im, mt, mmin, msad, par ? 1 : 0);
      } else {
        const double factor = ipm_triangle_factor<T, double>(p);
        ipm_deposit_cells<double><<<grid, kDepositThreads, 0, stream_>>>(d_verts_.p, ncx, ncy, factor, p.num_pixels_y.re,
                                                             p.num_pixels_y.im, mt, mmin, msad, par ? 1 : 0);
      }
      IRSB_LAUNCH_CK("ipm_deposit_cells");
      IRSB_CKR(cudaEventRecord(ev_dep1_, stream_));
      {
        int gr = std::max(1, std::min(ceil_div((long long)p.num_pixels_y.im * 32, 256), 148 * 8));
        if (par) {
          ipm_resolve_rows<<<gr, 256, 0, stream_>>>(p.num_pixels_y.re, p.num_pixels_y.im, mmin);
          ipm_resolve_rows<<<gr, 256, 0, stream_>>>(p.num_pixels_y.re, p.num_pixels_y.im, msad);
        } else {  // resolve and convert in one pass
          ipm_resolve_rows_out<T><<<gr, 256, 0, stream_>>>(p.num_pixels_y.re, p.num_pixels_y.im, mt, d_map_.p);
        }
        IRSB_LAUNCH_CK("ipm_resolve_rows");
      }
      launches += par ? 4 : 2;
      if (par) {
        int g2 = int(std::max<long long>(1, std::min<long long>((npix + 255) / 256, 148LL * 16)));
        ipm_finalize<T><<<g2, 256, 0, stream_>>>(npix, d_acc_.p, d_acc_min_.p, d_acc_sad_.p, d_map_.p,
                                                   d_map_min_.p, d_map_sad_.p, 1);
        IRSB_LAUNCH_CK("ipm_finalize");
      }
    }
    return true;
  }

  // Mean near-field size over the lattice points (algorithmic work per point).
  bool mean_near_count() {
    std::vector<int4> r(leaves_.n);
    std::vector<int> nn(leaves_.n);
    if (leaves_.n == 0) {
      mean_near = 0;
      return true;
    }
    IRSB_CKR(cudaMemcpyAsync(r.data(), tiles_.rect.p, r.size() * sizeof(int4), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaMemcpyAsync(nn.data(), leaves_.nnear.p, nn.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    double acc = 0, pts = 0;
    for (int l = 0; l < leaves_.n; l++) {
      double c = double(std::max(0, r[l].y - r[l].x)) * double(std::max(0, r[l].w - r[l].z));
      acc += c * nn[l];
      pts += c;
    }
    mean_near = pts > 0 ? acc / pts : 0;
    return true;
  }

  template <typename V>
  bool minmax(const V* v, long long n, long long& lo, long long& hi) {
    using K = typename OrderedKey<V>::K;
    if (!d_mm_.alloc_exact(2)) return false;
    K init[2];
    if constexpr (sizeof(K) == 4) {
      init[0] = 0x7fffffff;
      init[1] = int(0x80000000);
    } else {
      init[0] = 0x7fffffffffffffffLL;
      init[1] = (long long)0x8000000000000000ULL;
    }
    K* dm = reinterpret_cast<K*>(d_mm_.p);
    IRSB_CKR(cudaMemcpyAsync(dm, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
    int g = int(std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 8)));
    minmax_nonneg<V><<<g, 256, 0, stream_>>>(v, n, dm);
    IRSB_LAUNCH_CK("minmax_nonneg");
    K out[2];
    IRSB_CKR(cudaMemcpyAsync(out, dm, sizeof(out), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    lo = (long long)out[0];
    hi = (long long)out[1];
    return true;
  }
  template <typename V>
  static V decode(long long k) {
    if constexpr (std::is_same<V, int>::value) return V(k);
    else if constexpr (std::is_same<V, float>::value) {
      int b = int(k);
      float f;
      std::memcpy(&f, &b, 4);
      return f;
    } else {
      double d;
      std::memcpy(&d, &k, 8);
      return d;
    }
  }

  template <typename V>
  bool value_range(const V* v, long long n, V& lo, V& hi) {
    long long a, b;
    if (!minmax<V>(v, n, a, b)) return false;
    lo = decode<V>(a);
    hi = decode<V>(b);
    return true;
  }

  // Histogram of a device map, counted on the device and kept there: `out`
  // is filled by fetch_hists() when save() writes it (the histograms are not
  // otherwise read), so run() does not copy them back.
  template <typename V>
  bool make_hist(const V* v, long long n, int hmin, int len, int factor, int use_log, std::vector<int>& out) {
    if (n_hist_ >= kMaxHists) return false;
    HistSlot& h = hist_slots_[n_hist_++];
    if (!h.dev.alloc_exact(len)) return false;
    IRSB_CKR(cudaMemsetAsync(h.dev.p, 0, size_t(len) * sizeof(int), stream_));
    if (len <= kHistSmemBins) {
      int g = int(std::max<long long>(1, std::min<long long>((n + 1023) / 1024, 148LL)));
      histogram_map_smem<V><<<g, 1024, size_t(len) * sizeof(int), stream_>>>(v, n, hmin, len, factor, use_log,
                                                                            h.dev.p);
    } else {
      int g = int(std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 8)));
      histogram_map<V><<<g, 256, 0, stream_>>>(v, n, hmin, len, factor, use_log, h.dev.p);
    }
    IRSB_LAUNCH_CK("histogram_map");
    h.out = &out;
    h.len = len;
    return true;
  }
  // device histograms of the last run -> result vectors
  bool fetch_hists() {
    for (int i = 0; i < n_hist_; i++) {
      HistSlot& h = hist_slots_[i];
      h.out->resize(h.len);
      if (!IRSB_CK(cudaMemcpy(h.out->data(), h.dev.p, size_t(h.len) * sizeof(int), cudaMemcpyDeviceToHost)))
        return false;
    }
    n_hist_ = 0;
    return true;
  }

  bool post(int verbose) {
    const Params<T>& p = prm;
    const long long npix = (long long)p.num_pixels_y.re * p.num_pixels_y.im;
    const bool par = p.write_parities != 0;
    const Pix* dmap = IS_IRS ? (const Pix*)d_pix_.p : (const Pix*)d_map_.p;
    const Pix* dmin = IS_IRS ? (const Pix*)d_pmin_.p : (const Pix*)d_map_min_.p;
    const Pix* dsad = IS_IRS ? (const Pix*)d_psad_.p : (const Pix*)d_map_sad_.p;
    bool copy_started = false;
    if (IS_IRS) {
      if (!d_red_.alloc_exact(1)) return false;
      IRSB_CKR(cudaMemsetAsync(d_red_.p, 0, sizeof(unsigned long long), stream_));
      int g = int(std::max<long long>(1, std::min<long long>((npix + 255) / 256, 148LL * 8)));
      sum_int_map<<<g, 256, 0, stream_>>>(d_pix_.p, npix, d_red_.p);
      IRSB_LAUNCH_CK("sum_int_map");
      IRSB_CKR(cudaMemcpyAsync(&num_rays_received, d_red_.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               stream_));
    }
    if (p.write_histograms) {
      const int factor = IS_IRS ? 1 : 1000;
      Pix lo, hi;
      if (!value_range<Pix>(dmap, npix, lo, hi)) return false;
      long long mn = llround(double(lo) * factor), mx = llround(double(hi) * factor);
      if (IS_IRS) {
        mn = (long long)lo;
        mx = (long long)hi;
      } else {
        mn = (long long)std::round(T(lo * factor));
        mx = (long long)std::round(T(hi * factor));
      }
      T mu_min_theory = 1 / ((1 - p.kappa_tot + p.kappa_star) * (1 - p.kappa_tot + p.kappa_star));
      T mu_min_actual = IS_IRS ? T(1.0 * mn / p.num_rays_y) : T(1.0 * mn / factor);
      if (p.mu_ave > 1 && mu_min_actual < mu_min_theory)
        std::cerr << "Warning. Minimum magnification after shooting is less than the theoretical minimum.\n";
      if (par) {
        Pix a, b, c, d;
        if (!value_range<Pix>(dmin, npix, a, b) || !value_range<Pix>(dsad, npix, c, d)) return false;
        long long mna, mxa, mnc, mxc;
        if (IS_IRS) {
          mna = a; mxa = b; mnc = c; mxc = d;
        } else {
          mna = (long long)std::round(T(a * factor));
          mxa = (long long)std::round(T(b * factor));
          mnc = (long long)std::round(T(c * factor));
          mxc = (long long)std::round(T(d * factor));
        }
        mn = std::min({mn, mna, mnc});
        mx = std::max({mx, mxa, mxc});
      }
      hist_min = int(mn);
      hist_len = int(mx - mn + 1);
      if (hist_len < 1 || hist_len > (1 << 28)) {
        std::cerr << "Error. Histogram range is not valid.\n";
        return false;
      }
      // the map's range is read: its transfer can run beside the histograms
      // (with parity maps, their range reads would queue behind it)
      if (!par) {
        if (!start_map_copy(dmap, npix, copy_stream_)) return false;
        copy_started = true;
      }
      if (!make_hist<Pix>(dmap, npix, hist_min, hist_len, factor, 0, hist)) return false;
      if (par) {
        if (!make_hist<Pix>(dmin, npix, hist_min, hist_len, factor, 0, hist_minima)) return false;
        if (!make_hist<Pix>(dsad, npix, hist_min, hist_len, factor, 0, hist_saddles)) return false;
      }
      if (!IS_IRS) {
        auto lg = [&](Pix v) -> long long {
          T l = T(std::log10(T(v)));
          return (long long)std::round(T(l * factor));
        };
        // empty pixels (mu = 0) have no logarithm; the range uses the smallest positive value
        long long lmn = (lo > 0) ? lg(lo) : lg(std::max<Pix>(hi * Pix(1e-6), Pix(1e-30)));
        long long lmx = (hi > 0) ? lg(hi) : 0;
        if (par) {
          Pix a, b, c, d;
          if (!value_range<Pix>(dmin, npix, a, b) || !value_range<Pix>(dsad, npix, c, d)) return false;
          if (a > 0) lmn = std::min(lmn, lg(a));
          if (c > 0) lmn = std::min(lmn, lg(c));
          if (b > 0) lmx = std::max(lmx, lg(b));
          if (d > 0) lmx = std::max(lmx, lg(d));
        }
        log_hist_min = int(lmn);
        log_hist_len = int(lmx - lmn + 1);
        if (log_hist_len < 1 || log_hist_len > (1 << 28)) log_hist_len = 1;
        if (!make_hist<Pix>(dmap, npix, log_hist_min, log_hist_len, factor, 1, log_hist)) return false;
        if (par) {
          if (!make_hist<Pix>(dmin, npix, log_hist_min, log_hist_len, factor, 1, log_hist_minima)) return false;
          if (!make_hist<Pix>(dsad, npix, log_hist_min, log_hist_len, factor, 1, log_hist_saddles)) return false;
        }
      }
    }
    // maps to the host (the total map's transfer may have started above)
    if (!copy_started && !start_map_copy(dmap, npix, stream_)) return false;
    if (par) {
      if (!h_pmin.alloc(npix) || !h_psad.alloc(npix)) return false;
      IRSB_CKR(cudaMemcpyAsync(h_pmin.p, dmin, npix * sizeof(Pix), cudaMemcpyDeviceToHost, stream_));
      IRSB_CKR(cudaMemcpyAsync(h_psad.p, dsad, npix * sizeof(Pix), cudaMemcpyDeviceToHost, stream_));
    }
    (void)verbose;
    return finish_map_copy(npix);
  }

  // The total map to pinned host memory in chunks on stream st (after the map
  // is final on stream_), an event per chunk.
  bool start_map_copy(const Pix* dmap, long long npix, cudaStream_t st) {
    if (!h_pix.alloc(npix)) return false;
    if (st != stream_) {
      IRSB_CKR(cudaEventRecord(ev_map_, stream_));
      IRSB_CKR(cudaStreamWaitEvent(st, ev_map_, 0));
    }
    out_chunk_ = std::max<long long>(1 << 19, (npix + kOutChunks - 1) / kOutChunks);
    out_nch_ = int((npix + out_chunk_ - 1) / out_chunk_);
    for (int i = 0; i < out_nch_; i++) {
      const long long a = i * out_chunk_, n = std::min(npix, a + out_chunk_) - a;
      IRSB_CKR(cudaMemcpyAsync(h_pix.p + a, dmap + a, n * sizeof(Pix), cudaMemcpyDeviceToHost, st));
      IRSB_CKR(cudaEventRecord(out_ev_[i], st));
    }
    return true;
  }
  // Waits for the chunks; with a caller buffer set (set_pixels_out), the host
  // threads copy each chunk on while the next ones are still in transfer.
  bool finish_map_copy(long long npix) {
    Pix* user = out_user_;
    out_user_ = nullptr;
    for (int i = 0; i < out_nch_; i++) {
      const long long a = i * out_chunk_, n = std::min(npix, a + out_chunk_) - a;
      IRSB_CKR(cudaEventSynchronize(out_ev_[i]));
      if (!user) continue;
      const long long sub = (n + 7) / 8;
#pragma omp parallel for schedule(static) num_threads(8)
      for (int t = 0; t < 8; t++) {
        const long long b = a + t * sub, e = std::min(a + n, b + sub);
        if (b < e) std::memcpy(user + b, h_pix.p + b, size_t(e - b) * sizeof(Pix));
      }
    }
    out_nch_ = 0;
    return true;
  }

  static bool write_hist(const std::string& fname, const std::vector<int>& h, int hmin) {
    std::ofstream f(fname);
    if (!f) {
      std::cerr << "Error. Failed to open file " << fname << "\n";
      return false;
    }
    for (size_t i = 0; i < h.size(); i++)
      if (h[i] != 0) f << (long long)i + hmin << " " << h[i] << "\n";
    return true;
  }
  bool write_map(const std::string& fname, const Pix* v) {
    std::ofstream f(fname, std::ios::binary);
    if (!f) {
      std::cerr << "Error. Failed to open file " << fname << "\n";
      return false;
    }
    int nrows = prm.num_pixels_y.im, ncols = prm.num_pixels_y.re;
    f.write(reinterpret_cast<const char*>(&nrows), sizeof(int));
    f.write(reinterpret_cast<const char*>(&ncols), sizeof(int));
    f.write(reinterpret_cast<const char*>(v), size_t(nrows) * ncols * sizeof(Pix));
    return bool(f);
  }
};

}  // namespace irsb
