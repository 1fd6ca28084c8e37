// CCF<T>: critical curves and caustics of a star field, the host side of
// include/ccf.cuh (class CCF). Same inputs, defaults, checks, derived values,
// star field, tree and expansion order, root layout, outputs and files; the
// root finding runs the kernels of ccf.cuh (FP64).
#pragma once
#include "ccf.cuh"
#include "params.hpp"
#include "stars.cuh"

#include <chrono>
#include <functional>
#include <fstream>
#include <iostream>

namespace irsb {

template <typename T>
class CCF {
 public:
  // ---- inputs (defaults of include/ccf.cuh:42-63) ----
  T kappa_tot = T(0.3);
  T shear = T(0.3);
  T kappa_star = T(0.27);
  T theta_star = T(1);
  std::string mass_function_str = "equal";
  T m_solar = T(1);
  T m_lower = T(0.01);
  T m_upper = T(50);
  int rectangular = 0;
  int approx = 1;
  T safety_scale = T(1.37);
  int num_stars = 137;
  std::string starfile = "";
  int num_phi = 100;
  int num_branches = 1;
  int random_seed = 0;
  int write_stars = 1;
  int write_critical_curves = 1;
  int write_caustics = 1;
  int write_mu_length_scales = 0;
  std::string outfile_prefix = "./";
  // extension: simultaneous-update iterations at the branch centres and per
  // phi step (the reference uses 30 and 20, ccf.cuh:913, :985); rounded up to
  // even counts (the update alternates between two buffers)
  int num_iters_init = 30;
  int num_iters_step = 20;

  // ---- results ----
  double t_init_roots = 0, t_ccs = 0, t_caustics = 0;
  T max_error = 0;
  T mu_ave = 0, kappa_star_actual = 0, m_lower_actual = 0, m_upper_actual = 0;
  T mean_mass = 0, mean_mass2 = 0, mean_mass2_ln_mass = 0;
  T mean_mass_actual = 0, mean_mass2_actual = 0, mean_mass2_ln_mass_actual = 0;
  cplx<T> corner = mk<T>(0, 0);
  int taylor_smooth = 1, expansion_order = 0, tree_levels = 0, num_roots = 0;
  T alpha_error = 0, root_half_length = 0;
  T m_lower_run = 0, m_upper_run = 0;  // mass limits of the last run in mass units
  std::vector<StarRec<T>> stars_out;
  std::vector<double2> ccs, caustics;
  std::vector<double> mu_length_scales;

  ~CCF() {
    for (cudaEvent_t* e : {&e0_, &e1_, &e2_, &e3_})
      if (*e) cudaEventDestroy(*e);
    if (stream_) cudaStreamDestroy(stream_);
  }

  int get_num_roots() const { return num_roots; }
  cplx<T> get_corner() const { return rectangular ? corner : mk<T>(cabs_(corner), T(0)); }
  T* stars_ptr() { return stars_out.empty() ? nullptr : &stars_out[0].x; }
  T* ccs_ptr() { return ccs.empty() ? nullptr : reinterpret_cast<T*>(ccs.data()); }
  T* caustics_ptr() { return caustics.empty() ? nullptr : reinterpret_cast<T*>(caustics.data()); }
  T* mu_ptr() { return mu_length_scales.empty() ? nullptr : reinterpret_cast<T*>(mu_length_scales.data()); }

  // include/ccf.cuh:218-346
  bool check_input_params() const {
    const T tmin = std::numeric_limits<T>::min();
    auto fail = [](const char* m) {
      std::cerr << "Error. " << m << "\n";
      return false;
    };
    if (kappa_tot < tmin) return fail("kappa_tot must be >= the smallest positive normal number");
    if (kappa_star < tmin) return fail("kappa_star must be >= the smallest positive normal number");
    if (starfile.empty() && kappa_star > kappa_tot) return fail("kappa_star must be <= kappa_tot");
    if (starfile.empty() && theta_star < tmin) return fail("theta_star must be >= the smallest positive normal number");
    if (starfile.empty() && mass_function_kind(mass_function_str.c_str()) < 0)
      return fail("mass_function must be equal, uniform, Salpeter, Kroupa, or optical_depth.");
    if (starfile.empty() && m_solar < tmin) return fail("m_solar must be >= the smallest positive normal number");
    if (starfile.empty() && m_lower < tmin) return fail("m_lower must be >= the smallest positive normal number");
    if (starfile.empty() && m_upper < m_lower) return fail("m_upper must be >= m_lower.");
    if (starfile.empty() && rectangular != 0 && rectangular != 1)
      return fail("rectangular must be 1 (rectangular) or 0 (circular).");
    if (approx != 0 && approx != 1) return fail("approx must be 1 (approximate) or 0 (exact).");
    if (safety_scale < T(1.1)) return fail("safety_scale must be >= 1.1");
    if (num_stars < 1) return fail("num_stars must be an integer > 0");
    if (num_phi < 1 || num_phi % 2 != 0) return fail("num_phi must be an even integer > 0");
    if (num_branches < 1) return fail("num_branches must be an integer > 0");
    if (num_phi % (2 * num_branches) != 0) return fail("num_phi must be a multiple of 2 * num_branches");
    for (int v : {write_stars, write_critical_curves, write_caustics, write_mu_length_scales})
      if (v != 0 && v != 1) return fail("write flags must be 1 (true) or 0 (false).");
    if (num_iters_init < 1 || num_iters_step < 1) return fail("iteration counts must be >= 1");
    return true;
  }

  bool run(int verbose) {
    if (!check_input_params()) return false;
    if (!stream_) {
      IRSB_CKR(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
      for (cudaEvent_t* e : {&e0_, &e1_, &e2_, &e3_}) IRSB_CKR(cudaEventCreate(e));
    }
    cudaStream_t s = stream_;
    // ---- derived parameters (include/ccf.cuh:348-497)
    std::vector<StarRec<T>> field;
    int mf = kMFEqual;
    if (starfile.empty()) {
      mf = mass_function_kind(mass_function_str.c_str());
      // mass limits in mass units (the inputs stay as given)
      m_lower_run = mf == kMFEqual ? T(1) : m_lower * m_solar;
      m_upper_run = mf == kMFEqual ? T(1) : m_upper * m_solar;
      mean_mass = mf_moment<T>(mf, m_lower_run, m_upper_run, m_solar, 0);
      mean_mass2 = mf_moment<T>(mf, m_lower_run, m_upper_run, m_solar, 1);
      mean_mass2_ln_mass = mf_moment<T>(mf, m_lower_run, m_upper_run, m_solar, 2);
    } else {
      const std::string ext = std::filesystem::path(starfile).extension().string();
      bool ok = false;
      if (ext == ".bin")
        ok = read_star_file_bin<T>(starfile, num_stars, rectangular, corner, theta_star, field);
      else if (ext == ".txt")
        ok = read_star_file_txt<T>(starfile, num_stars, rectangular, corner, theta_star, field);
      if (!ok) {
        std::cerr << "Error. Unable to read star field parameters from file " << starfile << "\n";
        return false;
      }
      star_field_moments<T>(num_stars, rectangular, corner, theta_star, field.data(), kappa_star, m_lower_run,
                            m_upper_run, mean_mass, mean_mass2, mean_mass2_ln_mass);
      if (kappa_star > kappa_tot) std::cerr << "Warning. kappa_star > kappa_tot\n";
    }
    mu_ave = T(1) / ((1 - kappa_tot) * (1 - kappa_tot) - shear * shear);
    if (starfile.empty()) {
      cplx<T> c = mk<T>(1 / std::abs(1 - kappa_tot + shear), 1 / std::abs(1 - kappa_tot - shear));
      corner = rectangular ? scaled_rect(c, mean_mass) : scaled_circle(c, mean_mass);
    }
    alpha_error = theta_star * T(0.0000001);  // 1e-7 Einstein radii
    taylor_smooth = 1;
    const T cab = cabs_(corner);
    while ((kappa_star * kInvPi<T> * 4 / (taylor_smooth + 1) * cab * (safety_scale + 1) / (safety_scale - 1) *
                std::pow(1 / safety_scale, taylor_smooth + 1) >
            alpha_error) &&
           taylor_smooth <= kMaxTaylorSmooth)
      taylor_smooth += 2;
    const T ca = carg(corner);
    while ((std::fmod(ca * (taylor_smooth - 1), kPi<T>) < 0.1 * kPi<T> ||
            std::fmod(ca * (taylor_smooth - 1), kPi<T>) > 0.9 * kPi<T>) &&
           taylor_smooth <= kMaxTaylorSmooth)
      taylor_smooth += 2;
    if (rectangular && taylor_smooth > kMaxTaylorSmooth) {
      std::cerr << "Error. taylor_smooth must be <= " << kMaxTaylorSmooth << "\n";
      return false;
    }
    num_roots = rectangular ? (approx ? 2 * num_stars + taylor_smooth - 1 : 2 * num_stars)
                            : (approx ? 2 * num_stars : 2 * num_stars + 2);

    // ---- star field (include/ccf.cuh:602-700)
    const int n = num_stars;
    if (!d_stars_.alloc_exact(n)) return false;
    if (starfile.empty()) {
      while (random_seed == 0) random_seed = int(std::chrono::system_clock::now().time_since_epoch().count());
      const int blocks = std::max(1, std::min(ceil_div(n, 256), 148 * 16));
      generate_stars_kernel<T><<<blocks, 256, 0, s>>>(d_stars_.p, n, random_seed, rectangular, corner, mf,
                                                       m_lower_run, m_upper_run, m_solar);
      IRSB_LAUNCH_CK("generate_stars_kernel");
      field.resize(n);
      IRSB_CKR(cudaMemcpyAsync(field.data(), d_stars_.p, size_t(n) * sizeof(StarRec<T>), cudaMemcpyDeviceToHost, s));
      IRSB_CKR(cudaStreamSynchronize(s));
    } else {
      random_seed = 0;
      IRSB_CKR(cudaMemcpyAsync(d_stars_.p, field.data(), size_t(n) * sizeof(StarRec<T>), cudaMemcpyHostToDevice, s));
    }
    star_field_moments<T>(n, rectangular, corner, theta_star, field.data(), kappa_star_actual, m_lower_actual,
                          m_upper_actual, mean_mass_actual, mean_mass2_actual, mean_mass2_ln_mass_actual);
    if (starfile.empty())  // the corner from the realised mean mass (include/ccf.cuh:684-697)
      corner = rectangular ? scaled_rect(corner, mean_mass_actual) : scaled_circle(corner, mean_mass_actual);
    // ---- initial roots at each branch centre: star +/- 1, the rest on the
    // circle of radius |corner| (include/ccf.cuh:706-726)
    const int rows = num_phi + num_branches;
    std::vector<double2> init((size_t)rows * num_roots, make_double2(0, 0));
    const CcfParams P = params();
    for (int c = 0; c < num_branches; c++) {
      double2* r = init.data() + (size_t)ccf_row(P, c, 0) * num_roots;
      for (int i = 0; i < n; i++) {
        r[i] = make_double2(double(field[i].x) + 1.0, double(field[i].y));
        r[i + n] = make_double2(double(field[i].x) - 1.0, double(field[i].y));
      }
      const int extra = num_roots - 2 * n;
      for (int i = 0; i < extra; i++) {
        const double ang = 2 * kPi<double> / extra * i;
        r[2 * n + i] = make_double2(double(cabs_(corner)) * std::cos(ang), double(cabs_(corner)) * std::sin(ang));
      }
    }
    // ---- tree and expansions (include/ccf.cuh:732-904)
    root_half_length = T((rectangular ? std::max(corner.re, corner.im) : cabs_(corner)) * 1.1);
    if (!build_tree<T>(tree_, d_stars_.p, n, root_half_length, s)) return false;
    tree_levels = tree_.levels;
    expansion_order = static_cast<int>(std::ceil(2 * std::log2(theta_star) + tree_levels -
                                                 std::log2(root_half_length) - std::log2(alpha_error)));
    if (expansion_order < 3) {
      std::cerr << "Error. Expansion order needs to be >= 3\n";
      return false;
    }
    if (expansion_order > kMaxOrder) {
      std::cerr << "Error. Maximum allowed expansion order is " << kMaxOrder << "\n";
      return false;
    }
    if (!compute_fmm<T>(fmm_, tree_, d_stars_.p, expansion_order, s)) return false;
    if (!build_leaves<T>(leaves_, tree_, fmm_, d_stars_.p, double(theta_star), s)) return false;
    stars_out.resize(n);
    IRSB_CKR(cudaMemcpyAsync(stars_out.data(), d_stars_.p, size_t(n) * sizeof(StarRec<T>), cudaMemcpyDeviceToHost,
                             s));
    IRSB_CKR(cudaStreamSynchronize(s));
    std::vector<double2> pos(n);  // star positions in tree order, for the sums over all stars
    for (int i = 0; i < n; i++) pos[i] = make_double2(double(stars_out[i].x), double(stars_out[i].y));
    if (!d_spos_.alloc_exact(n)) return false;
    IRSB_CKR(cudaMemcpyAsync(d_spos_.p, pos.data(), n * sizeof(double2), cudaMemcpyHostToDevice, s));

    // ---- roots
    const CcfParams Q = params();
    const int nch = 2 * num_branches;
    if (!d_roots_.alloc_exact(init.size()) || !d_scratch_.alloc_exact((size_t)nch * num_roots) ||
        !d_fin_.alloc_exact((size_t)nch * num_roots) || !d_stat_.alloc_exact(2))
      return false;
    IRSB_CKR(cudaMemcpyAsync(d_roots_.p, init.data(), init.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemsetAsync(d_fin_.p, 0, (size_t)nch * num_roots, s));
    const LeafPtrs lp = leaf_ptrs();
    const DescentPtrs<T> dp{tree_.cx.p, tree_.cy.p, tree_.child0.p, leaves_.pos.p, nullptr};
    const int rpb = kCcfThreads / 32;  // roots per CTA (a warp each)
    const dim3 g0(ceil_div(num_roots, rpb), num_branches), g1(ceil_div(num_roots, rpb), nch);
    const int it0 = num_iters_init + (num_iters_init & 1), it1 = num_iters_step + (num_iters_step & 1);
    // The root finding is ~1000 short launches: each part is captured as a
    // CUDA graph and replayed, so the launches cost no host round trips.
    const int half = num_phi / (2 * num_branches);
    const int gp = std::max(1, std::min(ceil_div(nch * num_roots, 256), 148 * 8));
    cudaGraphExec_t centres = nullptr, steps = nullptr;
    auto capture = [&](cudaGraphExec_t& exec, const std::function<void()>& launches) -> bool {
      cudaGraph_t g = nullptr;
      IRSB_CKR(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      launches();
      const cudaError_t le = cudaGetLastError();
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (le != cudaSuccess || ce != cudaSuccess) {
        std::cerr << "Error. Capturing the root finding failed: " << cudaGetErrorString(le != cudaSuccess ? le : ce)
                  << "\n";
        if (g) cudaGraphDestroy(g);
        return false;
      }
      const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      return IRSB_CK(ie);
    };
    const bool ok_graphs =
        capture(centres,
                [&] {
                  for (int i = 0; i < it0; i++)  // branch centres (include/ccf.cuh:906-977)
                    ccf_iterate<T><<<g0, kCcfThreads, 0, s>>>(Q, lp, dp, d_stars_.p, d_spos_.p, 0, 1, i & 1,
                                                              d_roots_.p, d_scratch_.p, d_fin_.p);
                }) &&
        capture(steps, [&] {
          for (int j = 1; j <= half; j++) {  // steps away from the centres (include/ccf.cuh:979-1037)
            ccf_prepare<<<gp, 256, 0, s>>>(Q, j, d_roots_.p, d_fin_.p);
            for (int i = 0; i < it1; i++)
              ccf_iterate<T><<<g1, kCcfThreads, 0, s>>>(Q, lp, dp, d_stars_.p, d_spos_.p, j, 2, i & 1, d_roots_.p,
                                                        d_scratch_.p, d_fin_.p);
          }
        });
    bool ok_run = ok_graphs;
    if (ok_run) {
      ok_run = IRSB_CK(cudaEventRecord(e0_, s)) && IRSB_CK(cudaGraphLaunch(centres, s)) &&
               IRSB_CK(cudaEventRecord(e1_, s)) && IRSB_CK(cudaGraphLaunch(steps, s)) &&
               IRSB_CK(cudaEventRecord(e2_, s)) && IRSB_CK(cudaStreamSynchronize(s));
    }
    if (centres) cudaGraphExecDestroy(centres);
    if (steps) cudaGraphExecDestroy(steps);
    if (!ok_run) return false;
    // ---- error bound in 1/mu over every root (include/ccf.cuh:1044-1069)
    IRSB_CKR(cudaMemsetAsync(d_stat_.p, 0, 2 * sizeof(unsigned long long), s));
    const long long total = (long long)rows * num_roots;
    const int ge = int(std::max<long long>(1, std::min<long long>(ceil_div(total, 256LL), 148LL * 8)));
    ccf_errors<T><<<ge, 256, 0, s>>>(Q, lp, dp, d_stars_.p, d_roots_.p, d_stat_.p,
                                     reinterpret_cast<int*>(d_stat_.p + 1));
    IRSB_LAUNCH_CK("ccf_errors");
    unsigned long long st[2] = {0, 0};
    IRSB_CKR(cudaMemcpyAsync(st, d_stat_.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    if (int(st[1] & 0xffffffffu)) {
      std::cerr << "Error. Errors in 1/mu contain values which are not positive real numbers.\n";
      return false;
    }
    double me;
    std::memcpy(&me, &st[0], sizeof(double));
    max_error = T(me);
    // ---- outputs: critical curves [root][row], caustics, length scales
    if (!d_ccs_.alloc_exact(total) || (write_caustics && !d_caus_.alloc_exact(total)) ||
        (write_mu_length_scales && !d_mu_.alloc_exact(total)))
      return false;
    IRSB_CKR(cudaEventRecord(e3_, s));
    ccf_outputs<T><<<ge, 256, 0, s>>>(Q, lp, dp, d_stars_.p, d_roots_.p, d_ccs_.p,
                                      write_caustics ? d_caus_.p : nullptr, write_mu_length_scales ? d_mu_.p : nullptr);
    IRSB_LAUNCH_CK("ccf_outputs");
    cudaEvent_t e4 = nullptr;
    IRSB_CKR(cudaEventCreate(&e4));
    IRSB_CKR(cudaEventRecord(e4, s));
    ccs.resize(total);
    IRSB_CKR(cudaMemcpyAsync(ccs.data(), d_ccs_.p, total * sizeof(double2), cudaMemcpyDeviceToHost, s));
    caustics.clear();
    mu_length_scales.clear();
    if (write_caustics) {
      caustics.resize(total);
      IRSB_CKR(cudaMemcpyAsync(caustics.data(), d_caus_.p, total * sizeof(double2), cudaMemcpyDeviceToHost, s));
    }
    if (write_mu_length_scales) {
      mu_length_scales.resize(total);
      IRSB_CKR(cudaMemcpyAsync(mu_length_scales.data(), d_mu_.p, total * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    IRSB_CKR(cudaStreamSynchronize(s));
    float m01 = 0, m12 = 0, m34 = 0;
    IRSB_CKR(cudaEventElapsedTime(&m01, e0_, e1_));
    IRSB_CKR(cudaEventElapsedTime(&m12, e1_, e2_));
    IRSB_CKR(cudaEventElapsedTime(&m34, e3_, e4));
    cudaEventDestroy(e4);
    t_init_roots = m01 * 1e-3;
    t_ccs = m12 * 1e-3;
    t_caustics = m34 * 1e-3;
    if (verbose >= 1)
      std::cout << "ccf: stars " << n << ", roots " << num_roots << ", tree levels " << tree_levels
                << ", expansion order " << expansion_order << ", max error in 1/mu " << max_error << ", t_ccs "
                << t_ccs << " s\n";
    return true;
  }

  // include/ccf.cuh:1123-1263
  bool save(int verbose) {
    if (ccs.empty()) {
      std::cerr << "Error. save() needs a completed run().\n";
      return false;
    }
    std::string fname = outfile_prefix + "ccf_parameter_info.txt";
    std::ofstream f(fname);
    if (!f) {
      std::cerr << "Error. Failed to open file " << fname << "\n";
      return false;
    }
    f.precision(9);
    f << "kappa_tot " << kappa_tot << "\n";
    f << "shear " << shear << "\n";
    f << "mu_ave " << mu_ave << "\n";
    f << "smooth_fraction " << (1 - kappa_star / kappa_tot) << "\n";
    f << "kappa_star " << kappa_star << "\n";
    if (starfile.empty()) f << "kappa_star_actual " << kappa_star_actual << "\n";
    f << "theta_star " << theta_star << "\n";
    f << "random_seed " << random_seed << "\n";
    if (starfile.empty()) {
      f << "mass_function " << mass_function_str << "\n";
      if (mass_function_str == "salpeter" || mass_function_str == "kroupa") f << "m_solar " << m_solar << "\n";
      f << "m_lower " << m_lower_run << "\n";
      f << "m_upper " << m_upper_run << "\n";
      f << "mean_mass " << mean_mass << "\n";
      f << "mean_mass2 " << mean_mass2 << "\n";
      f << "mean_mass2_ln_mass " << mean_mass2_ln_mass << "\n";
    }
    f << "m_lower_actual " << m_lower_actual << "\n";
    f << "m_upper_actual " << m_upper_actual << "\n";
    f << "mean_mass_actual " << mean_mass_actual << "\n";
    f << "mean_mass2_actual " << mean_mass2_actual << "\n";
    f << "mean_mass2_ln_mass_actual " << mean_mass2_ln_mass_actual << "\n";
    f << "num_stars " << num_stars << "\n";
    if (rectangular) {
      f << "corner_x1 " << corner.re << "\n";
      f << "corner_x2 " << corner.im << "\n";
      if (approx) f << "taylor_smooth " << taylor_smooth << "\n";
    } else {
      f << "rad " << cabs_(corner) << "\n";
    }
    f << "num_roots " << num_roots << "\n";
    f << "num_phi " << num_phi << "\n";
    f << "num_branches " << num_branches << "\n";
    f << "max_error_1/mu " << max_error << "\n";
    f << "t_init_roots " << t_init_roots << "\n";
    f << "t_ccs " << t_ccs << "\n";
    f << "t_caustics " << t_caustics << "\n";
    f.close();
    if (!f) return false;
    if (verbose >= 1) std::cout << "Done writing parameter info to file " << fname << "\n";
    if (write_stars &&
        !write_star_file_bin<T>(outfile_prefix + "ccf_stars.bin", num_stars, rectangular, corner, theta_star,
                                stars_out.data()))
      return false;
    const int nrows = num_roots * num_branches, ncols = num_phi / num_branches + 1;
    if (write_critical_curves && !write_array(outfile_prefix + "ccf_ccs.bin", nrows, ncols, ccs.data(), sizeof(double2)))
      return false;
    if (write_caustics &&
        !write_array(outfile_prefix + "ccf_caustics.bin", nrows, ncols, caustics.data(), sizeof(double2)))
      return false;
    if (write_mu_length_scales && !write_array(outfile_prefix + "ccf_mu_length_scales.bin", nrows, ncols,
                                               mu_length_scales.data(), sizeof(double)))
      return false;
    return true;
  }

 private:
  cudaStream_t stream_ = nullptr;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr, e2_ = nullptr, e3_ = nullptr;
  DevVec<StarRec<T>> d_stars_;
  TreeDev<T> tree_;
  FmmDev fmm_;
  LeafSet leaves_;
  DevVec<double2> d_roots_, d_scratch_, d_ccs_, d_caus_, d_spos_;
  DevVec<double> d_mu_;
  DevVec<unsigned char> d_fin_;
  DevVec<unsigned long long> d_stat_;

  // Corner of a circular field of num_stars stars (include/ccf.cuh:427-432).
  cplx<T> scaled_circle(cplx<T> c, T mm) const {
    const T a = cabs_(c);
    const T sc = std::sqrt(theta_star * theta_star * num_stars * mm / kappa_star);
    return mk<T>(c.re / a * sc, c.im / a * sc);
  }
  // Corner of a rectangular field (include/ccf.cuh:421-425): the shape
  // (sqrt(re / im), sqrt(im / re)) of c, which a scaled corner keeps.
  cplx<T> scaled_rect(cplx<T> c, T mm) const {
    const cplx<T> sh = mk<T>(std::sqrt(c.re / c.im), std::sqrt(c.im / c.re));
    const T sc = std::sqrt(kPi<T> * theta_star * theta_star * num_stars * mm / (4 * kappa_star));
    return mk<T>(sh.re * sc, sh.im * sc);
  }

  CcfParams params() const {
    CcfParams P;
    P.kappa = double(kappa_tot);
    P.gamma = double(shear);
    P.kstar = double(kappa_star);
    P.theta2 = double(theta_star) * double(theta_star);
    P.inv_pi = kInvPi<double>;
    P.rect = rectangular;
    P.approx = approx;
    P.taylor_smooth = taylor_smooth;
    P.p = expansion_order;
    P.corner_re = double(corner.re);
    P.corner_im = double(corner.im);
    P.root_hl = double(root_half_length);
    P.nstars = num_stars;
    P.nroots = num_roots;
    P.nphi = num_phi;
    P.nbranches = num_branches;
    return P;
  }

  LeafPtrs leaf_ptrs() const {
    LeafPtrs lp{};
    lp.cx = leaves_.cx.p;
    lp.cy = leaves_.cy.p;
    lp.hl = leaves_.hl.p;
    lp.nnear = leaves_.nnear.p;
    lp.near64 = leaves_.near64.p;
    lp.near32 = leaves_.near32.p;
    lp.coef64 = leaves_.coef64.p;
    lp.coef32 = leaves_.coef32.p;
    lp.nleaves = leaves_.n;
    return lp;
  }

  // write_array (include/array_functions.cuh:280-306): int nrows, int ncols,
  // then the row-major values.
  static bool write_array(const std::string& fname, int nrows, int ncols, const void* data, size_t elem) {
    std::ofstream f(fname, std::ios::binary);
    if (!f) {
      std::cerr << "Error. Failed to open file " << fname << "\n";
      return false;
    }
    f.write(reinterpret_cast<const char*>(&nrows), sizeof(int));
    f.write(reinterpret_cast<const char*>(&ncols), sizeof(int));
    f.write(reinterpret_cast<const char*>(data), size_t(nrows) * ncols * elem);
    return bool(f);
  }
};

}  // namespace irsb
