// Host-side parameter handling: input validation, derived quantities and the
// star-field moments, restated from the reference pipeline driver
//   check_input_params       include/ipm.cuh:235-368
//   calculate_derived_params include/ipm.cuh:370-565
//   calculate_star_params    include/star.cuh:124-161
//   corner recomputation     include/ipm.cuh:717-731
// and the star-file formats (.bin: include/star.cuh:175-320 and 498-534,
// .txt: include/star.cuh:334-434).
//
// Every expression keeps the reference's precision semantics for the template
// type T (float for lib_ipm.so, double for lib_ipm_double.so), including the
// places where the reference promotes to double, so that num_stars, corner,
// half_length_x and num_ray_threads come out identical.
#pragma once
#include "common.cuh"
#include "massfn.cuh"

#include <algorithm>
#include <cmath>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

namespace irsb {

template <typename T>
constexpr T kPi = T(3.141592653589793238462643383279502884L);
template <typename T>
constexpr T kInvPi = T(0.318309886183790671537767526745028724L);

// Star as stored by the reference (position re, im, then mass): 3 x T.
template <typename T>
struct StarRec {
  T x, y, m;
};

template <typename T>
struct Params {
  // ---- inputs (defaults of IPM<T>, include/ipm.cuh:42-64) ----
  T kappa_tot = T(0.3);
  T shear = T(0.3);
  T kappa_star = T(0.27);
  T theta_star = T(1);
  std::string mass_function = "equal";
  T m_solar = T(1);
  T m_lower = T(0.01);
  T m_upper = T(50);
  T light_loss = T(0.001);
  int rectangular = 0;
  int approx = 1;
  T safety_scale = T(1.37);
  std::string starfile = "";
  cplx<T> center_y = mk<T>(0, 0);
  cplx<T> half_length_y = mk<T>(5, 5);
  cplx<int> num_pixels_y = mk<int>(1000, 1000);
  int num_rays_y = 1;
  int random_seed = 0;
  int write_stars = 1;
  int write_maps = 1;
  int write_parities = 0;
  int write_histograms = 1;
  std::string outfile_prefix = "./";
  // extension: 0 -> expansion order from the reference formula
  int expansion_order_override = 0;

  // ---- derived ----
  int mf_kind = kMFEqual;
  T mean_mass = 0, mean_mass2 = 0, mean_mass2_ln_mass = 0;
  int num_stars = 0;
  T kappa_star_actual = 0, m_lower_actual = 0, m_upper_actual = 0;
  T mean_mass_actual = 0, mean_mass2_actual = 0, mean_mass2_ln_mass_actual = 0;
  T mu_ave = 0;
  T num_rays_x = 0;
  cplx<T> ray_half_sep = mk<T>(0, 0);
  cplx<T> center_x = mk<T>(0, 0);
  cplx<T> half_length_x = mk<T>(0, 0);
  cplx<int> num_ray_threads = mk<int>(0, 0);
  cplx<T> corner = mk<T>(0, 0);
  int taylor_smooth = 1;
  T alpha_error = 0;
  int expansion_order = 0;
  T root_half_length = 0;
  int tree_levels = 0;
};

static const int kMaxTaylorSmooth = 101;  // include/ipm.cuh:81

template <typename T>
bool check_input_params(const Params<T>& p) {
  const T tmin = std::numeric_limits<T>::min();
  auto fail = [](const char* msg) {
    std::cerr << "Error. " << msg << "\n";
    return false;
  };
  if (p.kappa_tot < tmin) return fail("kappa_tot must be >= the smallest positive normal number");
  if (p.kappa_star < tmin) return fail("kappa_star must be >= the smallest positive normal number");
  if (p.starfile.empty() && p.kappa_star > p.kappa_tot) return fail("kappa_star must be <= kappa_tot");
  if (p.starfile.empty() && p.theta_star < tmin) return fail("theta_star must be > 0");
  if (p.starfile.empty() && mass_function_kind(p.mass_function.c_str()) == kMFInvalid)
    return fail("mass_function must be equal, uniform, Salpeter, Kroupa, or optical_depth.");
  if (p.starfile.empty() && p.m_solar < tmin) return fail("m_solar must be > 0");
  if (p.starfile.empty() && p.m_lower < tmin) return fail("m_lower must be > 0");
  if (p.starfile.empty() && p.m_upper < p.m_lower) return fail("m_upper must be >= m_lower.");
  if (p.light_loss < tmin) return fail("light_loss must be > 0");
  if (p.light_loss > 0.01) return fail("light_loss must be <= 0.01");
  if (p.starfile.empty() && p.rectangular != 0 && p.rectangular != 1)
    return fail("rectangular must be 1 (rectangular) or 0 (circular).");
  if (p.approx != 0 && p.approx != 1) return fail("approx must be 1 (approximate) or 0 (exact).");
  if (p.safety_scale < 1.1) return fail("safety_scale must be >= 1.1");
  if (p.half_length_y.re < tmin || p.half_length_y.im < tmin)
    return fail("half_length_y1 and half_length_y2 must both be > 0");
  if (p.num_pixels_y.re < 1 || p.num_pixels_y.im < 1)
    return fail("num_pixels_y1 and num_pixels_y2 must both be integers > 0");
  if (p.num_rays_y < 1) return fail("num_rays_y must be an integer > 0");
  const int flags[4] = {p.write_stars, p.write_maps, p.write_parities, p.write_histograms};
  for (int v : flags)
    if (v != 0 && v != 1) return fail("write_* flags must be 1 (true) or 0 (false).");
  if (p.expansion_order_override < 0 || p.expansion_order_override > kMaxOrder)
    return fail("expansion_order override must be in [0, 31]");
  return true;
}

// Moments and kappa_star of a concrete star field (include/star.cuh:124-161):
// sums in double, in star order.
template <typename T>
void star_field_moments(int n, int rectangular, cplx<T> corner, T theta, const StarRec<T>* s,
                        T& kappastar, T& m_lower, T& m_upper, T& mean_mass, T& mean_mass2,
                        T& mean_mass2_ln_mass) {
  m_lower = std::numeric_limits<T>::max();
  m_upper = std::numeric_limits<T>::min();
  double m_tot = 0, m2_tot = 0, m2_ln_tot = 0;
  for (int i = 0; i < n; i++) {
    T m = s[i].m;
    m_tot += m;
    m2_tot += m * m;
    m2_ln_tot += m * m * std::log(m);
    m_lower = std::min(m_lower, m);
    m_upper = std::max(m_upper, m);
  }
  mean_mass = T(m_tot / n);
  mean_mass2 = T(m2_tot / n);
  mean_mass2_ln_mass = T(m2_ln_tot / n);
  if (rectangular)
    kappastar = T(m_tot * kPi<T> * theta * theta / (4 * corner.re * corner.im));
  else
    kappastar = T(m_tot * theta * theta / (cabs_(corner) * cabs_(corner)));
}

// ---------------------------------------------------------------- star files
template <typename T>
bool read_star_file_bin(const std::string& path, int& n, int& rect, cplx<T>& corner, T& theta,
                        std::vector<StarRec<T>>& stars) {
  std::error_code ec;
  auto fsize = std::filesystem::file_size(path, ec);
  if (ec) {
    std::cerr << "Error determining size of star input file " << path << "\n";
    return false;
  }
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    std::cerr << "Error. Failed to open file " << path << "\n";
    return false;
  }
  in.read(reinterpret_cast<char*>(&n), sizeof(int));
  if (n < 1) {
    std::cerr << "Error. Invalid num_stars input. num_stars must be an integer > 0\n";
    return false;
  }
  in.read(reinterpret_cast<char*>(&rect), sizeof(int));
  if (rect != 0 && rect != 1) {
    std::cerr << "Error. Invalid rectangular input.\n";
    return false;
  }
  stars.resize(n);
  auto body = [&](auto tag) -> bool {
    using U = decltype(tag);
    U c[2], th;
    in.read(reinterpret_cast<char*>(c), sizeof(c));
    in.read(reinterpret_cast<char*>(&th), sizeof(U));
    std::vector<U> raw(size_t(n) * 3);
    in.read(reinterpret_cast<char*>(raw.data()), raw.size() * sizeof(U));
    corner = mk<T>(T(c[0]), T(c[1]));
    theta = T(th);
    for (int i = 0; i < n; i++) stars[i] = {T(raw[3 * i]), T(raw[3 * i + 1]), T(raw[3 * i + 2])};
    return bool(in);
  };
  const size_t hdr = 2 * sizeof(int);
  bool ok;
  if (fsize == hdr + 3 * sizeof(T) + size_t(n) * 3 * sizeof(T))
    ok = body(T(0));
  else if (fsize == hdr + 3 * sizeof(float) + size_t(n) * 3 * sizeof(float))
    ok = body(float(0));
  else if (fsize == hdr + 3 * sizeof(double) + size_t(n) * 3 * sizeof(double))
    ok = body(double(0));
  else {
    std::cerr << "Error. Star input file " << path
              << " does not contain validly formatted single or double precision stars.\n";
    return false;
  }
  if (!ok) {
    std::cerr << "Error. Failed reading star file " << path << "\n";
    return false;
  }
  if (corner.re < 0 || corner.im < 0) {
    std::cerr << "Error. Real and imaginary parts of the corner of the star field must both be >= 0\n";
    return false;
  }
  if (theta < std::numeric_limits<T>::min()) {
    std::cerr << "Error. theta_star must be > 0\n";
    return false;
  }
  return true;
}

// Whitespace-delimited "x1 x2 m" lines in units where theta_star = 1; the
// field shape is chosen by comparing the moment of inertia with that of a disk
// and of a rectangle (include/star.cuh:398-431).
template <typename T>
bool read_star_file_txt(const std::string& path, int& n, int& rect, cplx<T>& corner, T& theta,
                        std::vector<StarRec<T>>& stars) {
  std::ifstream in(path);
  if (!in) {
    std::cerr << "Error. Failed to open file " << path << "\n";
    return false;
  }
  stars.clear();
  T x1, x2, m;
  T max_x1 = 0, max_x2 = 0, max_rad = 0;
  double total_mass = 0, I_stars = 0;
  while (in >> x1 >> x2 >> m) {
    stars.push_back({x1, x2, m});
    total_mass += m;
    I_stars += m * (x1 * x1 + x2 * x2);
    max_x1 = std::max(max_x1, std::abs(x1));
    max_x2 = std::max(max_x2, std::abs(x2));
    max_rad = std::max(max_rad, std::hypot(x1, x2));
  }
  n = int(stars.size());
  if (n < 1) {
    std::cerr << "Error. Invalid num_stars input. num_stars must be an integer > 0\n";
    return false;
  }
  double I_circ = total_mass * max_rad * max_rad / 2;
  double I_rect = total_mass * (max_x1 * max_x1 + max_x2 * max_x2) / 3;
  if (I_stars / I_circ > I_stars / I_rect) {
    rect = 0;
    corner = mk<T>(max_rad, T(0));
  } else {
    rect = 1;
    corner = mk<T>(max_x1, max_x2);
  }
  theta = T(1);
  return true;
}

template <typename T>
bool write_star_file_bin(const std::string& path, int n, int rect, cplx<T> corner, T theta,
                         const StarRec<T>* stars) {
  if (std::filesystem::path(path).extension() != ".bin") {
    std::cerr << "Error. Star file " << path << " is not a .bin file.\n";
    return false;
  }
  std::ofstream out(path, std::ios::binary);
  if (!out) {
    std::cerr << "Error. Failed to open file " << path << "\n";
    return false;
  }
  cplx<T> c = rect ? corner : mk<T>(cabs_(corner), T(0));
  out.write(reinterpret_cast<const char*>(&n), sizeof(int));
  out.write(reinterpret_cast<const char*>(&rect), sizeof(int));
  out.write(reinterpret_cast<const char*>(&c), sizeof(c));
  out.write(reinterpret_cast<const char*>(&theta), sizeof(T));
  out.write(reinterpret_cast<const char*>(stars), size_t(n) * sizeof(StarRec<T>));
  return bool(out);
}

// calculate_derived_params (include/ipm.cuh:370-565). `stars_io` receives the
// star field when a star file is given.
// With `preloaded`, stars_io already holds the field and num_stars,
// rectangular, corner and theta_star are set (a star field passed in memory);
// it then follows the star-file branch without reading a file.
template <typename T>
bool derive_params(Params<T>& p, std::vector<StarRec<T>>& stars_io, bool preloaded = false) {
  const bool from_stars = preloaded || !p.starfile.empty();
  if (!from_stars) {
    p.mf_kind = mass_function_kind(p.mass_function.c_str());
    if (p.mf_kind == kMFEqual) {
      p.m_lower = T(1);
      p.m_upper = T(1);
    } else {
      p.m_lower = p.m_lower * p.m_solar;
      p.m_upper = p.m_upper * p.m_solar;
    }
    p.mean_mass = mf_moment<T>(p.mf_kind, p.m_lower, p.m_upper, p.m_solar, 0);
    p.mean_mass2 = mf_moment<T>(p.mf_kind, p.m_lower, p.m_upper, p.m_solar, 1);
    p.mean_mass2_ln_mass = mf_moment<T>(p.mf_kind, p.m_lower, p.m_upper, p.m_solar, 2);
  } else {
    std::string ext = std::filesystem::path(p.starfile).extension().string();
    bool ok;
    if (preloaded)
      ok = true;
    else if (ext == ".bin")
      ok = read_star_file_bin<T>(p.starfile, p.num_stars, p.rectangular, p.corner, p.theta_star, stars_io);
    else if (ext == ".txt")
      ok = read_star_file_txt<T>(p.starfile, p.num_stars, p.rectangular, p.corner, p.theta_star, stars_io);
    else {
      std::cerr << "Error. Star input file " << p.starfile << " is not a .bin or .txt file.\n";
      ok = false;
    }
    if (!ok) {
      std::cerr << "Error. Unable to read star field parameters from file " << p.starfile << "\n";
      return false;
    }
    star_field_moments<T>(p.num_stars, p.rectangular, p.corner, p.theta_star, stars_io.data(), p.kappa_star,
                          p.m_lower, p.m_upper, p.mean_mass, p.mean_mass2, p.mean_mass2_ln_mass);
    if (p.kappa_star > p.kappa_tot) std::cerr << "Warning. kappa_star > kappa_tot\n";
  }

  p.mu_ave = T(1) / ((1 - p.kappa_tot) * (1 - p.kappa_tot) - p.shear * p.shear);
  p.num_rays_x = T(1.0 * p.num_rays_y * p.num_pixels_y.re * p.num_pixels_y.im /
                   (2 * p.half_length_y.re * 2 * p.half_length_y.im));

  cplx<T> rhs = mk<T>(std::sqrt(p.half_length_y.re / p.half_length_y.im * p.num_pixels_y.im / p.num_pixels_y.re),
                      std::sqrt(p.half_length_y.im / p.half_length_y.re * p.num_pixels_y.re / p.num_pixels_y.im));
  T div = 2 * std::sqrt(p.num_rays_x);
  rhs.re /= div;
  rhs.im /= div;
  p.ray_half_sep = rhs;

  T t = p.theta_star * std::sqrt(p.kappa_star * p.mean_mass2 / (p.mean_mass * p.light_loss));
  cplx<T> hlx = mk<T>(p.half_length_y.re + t, p.half_length_y.im + t);
  hlx = mk<T>(hlx.re / std::abs(1 - p.kappa_tot + p.shear), hlx.im / std::abs(1 - p.kappa_tot - p.shear));
  cplx<int> nrt = mk<int>(static_cast<int>(hlx.re / (2 * rhs.re)) + 1, static_cast<int>(hlx.im / (2 * rhs.im)) + 1);
  hlx = mk<T>(2 * rhs.re * nrt.re, 2 * rhs.im * nrt.im);
  p.half_length_x = hlx;
  p.num_ray_threads = mk<int>(2 * nrt.re, 2 * nrt.im);
  if (!(hlx.re > 0 && hlx.im > 0) || !std::isfinite(double(hlx.re)) || !std::isfinite(double(hlx.im)) ||
      nrt.re <= 0 || nrt.im <= 0) {
    std::cerr << "Error. The shooting region is not finite (|1 - kappa_tot -/+ shear| must be > 0).\n";
    return false;
  }

  p.center_x = mk<T>(p.center_y.re / (1 - p.kappa_tot + p.shear), p.center_y.im / (1 - p.kappa_tot - p.shear));

  if (!from_stars) {
    cplx<T> c = mk<T>(std::abs(p.center_x.re) + hlx.re, std::abs(p.center_x.im) + hlx.im);
    if (p.rectangular) {
      T v = std::ceil(p.safety_scale * 2 * c.re * p.safety_scale * 2 * c.im * p.kappa_star /
                      (kPi<T> * p.theta_star * p.theta_star * p.mean_mass));
      p.num_stars = static_cast<int>(v);
      c = mk<T>(std::sqrt(c.re / c.im), std::sqrt(c.im / c.re));
      T s = std::sqrt(kPi<T> * p.theta_star * p.theta_star * p.num_stars * p.mean_mass / (4 * p.kappa_star));
      c = mk<T>(c.re * s, c.im * s);
    } else {
      T ca = cabs_(c);
      T v = std::ceil(p.safety_scale * ca * p.safety_scale * ca * p.kappa_star /
                      (p.theta_star * p.theta_star * p.mean_mass));
      p.num_stars = static_cast<int>(v);
      c = mk<T>(c.re / ca, c.im / ca);
      T s = std::sqrt(p.theta_star * p.theta_star * p.num_stars * p.mean_mass / p.kappa_star);
      c = mk<T>(c.re * s, c.im * s);
    }
    p.corner = c;
  } else {
    cplx<T> tc = mk<T>(std::abs(p.center_x.re) + hlx.re, std::abs(p.center_x.im) + hlx.im);
    if (!p.rectangular) {
      T tca = cabs_(tc);
      T ca = cabs_(p.corner);
      p.corner = mk<T>(tc.re / tca * ca, tc.im / tca * ca);
    }
    if ((p.rectangular && (p.corner.re < p.safety_scale * tc.re || p.corner.im < p.safety_scale * tc.im)) ||
        (!p.rectangular && (cabs_(p.corner) < p.safety_scale * cabs_(tc)))) {
      std::cerr << "Error. The provided star field is not large enough to cover the desired source plane region.\n";
      return false;
    }
  }
  if (p.num_stars < 1) {
    std::cerr << "Error. num_stars must be >= 1\n";
    return false;
  }

  p.alpha_error = std::min(p.half_length_y.re / (10 * p.num_pixels_y.re), p.half_length_y.im / (10 * p.num_pixels_y.im));

  int ts = 1;
  T cabs = cabs_(p.corner);
  while ((p.kappa_star * kInvPi<T> * 4 / (ts + 1) * cabs * (p.safety_scale + 1) / (p.safety_scale - 1) *
              std::pow(1 / p.safety_scale, ts + 1) >
          p.alpha_error) &&
         ts <= kMaxTaylorSmooth)
    ts += 2;
  T carg_ = carg(p.corner);
  while ((std::fmod(carg_ * (ts - 1), kPi<T>) < 0.1 * kPi<T> || std::fmod(carg_ * (ts - 1), kPi<T>) > 0.9 * kPi<T>) &&
         ts <= kMaxTaylorSmooth)
    ts += 2;
  p.taylor_smooth = ts;
  if (p.rectangular && ts > kMaxTaylorSmooth) {
    std::cerr << "Error. taylor_smooth must be <= " << kMaxTaylorSmooth << "\n";
    return false;
  }
  return true;
}

// Corner recomputed from the realised mean mass (include/ipm.cuh:717-731).
template <typename T>
void recompute_corner(Params<T>& p) {
  cplx<T> c = p.corner;
  if (p.rectangular) {
    c = mk<T>(std::sqrt(c.re / c.im), std::sqrt(c.im / c.re));
    T s = std::sqrt(kPi<T> * p.theta_star * p.theta_star * p.num_stars * p.mean_mass_actual / (4 * p.kappa_star));
    c = mk<T>(c.re * s, c.im * s);
  } else {
    T ca = cabs_(c);
    c = mk<T>(c.re / ca, c.im / ca);
    T s = std::sqrt(p.theta_star * p.theta_star * p.num_stars * p.mean_mass_actual / p.kappa_star);
    c = mk<T>(c.re * s, c.im * s);
  }
  p.corner = c;
}

template <typename T>
T root_half_length_of(const Params<T>& p) {
  T r = p.rectangular ? (p.corner.re > p.corner.im ? p.corner.re : p.corner.im) : cabs_(p.corner);
  return T(r * 1.1);
}

// Expansion order from the reference formula (include/ipm.cuh:848-849).
template <typename T>
int expansion_order_of(const Params<T>& p) {
  return static_cast<int>(std::ceil(2 * std::log2(p.theta_star) + p.tree_levels - std::log2(p.root_half_length) -
                                    std::log2(p.alpha_error)));
}

}  // namespace irsb
