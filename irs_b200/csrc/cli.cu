// Command-line map makers: ipm_gpu / ipm_gpu_double / irs_gpu / irs_gpu_double.
//
// Same option table and conventions as the reference's src/main_ipm_irs.cu
// (lines 41-72, 169-606): every option takes one value; -s / --smooth_fraction
// sets kappa_star = (1 - s) kappa_tot unless kappa_star or a star file is
// given; -h prints the usage; an invalid option or value is an error (exit
// status 255). The map is made with run() and written with save(). Extension
// options: -p / --expansion_order (0 = the reference formula) and
// --precision (0 default, 1 FP64, 2 FP32).
#include "engine.cuh"

#include <cstdlib>
#include <functional>
#include <iostream>
#include <map>
#include <string>

#ifndef IRSB_DOUBLE
#define IRSB_DOUBLE 0
#endif
#ifndef IRSB_IRS
#define IRSB_IRS 0
#endif
#if IRSB_DOUBLE
using dtype = double;
#else
using dtype = float;
#endif
using Maker = irsb::MapMaker<dtype, bool(IRSB_IRS)>;

namespace {

struct Opt {
  const char* shrt;
  const char* lng;
  const char* help;
};

const Opt kOpts[] = {
    {"-h", "--help", "show this message"},
    {"-v", "--verbose", "verbosity 0..3"},
    {"-k", "--kappa_tot", "total convergence"},
    {"-y", "--shear", "external shear"},
    {"-s", "--smooth_fraction", "fraction of the convergence in smooth matter"},
    {"-ks", "--kappa_star", "convergence in point masses"},
    {"-t", "--theta_star", "Einstein radius of a unit mass"},
    {"-mf", "--mass_function", "equal, uniform, salpeter, kroupa or optical_depth"},
    {"-ms", "--m_solar", "solar mass in arbitrary units"},
    {"-ml", "--m_lower", "lower mass cutoff (solar masses)"},
    {"-mh", "--m_upper", "upper mass cutoff (solar masses)"},
    {"-ll", "--light_loss", "average fraction of light lost to large deflections"},
    {"-r", "--rectangular", "1 rectangular star field, 0 circular"},
    {"-a", "--approx", "1 approximate smooth-matter deflection, 0 exact"},
    {"-ss", "--safety_scale", "star field size over shooting region size"},
    {"-sf", "--starfile", "star field file (.bin or .txt)"},
    {"-cy1", "--center_y1", "source region centre, y1"},
    {"-cy2", "--center_y2", "source region centre, y2"},
    {"-hly1", "--half_length_y1", "source region half length, y1"},
    {"-hly2", "--half_length_y2", "source region half length, y2"},
    {"-npy1", "--num_pixels_y1", "pixels along y1"},
    {"-npy2", "--num_pixels_y2", "pixels along y2"},
    {"-nry", "--num_rays_y", "rays (IRS) or cells (IPM) per pixel without lensing"},
    {"-rs", "--random_seed", "seed of the star field (0: from the clock)"},
    {"-ws", "--write_stars", "1 write the star field"},
    {"-wm", "--write_maps", "1 write the maps"},
    {"-wp", "--write_parities", "1 keep minima / saddle maps"},
    {"-wh", "--write_histograms", "1 write histograms"},
    {"-o", "--outfile_prefix", "prefix of the output files"},
    {"-p", "--expansion_order", "(extension) expansion order, 0 = reference formula"},
    {"-pr", "--precision", "(extension) 0 default, 1 FP64, 2 FP32"},
};

void usage(const char* name) {
  std::cout << "Usage: " << (name ? name : "map_maker") << " opt1 val1 opt2 val2 ...\n\nOptions:\n";
  for (const Opt& o : kOpts) std::cout << "  " << o.shrt << "," << o.lng << "  " << o.help << "\n";
}

const Opt* find_opt(const std::string& a) {
  for (const Opt& o : kOpts)
    if (a == o.shrt || a == o.lng) return &o;
  return nullptr;
}

}  // namespace

int main(int argc, char* argv[]) {
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-h" || a == "--help") {
      usage(argv[0]);
      return -1;
    }
  }
  if ((argc - 1) % 2 != 0) {
    std::cerr << "Error. Invalid input syntax.\n";
    usage(argv[0]);
    return -1;
  }
  Maker m;
  auto& p = m.prm;
  int verbose = 1;
  bool have_ks = false, have_sf = false, have_s = false;
  dtype smooth_fraction = dtype(1 - p.kappa_star / p.kappa_tot);
  std::map<std::string, std::function<void(const std::string&)>> set = {
      {"--verbose", [&](const std::string& v) { verbose = std::stoi(v); }},
      {"--kappa_tot", [&](const std::string& v) { p.kappa_tot = dtype(std::stod(v)); }},
      {"--shear", [&](const std::string& v) { p.shear = dtype(std::stod(v)); }},
      {"--smooth_fraction", [&](const std::string& v) { smooth_fraction = dtype(std::stod(v)); have_s = true; }},
      {"--kappa_star", [&](const std::string& v) { p.kappa_star = dtype(std::stod(v)); have_ks = true; }},
      {"--theta_star", [&](const std::string& v) { p.theta_star = dtype(std::stod(v)); }},
      {"--mass_function", [&](const std::string& v) { p.mass_function = v; }},
      {"--m_solar", [&](const std::string& v) { p.m_solar = dtype(std::stod(v)); }},
      {"--m_lower", [&](const std::string& v) { p.m_lower = dtype(std::stod(v)); }},
      {"--m_upper", [&](const std::string& v) { p.m_upper = dtype(std::stod(v)); }},
      {"--light_loss", [&](const std::string& v) { p.light_loss = dtype(std::stod(v)); }},
      {"--rectangular", [&](const std::string& v) { p.rectangular = std::stoi(v); }},
      {"--approx", [&](const std::string& v) { p.approx = std::stoi(v); }},
      {"--safety_scale", [&](const std::string& v) { p.safety_scale = dtype(std::stod(v)); }},
      {"--starfile", [&](const std::string& v) { p.starfile = v; have_sf = true; }},
      {"--center_y1", [&](const std::string& v) { p.center_y.re = dtype(std::stod(v)); }},
      {"--center_y2", [&](const std::string& v) { p.center_y.im = dtype(std::stod(v)); }},
      {"--half_length_y1", [&](const std::string& v) { p.half_length_y.re = dtype(std::stod(v)); }},
      {"--half_length_y2", [&](const std::string& v) { p.half_length_y.im = dtype(std::stod(v)); }},
      {"--num_pixels_y1", [&](const std::string& v) { p.num_pixels_y.re = std::stoi(v); }},
      {"--num_pixels_y2", [&](const std::string& v) { p.num_pixels_y.im = std::stoi(v); }},
      {"--num_rays_y", [&](const std::string& v) { p.num_rays_y = std::stoi(v); }},
      {"--random_seed", [&](const std::string& v) { p.random_seed = std::stoi(v); }},
      {"--write_stars", [&](const std::string& v) { p.write_stars = std::stoi(v); }},
      {"--write_maps", [&](const std::string& v) { p.write_maps = std::stoi(v); }},
      {"--write_parities", [&](const std::string& v) { p.write_parities = std::stoi(v); }},
      {"--write_histograms", [&](const std::string& v) { p.write_histograms = std::stoi(v); }},
      {"--outfile_prefix", [&](const std::string& v) { p.outfile_prefix = v; }},
      {"--expansion_order", [&](const std::string& v) { p.expansion_order_override = std::stoi(v); }},
      {"--precision", [&](const std::string& v) { m.precision = std::stoi(v); }},
  };
  for (int i = 1; i < argc; i += 2) {
    const Opt* o = find_opt(argv[i]);
    if (!o) {
      std::cerr << "Error. Invalid input syntax. Unknown option " << argv[i] << "\n";
      usage(argv[0]);
      return -1;
    }
    try {
      set.at(o->lng)(argv[i + 1]);
    } catch (...) {
      std::cerr << "Error. Invalid " << (o->lng + 2) << " input.\n";
      return -1;
    }
  }
  if (!have_sf && !have_ks && have_s) p.kappa_star = dtype((1 - smooth_fraction) * p.kappa_tot);
  if (!m.run(verbose)) return -1;
  if (!m.save(verbose)) return -1;
  return 0;
}
