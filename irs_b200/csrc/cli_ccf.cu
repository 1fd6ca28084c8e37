// Command-line critical-curve finder: ccf_gpu.
//
// Same option table and conventions as the reference's src/main_ccf.cu
// (lines 28-58, 150-520): every option takes one value; -s / --smooth_fraction
// sets kappa_star = (1 - s) kappa_tot unless kappa_star or a star file is
// given; -h prints the usage; an invalid option or value is an error (exit
// status 255). The curves are found with run() and written with save().
#include "ccf_host.cuh"

#include <functional>
#include <iostream>
#include <map>
#include <string>

using dtype = double;

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
    {"-r", "--rectangular", "1 rectangular star field, 0 circular"},
    {"-a", "--approx", "1 approximate smooth-matter deflection, 0 exact"},
    {"-ss", "--safety_scale", "star field size over the radius of convergence of alpha_smooth"},
    {"-ns", "--num_stars", "number of stars"},
    {"-sf", "--starfile", "star field file (.bin or .txt)"},
    {"-np", "--num_phi", "steps of phi in [0, 2 pi]"},
    {"-nb", "--num_branches", "branches of phi in [0, 2 pi]"},
    {"-rs", "--random_seed", "seed of the star field (0: from the clock)"},
    {"-ws", "--write_stars", "1 write the star field"},
    {"-wcc", "--write_critical_curves", "1 write the critical curves"},
    {"-wc", "--write_caustics", "1 write the caustics"},
    {"-wls", "--write_length_scales", "1 write the magnification length scales"},
    {"-o", "--outfile_prefix", "prefix of the output files"},
};

void usage(const char* name) {
  std::cout << "Usage: " << (name ? name : "ccf_gpu") << " opt1 val1 opt2 val2 ...\n\nOptions:\n";
  for (const Opt& o : kOpts) std::cout << "  " << o.shrt << "," << o.lng << "  " << o.help << "\n";
}

const Opt* find_opt(const std::string& a) {
  for (const Opt& o : kOpts)
    if (a == o.shrt || a == o.lng) return &o;
  return nullptr;
}

std::string lower(std::string s) {
  for (char& c : s) c = char(std::tolower(static_cast<unsigned char>(c)));
  return s;
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
  irsb::CCF<dtype> c;
  int verbose = 1;
  bool have_ks = false, have_sf = false, have_s = false;
  dtype smooth_fraction = 1 - c.kappa_star / c.kappa_tot;
  std::map<std::string, std::function<void(const std::string&)>> set = {
      {"--verbose", [&](const std::string& v) { verbose = std::stoi(v); }},
      {"--kappa_tot", [&](const std::string& v) { c.kappa_tot = std::stod(v); }},
      {"--shear", [&](const std::string& v) { c.shear = std::stod(v); }},
      {"--smooth_fraction",
       [&](const std::string& v) {
         smooth_fraction = std::stod(v);
         have_s = true;
         if (smooth_fraction < 0 || smooth_fraction >= 1) throw std::invalid_argument("smooth_fraction");
       }},
      {"--kappa_star", [&](const std::string& v) { c.kappa_star = std::stod(v); have_ks = true; }},
      {"--theta_star", [&](const std::string& v) { c.theta_star = std::stod(v); }},
      {"--mass_function", [&](const std::string& v) { c.mass_function_str = lower(v); }},
      {"--m_solar", [&](const std::string& v) { c.m_solar = std::stod(v); }},
      {"--m_lower", [&](const std::string& v) { c.m_lower = std::stod(v); }},
      {"--m_upper", [&](const std::string& v) { c.m_upper = std::stod(v); }},
      {"--rectangular", [&](const std::string& v) { c.rectangular = std::stoi(v); }},
      {"--approx", [&](const std::string& v) { c.approx = std::stoi(v); }},
      {"--safety_scale", [&](const std::string& v) { c.safety_scale = std::stod(v); }},
      {"--num_stars", [&](const std::string& v) { c.num_stars = std::stoi(v); }},
      {"--starfile", [&](const std::string& v) { c.starfile = v; have_sf = true; }},
      {"--num_phi", [&](const std::string& v) { c.num_phi = std::stoi(v); }},
      {"--num_branches", [&](const std::string& v) { c.num_branches = std::stoi(v); }},
      {"--random_seed", [&](const std::string& v) { c.random_seed = std::stoi(v); }},
      {"--write_stars", [&](const std::string& v) { c.write_stars = std::stoi(v); }},
      {"--write_critical_curves", [&](const std::string& v) { c.write_critical_curves = std::stoi(v); }},
      {"--write_caustics", [&](const std::string& v) { c.write_caustics = std::stoi(v); }},
      {"--write_length_scales", [&](const std::string& v) { c.write_mu_length_scales = std::stoi(v); }},
      {"--outfile_prefix", [&](const std::string& v) { c.outfile_prefix = v; }},
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
  if (!have_sf && !have_ks && have_s) c.kappa_star = (1 - smooth_fraction) * c.kappa_tot;
  if (!c.run(verbose)) return -1;
  if (!c.save(verbose)) return -1;
  return 0;
}
