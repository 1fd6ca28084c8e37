// Command-line caustic-crossing maps: ncc_gpu.
//
// Same option table and conventions as the reference's src/main_ncc.cu
// (lines 28-44, 120-296): every option takes one value; -h prints the usage;
// an invalid option or value is an error (exit status 255). The map is made
// from <infile_prefix>ccf_caustics.bin with run() and written with save().
#include "ncc_host.cuh"

#include <functional>
#include <iostream>
#include <map>
#include <string>

namespace {

struct Opt {
  const char* shrt;
  const char* lng;
  const char* help;
};

const Opt kOpts[] = {
    {"-h", "--help", "show this message"},
    {"-v", "--verbose", "verbosity 0..3"},
    {"-ip", "--infile_prefix", "prefix of the input ccf_caustics.bin"},
    {"-cy1", "--center_y1", "source region centre, y1"},
    {"-cy2", "--center_y2", "source region centre, y2"},
    {"-hly1", "--half_length_y1", "source region half length, y1"},
    {"-hly2", "--half_length_y2", "source region half length, y2"},
    {"-npy1", "--num_pixels_y1", "pixels along y1"},
    {"-npy2", "--num_pixels_y2", "pixels along y2"},
    {"-os", "--over_sample", "sampling 2^over_sample times finer before the block maximum"},
    {"-wm", "--write_maps", "1 write the map"},
    {"-wh", "--write_histograms", "1 write the histogram"},
    {"-o", "--outfile_prefix", "prefix of the output files"},
};

void usage(const char* name) {
  std::cout << "Usage: " << (name ? name : "ncc_gpu") << " opt1 val1 opt2 val2 ...\n\nOptions:\n";
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
  irsb::NCC<double> n;
  int verbose = 1;
  std::map<std::string, std::function<void(const std::string&)>> set = {
      {"--verbose", [&](const std::string& v) { verbose = std::stoi(v); }},
      {"--infile_prefix", [&](const std::string& v) { n.infile_prefix = v; }},
      {"--center_y1", [&](const std::string& v) { n.center_y.re = std::stod(v); }},
      {"--center_y2", [&](const std::string& v) { n.center_y.im = std::stod(v); }},
      {"--half_length_y1", [&](const std::string& v) { n.half_length_y.re = std::stod(v); }},
      {"--half_length_y2", [&](const std::string& v) { n.half_length_y.im = std::stod(v); }},
      {"--num_pixels_y1", [&](const std::string& v) { n.num_pixels_y.re = std::stoi(v); }},
      {"--num_pixels_y2", [&](const std::string& v) { n.num_pixels_y.im = std::stoi(v); }},
      {"--over_sample", [&](const std::string& v) { n.over_sample = std::stoi(v); }},
      {"--write_maps", [&](const std::string& v) { n.write_maps = std::stoi(v); }},
      {"--write_histograms", [&](const std::string& v) { n.write_histograms = std::stoi(v); }},
      {"--outfile_prefix", [&](const std::string& v) { n.outfile_prefix = v; }},
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
  if (!n.run(verbose)) return -1;
  if (!n.save(verbose)) return -1;
  return 0;
}
