// NCC<T>: the number-of-caustic-crossings map, the host side of
// include/ncc.cuh (class NCC). Same inputs, defaults, checks, input file
// (<infile_prefix>ccf_caustics.bin, float or double), outputs and files;
// the map is built by the kernels of ncc.cuh.
#pragma once
#include "devutil.cuh"
#include "ncc.cuh"
#include "post.cuh"

#include <algorithm>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <vector>

namespace irsb {

template <typename T>
class NCC {
 public:
  // ---- inputs (defaults of include/ncc.cuh:27-35) ----
  std::string infile_prefix = "./";
  cplx<T> center_y = mk<T>(0, 0);
  cplx<T> half_length_y = mk<T>(5, 5);
  cplx<int> num_pixels_y = mk<int>(1000, 1000);
  int over_sample = 2;
  int write_maps = 1;
  int write_histograms = 1;
  std::string outfile_prefix = "./";
  // extension: caustics from host memory (rows x cols complex values) instead
  // of the input file
  std::vector<double2> host_caustics;
  int host_rows = 0, host_cols = 0;

  // ---- results ----
  double t_ncc = 0, t_reduce = 0;
  int num_rows = 0, num_cols = 0, min_num = 0, max_num = 0, errors = 0;
  std::vector<int> map, histogram;

  ~NCC() {
    for (cudaEvent_t* e : {&e0_, &e1_, &e2_})
      if (*e) cudaEventDestroy(*e);
    if (stream_) cudaStreamDestroy(stream_);
  }

  int* num_crossings() { return map.empty() ? nullptr : map.data(); }

  // include/ncc.cuh:131-171
  bool check_input_params() const {
    auto fail = [](const char* m) {
      std::cerr << "Error. " << m << "\n";
      return false;
    };
    if (half_length_y.re < std::numeric_limits<T>::min() || half_length_y.im < std::numeric_limits<T>::min())
      return fail("half_length_y1 and half_length_y2 must both be >= the smallest positive normal number");
    if (num_pixels_y.re < 1 || num_pixels_y.im < 1)
      return fail("num_pixels_y1 and num_pixels_y2 must both be integers > 0");
    if (over_sample < 0) return fail("over_sample must be an integer >= 0");
    if (over_sample > 10) return fail("over_sample must be <= 10");
    if (write_maps != 0 && write_maps != 1) return fail("write_maps must be 1 (true) or 0 (false).");
    if (write_histograms != 0 && write_histograms != 1) return fail("write_histograms must be 1 (true) or 0 (false).");
    return true;
  }

  bool run(int verbose) {
    if (!check_input_params()) return false;
    if (!stream_) {
      IRSB_CKR(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
      for (cudaEvent_t* e : {&e0_, &e1_, &e2_}) IRSB_CKR(cudaEventCreate(e));
    }
    cudaStream_t s = stream_;
    std::vector<double2> caus;
    if (host_rows > 0) {
      caus = host_caustics;
      num_rows = host_rows;
      num_cols = host_cols;
    } else if (!read_caustics(infile_prefix + "ccf_caustics.bin", caus)) {
      return false;
    }
    if (num_rows < 1 || num_cols < 2) {
      std::cerr << "Error. Need at least 1 row and 2 columns of caustic positions.\n";
      return false;
    }
    const int B = 1 << over_sample;
    const long long fx = (long long)num_pixels_y.re * B, fy = (long long)num_pixels_y.im * B;
    if (fx > (1 << 30) || fy > (1 << 30) || fx * fy > (1LL << 34)) {
      std::cerr << "Error. The oversampled map is too large.\n";
      return false;
    }
    const long long nfine = fx * fy, ndiff = fy * (fx + 1), nout = (long long)num_pixels_y.re * num_pixels_y.im;
    if (!d_caus_.alloc_exact(caus.size()) || !d_diff_.alloc_exact(ndiff) || !d_fine_.alloc_exact(nfine) ||
        !d_out_.alloc_exact(nout) || !d_err_.alloc_exact(1))
      return false;
    IRSB_CKR(cudaMemcpyAsync(d_caus_.p, caus.data(), caus.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemsetAsync(d_diff_.p, 0, ndiff * sizeof(int), s));
    IRSB_CKR(cudaMemsetAsync(d_err_.p, 0, sizeof(int), s));
    const NccGeom g{double(center_y.re), double(center_y.im), double(half_length_y.re), double(half_length_y.im),
                    int(fx), int(fy)};
    const long long nseg = (long long)num_rows * (num_cols - 1);
    IRSB_CKR(cudaEventRecord(e0_, s));
    ncc_segments<<<int(std::max<long long>(1, std::min<long long>(ceil_div(nseg, 256LL), 148LL * 16))), 256, 0, s>>>(
        d_caus_.p, num_rows, num_cols, g, d_diff_.p, d_err_.p);
    IRSB_LAUNCH_CK("ncc_segments");
    ncc_rows<<<int(std::max<long long>(1, std::min<long long>(ceil_div(fy * 32, 256LL), 148LL * 16))), 256, 0, s>>>(
        d_diff_.p, int(fx), int(fy), d_fine_.p);
    IRSB_LAUNCH_CK("ncc_rows");
    IRSB_CKR(cudaEventRecord(e1_, s));
    ncc_pool<<<int(std::max<long long>(1, std::min<long long>(ceil_div(nout, 256LL), 148LL * 16))), 256, 0, s>>>(
        d_fine_.p, num_pixels_y.re, num_pixels_y.im, B, d_out_.p);
    IRSB_LAUNCH_CK("ncc_pool");
    IRSB_CKR(cudaEventRecord(e2_, s));
    map.resize(nout);
    IRSB_CKR(cudaMemcpyAsync(map.data(), d_out_.p, nout * sizeof(int), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaMemcpyAsync(&errors, d_err_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    float m01 = 0, m12 = 0;
    IRSB_CKR(cudaEventElapsedTime(&m01, e0_, e1_));
    IRSB_CKR(cudaEventElapsedTime(&m12, e1_, e2_));
    t_ncc = m01 * 1e-3;
    t_reduce = m12 * 1e-3;
    if (errors) std::cerr << "Error. Caustic crossing takes place outside the desired region.\n";
    min_num = *std::min_element(map.begin(), map.end());
    max_num = *std::max_element(map.begin(), map.end());
    if (min_num < 0) {
      std::cerr << "Error. Number of caustic crossings should be >= 0\n";
      return false;
    }
    histogram.clear();
    if (write_histograms) {  // include/ncc.cuh:330-355
      histogram.assign(max_num - min_num + 1, 0);
      for (int v : map) histogram[v - min_num]++;
    }
    if (verbose >= 1)
      std::cout << "ncc: " << num_rows << " x " << num_cols << " caustic points, map " << num_pixels_y.re << " x "
                << num_pixels_y.im << " (x" << B << " oversampled), crossings " << min_num << " .. " << max_num
                << ", t_ncc " << t_ncc << " s\n";
    return true;
  }

  // include/ncc.cuh:357-440
  bool save(int verbose) {
    if (map.empty()) {
      std::cerr << "Error. save() needs a completed run().\n";
      return false;
    }
    std::string fname = outfile_prefix + "ncc_parameter_info.txt";
    std::ofstream f(fname);
    if (!f) {
      std::cerr << "Error. Failed to open file " << fname << "\n";
      return false;
    }
    f.precision(9);
    f << "center_y1 " << center_y.re << "\n";
    f << "center_y2 " << center_y.im << "\n";
    f << "half_length_y1 " << half_length_y.re << "\n";
    f << "half_length_y2 " << half_length_y.im << "\n";
    f << "num_pixels_y1 " << num_pixels_y.re << "\n";
    f << "num_pixels_y2 " << num_pixels_y.im << "\n";
    f << "over_sample " << over_sample << "\n";
    f << "t_ncc " << t_ncc << "\n";
    f << "t_reduce " << t_reduce << "\n";
    f.close();
    if (!f) return false;
    if (write_histograms) {  // write_histogram (array_functions.cuh:318-349): "value count" for nonzero counts
      std::ofstream h(outfile_prefix + "ncc_ncc_numpixels.txt");
      if (!h) return false;
      for (size_t k = 0; k < histogram.size(); k++)
        if (histogram[k] != 0) h << (int(k) + min_num) << " " << histogram[k] << "\n";
    }
    if (write_maps) {  // write_array: int nrows, int ncols, row-major int32
      std::ofstream m(outfile_prefix + "ncc_ncc.bin", std::ios::binary);
      if (!m) return false;
      const int nr = num_pixels_y.im, nc = num_pixels_y.re;
      m.write(reinterpret_cast<const char*>(&nr), sizeof(int));
      m.write(reinterpret_cast<const char*>(&nc), sizeof(int));
      m.write(reinterpret_cast<const char*>(map.data()), map.size() * sizeof(int));
      if (!m) return false;
    }
    if (verbose >= 1) std::cout << "Done writing NCC files with prefix " << outfile_prefix << "\n";
    return true;
  }

 private:
  cudaStream_t stream_ = nullptr;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr, e2_ = nullptr;
  DevVec<double2> d_caus_;
  DevVec<int> d_diff_, d_fine_, d_out_, d_err_;

  // read_complex_array (include/array_functions.cuh:172-268): int nrows, int
  // ncols, then complex values in T, float or double (by the file size).
  bool read_caustics(const std::string& fname, std::vector<double2>& out) {
    if (std::filesystem::path(fname).extension() != ".bin") {
      std::cerr << "Error. File " << fname << " is not a .bin file.\n";
      return false;
    }
    std::error_code ec;
    const auto fsize = std::filesystem::file_size(fname, ec);
    if (ec) {
      std::cerr << "Error determining size of input file " << fname << "\n";
      return false;
    }
    std::ifstream in(fname, std::ios::binary);
    if (!in) {
      std::cerr << "Error. Failed to open file " << fname << "\n";
      return false;
    }
    int nr = 0, nc = 0;
    in.read(reinterpret_cast<char*>(&nr), sizeof(int));
    in.read(reinterpret_cast<char*>(&nc), sizeof(int));
    if (nr < 1 || nc < 1) {
      std::cerr << "Error. File " << fname << " does not contain valid values for num_rows and num_cols.\n";
      return false;
    }
    const size_t n = size_t(nr) * nc;
    out.resize(n);
    if (fsize == 2 * sizeof(int) + n * 2 * sizeof(double)) {
      in.read(reinterpret_cast<char*>(out.data()), n * sizeof(double2));
    } else if (fsize == 2 * sizeof(int) + n * 2 * sizeof(float)) {
      std::vector<float> tmp(2 * n);
      in.read(reinterpret_cast<char*>(tmp.data()), tmp.size() * sizeof(float));
      for (size_t k = 0; k < n; k++) out[k] = make_double2(tmp[2 * k], tmp[2 * k + 1]);
    } else {
      std::cerr << "Error. Binary file " << fname << " does not contain valid single or double precision numbers.\n";
      return false;
    }
    if (!in) {
      std::cerr << "Error. Failed reading file " << fname << "\n";
      return false;
    }
    num_rows = nr;
    num_cols = nc;
    return true;
  }
};

}  // namespace irsb
