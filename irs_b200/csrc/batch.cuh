// Many IPM realizations in one device pipeline, captured in one CUDA graph.
//
// Realizations of uneven size (own seed, convergence, shear, smooth fraction,
// mass function; one map size for the batch) share every launch:
//   * stars: one generation kernel per realization into one star buffer, then
//     one thread per realization sums its masses in star order (the host
//     summation of star_field_moments, so the corner and the tree root are
//     those of a single run); the host recomputes the corners;
//   * tree: one level-synchronous build over all roots (level l of every
//     realization in the same launches), level sizes kept on the device, a
//     fixed number of levels and fixed capacities checked on the device, so
//     that no host synchronisation is needed and the whole build is captured;
//   * expansions: the per-level FMM kernels over all realizations' nodes;
//   * leaves: one record set for all realizations (theta per realization);
//   * shooting: passes over a bounded corner buffer; a pass holds row bands of
//     one or more realizations, its tile list covers the leaves of all of them
//     (one persistent launch of shoot_f32_batch) and its deposition covers all
//     their 32-cell chunks (one persistent launch of ipm_deposit_batch);
//   * maps: one fixed-point map per realization, resolved and converted in
//     two launches.
// Tree build through deposition is captured once per batch shape and replayed.
// Each realization's map is bit-identical to a single run of the same inputs at
// the same expansion order: the per-node, per-leaf, per-point and per-cell
// arithmetic is the single run's, and the fixed-point deposition does not
// depend on the order of work.
#pragma once
#include "engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace irsb {

// ---------------------------------------------------------------- kernels

// Sequential mass sums per realization in star order (one thread each), as
// star_field_moments sums them on the host.
template <typename T>
__global__ void batch_star_moments(int R, const StarRec<T>* __restrict__ stars, const long long* __restrict__ off,
                                   double* __restrict__ out /* [R][2]: m_tot, m2_tot */,
                                   T* __restrict__ mlo, T* __restrict__ mhi) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    double m_tot = 0, m2_tot = 0;
    T lo = std::numeric_limits<T>::max(), hi = std::numeric_limits<T>::min();
    for (long long i = off[r]; i < off[r + 1]; i++) {
      const T m = stars[i].m;
      const T mm = sizeof(T) == 4 ? T(__fmul_rn(float(m), float(m))) : T(__dmul_rn(double(m), double(m)));
      m_tot = __dadd_rn(m_tot, double(m));
      m2_tot = __dadd_rn(m2_tot, double(mm));
      lo = m < lo ? m : lo;
      hi = m > hi ? m : hi;
    }
    out[2 * r] = m_tot;
    out[2 * r + 1] = m2_tot;
    mlo[r] = lo;
    mhi[r] = hi;
  }
}

// Roots of all realizations (level 0), level bookkeeping and flags reset.
template <typename T>
__global__ void batch_tree_roots(int R, const T* __restrict__ root_hl, const long long* __restrict__ star_off,
                                 T* cx, T* cy, T* hl, int* level, int* parent, int* child0, int* sbeg, int* scnt,
                                 int* rid, int* n_nbr, int* n_sil, int* n_dil, double* lox, double* hix, double* loy,
                                 double* hiy, int* off, int* lvl_n, int nlev, int* stop, int* dstat,
                                 int* levels_r) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    cx[r] = T(0);
    cy[r] = T(0);
    hl[r] = root_hl[r];
    level[r] = 0;
    parent[r] = -1;
    child0[r] = -1;
    sbeg[r] = int(star_off[r]);
    scnt[r] = int(star_off[r + 1] - star_off[r]);
    rid[r] = r;
    n_nbr[r] = n_sil[r] = n_dil[r] = 0;
    lox[r] = -INFINITY;
    hix[r] = INFINITY;
    loy[r] = -INFINITY;
    hiy[r] = INFINITY;
    levels_r[r] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    off[0] = 0;
    off[1] = R;
    for (int l = 2; l <= nlev + 1; l++) off[l] = R;
    lvl_n[0] = R;
    for (int l = 1; l <= nlev; l++) lvl_n[l] = 0;
    *stop = 0;
    dstat[0] = dstat[1] = 0;
  }
}

__global__ void batch_levels(const int* __restrict__ off, int nlev, const int* __restrict__ level,
                             const int* __restrict__ rid, int* levels_r) {
  const int n = off[nlev];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    atomicMax(&levels_r[rid[k]], level[k]);
}

__global__ void batch_set_count(const long long* __restrict__ sum, int* __restrict__ n) { *n = int(*sum); }

__global__ void batch_tile_end(const int* __restrict__ nleaves, const long long* __restrict__ sum,
                               long long* __restrict__ tile_off) {
  tile_off[*nleaves] = *sum;
}

// ---------------------------------------------------------------- host driver

template <typename T>
class BatchMaker {
 public:
  std::vector<Params<T>> in;  // inputs of each realization
  int expansion_order = 0;    // 0: the largest reference-formula order over the batch
  long long corner_cap = 0;   // corner positions per pass (0: chosen from free memory)
  int nlev = 24;              // tree levels the captured build holds

  // results
  std::vector<Params<T>> prm;  // derived parameters of each realization
  std::vector<int> levels;     // tree levels of each realization
  int order = 0;               // expansion order used
  int passes = 0;
  long long total_cells = 0, total_pixels = 0, total_stars = 0;
  double t_stars = 0, t_graph = 0;  // seconds: star generation + moments, graph replay
  int graph_nodes = 0;
  bool graph_used = false;

  ~BatchMaker() { release(); }

  int size() const { return int(in.size()); }

  // Star field, tree, expansions, leaves, shooting and deposition of every
  // realization; maps stay on the device (maps_device) until copied.
  bool run(int verbose) {
    if (in.empty()) {
      std::cerr << "Error. The batch holds no realization.\n";
      return false;
    }
    if (!stream_ && !IRSB_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking))) return false;
    if (!ev0_) {
      IRSB_CKR(cudaEventCreate(&ev0_));
      IRSB_CKR(cudaEventCreate(&ev1_));
      IRSB_CKR(cudaEventCreate(&ev2_));
    }
    if (!derive()) return false;
    IRSB_CKR(cudaEventRecord(ev0_, stream_));
    if (!make_stars()) return false;
    IRSB_CKR(cudaEventRecord(ev1_, stream_));
    const std::vector<long long> shape = shape_key();
    if (!graph_ || shape != shape_) {
      if (!plan()) return false;
      for (int attempt = 0; attempt < 3; attempt++) {
        if (!capture()) return false;
        shape_ = shape;
        if (!replay()) return false;
        int st = 0;
        if (!check(&st)) return false;
        if (!(st & (kErrNodeOverflow | kErrLevelOverflow | kErrTableOverflow))) break;
        // grow the capacity that ran out and capture again
        if (st & kErrNodeOverflow) node_cap_ *= 2;
        if (st & kErrLevelOverflow) nlev = std::min(kMaxLevels, nlev + 8);
        if (st & kErrTableOverflow) table_cap_ *= 2;
        if (attempt == 2) {
          std::cerr << "Error. Batch capacities exceeded (code " << st << ").\n";
          return false;
        }
        if (!plan_buffers()) return false;
      }
    } else {
      if (!replay()) return false;
      int st = 0;
      if (!check(&st)) return false;
      if (st) {
        std::cerr << "Error. Batch pipeline failed (code " << st << ").\n";
        return false;
      }
    }
    float ms_stars = 0, ms_graph = 0;
    IRSB_CKR(cudaEventElapsedTime(&ms_stars, ev0_, ev1_));
    IRSB_CKR(cudaEventElapsedTime(&ms_graph, ev1_, ev2_));
    t_stars = ms_stars * 1e-3;
    t_graph = ms_graph * 1e-3;
    if (!read_levels()) return false;
    if (verbose >= 1)
      std::cout << "batch: " << size() << " realizations, " << total_stars << " stars, " << total_cells
                << " cells, order " << order << ", passes " << passes << ", graph " << t_graph << " s\n";
    return true;
  }

  // Replays the captured pipeline `repeats` times on the star fields of the last
  // run (the build is idempotent on them); summed device seconds.
  bool rerun(int repeats, double* seconds) {
    if (!graph_) {
      std::cerr << "Error. rerun() needs a completed run().\n";
      return false;
    }
    double tot = 0;
    for (int i = 0; i < repeats; i++) {
      IRSB_CKR(cudaEventRecord(ev1_, stream_));
      if (!replay()) return false;
      int st = 0;
      if (!check(&st)) return false;
      if (st) return false;
      float ms = 0;
      IRSB_CKR(cudaEventElapsedTime(&ms, ev1_, ev2_));
      tot += ms * 1e-3;
    }
    t_graph = tot / std::max(1, repeats);
    if (seconds) *seconds = tot;
    return true;
  }

  // Maps of all realizations, [R][npy][npx] in T, on the device.
  const T* maps_device() const { return d_out_.p; }
  bool copy_maps(T* host) {
    IRSB_CKR(cudaMemcpyAsync(host, d_out_.p, size_t(total_pixels) * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    return true;
  }
  bool copy_stars(T* host) {  // [N][3], realizations in order, each in tree order
    IRSB_CKR(cudaMemcpyAsync(host, d_stars_.p, size_t(total_stars) * sizeof(StarRec<T>), cudaMemcpyDeviceToHost,
                             stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    return true;
  }
  long long star_offset(int r) const { return star_off_[r]; }
  int npx() const { return npx_; }
  int npy() const { return npy_; }

 private:
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, ev2_ = nullptr;
  cudaGraph_t graph_src_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  std::vector<long long> shape_;
  int npx_ = 0, npy_ = 0;
  bool generic_ = false;
  long long node_cap_ = 0, table_cap_ = 0, vcap_ = 0;
  std::vector<long long> star_off_;
  // device
  DevVec<StarRec<T>> d_stars_;
  DevVec<long long> d_star_off_;
  DevVec<double> d_msum_;
  DevVec<T> d_mlo_, d_mhi_, d_root_hl_;
  DevVec<double> d_theta_;
  DevVec<int> d_off_, d_lvl_n_, d_stop_, d_levels_;
  TreeDev<T> tree_;
  FmmDev fmm_;
  LeafSet leaves_;
  DevVec<int> d_leaf_rid_, d_nleaves_;
  LatticeTiles tiles_;
  DevVec<ShootParams> d_sps_;
  DevVec<LatticeGeom> d_geom_;
  DevVec<long long> d_jlo_, d_jhi_, d_voff_;  // [passes][R]
  DevVec<double2> d_verts_;
  HostVec<double> h_msum_;
  HostVec<T> h_mlo_, h_mhi_;
  // deposition
  struct PassPlan {
    long long nchunks = 0, poff = 0;
    int npieces = 0;
  };
  std::vector<PassPlan> pass_;
  DevVec<DepositPiece<float>> d_pieces_;
  DevVec<unsigned long long> d_acc_, d_diff_;
  DevVec<T> d_out_;

  void release() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (graph_src_) cudaGraphDestroy(graph_src_);
    graph_ = nullptr;
    graph_src_ = nullptr;
    if (stream_) cudaStreamDestroy(stream_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (ev2_) cudaEventDestroy(ev2_);
    stream_ = nullptr;
    ev0_ = ev1_ = ev2_ = nullptr;
  }

  bool derive() {
    const int R = size();
    prm.assign(in.begin(), in.end());
    npx_ = prm[0].num_pixels_y.re;
    npy_ = prm[0].num_pixels_y.im;
    total_cells = 0;
    total_stars = 0;
    generic_ = false;
    star_off_.assign(R + 1, 0);
    for (int r = 0; r < R; r++) {
      Params<T>& p = prm[r];
      if (!p.starfile.empty()) {
        std::cerr << "Error. Batched realizations draw their own star fields (no star file).\n";
        return false;
      }
      if (p.num_pixels_y.re != npx_ || p.num_pixels_y.im != npy_) {
        std::cerr << "Error. All realizations of a batch need the same number of pixels.\n";
        return false;
      }
      if (!check_input_params(p)) return false;
      std::vector<StarRec<T>> none;
      if (!derive_params<T>(p, none, false)) return false;
      if (p.random_seed == 0) {
        std::cerr << "Error. Batched realizations need a nonzero random seed.\n";
        return false;
      }
      if (!(p.approx && !p.rectangular)) generic_ = true;
      star_off_[r + 1] = star_off_[r] + p.num_stars;
      total_cells += (long long)p.num_ray_threads.re * p.num_ray_threads.im;
    }
    total_stars = star_off_[R];
    total_pixels = (long long)R * npx_ * npy_;
    return true;
  }

  // Star fields, mass sums, corners and tree roots (eager: the corners are
  // computed on the host exactly as for a single run).
  bool make_stars() {
    const int R = size();
    if (!d_stars_.alloc_exact(total_stars) || !d_star_off_.alloc_exact(R + 1) || !d_msum_.alloc_exact(2 * R) ||
        !d_mlo_.alloc_exact(R) || !d_mhi_.alloc_exact(R) || !h_msum_.alloc(2 * R) || !h_mlo_.alloc(R) ||
        !h_mhi_.alloc(R))
      return false;
    IRSB_CKR(cudaMemcpyAsync(d_star_off_.p, star_off_.data(), (R + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                             stream_));
    for (int r = 0; r < R; r++) {
      const Params<T>& p = prm[r];
      const int n = p.num_stars;
      const int blocks = std::max(1, std::min(ceil_div(n, 256), 148 * 16));
      generate_stars_kernel<T><<<blocks, 256, 0, stream_>>>(d_stars_.p + star_off_[r], n, p.random_seed,
                                                             p.rectangular, p.corner, p.mf_kind, p.m_lower,
                                                             p.m_upper, p.m_solar);
      IRSB_LAUNCH_CK("generate_stars_kernel");
    }
    batch_star_moments<T><<<ceil_div(R, 64), 64, 0, stream_>>>(R, d_stars_.p, d_star_off_.p, d_msum_.p, d_mlo_.p,
                                                                d_mhi_.p);
    IRSB_LAUNCH_CK("batch_star_moments");
    IRSB_CKR(cudaMemcpyAsync(h_msum_.p, d_msum_.p, 2 * R * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaMemcpyAsync(h_mlo_.p, d_mlo_.p, R * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaMemcpyAsync(h_mhi_.p, d_mhi_.p, R * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    for (int r = 0; r < R; r++) {
      Params<T>& p = prm[r];
      const double m_tot = h_msum_.p[2 * r], m2_tot = h_msum_.p[2 * r + 1];
      const int n = p.num_stars;
      p.m_lower_actual = h_mlo_.p[r];
      p.m_upper_actual = h_mhi_.p[r];
      p.mean_mass_actual = T(m_tot / n);
      p.mean_mass2_actual = T(m2_tot / n);
      if (p.rectangular)
        p.kappa_star_actual = T(m_tot * kPi<T> * p.theta_star * p.theta_star / (4 * p.corner.re * p.corner.im));
      else
        p.kappa_star_actual = T(m_tot * p.theta_star * p.theta_star / (cabs_(p.corner) * cabs_(p.corner)));
      recompute_corner(p);
      p.root_half_length = root_half_length_of(p);
    }
    return true;
  }

  std::vector<long long> shape_key() const {
    std::vector<long long> k;
    for (const Params<T>& p : prm) {
      k.push_back(p.num_stars);
      k.push_back(p.num_ray_threads.re);
      k.push_back(p.num_ray_threads.im);
      k.push_back(p.random_seed);
      for (double v : {double(p.kappa_tot), double(p.shear), double(p.kappa_star), double(p.theta_star),
                       double(p.corner.re), double(p.corner.im), double(p.half_length_y.re),
                       double(p.half_length_y.im)}) {
        long long b;
        std::memcpy(&b, &v, sizeof b);
        k.push_back(b);
      }
    }
    k.push_back(expansion_order);
    k.push_back(corner_cap);
    return k;
  }

  // Expansion order, capacities, passes and all device tables.
  bool plan() {
    const int R = size();
    node_cap_ = 2 * total_stars + 8LL * R + 1024;
    // the reference formula needs the tree depth: estimate it from the star
    // count (a level per factor 4 beyond 32 stars); the order used is
    // reported, and a fixed expansion_order replaces the estimate
    order = expansion_order;
    if (order <= 0) {
      for (const Params<T>& p0 : prm) {
        Params<T> p = p0;
        p.tree_levels = int(std::ceil(std::log(std::max(1.0, p.num_stars / 32.0)) / std::log(4.0))) + 2;
        order = std::max(order, expansion_order_of(p));
      }
    }
    order = std::max(3, std::min(kMaxOrder, order));
    for (Params<T>& p : prm) p.expansion_order = order;
    // corner buffer: bounded by free memory, at least two corner rows of the
    // widest realization
    long long widest = 0, needed = 0;
    for (const Params<T>& p : prm) {
      widest = std::max<long long>(widest, p.num_ray_threads.re + 1);
      needed += ((long long)p.num_ray_threads.re + 1) * (p.num_ray_threads.im + 1);
    }
    vcap_ = corner_cap;
    if (vcap_ <= 0) {
      size_t fr = 0, tot = 0;
      IRSB_CKR(cudaMemGetInfo(&fr, &tot));
      vcap_ = std::min<long long>(needed, (long long)(fr / 4) / (long long)sizeof(double2));
      vcap_ = std::min<long long>(vcap_, 512LL << 20);  // 8 GB
    }
    vcap_ = std::max(vcap_, 2 * widest);
    // passes: realizations in order, cut into row pieces that fill the buffer
    std::vector<std::vector<long long>> jlo(1, std::vector<long long>(R, 0)), jhi(1, std::vector<long long>(R, 0)),
        voff(1, std::vector<long long>(R, 0));
    std::vector<DepositPiece<float>> pieces;
    pass_.assign(1, PassPlan{});
    long long used = 0;
    for (int r = 0; r < R; r++) {
      const Params<T>& p = prm[r];
      const long long ncx = p.num_ray_threads.re, ncy = p.num_ray_threads.im, w = ncx + 1;
      const float factor = ipm_triangle_factor<T, float>(p);
      long long row = 0;
      while (row < ncy) {
        long long room = (vcap_ - used) / w - 1;  // cell rows that fit (corner rows - 1)
        if (room <= 0) {
          jlo.emplace_back(R, 0);
          jhi.emplace_back(R, 0);
          voff.emplace_back(R, 0);
          pass_.push_back(PassPlan{});
          pass_.back().poff = (long long)pieces.size();
          used = 0;
          continue;
        }
        const long long take = std::min(room, ncy - row);
        PassPlan& pp = pass_.back();
        DepositPiece<float> pc;
        pc.voff = used;
        pc.vstride = ncx + 1;
        pc.vstep = 1;
        pc.ox = pc.oy = 0.0;
        pc.inv_scale = 1.0;
        pc.ncx = ncx;
        pc.ncy = take;
        pc.chunk0 = pp.nchunks;
        pc.factor = factor;
        pc.r = r;
        pieces.push_back(pc);
        pp.npieces++;
        pp.nchunks += (ncx * take + 31) / 32;
        jlo.back()[r] = row;
        jhi.back()[r] = row + take + 1;
        voff.back()[r] = used;
        used += (take + 1) * w;
        row += take;
      }
    }
    passes = int(pass_.size());
    table_cap_ = 2 * (vcap_ / (kTileX * kTileY)) + 2 * node_cap_ + 1024;
    // tables
    std::vector<ShootParams> sps(R);
    std::vector<LatticeGeom> geom(R);
    std::vector<double> theta(R);
    std::vector<T> root_hl(R);
    for (int r = 0; r < R; r++) {
      sps[r] = make_shoot_params(prm[r], true, 0);
      geom[r] = LatticeGeom{sps[r].base_x, sps[r].base_y, sps[r].rhs_x, sps[r].rhs_y, sps[r].nx, sps[r].ny};
      theta[r] = double(prm[r].theta_star);
      root_hl[r] = prm[r].root_half_length;
    }
    std::vector<long long> fjlo, fjhi, fvoff;
    for (int c = 0; c < passes; c++) {
      fjlo.insert(fjlo.end(), jlo[c].begin(), jlo[c].end());
      fjhi.insert(fjhi.end(), jhi[c].begin(), jhi[c].end());
      fvoff.insert(fvoff.end(), voff[c].begin(), voff[c].end());
    }
    if (!d_sps_.alloc_exact(R) || !d_geom_.alloc_exact(R) || !d_theta_.alloc_exact(R) ||
        !d_root_hl_.alloc_exact(R) || !d_jlo_.alloc_exact(fjlo.size()) || !d_jhi_.alloc_exact(fjhi.size()) ||
        !d_voff_.alloc_exact(fvoff.size()) || !d_pieces_.alloc_exact(pieces.size()))
      return false;
    IRSB_CKR(cudaMemcpyAsync(d_sps_.p, sps.data(), R * sizeof(ShootParams), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaMemcpyAsync(d_geom_.p, geom.data(), R * sizeof(LatticeGeom), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaMemcpyAsync(d_theta_.p, theta.data(), R * sizeof(double), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaMemcpyAsync(d_root_hl_.p, root_hl.data(), R * sizeof(T), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaMemcpyAsync(d_jlo_.p, fjlo.data(), fjlo.size() * sizeof(long long), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaMemcpyAsync(d_jhi_.p, fjhi.data(), fjhi.size() * sizeof(long long), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(
        cudaMemcpyAsync(d_voff_.p, fvoff.data(), fvoff.size() * sizeof(long long), cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaMemcpyAsync(d_pieces_.p, pieces.data(), pieces.size() * sizeof(DepositPiece<float>),
                             cudaMemcpyHostToDevice, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));  // host tables go out of scope
    return plan_buffers();
  }

  bool plan_buffers() {
    const int R = size();
    const long long ncoef = node_cap_ * (order + 1);
    if (!tree_reserve(tree_, int(node_cap_), stream_) || !tree_.tmp_stars.reserve(total_stars, stream_) ||
        !tree_.dstat.reserve(2, stream_) || !tree_.split.reserve(node_cap_, stream_) ||
        !tree_.rank.reserve(node_cap_ + 1, stream_) || !scan_reserve(tree_.scan, node_cap_, stream_))
      return false;
    if (!d_off_.alloc_exact(kMaxLevels + 2) || !d_lvl_n_.alloc_exact(kMaxLevels + 1) || !d_stop_.alloc_exact(1) ||
        !d_levels_.alloc_exact(R))
      return false;
    if (!fmm_.mult.alloc_exact(ncoef) || !fmm_.loc.alloc_exact(ncoef)) return false;
    fmm_.p = order;
    std::vector<double> bt = binomial_table(2 * kMaxOrder);
    if (!fmm_.btab.alloc_exact(bt.size())) return false;
    IRSB_CKR(cudaMemcpyAsync(fmm_.btab.p, bt.data(), bt.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
    LeafSet& L = leaves_;
    if (!L.flag.alloc_exact(node_cap_) || !L.pos.alloc_exact(node_cap_ + 1) || !L.node.alloc_exact(node_cap_) ||
        !L.cx.alloc_exact(node_cap_) || !L.cy.alloc_exact(node_cap_) || !L.hl.alloc_exact(node_cap_) ||
        !L.nnear.alloc_exact(node_cap_) || !L.near32.alloc_exact(node_cap_ * kMaxStarsDirect) ||
        !L.coef32.alloc_exact(node_cap_ * kMaxOrder) || !d_leaf_rid_.alloc_exact(node_cap_) ||
        !d_nleaves_.alloc_exact(1) || !scan_reserve(L.scan, node_cap_, stream_))
      return false;
    LatticeTiles& W = tiles_;
    if (!W.rect.alloc_exact(node_cap_) || !W.tiles.alloc_exact(node_cap_) || !W.tile_off.alloc_exact(node_cap_ + 1) ||
        !W.table.alloc_exact(table_cap_) || !scan_reserve(W.scan, node_cap_, stream_))
      return false;
    IRSB_CKR(cudaMemsetAsync(W.table.p, 0, table_cap_ * sizeof(int4), stream_));
    if (!d_verts_.alloc_exact(vcap_)) return false;
    const long long npix = (long long)npx_ * npy_, ndiff = (long long)npy_ * (npx_ + 1);
    if (!d_acc_.alloc_exact(npix * R) || !d_diff_.alloc_exact(ndiff * R) || !d_out_.alloc_exact(npix * R))
      return false;
    IRSB_CKR(cudaStreamSynchronize(stream_));
    return true;
  }

  LeafPtrs leaf_ptrs() const {
    LeafPtrs lp{};
    lp.cx = leaves_.cx.p;
    lp.cy = leaves_.cy.p;
    lp.hl = leaves_.hl.p;
    lp.nnear = leaves_.nnear.p;
    lp.near32 = leaves_.near32.p;
    lp.coef32 = leaves_.coef32.p;
    lp.rect = tiles_.rect.p;
    lp.tile_off = tiles_.tile_off.p;
    lp.table = tiles_.table.p;
    lp.nleaves = 0;
    return lp;
  }

  // The device pipeline after the star fields, as one stream of launches with
  // no host synchronisation (recorded into the graph).
  bool record() {
    const int R = size();
    cudaStream_t s = stream_;
    TreeDev<T>& t = tree_;
    const int G = 148 * 8;  // grid of the level kernels (grid-stride)
    const int ncap = int(node_cap_);
    int* dstat = t.dstat.p;
    batch_tree_roots<T><<<ceil_div(R, 128), 128, 0, s>>>(
        R, d_root_hl_.p, d_star_off_.p, t.cx.p, t.cy.p, t.hl.p, t.level.p, t.parent.p, t.child0.p, t.sbeg.p,
        t.scnt.p, t.rid.p, t.n_nbr.p, t.n_sil.p, t.n_dil.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p, d_off_.p, d_lvl_n_.p,
        nlev, d_stop_.p, dstat, d_levels_.p);
    IRSB_LAUNCH_CK("batch_tree_roots");
    for (int l = 0; l < nlev; l++) {
      const LevelRange lr{d_off_.p, l};
      tree_near_count<<<G, 256, 0, s>>>(0, 0, lr, t.scnt.p, t.nbr.p, t.n_nbr.p, t.split.p, dstat);
      if (!exclusive_scan_dev<int>(t.split.p, d_lvl_n_.p + l, node_cap_, t.rank.p, t.scan, s)) return false;
      tree_advance_level<<<1, 1, 0, s>>>(l, nlev, d_off_.p, d_lvl_n_.p, t.scan.sum.p, ncap, d_stop_.p, dstat);
      tree_make_children<T><<<G, 256, 0, s>>>(0, 0, 0, lr, d_stop_.p, t.split.p, t.rank.p, t.cx.p, t.cy.p, t.hl.p,
                                              t.level.p, t.parent.p, t.child0.p, t.sbeg.p, t.scnt.p, t.rid.p,
                                              t.n_nbr.p, t.n_sil.p, t.n_dil.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p);
      if (l + 1 < nlev) {
        if (l < 2)  // a few nodes per realization, many stars each
          tree_partition_stars<T, 1024><<<G, 1024, 0, s>>>(0, 0, lr, d_stop_.p, t.split.p, t.cx.p, t.cy.p,
                                                            t.child0.p, t.sbeg.p, t.scnt.p, d_stars_.p,
                                                            t.tmp_stars.p);
        else
          tree_partition_stars<T><<<G, 256, 0, s>>>(0, 0, lr, d_stop_.p, t.split.p, t.cx.p, t.cy.p, t.child0.p,
                                                    t.sbeg.p, t.scnt.p, d_stars_.p, t.tmp_stars.p);
        tree_set_neighbors<T><<<G, 256, 0, s>>>(0, 0, LevelRange{d_off_.p, l + 1}, t.cx.p, t.cy.p, t.hl.p,
                                                t.parent.p, t.child0.p, t.scnt.p, t.nbr.p, t.n_nbr.p, t.sil.p,
                                                t.n_sil.p, t.dil.p, t.n_dil.p, dstat);
      }
      IRSB_LAUNCH_CK("batch tree level");
    }
    batch_levels<<<G, 256, 0, s>>>(d_off_.p, nlev, t.level.p, t.rid.p, d_levels_.p);
    // expansions
    const long long ncoef = node_cap_ * (order + 1);
    IRSB_CKR(cudaMemsetAsync(fmm_.mult.p, 0, ncoef * sizeof(double2), s));
    IRSB_CKR(cudaMemsetAsync(fmm_.loc.p, 0, ncoef * sizeof(double2), s));
    const int GF = 148 * 16;
    for (int l = nlev - 1; l >= 0; l--) {
      const LevelRange lr{d_off_.p, l};
      fmm_p2m<T><<<GF, 256, 0, s>>>(0, 0, lr, order, t.cx.p, t.cy.p, t.hl.p, t.child0.p, t.sbeg.p, t.scnt.p,
                                     d_stars_.p, fmm_.mult.p);
      fmm_m2m<T><<<GF, 256, 0, s>>>(0, 0, lr, order, t.cx.p, t.cy.p, t.hl.p, t.child0.p, fmm_.btab.p, fmm_.mult.p);
    }
    for (int l = 2; l < nlev; l++) {
      fmm_local<T><<<GF, 256, 0, s>>>(0, 0, LevelRange{d_off_.p, l}, order, t.cx.p, t.cy.p, t.hl.p, t.parent.p,
                                       t.sbeg.p, t.scnt.p, t.sil.p, t.n_sil.p, t.dil.p, t.n_dil.p, d_stars_.p,
                                       fmm_.btab.p, fmm_.mult.p, fmm_.loc.p);
    }
    IRSB_LAUNCH_CK("batch fmm");
    // leaves
    LeafSet& L = leaves_;
    const int* dnodes = d_off_.p + nlev;
    leaf_flags<<<G, 256, 0, s>>>(0, dnodes, t.child0.p, L.flag.p);
    if (!exclusive_scan_dev<int>(L.flag.p, dnodes, node_cap_, L.pos.p, L.scan, s)) return false;
    batch_set_count<<<1, 1, 0, s>>>(L.scan.sum.p, d_nleaves_.p);
    leaf_compact<<<G, 256, 0, s>>>(0, dnodes, L.flag.p, L.pos.p, L.node.p);
    leaf_build<T><<<GF, 256, 0, s>>>(0, d_nleaves_.p, order, 1.0, d_theta_.p, t.rid.p, L.node.p, t.cx.p, t.cy.p,
                                     t.hl.p, t.sbeg.p, t.scnt.p, t.nbr.p, t.n_nbr.p, d_stars_.p, fmm_.loc.p, L.cx.p,
                                     L.cy.p, L.hl.p, L.nnear.p, nullptr, L.near32.p, nullptr, L.coef32.p,
                                     d_leaf_rid_.p, dstat + 1);
    IRSB_LAUNCH_CK("batch leaves");
    // maps
    const long long npix = (long long)npx_ * npy_, ndiff = (long long)npy_ * (npx_ + 1);
    IRSB_CKR(cudaMemsetAsync(d_acc_.p, 0, npix * R * sizeof(unsigned long long), s));
    IRSB_CKR(cudaMemsetAsync(d_diff_.p, 0, ndiff * R * sizeof(unsigned long long), s));
    // passes
    LatticeTiles& W = tiles_;
    const LeafPtrs lp = leaf_ptrs();
    for (int c = 0; c < passes; c++) {
      leaf_rects_batch<<<G, 256, 0, s>>>(d_nleaves_.p, L.node.p, t.rid.p, t.lox.p, t.hix.p, t.loy.p, t.hiy.p,
                                         d_geom_.p, d_jlo_.p + (long long)c * R, d_jhi_.p + (long long)c * R, kTileX,
                                         kTileY, W.rect.p, W.tiles.p);
      if (!exclusive_scan_dev<long long>(W.tiles.p, d_nleaves_.p, node_cap_, W.tile_off.p, W.scan, s)) return false;
      batch_tile_end<<<1, 1, 0, s>>>(d_nleaves_.p, W.scan.sum.p, W.tile_off.p);
      leaf_tile_table<<<G, 256, 0, s>>>(0, d_nleaves_.p, W.rect.p, W.tile_off.p, kTileX, kTileY, W.table.p,
                                        table_cap_, dstat + 1);
      BatchShoot bs{d_sps_.p, d_leaf_rid_.p, d_jlo_.p + (long long)c * R, d_voff_.p + (long long)c * R,
                    W.scan.sum.p, table_cap_, dstat + 1};
      if (generic_)
        shoot_f32_batch<true><<<148 * 64, kShootBatchThreads, 0, s>>>(bs, lp, d_verts_.p);
      else
        shoot_f32_batch<false><<<148 * 64, kShootBatchThreads, 0, s>>>(bs, lp, d_verts_.p);
      const PassPlan& pp = pass_[c];
      const int grid = deposit_grid(pp.nchunks);
      ipm_deposit_batch<float><<<grid, kDepositThreads, 0, s>>>(d_verts_.p, d_pieces_.p + pp.poff, pp.npieces, pp.nchunks, npx_,
                                                    npy_, DepositMaps{d_acc_.p, d_diff_.p}, npix, ndiff);
      IRSB_LAUNCH_CK("batch pass");
    }
    const DepositMaps mt{d_acc_.p, d_diff_.p};
    const int gr = std::max(1, std::min(ceil_div((long long)npy_ * R * 32, 256), 148 * 8));
    ipm_resolve_rows_out<T><<<gr, 256, 0, s>>>(npx_, npy_ * R, mt, d_out_.p);  // resolve and convert
    IRSB_LAUNCH_CK("batch maps");
    return true;
  }

  bool capture() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (graph_src_) cudaGraphDestroy(graph_src_);
    graph_ = nullptr;
    graph_src_ = nullptr;
    IRSB_CKR(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    const bool ok = record();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (!ok || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      std::cerr << "Error. Capturing the batch pipeline failed: " << cudaGetErrorString(e) << "\n";
      return false;
    }
    graph_src_ = g;
    size_t n = 0;
    IRSB_CKR(cudaGraphGetNodes(g, nullptr, &n));
    graph_nodes = int(n);
    IRSB_CKR(cudaGraphInstantiate(&graph_, g, 0));
    graph_used = true;
    return true;
  }

  bool replay() {
    IRSB_CKR(cudaGraphLaunch(graph_, stream_));
    IRSB_CKR(cudaEventRecord(ev2_, stream_));
    return true;
  }

  bool check(int* st) {
    int h[2] = {0, 0};
    IRSB_CKR(cudaMemcpyAsync(h, tree_.dstat.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    *st = h[1];
    if (h[1] & (kErrNeighborOverflow | kErrSameLevelOverflow | kErrDiffLevelOverflow | kErrNearOverflow)) {
      std::cerr << "Error. Tree list overflow in the batch (code " << h[1] << ").\n";
      return false;
    }
    return true;
  }

  bool read_levels() {
    const int R = size();
    levels.assign(R, 0);
    IRSB_CKR(cudaMemcpyAsync(levels.data(), d_levels_.p, R * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    IRSB_CKR(cudaStreamSynchronize(stream_));
    for (int r = 0; r < R; r++) prm[r].tree_levels = levels[r];
    return true;
  }
};

}  // namespace irsb
