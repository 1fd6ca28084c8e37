// Host driver of the adaptive IPM (kernels in adaptive.cuh and mlp.cuh).
//
// run():
//   1. the base pass of MapMaker in the FP32 form, stopped after the corner
//      lattice (tree, expansions, leaf records, tiled lens equation);
//   2. per-tile features and the level of every tile: from the network, one
//      uniform level, or levels given by the caller;
//   3. audit: a seeded random sample of tiles is deposited on its own at its
//      chosen level and at level 16 (ada_window_errors); a tile whose deposit
//      differs by more than the tolerance falls back to level 16;
//   4. deposition: level-1 tiles straight from the base lattice, refined tiles
//      level by level through a bounded corner buffer (conforming corners,
//      factor / s^2 per subcell), all into one fixed-point map;
//   5. resolve and convert the map.
// Steps 2-5 are timed as t_adapt, step 1 as t_base.
#pragma once
#include "adaptive.cuh"
#include "engine.cuh"
#include "mlp.cuh"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace irsb {

enum AdaPolicy : int { kAdaNetwork = 0, kAdaUniform = 1, kAdaGiven = 2 };

template <typename T>
class AdaptiveIPM {
 public:
  MapMaker<T, false> base;
  int policy = kAdaNetwork;
  int uniform_level = 1;
  std::vector<int> given_levels;
  double eps = 1e-3;             // tolerance of a tile's deposit error (err_mode)
  int max_level = 8;  // labels and network choices stop here; only the audit sends tiles to 16
  int err_mode = 0;  // 0: share of the tile's own flux; 1: of the map's flux where it lands; 2: the smaller (ada_window_errors)
  double audit_fraction = 0.01;  // share of tiles audited per run
  unsigned audit_seed = 1;
  long long refine_cap = 0;      // corner positions in the refinement buffer (0: automatic)
  // chunks of at least this many tiles of one level are refined by the tiled
  // lens kernel over the level-s lattice (refine_tiled), smaller ones point by
  // point (ada_refine_tiles)
  int tiled_min = 1 << 30;
  std::vector<float> net_w, net_mu, net_sig;  // FP32 master weights, feature standardisation
  float net_quantile = 0.8f;  // a tile takes the smallest level whose cumulative probability reaches this
  // audit bound: when more than this share of the audited tiles misses eps at
  // its chosen level, the choice escalates (network quantiles 0.9, 0.95,
  // 0.99, then every tile one level finer, up to max_level) to the first
  // choice whose audited share is within the bound; audited tiles that still
  // miss go to level 16
  double fail_bound = 0.05;

  // results
  int ntx = 0, nty = 0;
  std::vector<int> level, predicted;  // per tile, subdivision 1..16
  long long cells_base = 0, cells_evaluated = 0, audit_cells = 0;
  int audited = 0, audit_failures = 0;
  double fail_rate_initial = 0, fail_rate = 0;  // audited share missing eps: the network's choice, the final choice
  int escalation = 0;  // 0: none; 1-3: network quantile 0.9 / 0.95 / 0.99; 4+: 3 + levels raised
  float quantile_used = 0.8f;
  double t_base = 0, t_adapt = 0;                          // seconds
  double t_select = 0, t_audit = 0, t_refine_deposit = 0;  // parts of t_adapt

  ~AdaptiveIPM() {
    if (e0_) cudaEventDestroy(e0_);
    if (e1_) cudaEventDestroy(e1_);
    if (ea_) cudaEventDestroy(ea_);
    if (eb_) cudaEventDestroy(eb_);
  }

  int num_tiles() const { return ntx * nty; }

  bool run(int verbose) {
    base.precision = kPrecisionFP32;
    base.verts_only = true;
    if (!base.run(verbose)) return false;
    t_base = base.t_pipeline;
    cudaStream_t s = base.stream_;
    if (!e0_) {
      IRSB_CKR(cudaEventCreate(&e0_));
      IRSB_CKR(cudaEventCreate(&e1_));
      IRSB_CKR(cudaEventCreate(&ea_));
      IRSB_CKR(cudaEventCreate(&eb_));
    }
    setup_geometry();
    base_map_ready_ = false;
    IRSB_CKR(cudaEventRecord(e0_, s));
    if (!features()) return false;
    if (!choose_levels()) return false;
    IRSB_CKR(cudaEventRecord(ea_, s));
    if (!audit()) return false;
    IRSB_CKR(cudaEventRecord(eb_, s));
    if (!deposit()) return false;
    IRSB_CKR(cudaEventRecord(e1_, s));
    IRSB_CKR(cudaEventSynchronize(e1_));
    float ms = 0, m1 = 0, m2 = 0;
    IRSB_CKR(cudaEventElapsedTime(&ms, e0_, e1_));
    IRSB_CKR(cudaEventElapsedTime(&m1, e0_, ea_));
    IRSB_CKR(cudaEventElapsedTime(&m2, ea_, eb_));
    t_adapt = ms * 1e-3;
    t_select = m1 * 1e-3;
    t_audit = m2 * 1e-3;
    t_refine_deposit = (ms - m1 - m2) * 1e-3;
    if (verbose >= 1) {
      long long hist[kAdaLevels] = {0};
      for (int v : level) hist[__builtin_ctz(v)]++;
      std::cout << "adaptive: " << num_tiles() << " tiles, levels 1/2/4/8/16 = " << hist[0] << "/" << hist[1] << "/"
                << hist[2] << "/" << hist[3] << "/" << hist[4] << ", audited " << audited << " (" << audit_failures
                << " fell back), cells " << cells_evaluated << " (base " << cells_base << ")\n";
    }
    return true;
  }

  // Labels of `tiles` (after run): smallest level within eps, at most
  // max_level, as a class 0..4, and the deposit errors of levels 1, 2, 4, 8
  // ([n][4]).
  bool labels(const std::vector<int>& tiles, std::vector<int>& lab, std::vector<float>& err) {
    lab.assign(tiles.size(), 0);
    err.assign(tiles.size() * 4, 0.f);
    if (!fine_errors(tiles, err)) return false;
    const int cmax = __builtin_ctz(std::max(1, std::min(kAdaMaxLevel, max_level)));
    for (size_t k = 0; k < tiles.size(); k++) {
      int c = 4;
      for (int q = 0; q < 4; q++)
        if (err[k * 4 + q] <= eps) {
          c = q;
          break;
        }
      lab[k] = std::min(c, cmax);
    }
    return true;
  }

  bool copy_features(float* out) {
    IRSB_CKR(cudaMemcpyAsync(out, d_feat_.p, size_t(num_tiles()) * kAdaFeatures * sizeof(float),
                             cudaMemcpyDeviceToHost, base.stream_));
    IRSB_CKR(cudaStreamSynchronize(base.stream_));
    return true;
  }
  bool copy_map(T* out) {
    const long long npix = (long long)base.prm.num_pixels_y.re * base.prm.num_pixels_y.im;
    IRSB_CKR(cudaMemcpyAsync(out, d_map_.p, npix * sizeof(T), cudaMemcpyDeviceToHost, base.stream_));
    IRSB_CKR(cudaStreamSynchronize(base.stream_));
    return true;
  }
  const T* map_device() const { return d_map_.p; }

 private:
  cudaEvent_t e0_ = nullptr, e1_ = nullptr, ea_ = nullptr, eb_ = nullptr;
  AdaGeom g_{};
  ShootParams sp_{};
  bool generic_ = false;
  DevVec<float> d_feat_, d_mu_, d_sig_, d_wf_, d_err_;
  DevVec<__nv_bfloat16> d_w_;
  DevVec<int> d_cls_, d_level_, d_list_;
  DevVec<double2> d_ref_;
  DevVec<DepositPiece<float>> d_pieces_;
  DevVec<int4> d_win_;
  DevVec<int> d_slot_;
  LatticeTiles rtiles_;  // lattice tiles of a refinement pass
  DevVec<unsigned long long> d_acc_, d_diff_, d_wacc_, d_wdiff_, d_bacc_, d_bdiff_;
  bool base_map_ready_ = false;
  DevVec<T> d_map_;
  DevVec<int> d_tile_leaf_;  // per tile: the leaf owning all its points, or -1
  bool tile_leaf_ready_ = false;

  void setup_geometry() {
    const Params<T>& p = base.prm;
    sp_ = make_shoot_params(p, true, 0);
    const long long ncx = p.num_ray_threads.re, ncy = p.num_ray_threads.im;
    ntx = int((ncx + kAdaTile - 1) / kAdaTile);
    nty = int((ncy + kAdaTile - 1) / kAdaTile);
    g_ = AdaGeom{sp_.base_x, sp_.base_y, sp_.rhs_x, sp_.rhs_y, ncx, ncy, ntx, nty, p.num_pixels_y.re,
                 p.num_pixels_y.im};
    generic_ = !(p.approx && !p.rectangular) && !base.smooth_folded();
    cells_base = ncx * ncy;
  }

  DescentPtrs<T> descent() const {
    return DescentPtrs<T>{base.tree_.cx.p, base.tree_.cy.p, base.tree_.child0.p, base.leaves_.pos.p,
                          tile_leaf_ready_ ? d_tile_leaf_.p : nullptr};
  }

  int tile_cells_x(int t) const { return int(std::min<long long>(kAdaTile, g_.ncx - (long long)(t % ntx) * kAdaTile)); }
  int tile_cells_y(int t) const { return int(std::min<long long>(kAdaTile, g_.ncy - (long long)(t / ntx) * kAdaTile)); }

  long long buffer_cap() {
    if (refine_cap > 0) return std::max<long long>(refine_cap, 513LL * 513);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 64LL << 20;
    return std::max<long long>(513LL * 513, std::min<long long>((long long)(fr / 4) / 16, 256LL << 20));
  }

  bool features() {
    const int nt = num_tiles();
    if (!d_feat_.alloc_exact((size_t)nt * kAdaFeatures) || !d_tile_leaf_.alloc_exact(nt)) return false;
    const int grid = std::max(1, std::min(ceil_div(nt, 128), 148 * 8));
    tile_leaf_ready_ = false;
    ada_features<T><<<grid, 128, 0, base.stream_>>>(g_, sp_, base.leaf_ptrs(), descent(), base.d_verts_.p,
                                                    d_feat_.p, d_tile_leaf_.p);
    IRSB_LAUNCH_CK("ada_features");
    tile_leaf_ready_ = true;
    return true;
  }

  bool choose_levels() {
    const int nt = num_tiles();
    level.assign(nt, 1);
    predicted.assign(nt, 1);
    if (policy == kAdaUniform) {
      level.assign(nt, uniform_level);
    } else if (policy == kAdaGiven) {
      if ((int)given_levels.size() != nt) {
        std::cerr << "Error. " << nt << " tile levels are needed, " << given_levels.size() << " were given.\n";
        return false;
      }
      level = given_levels;
    } else {
      if ((int)net_w.size() != kMlpParams || net_mu.size() != kMlpIn || net_sig.size() != kMlpIn) {
        std::cerr << "Error. The adaptive IPM has no level network.\n";
        return false;
      }
      if (!d_wf_.alloc_exact(kMlpParams) || !d_w_.alloc_exact(kMlpParams) || !d_mu_.alloc_exact(kMlpIn) ||
          !d_sig_.alloc_exact(kMlpIn) || !d_cls_.alloc_exact(nt))
        return false;
      cudaStream_t s = base.stream_;
      IRSB_CKR(cudaMemcpyAsync(d_wf_.p, net_w.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, s));
      IRSB_CKR(cudaMemcpyAsync(d_mu_.p, net_mu.data(), kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
      IRSB_CKR(cudaMemcpyAsync(d_sig_.p, net_sig.data(), kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
      mlp_to_bf16<<<ceil_div(kMlpParams, 256), 256, 0, s>>>(d_wf_.p, d_w_.p);
      if (!classify(net_quantile, level)) return false;
      quantile_used = net_quantile;
    }
    for (int v : level)
      if (v != 1 && v != 2 && v != 4 && v != 8 && v != 16) {
        std::cerr << "Error. Tile levels must be 1, 2, 4, 8 or 16.\n";
        return false;
      }
    predicted = level;
    return true;
  }

  // The network's levels of all tiles at cumulative-probability quantile q.
  bool classify(float q, std::vector<int>& lv) {
    const int nt = num_tiles();
    cudaStream_t s = base.stream_;
    mlp_classify<<<std::max(1, std::min(ceil_div(nt, 128), 148 * 4)), 128, 0, s>>>(d_w_.p, d_mu_.p, d_sig_.p,
                                                                                   d_feat_.p, nt, q, d_cls_.p);
    IRSB_LAUNCH_CK("mlp_classify");
    std::vector<int> cls(nt);
    IRSB_CKR(cudaMemcpyAsync(cls.data(), d_cls_.p, nt * sizeof(int), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    lv.resize(nt);
    for (int t = 0; t < nt; t++) lv[t] = std::min(ada_level_of(cls[t]), std::max(1, max_level));
    return true;
  }

  // Deposit errors of levels 1..8 against level 16 for isolated tiles
  // (ada_window_errors), [tiles][4].
  bool fine_errors(const std::vector<int>& tiles, std::vector<float>& err) {
    if (tiles.empty()) return true;
    cudaStream_t s = base.stream_;
    const Params<T>& p = base.prm;
    const float factor = ipm_triangle_factor<T, float>(p);
    if (err_mode >= 1 && !base_map_ready_ && !base_map()) return false;
    const long long per = 513LL * 513;
    const int chunk = int(std::max<long long>(1, std::min<long long>(64, buffer_cap() / per)));
    const int nc = int(std::min<size_t>(chunk, tiles.size()));
    if (!d_ref_.alloc_exact(nc * per) || !d_list_.alloc_exact(tiles.size()) || !d_err_.alloc_exact(tiles.size() * 4) ||
        !d_win_.alloc_exact(nc) || !d_pieces_.alloc_exact(nc * 5))
      return false;
    IRSB_CKR(cudaMemcpyAsync(d_list_.p, tiles.data(), tiles.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    std::vector<int4> win(nc);
    std::vector<DepositPiece<float>> pieces;
    for (size_t k0 = 0; k0 < tiles.size(); k0 += chunk) {
      const int n = int(std::min<size_t>(chunk, tiles.size() - k0));
      const int grid = int(std::max<long long>(1, std::min<long long>(ada_band_items(n, kAdaMaxLevel), 148LL * 8)));
      if (generic_)
        ada_refine_tiles<T, true><<<grid, 256, 0, s>>>(g_, sp_, base.leaf_ptrs(), descent(), base.d_verts_.p,
                                                       nullptr, d_list_.p + k0, n, kAdaMaxLevel, per, d_ref_.p);
      else
        ada_refine_tiles<T, false><<<grid, 256, 0, s>>>(g_, sp_, base.leaf_ptrs(), descent(), base.d_verts_.p,
                                                        nullptr, d_list_.p + k0, n, kAdaMaxLevel, per, d_ref_.p);
      ada_tile_windows<<<std::min(n, 148 * 8), 256, 0, s>>>(g_, d_list_.p + k0, n, per, d_ref_.p, d_win_.p);
      IRSB_LAUNCH_CK("ada windows");
      IRSB_CKR(cudaMemcpyAsync(win.data(), d_win_.p, n * sizeof(int4), cudaMemcpyDeviceToHost, s));
      IRSB_CKR(cudaStreamSynchronize(s));
      // window side of this chunk: the small one unless a tile needs more
      int ws = kAdaWindow;
      for (int k = 0; k < n; k++)
        if (win[k].z > kAdaWindow || win[k].w > kAdaWindow) ws = kAdaWindowLarge;
      const long long W2 = (long long)ws * ws, WD = (long long)ws * (ws + 1);
      if (!d_wacc_.alloc_exact(n * 5 * W2) || !d_wdiff_.alloc_exact(n * 5 * WD)) return false;
      pieces.clear();
      long long nchunks = 0;
      for (int k = 0; k < n; k++) {
        if (win[k].z <= 0) continue;
        const int t = tiles[k0 + k];
        const int cx = tile_cells_x(t), cy = tile_cells_y(t);
        for (int c = 0; c < kAdaLevels; c++) {
          const int sl = ada_level_of(c);
          DepositPiece<float> pc;
          pc.voff = (long long)k * per;
          pc.vstride = (long long)cx * kAdaMaxLevel + 1;
          pc.vstep = kAdaMaxLevel / sl;
          pc.ox = win[k].x;
          pc.oy = win[k].y;
          pc.inv_scale = 1.0 / ada_window_scale(win[k], ws);
          pc.ncx = (long long)cx * sl;
          pc.ncy = (long long)cy * sl;
          pc.chunk0 = nchunks;
          pc.factor = factor / float(sl * sl);
          pc.r = k * kAdaLevels + c;
          pieces.push_back(pc);
          nchunks += (pc.ncx * pc.ncy + 31) / 32;
        }
      }
      IRSB_CKR(cudaMemsetAsync(d_wacc_.p, 0, n * 5 * W2 * sizeof(unsigned long long), s));
      IRSB_CKR(cudaMemsetAsync(d_wdiff_.p, 0, n * 5 * WD * sizeof(unsigned long long), s));
      const DepositMaps M{d_wacc_.p, d_wdiff_.p};
      if (!pieces.empty()) {
        IRSB_CKR(cudaMemcpyAsync(d_pieces_.p, pieces.data(), pieces.size() * sizeof(DepositPiece<float>),
                                 cudaMemcpyHostToDevice, s));
        const int gd = deposit_grid(nchunks);
        ipm_deposit_batch<float><<<gd, kDepositThreads, 0, s>>>(d_ref_.p, d_pieces_.p, int(pieces.size()), nchunks, ws, ws, M,
                                                    W2, WD);
        const int gr = std::max(1, std::min(ceil_div((long long)ws * 5 * n * 32, 256), 148 * 8));
        ipm_resolve_rows<<<gr, 256, 0, s>>>(ws, ws * 5 * n, M);
      }
      ada_window_errors<<<std::min(n, 148 * 8), 256, 0, s>>>(g_, d_list_.p + k0, n, ws, factor, err_mode, d_win_.p,
                                                            d_wacc_.p, d_bacc_.p, d_err_.p + k0 * 4);
      IRSB_LAUNCH_CK("ada window errors");
      IRSB_CKR(cudaStreamSynchronize(s));  // the host pieces are rebuilt for the next chunk
    }
    IRSB_CKR(cudaMemcpyAsync(err.data(), d_err_.p, tiles.size() * 4 * sizeof(float), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    return true;
  }

  // The plain (level 1) map in fixed point, the reference of the tile errors.
  bool base_map() {
    cudaStream_t s = base.stream_;
    const Params<T>& p = base.prm;
    const int npx = p.num_pixels_y.re, npy = p.num_pixels_y.im;
    const long long npix = (long long)npx * npy, ndiff = (long long)npy * (npx + 1);
    if (!d_bacc_.alloc_exact(npix) || !d_bdiff_.alloc_exact(ndiff)) return false;
    IRSB_CKR(cudaMemsetAsync(d_bacc_.p, 0, npix * sizeof(unsigned long long), s));
    IRSB_CKR(cudaMemsetAsync(d_bdiff_.p, 0, ndiff * sizeof(unsigned long long), s));
    const DepositMaps M{d_bacc_.p, d_bdiff_.p};
    const long long ncells = g_.ncx * g_.ncy;
    const int grid = deposit_grid((ncells + 31) / 32);
    ipm_deposit_cells<float><<<grid, kDepositThreads, 0, s>>>(base.d_verts_.p, g_.ncx, g_.ncy, ipm_triangle_factor<T, float>(p),
                                                  npx, npy, M, M, M, 0);
    const int gr = std::max(1, std::min(ceil_div((long long)npy * 32, 256), 148 * 8));
    ipm_resolve_rows<<<gr, 256, 0, s>>>(npx, npy, M);
    IRSB_LAUNCH_CK("ada base map");
    base_map_ready_ = true;
    return true;
  }

  bool audit() {
    audited = audit_failures = 0;
    audit_cells = 0;
    if (audit_fraction <= 0) return true;
    std::mt19937_64 rng(audit_seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::vector<int> tiles;
    for (int t = 0; t < num_tiles(); t++)
      if (u(rng) < audit_fraction) tiles.push_back(t);
    if (tiles.empty()) return true;
    std::vector<float> err(tiles.size() * 4);
    if (!fine_errors(tiles, err)) return false;
    audited = int(tiles.size());
    // share of the audited tiles that a level assignment leaves above eps
    auto miss_rate = [&](const std::vector<int>& lv) {
      int miss = 0;
      for (size_t k = 0; k < tiles.size(); k++) {
        const int c = __builtin_ctz(lv[tiles[k]]);
        if (c < 4 && err[k * 4 + c] > eps) miss++;
      }
      return double(miss) / double(tiles.size());
    };
    fail_rate_initial = fail_rate = miss_rate(level);
    escalation = 0;
    if (policy == kAdaNetwork && fail_rate > fail_bound) {
      const float qs[3] = {0.9f, 0.95f, 0.99f};
      std::vector<int> lv;
      for (int e = 0; e < 3 && fail_rate > fail_bound; e++) {
        if (qs[e] <= quantile_used) continue;
        if (!classify(qs[e], lv)) return false;
        const double r = miss_rate(lv);
        if (r < fail_rate || r <= fail_bound) {
          level = lv, fail_rate = r, escalation = e + 1, quantile_used = qs[e];
        }
      }
      for (int up = 1; fail_rate > fail_bound && up <= 4; up++) {  // every tile finer, capped at max_level
        lv = level;
        bool changed = false;
        for (int& v : lv) {
          const int w = std::min(v * 2, std::max(1, max_level));
          changed = changed || w != v;
          v = w;
        }
        if (!changed) break;
        level = lv, fail_rate = miss_rate(lv), escalation = 3 + up;
      }
    }
    for (size_t k = 0; k < tiles.size(); k++) {
      const int t = tiles[k];
      audit_cells += (long long)tile_cells_x(t) * tile_cells_y(t) * kAdaMaxLevel * kAdaMaxLevel;
      const int c = __builtin_ctz(level[t]);
      if (c < 4 && err[k * 4 + c] > eps) {
        level[t] = kAdaMaxLevel;
        audit_failures++;
      }
    }
    return true;
  }


  // Corner grids of the tiles `tl` (host, row-major tile order) / `d_tl`
  // (device) at level sl into d_ref_: the leaf-tiled FP32 lens kernel over
  // the rows of the level-sl corner lattice that these tiles span, each point
  // stored in the grids holding it, then ada_fixup_corners.
  bool refine_tiled(int sl, const int* tl, const int* d_tl, int n) {
    cudaStream_t s = base.stream_;
    const int nt = num_tiles();
    const long long per = (long long)(kAdaTile * sl + 1) * (kAdaTile * sl + 1);
    if (!d_slot_.alloc_exact(nt)) return false;
    ada_slots_clear<<<std::max(1, std::min(ceil_div(nt, 256), 148 * 8)), 256, 0, s>>>(nt, d_slot_.p);
    ada_slots_set<<<std::max(1, ceil_div(n, 256)), 256, 0, s>>>(d_tl, n, d_slot_.p);
    const int ty_a = tl[0] / ntx, ty_b = tl[n - 1] / ntx;
    const long long nxs = g_.ncx * sl + 1, nys = g_.ncy * sl + 1;
    const long long jlo = (long long)ty_a * kAdaTile * sl;
    const long long jhi = std::min<long long>(((long long)ty_b + 1) * kAdaTile * sl + 1, nys);
    ShootParams sps = sp_;
    sps.rhs_x = sp_.rhs_x / sl;  // exact: sl is a power of two
    sps.rhs_y = sp_.rhs_y / sl;
    sps.nx = nxs;
    sps.ny = nys;
    sps.jbase = 0;
    if (!build_lattice_tiles<T>(rtiles_, base.leaves_, base.tree_, sps.base_x, sps.base_y, sps.rhs_x, sps.rhs_y, nxs,
                                nys, jlo, jhi, s))
      return false;
    LeafPtrs lp = base.leaf_ptrs();
    lp.rect = rtiles_.rect.p;
    lp.tile_off = rtiles_.tile_off.p;
    lp.table = rtiles_.table.p;
    const TileStore st{d_slot_.p, sl, ntx, nty, g_.ncx, g_.ncy, per, d_ref_.p};
    if (rtiles_.total > 0) {
      const int grid = int(std::max<long long>(1, std::min<long long>(rtiles_.total, 148LL * 8)));
      if (generic_)
        shoot_f32_tiles<true><<<grid, kShootThreads, 0, s>>>(sps, lp, rtiles_.total, st);
      else
        shoot_f32_tiles<false><<<grid, kShootThreads, 0, s>>>(sps, lp, rtiles_.total, st);
      IRSB_LAUNCH_CK("shoot_f32_tiles");
    }
    const long long total = per * n;
    const int grid = int(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32)));
    ada_fixup_corners<<<grid, 256, 0, s>>>(g_, base.d_verts_.p, d_level_.p, d_tl, n, sl, per, d_ref_.p);
    IRSB_LAUNCH_CK("ada_fixup_corners");
    return true;
  }

  bool deposit() {
    cudaStream_t s = base.stream_;
    const Params<T>& p = base.prm;
    const int nt = num_tiles();
    const int npx = p.num_pixels_y.re, npy = p.num_pixels_y.im;
    const long long npix = (long long)npx * npy, ndiff = (long long)npy * (npx + 1);
    const float factor = ipm_triangle_factor<T, float>(p);
    if (!d_acc_.alloc_exact(npix) || !d_diff_.alloc_exact(ndiff) || !d_map_.alloc_exact(npix) ||
        !d_level_.alloc_exact(nt))
      return false;
    IRSB_CKR(cudaMemcpyAsync(d_level_.p, level.data(), nt * sizeof(int), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemsetAsync(d_acc_.p, 0, npix * sizeof(unsigned long long), s));
    IRSB_CKR(cudaMemsetAsync(d_diff_.p, 0, ndiff * sizeof(unsigned long long), s));
    // pieces and tile lists of every launch, built first and uploaded once
    struct Launch {
      int s, nlist;
      long long list_off, piece_off, npieces, nchunks;
    };
    std::vector<Launch> launches;
    std::vector<DepositPiece<float>> pieces;
    std::vector<int> lists;
    cells_evaluated = 0;
    const long long cap = buffer_cap();
    long long max_ref = 0;
    for (int c = 0; c < kAdaLevels; c++) {
      const int sl = ada_level_of(c);
      std::vector<int> tl;
      for (int t = 0; t < nt; t++)
        if (level[t] == sl) tl.push_back(t);
      if (tl.empty()) continue;
      const long long per = (long long)(kAdaTile * sl + 1) * (kAdaTile * sl + 1);
      const int chunk = sl == 1 ? int(tl.size()) : int(std::max<long long>(1, cap / per));
      for (size_t k0 = 0; k0 < tl.size(); k0 += chunk) {
        const int n = int(std::min<size_t>(chunk, tl.size() - k0));
        Launch L{sl, n, (long long)lists.size(), (long long)pieces.size(), n, 0};
        for (int k = 0; k < n; k++) {
          const int t = tl[k0 + k];
          lists.push_back(t);
          const int cx = tile_cells_x(t), cy = tile_cells_y(t);
          DepositPiece<float> pc;
          if (sl == 1) {
            pc.voff = (long long)(t / ntx) * kAdaTile * (g_.ncx + 1) + (long long)(t % ntx) * kAdaTile;
            pc.vstride = g_.ncx + 1;
          } else {
            pc.voff = (long long)k * per;
            pc.vstride = (long long)cx * sl + 1;
          }
          pc.vstep = 1;
          pc.ox = pc.oy = 0.0;
        pc.inv_scale = 1.0;
          pc.ncx = (long long)cx * sl;
          pc.ncy = (long long)cy * sl;
          pc.chunk0 = L.nchunks;
          pc.factor = factor / float(sl * sl);
          pc.r = 0;
          pieces.push_back(pc);
          L.nchunks += (pc.ncx * pc.ncy + 31) / 32;
          cells_evaluated += pc.ncx * pc.ncy;
        }
        if (sl > 1) max_ref = std::max(max_ref, per * n);
        launches.push_back(L);
      }
    }
    if (!d_pieces_.alloc_exact(std::max<size_t>(pieces.size(), 1)) || !d_list_.alloc_exact(std::max<size_t>(lists.size(), 1)))
      return false;
    if (max_ref > 0 && !d_ref_.alloc_exact(max_ref)) return false;
    IRSB_CKR(cudaMemcpyAsync(d_pieces_.p, pieces.data(), pieces.size() * sizeof(DepositPiece<float>),
                             cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(d_list_.p, lists.data(), lists.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    const DepositMaps M{d_acc_.p, d_diff_.p};
    for (const Launch& L : launches) {
      const double2* verts = base.d_verts_.p;
      if (L.s > 1 && L.nlist >= tiled_min) {
        if (!refine_tiled(L.s, lists.data() + L.list_off, d_list_.p + L.list_off, L.nlist)) return false;
        verts = d_ref_.p;
      } else if (L.s > 1) {
        const long long per = (long long)(kAdaTile * L.s + 1) * (kAdaTile * L.s + 1);
        const int grid = int(std::max<long long>(1, std::min<long long>(ada_band_items(L.nlist, L.s), 148LL * 8)));
        if (generic_)
          ada_refine_tiles<T, true><<<grid, 256, 0, s>>>(g_, sp_, base.leaf_ptrs(), descent(), base.d_verts_.p,
                                                         d_level_.p, d_list_.p + L.list_off, L.nlist, L.s, per,
                                                         d_ref_.p);
        else
          ada_refine_tiles<T, false><<<grid, 256, 0, s>>>(g_, sp_, base.leaf_ptrs(), descent(), base.d_verts_.p,
                                                          d_level_.p, d_list_.p + L.list_off, L.nlist, L.s, per,
                                                          d_ref_.p);
        IRSB_LAUNCH_CK("ada_refine_tiles");
        verts = d_ref_.p;
      }
      const int grid = deposit_grid(L.nchunks);
      ipm_deposit_batch<float><<<grid, kDepositThreads, 0, s>>>(verts, d_pieces_.p + L.piece_off, int(L.npieces), L.nchunks, npx,
                                                    npy, M, 0, 0);
      IRSB_LAUNCH_CK("ada deposit");
    }
    const int gr = std::max(1, std::min(ceil_div((long long)npy * 32, 256), 148 * 8));
    ipm_resolve_rows<<<gr, 256, 0, s>>>(npx, npy, M);
    const int g2 = int(std::max<long long>(1, std::min<long long>((npix + 255) / 256, 148LL * 16)));
    ipm_finalize<T><<<g2, 256, 0, s>>>(npix, d_acc_.p, nullptr, nullptr, d_map_.p, nullptr, nullptr, 0);
    IRSB_LAUNCH_CK("ada maps");
    return true;
  }
};

// Training and evaluation of the level network on the device.
class MlpTrainer {
 public:
  // Standardises the features, initialises the weights (He normal, seeded),
  // then runs `epochs` passes of seeded-shuffled minibatches of Adam.
  // epoch_loss[e] receives the mean cross-entropy seen during epoch e.
  static bool train(const float* feat, const int* lab, int n, int epochs, int batch, float lr, unsigned seed,
                    float* w_out, float* mu_out, float* sig_out, float* epoch_loss) {
    if (n <= 0 || batch <= 0 || epochs <= 0) return false;
    for (int i = 0; i < kMlpIn; i++) {
      double m = 0, q = 0;
      for (int k = 0; k < n; k++) m += feat[(long long)k * kMlpIn + i];
      m /= n;
      for (int k = 0; k < n; k++) {
        const double d = feat[(long long)k * kMlpIn + i] - m;
        q += d * d;
      }
      mu_out[i] = float(m);
      sig_out[i] = float(std::max(std::sqrt(q / n), 1e-3));
    }
    std::mt19937_64 rng(seed);
    std::vector<float> w(kMlpParams, 0.f);
    auto init = [&](int off, int fan_out, int fan_in) {
      std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / fan_in));
      for (int k = 0; k < fan_out * fan_in; k++) w[off + k] = float(nd(rng));
    };
    init(kOffW1, kMlpH, kMlpIn);
    init(kOffW2, kMlpH, kMlpH);
    init(kOffW3, kMlpOut, kMlpH);
    Buffers b;
    if (!b.alloc(n, batch)) return false;
    cudaStream_t s = b.s;
    IRSB_CKR(cudaMemcpyAsync(b.feat.p, feat, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.lab.p, lab, n * sizeof(int), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.w.p, w.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.mu.p, mu_out, kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.sig.p, sig_out, kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemsetAsync(b.m.p, 0, kMlpParams * sizeof(float), s));
    IRSB_CKR(cudaMemsetAsync(b.v.p, 0, kMlpParams * sizeof(float), s));
    mlp_to_bf16<<<ceil_div(kMlpParams, 256), 256, 0, s>>>(b.w.p, b.wb.p);
    std::vector<int> perm(n);
    std::vector<float> loss(n);
    int step = 0;
    for (int e = 0; e < epochs; e++) {
      for (int k = 0; k < n; k++) perm[k] = k;
      std::shuffle(perm.begin(), perm.end(), rng);
      IRSB_CKR(cudaMemcpyAsync(b.perm.p, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
      for (int b0 = 0; b0 < n; b0 += batch) {
        const int B = std::min(batch, n - b0);
        if (!b.step(B, b.perm.p + b0, b.loss.p + b0)) return false;
        mlp_adam<<<ceil_div(kMlpParams, 256), 256, 0, s>>>(++step, lr, b.w.p, b.m.p, b.v.p, b.grad.p, b.wb.p);
      }
      IRSB_LAUNCH_CK("mlp training");
      IRSB_CKR(cudaMemcpyAsync(loss.data(), b.loss.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
      IRSB_CKR(cudaStreamSynchronize(s));
      double acc = 0;
      for (float v : loss) acc += v;
      if (epoch_loss) epoch_loss[e] = float(acc / n);
    }
    IRSB_CKR(cudaMemcpyAsync(w_out, b.w.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    return true;
  }

  // Gradient of the mean cross-entropy over all n samples (one minibatch) at
  // weights w (used as BF16), and that mean loss.
  static bool gradients(const float* w, const float* mu, const float* sig, const float* feat, const int* lab, int n,
                        float* grad, float* mean_loss) {
    Buffers b;
    if (!b.alloc(n, n)) return false;
    cudaStream_t s = b.s;
    std::vector<int> idx(n);
    for (int k = 0; k < n; k++) idx[k] = k;
    IRSB_CKR(cudaMemcpyAsync(b.feat.p, feat, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.lab.p, lab, n * sizeof(int), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.perm.p, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.w.p, w, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.mu.p, mu, kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.sig.p, sig, kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    mlp_to_bf16<<<ceil_div(kMlpParams, 256), 256, 0, s>>>(b.w.p, b.wb.p);
    if (!b.step(n, b.perm.p, b.loss.p)) return false;
    std::vector<float> loss(n);
    IRSB_CKR(cudaMemcpyAsync(grad, b.grad.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaMemcpyAsync(loss.data(), b.loss.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    double acc = 0;
    for (float v : loss) acc += v;
    if (mean_loss) *mean_loss = float(acc / n);
    return true;
  }

  static bool predict(const float* w, const float* mu, const float* sig, const float* feat, int n, int* cls) {
    Buffers b;
    if (!b.alloc(n, 1)) return false;
    cudaStream_t s = b.s;
    IRSB_CKR(cudaMemcpyAsync(b.feat.p, feat, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.w.p, w, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.mu.p, mu, kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    IRSB_CKR(cudaMemcpyAsync(b.sig.p, sig, kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s));
    mlp_to_bf16<<<ceil_div(kMlpParams, 256), 256, 0, s>>>(b.w.p, b.wb.p);
    mlp_classify<<<std::max(1, std::min(ceil_div(n, 128), 148 * 4)), 128, 0, s>>>(b.wb.p, b.mu.p, b.sig.p, b.feat.p,
                                                                                  n, 0.f, b.lab.p);
    IRSB_LAUNCH_CK("mlp_classify");
    IRSB_CKR(cudaMemcpyAsync(cls, b.lab.p, n * sizeof(int), cudaMemcpyDeviceToHost, s));
    IRSB_CKR(cudaStreamSynchronize(s));
    return true;
  }

 private:
  struct Buffers {
    cudaStream_t s = nullptr;
    DevVec<float> feat, X, H1, H2, D1, D2, D3, loss, w, m, v, grad, mu, sig;
    DevVec<int> lab, perm;
    DevVec<__nv_bfloat16> wb;
    ~Buffers() {
      if (s) cudaStreamDestroy(s);
    }
    bool alloc(int n, int B) {
      if (!IRSB_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))) return false;
      return feat.alloc_exact((size_t)n * kMlpIn) && lab.alloc_exact(n) && perm.alloc_exact(n) &&
             loss.alloc_exact(n) && X.alloc_exact((size_t)B * kMlpIn) && H1.alloc_exact((size_t)B * kMlpH) &&
             H2.alloc_exact((size_t)B * kMlpH) && D1.alloc_exact((size_t)B * kMlpH) &&
             D2.alloc_exact((size_t)B * kMlpH) && D3.alloc_exact((size_t)B * kMlpOut) && w.alloc_exact(kMlpParams) &&
             m.alloc_exact(kMlpParams) && v.alloc_exact(kMlpParams) && grad.alloc_exact(kMlpParams) &&
             mu.alloc_exact(kMlpIn) && sig.alloc_exact(kMlpIn) && wb.alloc_exact(kMlpParams);
    }
    // forward, backward and gradient of one minibatch idx[0..B)
    bool step(int B, const int* idx, float* loss_out) {
      const int g = std::max(1, ceil_div(B, 128));
      mlp_train_forward<<<g, 128, 0, s>>>(wb.p, mu.p, sig.p, feat.p, lab.p, idx, B, X.p, H1.p, H2.p, D3.p, loss_out);
      mlp_train_backward<<<g, 128, 0, s>>>(wb.p, B, H1.p, H2.p, D3.p, D2.p, D1.p);
      mlp_grad<<<ceil_div(kMlpParams, 128), 128, 0, s>>>(B, X.p, H1.p, H2.p, D1.p, D2.p, D3.p, grad.p);
      return IRSB_CK(cudaGetLastError());
    }
  };
};

}  // namespace irsb
