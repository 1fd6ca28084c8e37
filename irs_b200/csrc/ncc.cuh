// Number of caustic crossings (NCC): for every source-plane pixel, how many
// caustic curves a ray from the pixel centre to +infinity along y1 crosses
// (entering minus leaving), i.e. the number of extra image pairs.
//
// Semantics of the reference (include/ncc_functions.cuh, include/ncc.cuh):
// the caustics of a CCF run are rows of points (curves traced clockwise);
// each segment between consecutive points of a row is clipped to the region
// y1 > -hl1, |y2| < hl2 (corrected_point, :100-142, points moved 1/100 pixel
// inside); in pixel units every pixel-centre line y = k + 1/2 that the segment
// crosses adds -1 (segment going up) or +1 (going down) to all pixels of that
// row left of the crossing, column int(x + 1/2) - 1 and below
// (find_num_caustic_crossings_kernel, :149-337); the map is computed at
// 2^over_sample times the resolution and reduced by the maximum over
// 2^over_sample x 2^over_sample blocks (reduce_pix_array_kernel, :349-367).
//
// How, differently by design:
//   * a crossing adds its +-1 to a per-row difference array (two integer
//     atomics: the row's first column and one past the crossing) instead of
//     one atomic per pixel left of it; one warp per row then turns the
//     differences into counts by a prefix sum. Integer sums: the map does not
//     depend on the order of the crossings;
//   * the intersection of a segment with y = const is x0 + ((y - y0) / dy) dx
//     in explicitly rounded FP64 (the reference evaluates the same quantity
//     through logarithms and exponentials, :62-98), so a host
//     restatement with the same operations gives the same map bit for bit;
//   * the block maximum is one pass over the fine map.
#pragma once
#include "common.cuh"

namespace irsb {

struct NccGeom {
  double cy_re, cy_im;    // centre of the source region
  double hl_re, hl_im;    // half lengths
  int npx, npy;           // pixels of the fine map (2^over_sample times the output)
};

__device__ __forceinline__ double ncc_sgn(double v) { return v < 0 ? -1.0 : (v > 0 ? 1.0 : 0.0); }

// x where the line through (x0, y0), (x1, y1) meets y = const (x0 for a
// vertical line); y where it meets x = const (y0 for a horizontal line).
__device__ __forceinline__ double ncc_x_at(double y, double x0, double y0, double x1, double y1) {
  const double dx = __dsub_rn(x1, x0);
  if (dx == 0.0) return x0;
  const double dy = __dsub_rn(y1, y0);
  return __dadd_rn(x0, __dmul_rn(__ddiv_rn(__dsub_rn(y, y0), dy), dx));
}
__device__ __forceinline__ double ncc_y_at(double x, double x0, double y0, double x1, double y1) {
  const double dy = __dsub_rn(y1, y0);
  if (dy == 0.0) return y0;
  const double dx = __dsub_rn(x1, x0);
  return __dadd_rn(y0, __dmul_rn(__ddiv_rn(__dsub_rn(x, x0), dx), dy));
}

__device__ __forceinline__ bool ncc_in_region(double x, double y, const NccGeom& g) {
  return x > -g.hl_re && fabs(y) < g.hl_im;
}

// (x, y) moved along the segment towards (xo, yo) to 1/100 of a fine pixel
// inside the region where it lies beyond an edge (corrected_point).
__device__ __forceinline__ void ncc_correct(double& x, double& y, double xo, double yo, const NccGeom& g) {
  const double x0 = x, y0 = y;
  if (x <= -g.hl_re) {
    x = __dadd_rn(-g.hl_re, __ddiv_rn(__dmul_rn(0.01 * 2, g.hl_re), double(g.npx)));
    y = ncc_y_at(x, x0, y0, xo, yo);
  }
  if (fabs(y) >= g.hl_im) {
    y = __dmul_rn(ncc_sgn(y), __dsub_rn(g.hl_im, __ddiv_rn(__dmul_rn(0.01 * 2, g.hl_im), double(g.npy))));
    x = ncc_x_at(y, x0, y0, xo, yo);
  }
}

// One thread per segment (row i, points j and j + 1) of the caustics.
// diff: [npy][npx + 1] row differences of the fine map; err counts crossings
// that would land outside the map (the reference prints an error for them).
__global__ void ncc_segments(const double2* __restrict__ caus, int nrows, int ncols, NccGeom g, int* __restrict__ diff,
                             int* __restrict__ err) {
  const long long nseg = (long long)nrows * (ncols - 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nseg; q += (long long)gridDim.x * blockDim.x) {
    const long long i = q / (ncols - 1), j = q - i * (ncols - 1);
    const double2 a = caus[i * ncols + j], b = caus[i * ncols + j + 1];
    double x0 = __dsub_rn(a.x, g.cy_re), y0 = __dsub_rn(a.y, g.cy_im);
    double x1 = __dsub_rn(b.x, g.cy_re), y1 = __dsub_rn(b.y, g.cy_im);
    bool use = ncc_in_region(x0, y0, g) || ncc_in_region(x1, y1, g);
    if (!use)  // a long segment whose line crosses into the region
      use = ncc_x_at(g.hl_im, x0, y0, x1, y1) >= -g.hl_re || ncc_x_at(-g.hl_im, x0, y0, x1, y1) >= -g.hl_re ||
            fabs(ncc_y_at(-g.hl_re, x0, y0, x1, y1)) <= g.hl_im;
    if (!use) continue;
    ncc_correct(x0, y0, x1, y1, g);
    ncc_correct(x1, y1, x0, y0, g);
    // pixel coordinates (point_to_pixel, array_functions.cuh:70-75)
    const double s_re = 2 * g.hl_re, s_im = 2 * g.hl_im;
    const double px0 = __ddiv_rn(__dmul_rn(__dadd_rn(x0, g.hl_re), double(g.npx)), s_re);
    const double py0 = __ddiv_rn(__dmul_rn(__dadd_rn(y0, g.hl_im), double(g.npy)), s_im);
    const double px1 = __ddiv_rn(__dmul_rn(__dadd_rn(x1, g.hl_re), double(g.npx)), s_re);
    const double py1 = __ddiv_rn(__dmul_rn(__dadd_rn(y1, g.hl_im), double(g.npy)), s_im);
    const int k0 = int(__dadd_rn(py0, 0.5)), k1 = int(__dadd_rn(py1, 0.5));
    const bool up = py0 < py1;
    if (py0 == py1) continue;
    // going up: rows k0 .. k1 - 1 at y = k + 1/2, -1; going down: rows
    // k0 - 1 .. k1 at y = k - 1/2, +1
    const int v = up ? -1 : 1;
    for (int k = k0; up ? k < k1 : k > k1; k += up ? 1 : -1) {
      const double yc = up ? __dadd_rn(double(k), 0.5) : __dsub_rn(double(k), 0.5);
      const double xc = ncc_x_at(yc, px0, py0, px1, py1);
      int col = int(__dadd_rn(xc, 0.5)) - 1;
      const int rk = up ? k : k - 1;
      const int row = g.npy - 1 - rk;
      if (col > g.npx - 1) col = g.npx - 1;
      if (col < 0) continue;
      if (row < 0 || row >= g.npy) {
        atomicAdd(err, 1);
        continue;
      }
      int* d = diff + (long long)row * (g.npx + 1);
      atomicAdd(d, v);
      atomicAdd(d + col + 1, -v);
    }
  }
}

// Fine map from the row differences: one warp per row, 32 columns per step
// with a carried running sum.
__global__ void ncc_rows(const int* __restrict__ diff, int npx, int npy, int* __restrict__ fine) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < npy; r += warps) {
    const int* d = diff + (long long)r * (npx + 1);
    int* out = fine + (long long)r * npx;
    int carry = 0;
    for (int c0 = 0; c0 < npx; c0 += 32) {
      const int c = c0 + lane;
      int v = c < npx ? d[c] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
      }
      if (c < npx) out[c] = carry + v;
      carry += __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// Output pixel = maximum over its B x B block of the fine map (B = 2^over_sample).
__global__ void ncc_pool(const int* __restrict__ fine, int npx, int npy, int B, int* __restrict__ out) {
  const long long n = (long long)npx * npy;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int r = int(q / npx), c = int(q - (long long)r * npx);
    int m = fine[(long long)r * B * npx * B + (long long)c * B];
    for (int dy = 0; dy < B; dy++)
      for (int dx = 0; dx < B; dx++) m = max(m, fine[((long long)r * B + dy) * npx * B + (long long)c * B + dx]);
    out[q] = m;
  }
}

}  // namespace irsb
