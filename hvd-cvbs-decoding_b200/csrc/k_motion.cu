// k_motion.cu -- block-matching motion estimation (kernel d) and the
// per-pixel vector field / warps / confidence upsampling that turn it into
// neighbour terms.
//
// Reference: EstimateMotion (hvd-core/src/engine/motion.cpp:397-488) with
// BoxBlur (:21-55, 391-395), Decimate (:59-78), BmPass (:105-260),
// RangeFromCentre (:286-298), CostAt (:309-315), MotionConfidence (:321-387);
// VectorsPerPixel / WarpByTiles / UpsampleConfidence[Fast]
// (engine/temporal.cpp:45-254).
//
// Bit-exact to the reference's float arithmetic: this file is compiled with
// FMA contraction off (--fmad=false), every float / double operation is
// issued in the reference's order, and each (pair, tile) visits the
// candidates in the reference's centre-out order with the same
// partial-distortion bail-out and strict-less update (one thread per tile,
// or for the refinement a warp per tile that replays the visit from
// per-row running sums), so the selected vectors, sub-pel fits and
// confidences equal the reference's bit for bit.
#include <cuda_runtime.h>

#include "hvdg_common.cuh"
#include "k_motion.h"
#include "per_device.h"

namespace hvdg {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// One line of BoxBlur (motion.cpp:21-55): prefix sums c_k = c_(k-1) +
// s_(k-1) in double, in order, and out_i = (c_min(i+r+1, n) - c_max(i-r, 0))
// * norm; samples `ss` apart in the source, outputs `ds` apart. Output i is
// written as soon as the prefix its window ends at exists (the ones cut by
// the line's end last). The last 32 prefix sums of each thread live in a
// shared-memory history (slot k & 31, one column per thread of a block of
// at most kBoxThreads), so no step divides or touches local memory; the
// samples are fetched kBoxChunk at a time ahead of their additions. The
// values are those of the sample-by-sample loop. Needs 2 r + 1 <= 31.
constexpr int kBoxChunk = 16;
constexpr int kBoxThreads = 128;

__device__ __forceinline__ void box_line(const float* __restrict__ s, int64_t ss,
                                         float* __restrict__ d, int64_t ds, int n, int r,
                                         double norm) {
  __shared__ double hist[32 * kBoxThreads];
  double* h = hist + threadIdx.x;
  double c = 0.0;
  for (int k0 = 1; k0 <= n; k0 += kBoxChunk) {
    float v[kBoxChunk];
#pragma unroll
    for (int j = 0; j < kBoxChunk; ++j) v[j] = k0 + j <= n ? s[(int64_t)(k0 - 1 + j) * ss] : 0.0f;
#pragma unroll
    for (int j = 0; j < kBoxChunk; ++j) {
      const int k = k0 + j;
      if (k <= n) {
        c = c + (double)v[j];
        h[(k & 31) * kBoxThreads] = c;
        const int i = k - r - 1;
        if (i >= 0) {
          const int i0 = i - r;
          const double c0v = i0 > 0 ? h[(i0 & 31) * kBoxThreads] : 0.0;
          d[(int64_t)i * ds] = (float)((c - c0v) * norm);
        }
      }
    }
  }
  for (int i = n - r > 0 ? n - r : 0; i < n; ++i) {
    const int i0 = i - r;
    d[(int64_t)i * ds] = (float)((c - (i0 > 0 ? h[(i0 & 31) * kBoxThreads] : 0.0)) * norm);
  }
}

// Shared memory of the row blur (declared once per kernel): the band's
// 32 x 32 sample / output tile and each lane's 64-slot prefix history.
struct RowBlurSmem {
  float tile[32][33];
  double hist[32][65];
};

// box_line along rows for one warp: lane l runs row l of a 32-row band
// (`rows` of them exist). The band's samples arrive 32 columns at a time
// through shared memory, each load instruction reading one row's 32
// consecutive columns. Per chunk, each lane first runs its row's prefix sums
// (the only serial chain: one double add per column, in column order, the
// loads and conversions ahead of it) into a 64-slot shared-memory history,
// then forms the chunk's window sums from that history with no chain at all
// (prefix k minus prefix k - 2 r - 1, the same doubles as a running ring),
// and the outputs leave through a shared tile as coalesced row segments.
// Needs 2 r + 1 <= 32.
__device__ __forceinline__ void box_rows_warp_any(RowBlurSmem& sm, const float* __restrict__ s,
                                                  float* __restrict__ d, int64_t pitch, int rows,
                                                  int n, int r, double norm) {
  float (&tile)[32][33] = sm.tile;
  double (&pre)[32][65] = sm.hist;  // prefix k of lane l at pre[l][k & 63]
  const int lane = threadIdx.x & 31;
  double* hist = pre[lane];
  double c = 0.0;
  hist[0] = 0.0;
  for (int c0 = 0; c0 < n; c0 += 32) {
    {
      // all 32 loads issued before the first store
      float v[32];
      const bool col = c0 + lane < n;
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] = col && q < rows ? s[(int64_t)q * pitch + c0 + lane] : 0.0f;
#pragma unroll
      for (int q = 0; q < 32; ++q) tile[q][lane] = v[q];
    }
    __syncwarp();
    const int m = min(32, n - c0);  // columns of this chunk
    {
      double v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = (double)tile[lane][j];
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < m) {
          c = c + v[j];
          hist[(c0 + j + 1) & 63] = c;
        }
    }
    __syncwarp();
    // window sums ending at prefix k = c0 + j + 1: output column i = k - r - 1
    // (window [max(i - r, 0), i + r]), staged in the tile at column j
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int k = c0 + j + 1, i = k - r - 1;
      float o = 0.0f;
      if (j < m && i >= 0) {
        const double c0v = i - r > 0 ? hist[(i - r) & 63] : 0.0;
        o = (float)((hist[k & 63] - c0v) * norm);
      }
      tile[lane][j] = o;
    }
    __syncwarp();
    // row q's outputs of this chunk: columns c0 - r .. c0 + m - 1 - r
#pragma unroll 4
    for (int q = 0; q < rows; ++q) {
      const int i = c0 - r + lane;
      if (lane < m && i >= 0) d[(int64_t)q * pitch + i] = tile[q][lane];
    }
    __syncwarp();
  }
  if (lane >= rows) return;
  // outputs whose window is cut by the end: prefix n is c
  float* drow = d + (int64_t)lane * pitch;
  for (int i = n - r > 0 ? n - r : 0; i < n; ++i) {
    const int i0 = i - r > 0 ? i - r : 0;
    drow[i] = (float)((c - (i0 > 0 ? hist[i0 & 63] : 0.0)) * norm);
  }
}

// The same blur for a radius known at compile time (the window's 2, 6 and
// 8): a chunk's prefix sums and the previous chunk's stay in registers (every
// index is a constant), so a column costs its one chained addition, a copy
// of the sum into a shared history (read only by the windows cut by the
// row's end) and its window sum.
template <int R>
__device__ __forceinline__ void box_rows_warp_r(RowBlurSmem& sm, const float* __restrict__ s,
                                                float* __restrict__ d, int64_t pitch, int rows,
                                                int n, double norm) {
  constexpr int kW = 2 * R + 1;  // window: prefix k minus prefix k - kW
  static_assert(kW <= 32, "window within two chunks");
  float (&tile)[32][33] = sm.tile;
  double (&hist)[32][65] = sm.hist;
  const int lane = threadIdx.x & 31;
  double* hrow = hist[lane];  // prefix k at slot k & 63, for the cut windows
  double c = 0.0, prev[32], cur[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) prev[j] = 0.0;
  for (int c0 = 0; c0 < n; c0 += 32) {
    {
      float v[32];
      const bool col = c0 + lane < n;
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] = col && q < rows ? s[(int64_t)q * pitch + c0 + lane] : 0.0f;
#pragma unroll
      for (int q = 0; q < 32; ++q) tile[q][lane] = v[q];
    }
    __syncwarp();
    const int m = min(32, n - c0);
    // the chain: cur[j] = prefix c0 + j + 1, in column order
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float x = tile[lane][j];
      if (j < m) {
        c = c + (double)x;
        hrow[(c0 + j + 1) & 63] = c;
      }
      cur[j] = c;
    }
    __syncwarp();
    // window sums ending at prefix k = c0 + j + 1 (output column k - R - 1),
    // starting at prefix k - kW (0 below 1)
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int k = c0 + j + 1, i = k - R - 1;
      const double c0v = k - kW > 0 ? (j - kW >= 0 ? cur[j - kW] : prev[j - kW + 32]) : 0.0;
      tile[lane][j] = (j < m && i >= 0) ? (float)((cur[j] - c0v) * norm) : 0.0f;
    }
    __syncwarp();
#pragma unroll 4
    for (int q = 0; q < rows; ++q) {
      const int i = c0 - R + lane;
      if (lane < m && i >= 0) d[(int64_t)q * pitch + i] = tile[q][lane];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; ++j) prev[j] = cur[j];
  }
  if (lane >= rows) return;
  // the windows cut by the row's end start within the last 2 R prefixes
  float* drow = d + (int64_t)lane * pitch;
  for (int i = n - R > 0 ? n - R : 0; i < n; ++i) {
    const int i0 = i - R;
    drow[i] = (float)((c - (i0 > 0 ? hrow[i0 & 63] : 0.0)) * norm);
  }
}

__device__ __forceinline__ void box_rows_warp(const float* __restrict__ s, float* __restrict__ d,
                                              int64_t pitch, int rows, int n, int r,
                                              double norm) {
  __shared__ RowBlurSmem sm;
  if (r == 2) return box_rows_warp_r<2>(sm, s, d, pitch, rows, n, norm);
  if (r == 6) return box_rows_warp_r<6>(sm, s, d, pitch, rows, n, norm);
  if (r == 8) return box_rows_warp_r<8>(sm, s, d, pitch, rows, n, norm);
  box_rows_warp_any(sm, s, d, pitch, rows, n, r, norm);
}

// ---- BoxBlur (motion.cpp:21-55): double prefix sums, constant 1/(2r+1) ----
// Vertical pass: one thread per (field, column).
__global__ void k_blur_v(const MeField* __restrict__ mf, int nf, const float* __restrict__ src,
                         float* __restrict__ dst, int r, int src_sel) {
  const int f = blockIdx.y;
  if (f >= nf) return;
  const MeField m = mf[f];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= m.w) return;
  const int64_t sb = src_sel == 0 ? m.y_off : m.b_off;
  const float* s = src + sb;
  float* d = dst + m.t_off;
  const double norm = (double)(1.0f / (float)(2 * r + 1));
  box_line(s + x, m.pitch, d + x, m.pitch, m.h, r, norm);
}

// Horizontal pass: one warp per (field, 32-row band).
__global__ void k_blur_h(const MeField* __restrict__ mf, int nf, const float* __restrict__ src,
                         float* __restrict__ dst, int r) {
  const int f = blockIdx.y;
  if (f >= nf) return;
  const MeField m = mf[f];
  const int y0 = blockIdx.x * 32;
  if (y0 >= m.h) return;
  const double norm = (double)(1.0f / (float)(2 * r + 1));
  box_rows_warp(src + m.t_off + (int64_t)y0 * m.pitch, dst + m.b_off + (int64_t)y0 * m.pitch,
                m.pitch, min(32, m.h - y0), m.w, r, norm);
}

// ---- Decimate (motion.cpp:59-78): 4 x 4 block mean ---------------------------
__global__ void k_decimate(const MeField* __restrict__ mf, int nf, const float* __restrict__ blur,
                           float* __restrict__ dec) {
  const int f = blockIdx.y;
  if (f >= nf) return;
  const MeField m = mf[f];
  const int hd = m.h / 4, wd = m.w / 4;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hd * wd) return;
  const int y = i / wd, x = i % wd;
  const float* b = blur + m.b_off;
  float acc = 0.0f;
  for (int dy = 0; dy < 4; ++dy)
    for (int dx = 0; dx < 4; ++dx) acc += b[(int64_t)(y * 4 + dy) * m.pitch + x * 4 + dx];
  dec[m.d_off + (int64_t)y * m.dpitch + x] = acc * (1.0f / 16.0f);
}

// Sum of squared differences over one tile, rows in order, with the
// reference's per-row partial-distortion bail-out (acc >= kill).
__device__ __forceinline__ float tile_ssd(const float* A, const float* B, int pitch, int h, int w,
                                          int ty0, int ty1, int tx0, int tx1, int sy, int sx,
                                          float kill) {
  float acc = 0.0f;
  for (int y = ty0; y < ty1; ++y) {
    const float* arow = A + (int64_t)y * pitch;
    const float* brow = B + (int64_t)clampi(y - sy, 0, h - 1) * pitch;
    for (int x = tx0; x < tx1; ++x) {
      const float diff = arow[x] - brow[clampi(x - sx, 0, w - 1)];
      acc += diff * diff;
    }
    if (acc >= kill) break;
  }
  return acc;
}

// centre-out candidate order (RangeFromCentre, motion.cpp:286-298) for a
// symmetric range [-r, r]: 0, -1, 1, -2, 2, ...
__device__ __forceinline__ int centre_out(int i) { return (i & 1) ? -((i + 1) >> 1) : (i >> 1); }

// ---- coarse absolute pass on the 4x-decimated planes (motion.cpp:406-413) --
__global__ void k_me_coarse(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                            int npairs, const float* __restrict__ dec, MeArgs a,
                            float* __restrict__ cdy, float* __restrict__ cdx) {
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int hd = mc.h / 4, wd = mc.w / 4;
  const int ct = a.tile / 4 > 4 ? a.tile / 4 : 4;
  const int th = (hd + ct - 1) / ct, tw = (wd + ct - 1) / ct;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= th * tw) return;
  const int ty = t / tw, tx = t % tw;
  const int cs = (a.search + 3) / 4 > 1 ? (a.search + 3) / 4 : 1;
  const float* A = dec + mc.d_off;
  const float* B = dec + mr.d_off;
  const int y0 = ty * ct, y1 = min((ty + 1) * ct, hd);
  const int x0 = tx * ct, x1 = min((tx + 1) * ct, wd);
  float best = __int_as_float(0x7f800000);
  float bdy = 0.0f, bdx = 0.0f;
  const int n = 2 * cs + 1;
  for (int i = 0; i < n; ++i) {
    const int dy = centre_out(i);
    for (int j = 0; j < n; ++j) {
      const int dx = centre_out(j);
      const float bias = 1.0f + 0.02f * (float)(abs(dy) + abs(dx));
      const float inv_bias = 1.0f / bias;
      const bool exact = dy == 0 && dx == 0;  // cost0 needs the full sum
      const float kill = exact ? __int_as_float(0x7f800000) : best * inv_bias;
      const float se = tile_ssd(A, B, mc.dpitch, hd, wd, y0, y1, x0, x1, dy, dx, kill);
      const float cost = se * bias;
      if (cost < best) {
        best = cost;
        bdy = (float)dy;
        bdx = (float)dx;
      }
    }
  }
  cdy[a.coarse_off * p + t] = bdy;
  cdx[a.coarse_off * p + t] = bdx;
}

// The coarse pass with a warp per (pair, coarse tile) when the candidates
// and tile rows fit (n^2 <= kCoarseWarpCands, ct <= kCoarseWarpRows): lanes
// sum the candidates' SSD row by row in the reference's order, one lane
// replays the visit from the per-row running sums (the zero vector, whose
// cost needs the full sum, is never cut), as in k_me_refine_warp.
constexpr int kCoarseWarpCands = 128;
constexpr int kCoarseWarpRows = 16;

__global__ void k_me_coarse_warp(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                                 int npairs, const float* __restrict__ dec, MeArgs a,
                                 float* __restrict__ cdy, float* __restrict__ cdx) {
  extern __shared__ float mc_part[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpc = blockDim.x >> 5;
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int hd = mc.h / 4, wd = mc.w / 4;
  const int ct = a.tile / 4 > 4 ? a.tile / 4 : 4;
  const int th = (hd + ct - 1) / ct, tw = (wd + ct - 1) / ct;
  const int t = blockIdx.x * wpc + warp;
  if (t >= th * tw) return;  // the whole warp; only warp-level sync below
  const int ty = t / tw, tx = t % tw;
  const int cs = (a.search + 3) / 4 > 1 ? (a.search + 3) / 4 : 1;
  const int n = 2 * cs + 1;
  const int ncand = n * n;
  float* part = mc_part + (size_t)warp * kCoarseWarpCands * kCoarseWarpRows;
  const float* A = dec + mc.d_off;
  const float* B = dec + mr.d_off;
  const int y0 = ty * ct, y1 = min((ty + 1) * ct, hd);
  const int x0 = tx * ct, x1 = min((tx + 1) * ct, wd);
  const int rows = y1 - y0;
  for (int c = lane; c < ncand; c += 32) {
    const int sy = centre_out(c / n), sx = centre_out(c % n);
    float acc = 0.0f;
    for (int y = y0; y < y1; ++y) {
      const float* arow = A + (int64_t)y * mc.dpitch;
      const float* brow = B + (int64_t)clampi(y - sy, 0, hd - 1) * mc.dpitch;
      for (int x = x0; x < x1; ++x) {
        const float diff = arow[x] - brow[clampi(x - sx, 0, wd - 1)];
        acc += diff * diff;
      }
      part[c * kCoarseWarpRows + (y - y0)] = acc;
    }
  }
  __syncwarp();
  if (lane != 0) return;
  float best = __int_as_float(0x7f800000);
  float bdy = 0.0f, bdx = 0.0f;
  for (int c = 0; c < ncand; ++c) {
    const int dy = centre_out(c / n), dx = centre_out(c % n);
    const float bias = 1.0f + 0.02f * (float)(abs(dy) + abs(dx));
    const float inv_bias = 1.0f / bias;
    const bool exact = dy == 0 && dx == 0;
    const float kill = exact ? __int_as_float(0x7f800000) : best * inv_bias;
    const float* pc = part + c * kCoarseWarpRows;
    float se = pc[rows - 1];
    for (int r = 0; r < rows; ++r) {
      if (pc[r] >= kill) {
        se = pc[r];
        break;
      }
    }
    const float cost = se * bias;
    if (cost < best) {
      best = cost;
      bdy = (float)dy;
      bdx = (float)dx;
    }
  }
  cdy[a.coarse_off * p + t] = bdy;
  cdx[a.coarse_off * p + t] = bdx;
}

// ---- full-res refinement, sub-pel fit, zero / margin rule (motion.cpp:415-473)
__global__ void k_me_refine(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                            int npairs, const float* __restrict__ blur, MeArgs a,
                            const float* __restrict__ cdy, const float* __restrict__ cdx,
                            float* __restrict__ out_mdy, float* __restrict__ out_mdx,
                            float* __restrict__ out_sdy, float* __restrict__ out_sdx,
                            float* __restrict__ out_best) {
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int h = mc.h, w = mc.w, tile = a.tile;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= th * tw) return;
  const int ty = t / tw, tx = t % tw;
  const int hd = h / 4, wd = w / 4;
  const int ct = tile / 4 > 4 ? tile / 4 : 4;
  const int hh = (hd + ct - 1) / ct, ww = (wd + ct - 1) / ct;
  const int gy = min((ty * hh) / th, hh - 1), gx = min((tx * ww) / tw, ww - 1);
  const float base_dy = cdy[a.coarse_off * p + gy * ww + gx] * 4.0f;
  const float base_dx = cdx[a.coarse_off * p + gy * ww + gx] * 4.0f;
  const float* A = blur + mc.b_off;
  const float* B = blur + mr.b_off;
  const int y0 = ty * tile, y1 = min((ty + 1) * tile, h);
  const int x0 = tx * tile, x1 = min((tx + 1) * tile, w);
  const float inf = __int_as_float(0x7f800000);
  // refine: relative candidates RangeFromCentre(-3, 3)^2, no cost0
  const int rby = (int)lroundf(base_dy), rbx = (int)lroundf(base_dx);
  float best = inf, mdy = 0.0f, mdx = 0.0f;
  for (int i = 0; i < 7; ++i) {
    const int dy = centre_out(i);
    for (int j = 0; j < 7; ++j) {
      const int dx = centre_out(j);
      const float bias = 1.0f + 0.02f * (float)(abs(dy) + abs(dx));
      const float inv_bias = 1.0f / bias;
      const float kill = best * inv_bias;
      const float se = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1, rby + dy, rbx + dx, kill);
      const float cost = se * bias;
      if (cost < best) {
        best = cost;
        mdy = base_dy + (float)dy;
        mdx = base_dx + (float)dx;
      }
    }
  }
  // CostAt at (+-1, 0), (0, +-1): single relative candidate, full sum, bias 1
  const int iy = (int)lroundf(mdy), ix = (int)lroundf(mdx);
  const float cym = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1,
                             (int)lroundf(mdy + -1.0f), ix, inf) * 1.0f;
  const float cyp = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1,
                             (int)lroundf(mdy + 1.0f), ix, inf) * 1.0f;
  const float cxm = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1, iy,
                             (int)lroundf(mdx + -1.0f), inf) * 1.0f;
  const float cxp = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1, iy,
                             (int)lroundf(mdx + 1.0f), inf) * 1.0f;
  auto parabolic = [](float cm, float c0, float cp) {
    const float den = cm - 2.0f * c0 + cp;
    float sub = 0.0f;
    if (den > 1e-9f) sub = 0.5f * (cm - cp) / fmaxf(den, 1e-9f);
    return fminf(fmaxf(sub, -0.5f), 0.5f);
  };
  float sdy = parabolic(cym, best, cyp);
  float sdx = parabolic(cxm, best, cxp);
  // explicit zero-motion evaluation + "prefer zero" margin rule
  const float cost0 = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1, 0, 0, inf);
  const float best0 = cost0 * 1.0f;
  if (best0 < best) {
    mdy = 0.0f;
    mdx = 0.0f;
    best = best0;
  }
  if (best > 0.85f * cost0) {
    mdy = 0.0f;
    mdx = 0.0f;
    best = cost0;
    sdy = 0.0f;
    sdx = 0.0f;
  }
  const int o = a.tiles_off * p + t;
  out_mdy[o] = mdy;
  out_mdx[o] = mdx;
  out_sdy[o] = sdy;
  out_sdx[o] = sdx;
  out_best[o] = best;
}

// The same refinement with a warp per (pair, tile), for tiles of up to
// kRefineWarpTile rows. Lane l computes the SSD of refine candidates l and
// l + 32 (visit order) row by row in the reference's order, without the
// bail-out, keeping the running sum after every row in shared memory. The
// warp then replays the reference's visit from those sums -- kill = best *
// (1 / bias), the first row whose running sum reaches it (a ballot over the
// rows) ends the candidate with that sum, strict-less update -- so every
// cost, decision and vector is the per-thread kernel's; lanes 0-4 then take
// the four CostAt sums and the zero-motion cost (full sums) at once.
constexpr int kRefineCands = 49;  // RangeFromCentre(-3, 3)^2
constexpr int kRefineWarpTile = 64;

__global__ void k_me_refine_warp(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                                 int npairs, const float* __restrict__ blur, MeArgs a,
                                 const float* __restrict__ cdy, const float* __restrict__ cdx,
                                 float* __restrict__ out_mdy, float* __restrict__ out_mdx,
                                 float* __restrict__ out_sdy, float* __restrict__ out_sdx,
                                 float* __restrict__ out_best) {
  extern __shared__ float me_part[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpc = blockDim.x >> 5;
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int h = mc.h, w = mc.w, tile = a.tile;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const int t = blockIdx.x * wpc + warp;
  if (t >= th * tw) return;  // the whole warp; only warp-level sync below
  float* part = me_part + (size_t)warp * kRefineCands * tile;
  const int ty = t / tw, tx = t % tw;
  const int hd = h / 4, wd = w / 4;
  const int ct = tile / 4 > 4 ? tile / 4 : 4;
  const int hh = (hd + ct - 1) / ct, ww = (wd + ct - 1) / ct;
  const int gy = min((ty * hh) / th, hh - 1), gx = min((tx * ww) / tw, ww - 1);
  const float base_dy = cdy[a.coarse_off * p + gy * ww + gx] * 4.0f;
  const float base_dx = cdx[a.coarse_off * p + gy * ww + gx] * 4.0f;
  const float* A = blur + mc.b_off;
  const float* B = blur + mr.b_off;
  const int y0 = ty * tile, y1 = min((ty + 1) * tile, h);
  const int x0 = tx * tile, x1 = min((tx + 1) * tile, w);
  const int rows = y1 - y0;
  const float inf = __int_as_float(0x7f800000);
  const int rby = (int)lroundf(base_dy), rbx = (int)lroundf(base_dx);
  for (int c = lane; c < kRefineCands; c += 32) {
    const int sy = rby + centre_out(c / 7), sx = rbx + centre_out(c % 7);
    float acc = 0.0f;
    for (int y = y0; y < y1; ++y) {
      const float* arow = A + (int64_t)y * mc.pitch;
      const float* brow = B + (int64_t)clampi(y - sy, 0, h - 1) * mc.pitch;
      for (int x = x0; x < x1; ++x) {
        const float diff = arow[x] - brow[clampi(x - sx, 0, w - 1)];
        acc += diff * diff;
      }
      part[c * tile + (y - y0)] = acc;
    }
  }
  __syncwarp();
  // the reference's visit, the whole warp in step: for each candidate the
  // first row whose running sum reaches kill is found by a ballot over the
  // rows (lane r holds row r, r + 32), so every lane makes the same decisions
  float best = inf, mdy = 0.0f, mdx = 0.0f;
  for (int c = 0; c < kRefineCands; ++c) {
    const int dy = centre_out(c / 7), dx = centre_out(c % 7);
    const float bias = 1.0f + 0.02f * (float)(abs(dy) + abs(dx));
    const float inv_bias = 1.0f / bias;
    const float kill = best * inv_bias;
    const float* pc = part + c * tile;
    float se = pc[rows - 1];
    for (int r0 = 0; r0 < rows; r0 += 32) {
      const bool hit = r0 + lane < rows && pc[r0 + lane] >= kill;
      const unsigned b = __ballot_sync(0xffffffffu, hit);
      if (b) {
        se = pc[r0 + __ffs(b) - 1];
        break;
      }
    }
    const float cost = se * bias;
    if (cost < best) {
      best = cost;
      mdy = base_dy + (float)dy;
      mdx = base_dx + (float)dx;
    }
  }
  // CostAt at (+-1, 0), (0, +-1) and the zero-motion cost: full sums
  const int iy = (int)lroundf(mdy), ix = (int)lroundf(mdx);
  float v = 0.0f;
  if (lane < 5) {
    int sy = iy, sx = ix;
    if (lane == 0) sy = (int)lroundf(mdy + -1.0f);
    if (lane == 1) sy = (int)lroundf(mdy + 1.0f);
    if (lane == 2) sx = (int)lroundf(mdx + -1.0f);
    if (lane == 3) sx = (int)lroundf(mdx + 1.0f);
    if (lane == 4) sy = sx = 0;
    v = tile_ssd(A, B, mc.pitch, h, w, y0, y1, x0, x1, sy, sx, inf) * 1.0f;
  }
  const float cym = __shfl_sync(0xffffffffu, v, 0);
  const float cyp = __shfl_sync(0xffffffffu, v, 1);
  const float cxm = __shfl_sync(0xffffffffu, v, 2);
  const float cxp = __shfl_sync(0xffffffffu, v, 3);
  const float cost0 = __shfl_sync(0xffffffffu, v, 4);
  if (lane != 0) return;
  auto parabolic = [](float cm, float c0, float cp) {
    const float den = cm - 2.0f * c0 + cp;
    float sub = 0.0f;
    if (den > 1e-9f) sub = 0.5f * (cm - cp) / fmaxf(den, 1e-9f);
    return fminf(fmaxf(sub, -0.5f), 0.5f);
  };
  float sdy = parabolic(cym, best, cyp);
  float sdx = parabolic(cxm, best, cxp);
  const float best0 = cost0 * 1.0f;
  if (best0 < best) {
    mdy = 0.0f;
    mdx = 0.0f;
    best = best0;
  }
  if (best > 0.85f * cost0) {
    mdy = 0.0f;
    mdx = 0.0f;
    best = cost0;
    sdy = 0.0f;
    sdx = 0.0f;
  }
  const int o = a.tiles_off * p + t;
  out_mdy[o] = mdy;
  out_mdx[o] = mdx;
  out_sdy[o] = sdy;
  out_sdx[o] = sdx;
  out_best[o] = best;
}

// ---- MotionConfidence (motion.cpp:321-387) + final vectors. One CTA per pair.
__global__ void __launch_bounds__(256) k_me_confidence(const MeField* __restrict__ mf,
                                                       const MePair* __restrict__ pairs,
                                                       int npairs, const float* __restrict__ blur,
                                                       MeArgs a, const float* __restrict__ mdy,
                                                       const float* __restrict__ mdx,
                                                       const float* __restrict__ sdy,
                                                       const float* __restrict__ sdx,
                                                       const float* __restrict__ bestv,
                                                       float* __restrict__ out_dy,
                                                       float* __restrict__ out_dx,
                                                       float* __restrict__ out_conf) {
  extern __shared__ float me_sm[];
  __shared__ unsigned hist[256];
  __shared__ unsigned bc[2];
  const int p = blockIdx.x;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur];
  const int h = mc.h, w = mc.w, tile = a.tile;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const int nt = th * tw;
  float* ratios = me_sm;         // nt
  float* conf0 = me_sm + nt;     // nt
  const float* A = blur + mc.b_off;
  const int o = a.tiles_off * p;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    const int ty = t / tw, tx = t % tw;
    // pixels of this tile: rows/cols mapped by min(y / tile, th - 1)
    const int y0 = ty * tile, y1 = (ty == th - 1) ? h : (ty + 1) * tile;
    const int x0 = tx * tile, x1 = (tx == tw - 1) ? w : (tx + 1) * tile;
    float sum = 0.0f, sum2 = 0.0f, np = 0.0f;
    for (int y = y0; y < y1; ++y) {
      const float* arow = A + (int64_t)y * mc.pitch;
      // eight samples' loads ahead of their additions, which stay in x order
      for (int xb = x0; xb < x1; xb += 8) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = arow[xb + q < x1 ? xb + q : x1 - 1];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (xb + q < x1) {
            sum += v[q];
            sum2 += v[q] * v[q];
            np += 1.0f;
          }
      }
    }
    const float norm = 1.0f / fmaxf(1.0f, np);
    const float tmean = sum * norm;
    const float tvar = sum2 * norm - tmean * tmean;
    const float best = bestv[o + t];
    const float energy = (tvar + 1.0f) * fmaxf(1.0f, np);
    conf0[t] = fminf(fmaxf(1.0f - best / energy, 0.0f), 1.0f);
    ratios[t] = best / fmaxf(1.0f, np);
  }
  __syncthreads();
  // Median (motion.cpp:80-91): nth_element at n/2, averaged with the (n/2-1)-th for even n
  const int k = nt / 2;
  float med = block_select_kth(ratios, nt, k, hist, bc);
  if (nt % 2 == 0) {
    const float lo = block_select_kth(ratios, nt, k - 1, hist, bc);
    med = 0.5f * (med + lo);
  }
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    const float excess = fmaxf(0.0f, ratios[t] - med);
    float c = conf0[t];
    c *= (med + 1.0f) / (med + 1.0f + excess);
    c *= 6.0f / (6.0f + med);
    out_conf[o + t] = c;
    out_dy[o + t] = mdy[o + t] + sdy[o + t];
    out_dx[o + t] = mdx[o + t] + sdx[o + t];
  }
}

void launch_motion_blur(const MeField* d_fields, int nf, int max_h, int max_w, const MeBuffers& b,
                        cudaStream_t st) {
  if (nf <= 0) return;
  k_blur_v<<<dim3((max_w + kBoxThreads - 1) / kBoxThreads, nf), kBoxThreads, 0, st>>>(
      d_fields, nf, b.luma, b.tmp, 2, 0);
  k_blur_h<<<dim3((max_h + 31) / 32, nf), 32, 0, st>>>(d_fields, nf, b.tmp, b.blur, 2);
}

void launch_motion(const MeField* d_fields, int nf, int max_h, int max_w, const MePair* d_pairs,
                   int npairs, const MeArgs& a, const MeBuffers& b, cudaStream_t st) {
  if (nf <= 0 || npairs <= 0) return;
  const int r = 2;
  // blur every field's luma (A = blur(y_cur), B = blur(y_ref) share per field)
  k_blur_v<<<dim3((max_w + kBoxThreads - 1) / kBoxThreads, nf), kBoxThreads, 0, st>>>(
      d_fields, nf, b.luma, b.tmp, r, 0);
  k_blur_h<<<dim3((max_h + 31) / 32, nf), 32, 0, st>>>(d_fields, nf, b.tmp, b.blur, r);
  k_decimate<<<dim3(((max_h / 4) * (max_w / 4) + 255) / 256, nf), 256, 0, st>>>(d_fields, nf, b.blur, b.dec);
  const int ct = a.tile / 4 > 4 ? a.tile / 4 : 4;
  const int cth = ((max_h / 4) + ct - 1) / ct, ctw = ((max_w / 4) + ct - 1) / ct;
  const int cn = 2 * ((a.search + 3) / 4 > 1 ? (a.search + 3) / 4 : 1) + 1;
  if (cn * cn <= kCoarseWarpCands && ct <= kCoarseWarpRows) {
    const int wpc = 4;
    const int csmem = wpc * kCoarseWarpCands * kCoarseWarpRows * (int)sizeof(float);
    k_me_coarse_warp<<<dim3((cth * ctw + wpc - 1) / wpc, npairs), 32 * wpc, csmem, st>>>(
        d_fields, d_pairs, npairs, b.dec, a, b.cdy, b.cdx);
  } else {
    k_me_coarse<<<dim3((cth * ctw + 63) / 64, npairs), 64, 0, st>>>(d_fields, d_pairs, npairs,
                                                                 b.dec, a, b.cdy, b.cdx);
  }
  const int th = (max_h + a.tile - 1) / a.tile, tw = (max_w + a.tile - 1) / a.tile;
  if (a.tile <= kRefineWarpTile) {
    const int wpc = a.tile <= 32 ? 4 : 2;
    const int rsmem = wpc * kRefineCands * a.tile * (int)sizeof(float);
    k_me_refine_warp<<<dim3((th * tw + wpc - 1) / wpc, npairs), 32 * wpc, rsmem, st>>>(
        d_fields, d_pairs, npairs, b.blur, a, b.cdy, b.cdx, b.mdy, b.mdx, b.sdy, b.sdx, b.best);
  } else {
    k_me_refine<<<dim3((th * tw + 63) / 64, npairs), 64, 0, st>>>(
        d_fields, d_pairs, npairs, b.blur, a, b.cdy, b.cdx, b.mdy, b.mdx, b.sdy, b.sdx, b.best);
  }
  const int smem = 2 * th * tw * (int)sizeof(float);
  k_me_confidence<<<npairs, 256, smem, st>>>(d_fields, d_pairs, npairs, b.blur, a, b.mdy, b.mdx,
                                             b.sdy, b.sdx, b.best, b.dy, b.dx, b.conf);
}

// ---------------------------------------------------------------------------
// Integer-SAD motion mode (me_mode 1): exhaustive +-range search of
// block x block tiles on uint16-quantised, integer-box-blurred luma. The
// cost has no reference counterpart (the reference matches float SSD); the
// control structure follows EstimateMotion (motion.cpp:397-488) -- visit
// order RangeFromCentre (:286-298), strict-less update (:244), bias
// 1 + 0.02 (|dy| + |dx|), zero-motion margin 0.85 (:455-473), parabolic
// sub-pel (:437-452), MotionConfidence (:321-387) -- with every decision
// exact in integers: SAD_a (50 + L1_a) < SAD_b (50 + L1_b), and
// 20 best > 17 cost0 for the margin. A parallel argmin over the key
// (biased cost, visit index) selects the same candidate as the reference's
// sequential strict-less scan.
// ---------------------------------------------------------------------------
constexpr float kQuantZero = 16384.0f;   // 0 IRE
constexpr float kQuantScale = 348.16f;   // codes per IRE
constexpr int kSadMaxBlock = 32;
constexpr int kSadMaxRange = 22;         // (2 range + 1)^2 visit indices fit in 11 bits
// block, window and the window's integral image at the largest block and range
constexpr int kSadMaxWin = kSadMaxBlock + 2 * (kSadMaxRange + 1);
// block, window, integral image, then the packed copies (16-bit pairs) of
// the block's rows and of the window's rows at even and odd starts
__host__ __device__ constexpr int sad_smem_ints(int b, int ww) {
  return b * b + ww * ww + (ww + 1) * (ww + 1) + b * (b / 2) + 2 * ww * (ww / 2 + 1);
}
constexpr int kSadMaxSmem = sad_smem_ints(kSadMaxBlock, kSadMaxWin) * (int)sizeof(int);
constexpr int kSadThreads = 224;

int sad_max_block() { return kSadMaxBlock; }
int sad_max_range() { return kSadMaxRange; }

__device__ __forceinline__ int quant_luma(float y) {
  const float t = kQuantZero + kQuantScale * y;  // multiply, then add (no FMA in this unit)
  return (int)fminf(fmaxf(rintf(t), 0.0f), 65535.0f);
}

// Vertical 5-row window sums of the quantised luma (zero outside the field).
// One thread per (field, column).
__global__ void k_sad_vsum(const MeField* __restrict__ mf, int nf, const float* __restrict__ luma,
                           int* __restrict__ vsum) {
  const int f = blockIdx.y;
  const MeField m = mf[f];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= m.w) return;
  const float* Y = luma + m.y_off;
  int* V = vsum + m.t_off;
  int ring[5] = {0, 0, 0, 0, 0};
  int acc = 0;
  // rows y - 2 .. y + 2; prime with rows 0 .. 1
  for (int y = 0; y < 2 && y < m.h; ++y) {
    ring[y] = quant_luma(Y[(int64_t)y * m.pitch + x]);
    acc += ring[y];
  }
  for (int y = 0; y < m.h; ++y) {
    const int yn = y + 2;
    if (yn < m.h) {
      const int q = quant_luma(Y[(int64_t)yn * m.pitch + x]);
      acc += q;
      ring[yn % 5] = q;
    }
    V[(int64_t)y * m.pitch + x] = acc;
    const int yo = y - 2;
    if (yo >= 0) {
      acc -= ring[yo % 5];
      ring[yo % 5] = 0;
    }
  }
}

// Horizontal 5-column sums of vsum, rounded division by 25. One thread per
// (field, row).
__global__ void k_sad_hsum(const MeField* __restrict__ mf, int nf, const int* __restrict__ vsum,
                           int* __restrict__ qblur) {
  const int f = blockIdx.y;
  const MeField m = mf[f];
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= m.h) return;
  const int* V = vsum + m.t_off + (int64_t)y * m.pitch;
  int* Q = qblur + m.b_off + (int64_t)y * m.pitch;
  int acc = 0;
  for (int x = 0; x < 2 && x < m.w; ++x) acc += V[x];
  for (int x = 0; x < m.w; ++x) {
    if (x + 2 < m.w) acc += V[x + 2];
    Q[x] = (acc + 12) / 25;
    if (x - 2 >= 0) acc -= V[x - 2];
  }
}

__device__ __forceinline__ int centre_out_index(int d) {
  return d == 0 ? 0 : (d > 0 ? 2 * d : -2 * d - 1);
}

// SAD (or SSD) over the tile of source offset (dy, dx), one warp (lanes over pixels).
__device__ __forceinline__ unsigned long long warp_tile_cost(const int* As, const int* Bs, int b,
                                                             int ww, int S, int bh, int bw,
                                                             int dy, int dx, bool squared,
                                                             int lane) {
  unsigned long long acc = 0;
  for (int i = lane; i < bh * bw; i += 32) {
    const int yy = i / bw, xx = i % bw;
    const int d = As[yy * b + xx] - Bs[(yy - dy + S) * ww + (xx - dx + S)];
    acc += squared ? (unsigned long long)((long long)d * d) : (unsigned long long)abs(d);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// The exhaustive scan. For integers |a - b| = 2 max(a, b) - a - b, so a
// candidate's SAD is 2 sum max(A, B) - sum A - sum B over its window, the
// last from the window's integral image: one max and one add per candidate
// pixel, all in exact integers. Each item is one dy and G consecutive dx;
// its rows are split between two adjacent lanes (their sums meet by one
// shuffle), which halves the dependent chain of a candidate's additions.
// Blocks of BW = 16 columns keep a register window of the G + 15 row values
// they read (one new load per pixel). Returns the thread's best key (biased
// cost << 11 | centre-out visit index); the lane holding (0, 0) stores its
// SAD in *sad0.
// Two 16-bit lanes at once (the quantised luma is a uint16 code): the
// per-lane maximum, and the sum of the two lanes added to an accumulator by
// a two-way dot product with (1, 1).
__device__ __forceinline__ unsigned vmax_u16x2(unsigned a, unsigned b) {
  unsigned d;
  asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// Rows [yb, ye) of one item of a 16-wide block, packed: Ap holds the block's
// rows as 8 pairs (columns 2k, 2k + 1), BpE / BpO each window row's pairs
// starting at even / odd columns. For candidate offset dxg + g the window
// pair under block pair k starts at column e_lo + (G - 1 - g) + 2 k, e_lo =
// S - dxg - (G - 1); a0 = e_lo - Q (even, Q = e_lo & 1) is where this row's
// words are loaded from, so every register index below is a constant.
template <int G, int Q>
__device__ __forceinline__ void sad_rows_packed(const unsigned* __restrict__ Ap,
                                                const unsigned* __restrict__ BpE,
                                                const unsigned* __restrict__ BpO, int hb, int wp,
                                                int yb, int ye, int dy, int S, int a0h,
                                                unsigned (&acc)[G]) {
  constexpr int kWords = (Q + G - 1 + 14) / 2 + 1;
  for (int yy = yb; yy < ye; ++yy) {
    const unsigned* ap = Ap + yy * hb;
    const int row = yy - dy + S;
    const unsigned* be = BpE + row * wp + a0h;
    const unsigned* bo = BpO + row * wp + a0h;
    unsigned wE[kWords], wO[kWords];
#pragma unroll
    for (int j = 0; j < kWords; ++j) {
      wE[j] = be[j];
      wO[j] = bo[j];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const unsigned av = ap[k];
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int off = Q + (G - 1 - g) + 2 * k;
        const unsigned bv = (off & 1) ? wO[off >> 1] : wE[off >> 1];
        acc[g] = __dp2a_lo(vmax_u16x2(av, bv), 0x0101u, acc[g]);
      }
    }
  }
}

template <int G, int BW>
__device__ __forceinline__ unsigned long long sad_scan(const int* As, const int* Bs,
                                                       const int* I, const unsigned* Ap,
                                                       const unsigned* BpE, const unsigned* BpO,
                                                       int b, int ww, int S, int bh, int bw, int s,
                                                       unsigned sum_a, unsigned long long* sad0,
                                                       unsigned one) {
  const int n = 2 * s + 1;
  const int ngroups = (n + G - 1) / G;
  const int items = n * ngroups;
  const int wi = ww + 1;
  const int hsplit = (bh + 1) / 2;
  unsigned long long bestkey = ~0ull;
  // items (dy, group of G offsets) ordered by the parity of their packed
  // window start (odd G alternates it from group to group), so the lanes of a
  // warp take the same packed code path
  const int c0 = (S + s - G + 1) & 1;  // parity of group 0's start
  const int n0 = (G & 1) ? (ngroups - c0 + 1) / 2 : (c0 == 0 ? ngroups : 0);
  for (int base = 0; base < 2 * items; base += blockDim.x) {
    const int it = base + threadIdx.x;
    const bool valid = it < 2 * items;
    const int item = it >> 1, half = it & 1;
    int dyi, grp;
    if (!(G & 1)) {
      dyi = item / ngroups;
      grp = item % ngroups;
    } else if (item < n * n0) {
      dyi = item / n0;
      grp = c0 + 2 * (item % n0);
    } else {
      const int i1 = item - n * n0, n1 = ngroups - n0;
      dyi = i1 / n1;
      grp = (1 - c0) + 2 * (i1 % n1);
    }
    const int dy = dyi - s;
    const int dxg = -s + grp * G;
    unsigned acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = 0u;
    if (valid) {
      const int yb = half ? hsplit : 0, ye = half ? bh : hsplit;
      if (BW == 16) {
        const int e_lo = S - dxg - (G - 1);
        const int a0h = (e_lo - (e_lo & 1)) >> 1;
        if (e_lo & 1)
          sad_rows_packed<G, 1>(Ap, BpE, BpO, b / 2, ww / 2 + 1, yb, ye, dy, S, a0h, acc);
        else
          sad_rows_packed<G, 0>(Ap, BpE, BpO, b / 2, ww / 2 + 1, yb, ye, dy, S, a0h, acc);
      } else {
        for (int yy = yb; yy < ye; ++yy) {
          const int* ar = As + yy * b;
          // window value under pixel xx at offset dxg + g: br[xx - g]
          const int* br = Bs + (yy - dy + S) * ww + (S - dxg);
          for (int xx = 0; xx < bw; ++xx) {
            const int av = ar[xx];
#pragma unroll
            for (int g = 0; g < G; ++g) acc[g] = (unsigned)max(av, br[xx - g]) * one + acc[g];
          }
        }
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] += __shfl_xor_sync(0xffffffffu, acc[g], 1);
    if (!valid || half) continue;
    const int r0 = S - dy;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int dx = dxg + g;
      if (dx > s) break;
      const int c0 = S - dx;
      const unsigned sum_b = (unsigned)(I[(r0 + bh) * wi + c0 + bw] - I[r0 * wi + c0 + bw] -
                                        I[(r0 + bh) * wi + c0] + I[r0 * wi + c0]);
      const unsigned sad = 2u * acc[g] - sum_a - sum_b;
      const unsigned long long cost =
          (unsigned long long)sad * (unsigned long long)(50 + abs(dy) + abs(dx));
      const unsigned long long ci =
          (unsigned long long)(centre_out_index(dy) * n + centre_out_index(dx));
      const unsigned long long key = (cost << 11) | ci;
      if (key < bestkey) bestkey = key;
      if (dy == 0 && dx == 0) *sad0 = sad;
    }
  }
  return bestkey;
}

// One CTA per (tile, pair).
__global__ void __launch_bounds__(kSadThreads, 6) k_sad_search(const MeField* __restrict__ mf,
                                                            const MePair* __restrict__ pairs,
                                                            const int* __restrict__ qblur,
                                                            SadArgs a, SadBuffers out) {
  const int p = blockIdx.y, t = blockIdx.x;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int h = mc.h, w = mc.w, b = a.block, s = a.range;
  const int th = (h + b - 1) / b, tw = (w + b - 1) / b;
  if (t >= th * tw) return;
  const int ty = t / tw, tx = t % tw;
  const int y0 = ty * b, x0 = tx * b;
  const int bh = min(b, h - y0), bw = min(b, w - x0);
  const int S = s + 1;          // window margin: the search range plus the sub-pel neighbours
  const int ww = b + 2 * S;
  const int wi = ww + 1;
  extern __shared__ int sad_sm[];
  int* As = sad_sm;             // b x b
  int* Bs = sad_sm + b * b;     // ww x ww, B(clamp(y0 - S + wy), clamp(x0 - S + wx))
  int* I = Bs + ww * ww;        // (ww + 1)^2 integral image of Bs
  // packed 16-bit pairs: the block's rows (b / 2 per row), the window's rows
  // from even columns (BpE) and from odd columns (BpO), ww / 2 + 1 per row
  unsigned* Ap = reinterpret_cast<unsigned*>(I + (ww + 1) * (ww + 1));
  unsigned* BpE = Ap + b * (b / 2);
  unsigned* BpO = BpE + ww * (ww / 2 + 1);
  __shared__ unsigned long long red[kSadThreads / 32];
  __shared__ unsigned long long sh_sad0, sh_best, sh_side[4], sh_ssd;
  __shared__ long long sh_s1, sh_s2;
  __shared__ unsigned sh_suma;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int* QA = qblur + mc.b_off;
  const int* QB = qblur + mr.b_off;
  for (int i = tid; i < bh * bw; i += blockDim.x)
    As[(i / bw) * b + i % bw] = QA[(int64_t)(y0 + i / bw) * mc.pitch + x0 + i % bw];
  for (int i = tid; i < ww * ww; i += blockDim.x) {
    const int wy = i / ww, wx = i % ww;
    const int sy = clampi(y0 - S + wy, 0, h - 1), sx = clampi(x0 - S + wx, 0, w - 1);
    Bs[i] = QB[(int64_t)sy * mr.pitch + sx];
  }
  __syncthreads();
  // integral image: row prefix sums, then column prefix sums (exact ints:
  // the whole window sums below 2^31)
  for (int r = tid; r <= ww; r += blockDim.x) {
    int* Ir = I + r * wi;
    Ir[0] = 0;
    int acc = 0;
    if (r == 0) {
      for (int c = 1; c <= ww; ++c) Ir[c] = 0;
    } else {
      const int* br = Bs + (r - 1) * ww;
      for (int c = 1; c <= ww; ++c) {
        acc += br[c - 1];
        Ir[c] = acc;
      }
    }
  }
  {
    // the packed copies (columns past the window's edge pack as 0)
    const int hb = b / 2, wp = ww / 2 + 1;
    for (int i = tid; i < b * hb; i += blockDim.x) {
      const int r = i / hb, k = i % hb;
      Ap[i] = (unsigned)As[r * b + 2 * k] | ((unsigned)As[r * b + 2 * k + 1] << 16);
    }
    for (int i = tid; i < ww * wp; i += blockDim.x) {
      const int r = i / wp, k = i % wp;
      const int* br = Bs + r * ww;
      const unsigned e0 = 2 * k < ww ? (unsigned)br[2 * k] : 0u;
      const unsigned e1 = 2 * k + 1 < ww ? (unsigned)br[2 * k + 1] : 0u;
      const unsigned e2 = 2 * k + 2 < ww ? (unsigned)br[2 * k + 2] : 0u;
      BpE[i] = e0 | (e1 << 16);
      BpO[i] = e1 | (e2 << 16);
    }
  }
  if (warp == 0) {
    unsigned sa = 0;
    for (int i = lane; i < bh * bw; i += 32) sa += (unsigned)As[(i / bw) * b + i % bw];
    for (int o = 16; o > 0; o >>= 1) sa += __shfl_xor_sync(0xffffffffu, sa, o);
    if (lane == 0) sh_suma = sa;
  }
  __syncthreads();
  for (int c = tid; c <= ww; c += blockDim.x)
    for (int r = 1; r <= ww; ++r) I[r * wi + c] += I[(r - 1) * wi + c];
  __syncthreads();
  const int n = 2 * s + 1;
  const unsigned sum_a = sh_suma;
  // 1, in a form the compiler cannot fold: the accumulations are issued as
  // multiply-adds, which run on the FMA pipe beside the max on the integer
  // pipe (a plain add would share the integer pipe with the max)
  const unsigned one = ((unsigned)a.block >> 30) | 1u;
  // G consecutive dx per thread: 11 when it divides the row of candidates
  // (no wasted candidates at +-16), else 8
  unsigned long long bestkey;
  if (n % 11 == 0)
    bestkey = bw == 16 ? sad_scan<11, 16>(As, Bs, I, Ap, BpE, BpO, b, ww, S, bh, bw, s, sum_a, &sh_sad0, one)
                       : sad_scan<11, 0>(As, Bs, I, Ap, BpE, BpO, b, ww, S, bh, bw, s, sum_a, &sh_sad0, one);
  else
    bestkey = bw == 16 ? sad_scan<8, 16>(As, Bs, I, Ap, BpE, BpO, b, ww, S, bh, bw, s, sum_a, &sh_sad0, one)
                       : sad_scan<8, 0>(As, Bs, I, Ap, BpE, BpO, b, ww, S, bh, bw, s, sum_a, &sh_sad0, one);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, bestkey, o);
    if (v < bestkey) bestkey = v;
  }
  if (lane == 0) red[warp] = bestkey;
  __syncthreads();
  if (tid == 0) {
    unsigned long long m = red[0];
    for (int i = 1; i < (int)(blockDim.x / 32); ++i) m = red[i] < m ? red[i] : m;
    sh_best = m;
  }
  __syncthreads();
  const unsigned long long best = sh_best >> 11;
  const int ci = (int)(sh_best & 2047ull);
  const int mdy = centre_out(ci / n), mdx = centre_out(ci % n);
  // the sub-pel neighbours' unbiased SADs, the zero-margin decision, then the
  // SSD at the final vector and the tile statistics of A (one warp each)
  const unsigned long long cost0 = 50ull * sh_sad0;
  const bool zero = 20ull * best > 17ull * cost0;
  const int fdy = zero ? 0 : mdy, fdx = zero ? 0 : mdx;
  if (warp < 4) {
    const int oy = warp == 0 ? -1 : (warp == 1 ? 1 : 0);
    const int ox = warp == 2 ? -1 : (warp == 3 ? 1 : 0);
    const unsigned long long v =
        warp_tile_cost(As, Bs, b, ww, S, bh, bw, mdy + oy, mdx + ox, false, lane);
    if (lane == 0) sh_side[warp] = v;
  } else if (warp == 4) {
    const unsigned long long v = warp_tile_cost(As, Bs, b, ww, S, bh, bw, fdy, fdx, true, lane);
    if (lane == 0) sh_ssd = v;
  } else if (warp == 5) {
    long long s1 = 0, s2 = 0;
    for (int i = lane; i < bh * bw; i += 32) {
      const long long v = As[(i / bw) * b + i % bw];
      s1 += v;
      s2 += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
      sh_s1 = s1;
      sh_s2 = s2;
    }
  }
  __syncthreads();
  if (tid == 0) {
    // parabola through (-1, 50 SAD_m), (0, best), (+1, 50 SAD_p): exact
    // integer numerator and denominator, one division
    auto parabolic = [&](unsigned long long sm, unsigned long long sp) -> double {
      const long long num = 50ll * (long long)sm - 50ll * (long long)sp;
      const long long den = 50ll * (long long)sm - 2ll * (long long)best + 50ll * (long long)sp;
      double sub = den > 0 ? 0.5 * (double)num / (double)den : 0.0;
      return fmin(fmax(sub, -0.5), 0.5);
    };
    double sdy = parabolic(sh_side[0], sh_side[1]);
    double sdx = parabolic(sh_side[2], sh_side[3]);
    if (zero) {
      sdy = 0.0;
      sdx = 0.0;
    }
    const int o = a.tiles_off * p + t;
    out.mdy[o] = (float)fdy;
    out.mdx[o] = (float)fdx;
    out.sdy[o] = (float)sdy;
    out.sdx[o] = (float)sdx;
    const double sc2 = (double)kQuantScale * (double)kQuantScale;
    out.bestv[o] = (double)(sh_ssd * (unsigned long long)(50 + abs(fdy) + abs(fdx))) / (50.0 * sc2);
    out.s1[o] = (double)sh_s1;
    out.s2[o] = (double)sh_s2;
    out.npx[o] = (double)(bh * bw);
    out.dy[o] = (float)((double)fdy + sdy);
    out.dx[o] = (float)((double)fdx + sdx);
  }
}

// Exact k-th smallest of v[0..n) (stable rank count), by the whole CTA.
__device__ double block_kth_double(const double* v, int n, int k, double* slot) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = v[i];
    int less = 0, eq_before = 0;
    for (int j = 0; j < n; ++j) {
      const double y = v[j];
      less += y < x;
      eq_before += (y == x) & (j < i);
    }
    if (less + eq_before == k) *slot = x;
  }
  __syncthreads();
  const double r = *slot;
  __syncthreads();
  return r;
}

// MotionConfidence on the IRE scale from the exact integer statistics. One
// CTA per pair.
__global__ void __launch_bounds__(256) k_sad_confidence(const MeField* __restrict__ mf,
                                                        const MePair* __restrict__ pairs,
                                                        SadArgs a, SadBuffers out) {
  extern __shared__ double sadc_sm[];
  __shared__ double slot;
  const int p = blockIdx.x;
  const MeField mc = mf[pairs[p].cur];
  const int b = a.block;
  const int th = (mc.h + b - 1) / b, tw = (mc.w + b - 1) / b, nt = th * tw;
  double* ratios = sadc_sm;
  const int o = a.tiles_off * p;
  for (int t = threadIdx.x; t < nt; t += blockDim.x)
    ratios[t] = out.bestv[o + t] / fmax(1.0, out.npx[o + t]);
  __syncthreads();
  const int k = nt / 2;
  double med = block_kth_double(ratios, nt, k, &slot);
  if (nt % 2 == 0) med = 0.5 * (med + block_kth_double(ratios, nt, k - 1, &slot));
  const double sc2 = (double)kQuantScale * (double)kQuantScale;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    const double npx = out.npx[o + t];
    const double norm = 1.0 / fmax(1.0, npx);
    const double tmean = out.s1[o + t] * norm;
    const double tvar = (out.s2[o + t] * norm - tmean * tmean) / sc2;
    const double energy = (tvar + 1.0) * fmax(1.0, npx);
    double c = fmin(fmax(1.0 - out.bestv[o + t] / energy, 0.0), 1.0);
    const double excess = fmax(0.0, ratios[t] - med);
    c = c * ((med + 1.0) / (med + 1.0 + excess));
    c = c * (6.0 / (6.0 + med));
    out.conf[o + t] = (float)c;
  }
}

void launch_motion_sad(const MeField* d_fields, int nf, int max_h, int max_w,
                       const MePair* d_pairs, int npairs, const SadArgs& a, const SadBuffers& b,
                       cudaStream_t st) {
  if (nf <= 0 || npairs <= 0) return;
  k_sad_vsum<<<dim3((max_w + 127) / 128, nf), 128, 0, st>>>(d_fields, nf, b.luma, b.vsum);
  k_sad_hsum<<<dim3((max_h + 127) / 128, nf), 128, 0, st>>>(d_fields, nf, b.vsum, b.qblur);
  const int th = (max_h + a.block - 1) / a.block, tw = (max_w + a.block - 1) / a.block;
  const int ww = a.block + 2 * (a.range + 1);
  const int smem = sad_smem_ints(a.block, ww) * (int)sizeof(int);
  static PerDeviceOnce sad_once;
  sad_once([] {
    cudaFuncSetAttribute(k_sad_search, cudaFuncAttributeMaxDynamicSharedMemorySize, kSadMaxSmem);
  });
  k_sad_search<<<dim3(th * tw, npairs), kSadThreads, smem, st>>>(d_fields, d_pairs, b.qblur, a, b);
  k_sad_confidence<<<npairs, 256, th * tw * (int)sizeof(double), st>>>(d_fields, d_pairs, a, b);
}

// ---------------------------------------------------------------------------
// VectorsPerPixel (temporal.cpp:45-112): 3x3 median outlier snap on the tile
// grid, then bilinear interpolation between tile centres.
// ---------------------------------------------------------------------------
__device__ float median9(float* v) {
  // exact middle of 9 values (nth_element(v, v + 4, v + 9))
  for (int i = 0; i < 5; ++i) {
    int mi = i;
    for (int j = i + 1; j < 9; ++j)
      if (v[j] < v[mi]) mi = j;
    const float t = v[i];
    v[i] = v[mi];
    v[mi] = t;
  }
  return v[4];
}

// Snapped tile vectors; one thread per (pair, tile).
__global__ void k_vec_snap(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                           int npairs, MeArgs a, const float* __restrict__ dy_in,
                           const float* __restrict__ dx_in, float* __restrict__ dy_out,
                           float* __restrict__ dx_out) {
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MeField mc = mf[pairs[p].cur];
  const int th = (mc.h + a.tile - 1) / a.tile, tw = (mc.w + a.tile - 1) / a.tile;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= th * tw) return;
  const int o = a.tiles_off * p;
  float vy = dy_in[o + t], vx = dx_in[o + t];
  if (th >= 3 && tw >= 3) {
    const int ty = t / tw, tx = t % tw;
    float ay[9], ax[9];
    int q = 0;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int yy = clampi(ty + dy, 0, th - 1), xx = clampi(tx + dx, 0, tw - 1);
        ay[q] = dy_in[o + yy * tw + xx];
        ax[q] = dx_in[o + yy * tw + xx];
        ++q;
      }
    const float my = median9(ay), mx = median9(ax);
    const float dis = fabsf(vy - my) + fabsf(vx - mx);
    if (dis > 3.0f) {
      vy = my;
      vx = mx;
    }
  }
  dy_out[o + t] = vy;
  dx_out[o + t] = vx;
}

__device__ __forceinline__ void bracket(int coord, int n_tiles, int tile, int* lo, float* frac) {
  if (n_tiles > 1) {
    const float rel = (float)coord / (float)tile - 0.5f;
    *lo = clampi((int)floorf(rel), 0, n_tiles - 2);
    const float centre_lo = ((float)*lo + 0.5f) * (float)tile;
    *frac = fminf(fmaxf(((float)coord - centre_lo) / (float)tile, 0.0f), 1.0f);
  } else {
    *lo = 0;
    *frac = 0.0f;
  }
}

__device__ __forceinline__ float interp_tiles(const float* v, int tw, int iy, int iy1, int ix,
                                              int ix1, float fy, float fx) {
  const float v00 = v[iy * tw + ix], v10 = v[iy1 * tw + ix];
  const float v01 = v[iy * tw + ix1], v11 = v[iy1 * tw + ix1];
  return v00 * (1 - fy) * (1 - fx) + v10 * fy * (1 - fx) + v01 * (1 - fy) * fx + v11 * fy * fx;
}

// Per-pixel vectors for one pair, written as the warp source indices
// (sy, sx) = (clamp(y - lround(vdy)), clamp(x - lround(vdx))) packed in an
// int2, plus (optionally) the interpolated squared confidence (fast mode).
__global__ void k_vec_pixels(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                             int npairs, MeArgs a, const float* __restrict__ sdy,
                             const float* __restrict__ sdx, int2* __restrict__ src_idx,
                             const int64_t* __restrict__ pix_off) {
  const int p = blockIdx.z;
  if (p >= npairs) return;
  const MeField mc = mf[pairs[p].cur];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= mc.w || y >= mc.h) return;
  const int th = (mc.h + a.tile - 1) / a.tile, tw = (mc.w + a.tile - 1) / a.tile;
  int iy, ix;
  float fy, fx;
  bracket(y, th, a.tile, &iy, &fy);
  bracket(x, tw, a.tile, &ix, &fx);
  const int iy1 = min(iy + 1, th - 1), ix1 = min(ix + 1, tw - 1);
  const int o = a.tiles_off * p;
  const float vy = interp_tiles(sdy + o, tw, iy, iy1, ix, ix1, fy, fx);
  const float vx = interp_tiles(sdx + o, tw, iy, iy1, ix, ix1, fy, fx);
  const int sy = clampi(y - (int)lroundf(vy), 0, mc.h - 1);
  const int sx = clampi(x - (int)lroundf(vx), 0, mc.w - 1);
  src_idx[pix_off[p] + (int64_t)y * mc.pitch + x] = make_int2(sy, sx);
}

// Squared per-tile confidence -> per pixel.
//   fast: VectorsPerPixel of conf^2 (snap + bilinear), temporal.cpp:245-254
//   slow: nearest tile, squared, then BoxBlur radius 8, temporal.cpp:227-243
__global__ void k_conf_sq(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                          int npairs, MeArgs a, const float* __restrict__ conf,
                          float* __restrict__ c2) {
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MeField mc = mf[pairs[p].cur];
  const int nt = ((mc.h + a.tile - 1) / a.tile) * ((mc.w + a.tile - 1) / a.tile);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const float c = conf[a.tiles_off * p + t];
  c2[a.tiles_off * p + t] = c * c;
}

__global__ void k_conf_pixels_fast(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                                   int npairs, MeArgs a, const float* __restrict__ c2s,
                                   float* __restrict__ out, const int64_t* __restrict__ pix_off) {
  const int p = blockIdx.z;
  if (p >= npairs) return;
  const MeField mc = mf[pairs[p].cur];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= mc.w || y >= mc.h) return;
  const int th = (mc.h + a.tile - 1) / a.tile, tw = (mc.w + a.tile - 1) / a.tile;
  int iy, ix;
  float fy, fx;
  bracket(y, th, a.tile, &iy, &fy);
  bracket(x, tw, a.tile, &ix, &fx);
  out[pix_off[p] + (int64_t)y * mc.pitch + x] =
      interp_tiles(c2s + a.tiles_off * p, tw, iy, min(iy + 1, th - 1), ix, min(ix + 1, tw - 1), fy, fx);
}

__global__ void k_conf_pixels_nearest(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                                      int npairs, MeArgs a, const float* __restrict__ conf,
                                      float* __restrict__ out, const int64_t* __restrict__ pix_off) {
  const int p = blockIdx.z;
  if (p >= npairs) return;
  const MeField mc = mf[pairs[p].cur];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= mc.w || y >= mc.h) return;
  const int th = (mc.h + a.tile - 1) / a.tile, tw = (mc.w + a.tile - 1) / a.tile;
  const int ty = min(y / a.tile, th - 1), tx = min(x / a.tile, tw - 1);
  const float c = conf[a.tiles_off * p + ty * tw + tx];
  out[pix_off[p] + (int64_t)y * mc.pitch + x] = c * c;
}

// BoxBlur radius r over per-pair planes (same prefix-sum arithmetic as the
// luma blur); in place through a scratch plane.
__global__ void k_pair_blur_v(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                              int npairs, const float* __restrict__ src, float* __restrict__ dst,
                              const int64_t* __restrict__ pix_off, int r) {
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MeField m = mf[pairs[p].cur];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= m.w) return;
  const float* s = src + pix_off[p];
  float* d = dst + pix_off[p];
  const double norm = (double)(1.0f / (float)(2 * r + 1));
  box_line(s + x, m.pitch, d + x, m.pitch, m.h, r, norm);
}

// one warp per (pair, 32-row band)
__global__ void k_pair_blur_h(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                              int npairs, const float* __restrict__ src, float* __restrict__ dst,
                              const int64_t* __restrict__ pix_off, int r) {
  const int p = blockIdx.y;
  if (p >= npairs) return;
  const MeField m = mf[pairs[p].cur];
  const int y0 = blockIdx.x * 32;
  if (y0 >= m.h) return;
  const double norm = (double)(1.0f / (float)(2 * r + 1));
  box_rows_warp(src + pix_off[p] + (int64_t)y0 * m.pitch, dst + pix_off[p] + (int64_t)y0 * m.pitch,
                m.pitch, min(32, m.h - y0), m.w, r, norm);
}

// ---------------------------------------------------------------------------
// Trajectory consensus, fast-mode verification, motion cache, coherence gate
// ---------------------------------------------------------------------------
// numpy.median of up to kTrajMaxPairs values (Median, motion.cpp:80-91 and
// MedianOf, sequence.cpp:29-39: the mean of the two middles for even n)
__device__ float median_small(float* v, int n) {
  for (int i = 1; i < n; ++i) {
    const float x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
  const int k = n / 2;
  float m = v[k];
  if (n % 2 == 0) m = 0.5f * (m + v[k - 1]);
  return m;
}

// TrajectorySnap (motion.cpp:565-601) with FitTrajectory (:532-563): one
// thread per (field group, tile).
__global__ void k_traj_snap(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                            const TrajGroup* __restrict__ groups, int ngroups,
                            const TrajPair* __restrict__ tp, int tile, int tiles_off,
                            float* __restrict__ dy, float* __restrict__ dx,
                            const float* __restrict__ conf) {
  const int g = blockIdx.y;
  if (g >= ngroups) return;
  const TrajGroup G = groups[g];
  if (G.count < 2) return;
  const MeField mc = mf[pairs[G.pair[0]].cur];
  const int th = (mc.h + tile - 1) / tile, tw = (mc.w + tile - 1) / tile;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= th * tw) return;
  float sy[kTrajMaxPairs], sx[kTrajMaxPairs];
  int n = 0;
  for (int i = 0; i < G.count; ++i) {
    const int p = G.pair[i];
    const TrajPair q = tp[p];
    if (q.offset == 0) continue;
    const int o = tiles_off * p + t;
    if (conf[o] <= 0.15f) continue;
    const float of = (float)q.offset;
    sy[n] = (dy[o] - q.parity_shift) / of;
    sx[n] = dx[o] / of;
    ++n;
  }
  float vym = 0.0f, vxm = 0.0f;
  if (n > 0) {
    vym = median_small(sy, n);
    vxm = median_small(sx, n);
  }
  // consensus: the snap applies where >= 3 offsets agree within 1.5 px
  float agree = 0.0f;
  for (int i = 0; i < G.count; ++i) {
    const int p = G.pair[i];
    const TrajPair q = tp[p];
    const int o = tiles_off * p + t;
    const float of = (float)q.offset;
    const float py = of * vym + q.parity_shift;
    const float px = of * vxm;
    const float dev = fabsf(dy[o] - py) + fabsf(dx[o] - px);
    if (dev <= 1.5f) agree += 1.0f;
  }
  if (agree < 3.0f) return;
  for (int i = 0; i < G.count; ++i) {
    const int p = G.pair[i];
    const TrajPair q = tp[p];
    const int o = tiles_off * p + t;
    const float of = (float)q.offset;
    const float py = of * vym + q.parity_shift;
    const float px = of * vxm;
    const float dev = fabsf(dy[o] - py) + fabsf(dx[o] - px);
    if (dev <= 1.5f) {
      dy[o] = py;
      dx[o] = px;
    }
  }
}

// Fast-mode prediction (sequence.cpp:714-763) + VerifyMotion (motion.cpp:490-530).
// Sum of squared differences over one tile with no bail-out (a lone
// candidate: BmPass's kill stays infinite), rows in order and each row in
// order -- the reference's float additions -- with each row's samples
// loaded ahead of its additions.
__device__ __forceinline__ float tile_ssd_full(const float* A, const float* B, int pitch, int h,
                                               int w, int ty0, int ty1, int tx0, int tx1, int sy,
                                               int sx) {
  float acc = 0.0f;
  for (int y = ty0; y < ty1; ++y) {
    const float* arow = A + (int64_t)y * pitch;
    const float* brow = B + (int64_t)clampi(y - sy, 0, h - 1) * pitch;
    int x = tx0;
    for (; x + 8 <= tx1; x += 8) {
      float d[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) d[k] = arow[x + k] - brow[clampi(x + k - sx, 0, w - 1)];
#pragma unroll
      for (int k = 0; k < 8; ++k) acc += d[k] * d[k];
    }
    for (; x < tx1; ++x) {
      const float diff = arow[x] - brow[clampi(x - sx, 0, w - 1)];
      acc += diff * diff;
    }
  }
  return acc;
}

// VerifyMotion (motion.cpp:490-530) of pair base + i: one SSD at the rounded
// prediction, one at zero, the prediction kept where it is strictly better.
// The prediction is the trajectory median over the searched pairs of its
// group (sequence.cpp:714-763), or, with pred_dy / pred_dx given, the
// caller's per-tile vectors. Two adjacent threads per tile: the even one
// evaluates the prediction, the odd one zero.
__global__ void k_traj_verify(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                              int base, int npred, const int* __restrict__ grp,
                              const TrajGroup* __restrict__ searched,
                              const TrajPair* __restrict__ tp, const float* __restrict__ blur,
                              MeArgs a, const float* __restrict__ dy_in,
                              const float* __restrict__ dx_in, const float* __restrict__ pred_dy,
                              const float* __restrict__ pred_dx, float* __restrict__ out_mdy,
                              float* __restrict__ out_mdx, float* __restrict__ out_sdy,
                              float* __restrict__ out_sdx, float* __restrict__ out_best) {
  const int i = blockIdx.y;
  if (i >= npred) return;  // uniform per block
  const int p = base + i;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int h = mc.h, w = mc.w, tile = a.tile;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const int tt = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = tt >> 1, cand = tt & 1;
  const bool valid = t < th * tw;
  float pdy = 0.0f, pdx = 0.0f, ssd = 0.0f;
  if (valid) {
    if (pred_dy) {
      pdy = pred_dy[a.tiles_off * i + t];
      pdx = pred_dx[a.tiles_off * i + t];
    } else {
      const TrajGroup S = searched[grp[i]];
      float sy[kTrajMaxPairs], sx[kTrajMaxPairs];
      for (int k = 0; k < S.count; ++k) {
        const int q = S.pair[k];
        const TrajPair m = tp[q];
        const float of = (float)m.offset;
        sy[k] = (dy_in[a.tiles_off * q + t] - m.parity_shift) / of;
        sx[k] = dx_in[a.tiles_off * q + t] / of;
      }
      const float vym0 = S.count > 0 ? median_small(sy, S.count) : 0.0f;
      const float vxm0 = S.count > 0 ? median_small(sx, S.count) : 0.0f;
      const TrajPair me = tp[p];
      pdy = (float)me.offset * vym0 + me.parity_shift;
      pdx = (float)me.offset * vxm0;
    }
    const int iy = cand == 0 ? (int)lroundf(pdy) : 0, ix = cand == 0 ? (int)lroundf(pdx) : 0;
    const int y0 = (t / tw) * tile, y1 = min(y0 + tile, h);
    const int x0 = (t % tw) * tile, x1 = min(x0 + tile, w);
    ssd = tile_ssd_full(blur + mc.b_off, blur + mr.b_off, mc.pitch, h, w, y0, y1, x0, x1, iy, ix);
  }
  const float zero = __shfl_down_sync(0xffffffffu, ssd, 1);
  if (!valid || cand != 0) return;
  const float pred = ssd;
  const int o = a.tiles_off * p + t;
  if (zero <= pred) {
    out_mdy[o] = 0.0f;
    out_mdx[o] = 0.0f;
    out_best[o] = zero;
  } else {
    // the full float prediction is kept where it won
    out_mdy[o] = pdy;
    out_mdx[o] = pdx;
    out_best[o] = pred;
  }
  out_sdy[o] = 0.0f;
  out_sdx[o] = 0.0f;
}

__global__ void k_motion_cache(const int* __restrict__ gid, int npairs, int nt, int tiles_off,
                               float* __restrict__ dy, float* __restrict__ dx,
                               float* __restrict__ conf, float* __restrict__ cache,
                               int64_t stride, int store) {
  const int i = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npairs || t >= nt) return;
  const int64_t c = (int64_t)gid[i] * nt + t;
  const int o = tiles_off * i + t;
  if (store) {
    cache[c] = dy[o];
    cache[stride + c] = dx[o];
    cache[2 * stride + c] = conf[o];
  } else {
    dy[o] = cache[c];
    dx[o] = cache[stride + c];
    conf[o] = cache[2 * stride + c];
  }
}

// Cross terms of chi_j and chi_k bilinearly warped by the snapped per-pixel
// vectors (WarpBilinearTiles, temporal.cpp:140-168, row offset 0).
__global__ void k_coh_terms(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                            int npairs, MeArgs a, CohBuffers b) {
  const int p = blockIdx.z;
  if (p >= npairs) return;
  const MePair pr = pairs[p];
  const MeField mc = mf[pr.cur], mr = mf[pr.ref];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= mc.w || y >= mc.h) return;
  const int th = (mc.h + a.tile - 1) / a.tile, tw = (mc.w + a.tile - 1) / a.tile;
  int iy, ix;
  float fyb, fxb;
  bracket(y, th, a.tile, &iy, &fyb);
  bracket(x, tw, a.tile, &ix, &fxb);
  const int iy1 = min(iy + 1, th - 1), ix1 = min(ix + 1, tw - 1);
  const int o = a.tiles_off * p;
  const float vy = interp_tiles(b.snap_dy + o, tw, iy, iy1, ix, ix1, fyb, fxb);
  const float vx = interp_tiles(b.snap_dx + o, tw, iy, iy1, ix, ix1, fyb, fxb);
  float sy = (float)y - vy + 0.0f;
  float sx = (float)x - vx;
  sy = fminf(fmaxf(sy, 0.0f), (float)mr.h - 1.001f);
  sx = fminf(fmaxf(sx, 0.0f), (float)mr.w - 1.001f);
  const int y0 = (int)sy, x0 = (int)sx;
  const float fy = sy - (float)y0, fx = sx - (float)x0;
  const int y1 = min(y0 + 1, mr.h - 1), x1 = min(x0 + 1, mr.w - 1);
  const float2* K = b.chi + mr.y_off;
  const float2 k00 = K[(int64_t)y0 * mr.pitch + x0], k10 = K[(int64_t)y1 * mr.pitch + x0];
  const float2 k01 = K[(int64_t)y0 * mr.pitch + x1], k11 = K[(int64_t)y1 * mr.pitch + x1];
  const float wre = k00.x * (1 - fy) * (1 - fx) + k10.x * fy * (1 - fx) + k01.x * (1 - fy) * fx +
                    k11.x * fy * fx;
  const float wim = k00.y * (1 - fy) * (1 - fx) + k10.y * fy * (1 - fx) + k01.y * (1 - fy) * fx +
                    k11.y * fy * fx;
  const float2 z1 = b.chi[mc.y_off + (int64_t)y * mc.pitch + x];
  // z1 * conj(cw)
  const float cre = z1.x * wre - z1.y * (-wim);
  const float cim = z1.x * (-wim) + z1.y * wre;
  const int64_t q = b.pix_off[p] + (int64_t)y * mc.pitch + x;
  b.terms[q] = cre;
  b.terms[b.chan_stride + q] = cim;
  b.terms[2 * b.chan_stride + q] = z1.x * z1.x + z1.y * z1.y;
  b.terms[3 * b.chan_stride + q] = wre * wre + wim * wim;
}

__global__ void k_coh_apply(const MeField* __restrict__ mf, const MePair* __restrict__ pairs,
                            int npairs, CohBuffers b, float gate) {
  const int p = blockIdx.z;
  if (p >= npairs) return;
  const MeField mc = mf[pairs[p].cur];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= mc.w || y >= mc.h) return;
  const int64_t q = b.pix_off[p] + (int64_t)y * mc.pitch + x;
  const float re = b.terms[q], im = b.terms[b.chan_stride + q];
  const float m1 = b.terms[2 * b.chan_stride + q], m2 = b.terms[3 * b.chan_stride + q];
  const float num = sqrtf(re * re + im * im);
  const float den = sqrtf(fmaxf(0.0f, m1 * m2)) + 1e-6f;
  const float gamma = fminf(fmaxf(num / den, 0.0f), 1.0f);
  b.conf_px[q] *= (1.0f - gate) + gate * gamma;
}

void launch_vectors(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                    int max_w, const MeArgs& a, const VecBuffers& v, bool fast_conf,
                    cudaStream_t st) {
  if (npairs <= 0) return;
  const int th = (max_h + a.tile - 1) / a.tile, tw = (max_w + a.tile - 1) / a.tile;
  const int nt = th * tw;
  k_vec_snap<<<dim3((nt + 63) / 64, npairs), 64, 0, st>>>(d_fields, d_pairs, npairs, a, v.dy, v.dx,
                                                          v.snap_dy, v.snap_dx);
  k_vec_pixels<<<dim3((max_w + 127) / 128, max_h, npairs), 128, 0, st>>>(
      d_fields, d_pairs, npairs, a, v.snap_dy, v.snap_dx, v.src_idx, v.pix_off);
  if (fast_conf) {
    k_conf_sq<<<dim3((nt + 63) / 64, npairs), 64, 0, st>>>(d_fields, d_pairs, npairs, a, v.conf, v.c2);
    k_vec_snap<<<dim3((nt + 63) / 64, npairs), 64, 0, st>>>(d_fields, d_pairs, npairs, a, v.c2, v.c2,
                                                            v.c2_snap, v.c2_snap2);
    k_conf_pixels_fast<<<dim3((max_w + 127) / 128, max_h, npairs), 128, 0, st>>>(
        d_fields, d_pairs, npairs, a, v.c2_snap, v.conf_px, v.pix_off);
  } else {
    k_conf_pixels_nearest<<<dim3((max_w + 127) / 128, max_h, npairs), 128, 0, st>>>(
        d_fields, d_pairs, npairs, a, v.conf, v.conf_tmp, v.pix_off);
    k_pair_blur_v<<<dim3((max_w + kBoxThreads - 1) / kBoxThreads, npairs), kBoxThreads, 0,
                    st>>>(d_fields, d_pairs, npairs,
                                                                     v.conf_tmp, v.conf_px,
                                                                     v.pix_off, 8);
    k_pair_blur_h<<<dim3((max_h + 31) / 32, npairs), 32, 0, st>>>(d_fields, d_pairs, npairs,
                                                                  v.conf_px, v.conf_tmp,
                                                                  v.pix_off, 8);
    cudaMemcpyAsync(v.conf_px, v.conf_tmp, v.conf_bytes, cudaMemcpyDeviceToDevice, st);
  }
}

void launch_traj_snap(const MeField* d_fields, const MePair* d_pairs, const TrajGroup* d_groups,
                      int ngroups, const TrajPair* d_tp, int max_h, int max_w, int tile,
                      int tiles_off, float* dy, float* dx, const float* conf, cudaStream_t st) {
  if (ngroups <= 0) return;
  const int nt = ((max_h + tile - 1) / tile) * ((max_w + tile - 1) / tile);
  k_traj_snap<<<dim3((nt + 63) / 64, ngroups), 64, 0, st>>>(d_fields, d_pairs, d_groups, ngroups,
                                                           d_tp, tile, tiles_off, dy, dx, conf);
}

void launch_traj_verify(const MeField* d_fields, const MePair* d_pairs, int base, int npred,
                        const int* d_grp, const TrajGroup* d_searched, const TrajPair* d_tp,
                        const float* blur, int max_h, int max_w, const MeArgs& a,
                        const float* dy_in, const float* dx_in, float* mdy, float* mdx,
                        float* sdy, float* sdx, float* best, cudaStream_t st,
                        const float* pred_dy, const float* pred_dx) {
  if (npred <= 0) return;
  const int nt = ((max_h + a.tile - 1) / a.tile) * ((max_w + a.tile - 1) / a.tile);
  k_traj_verify<<<dim3((2 * nt + 63) / 64, npred), 64, 0, st>>>(
      d_fields, d_pairs, base, npred, d_grp, d_searched, d_tp, blur, a, dy_in, dx_in, pred_dy,
      pred_dx, mdy, mdx, sdy, sdx, best);
}

void launch_me_confidence(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                          int max_w, const MeArgs& a, const float* blur, const float* mdy,
                          const float* mdx, const float* sdy, const float* sdx, const float* best,
                          float* dy, float* dx, float* conf, cudaStream_t st) {
  if (npairs <= 0) return;
  const int th = (max_h + a.tile - 1) / a.tile, tw = (max_w + a.tile - 1) / a.tile;
  const int smem = 2 * th * tw * (int)sizeof(float);
  k_me_confidence<<<npairs, 256, smem, st>>>(d_fields, d_pairs, npairs, blur, a, mdy, mdx, sdy, sdx,
                                             best, dy, dx, conf);
}

void launch_motion_cache(const int* d_gid, int npairs, int nt, int tiles_off, float* dy, float* dx,
                         float* conf, float* cache, int64_t cache_stride, bool store,
                         cudaStream_t st) {
  if (npairs <= 0) return;
  k_motion_cache<<<dim3((nt + 127) / 128, npairs), 128, 0, st>>>(d_gid, npairs, nt, tiles_off, dy,
                                                                dx, conf, cache, cache_stride,
                                                                store ? 1 : 0);
}

void launch_coherence_gate(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                           int max_w, const MeArgs& a, const CohBuffers& b, float gate,
                           cudaStream_t st) {
  if (npairs <= 0) return;
  const dim3 grid((max_w + 127) / 128, max_h, npairs);
  k_coh_terms<<<grid, 128, 0, st>>>(d_fields, d_pairs, npairs, a, b);
  // ComplexCoherence's four BoxBlur(r = 6) passes (temporal.cpp:186-189)
  for (int c = 0; c < 4; ++c) {
    float* ch = b.terms + c * b.chan_stride;
    k_pair_blur_v<<<dim3((max_w + kBoxThreads - 1) / kBoxThreads, npairs), kBoxThreads, 0,
                    st>>>(d_fields, d_pairs, npairs, ch,
                                                                    b.tmp, b.pix_off, 6);
    k_pair_blur_h<<<dim3((max_h + 31) / 32, npairs), 32, 0, st>>>(d_fields, d_pairs, npairs,
                                                                 b.tmp, ch, b.pix_off, 6);
  }
  k_coh_apply<<<grid, 128, 0, st>>>(d_fields, d_pairs, npairs, b, gate);
}

// ---------------------------------------------------------------------------
// DrizzleFrame (sequence.cpp:283-421). Compiled with the rest of this file
// without multiply-add contraction, so every deposit position, weight and
// blend is the reference's float arithmetic; only the order of the float
// accumulations differs (atomics), i.e. the sums agree to rounding.
// ---------------------------------------------------------------------------

// One thread per (pair, source sample): robust agreement weight with the
// target's own decode at the rounded warp, linear split between the two
// fine rows around (2 (y + vy) + p_k) scale.
__global__ void k_drizzle_deposit(const DrizzlePair* __restrict__ pairs, int npairs, DrizzleArgs a) {
  const int pi = blockIdx.z;
  if (pi >= npairs) return;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= a.w || y >= a.h) return;
  const DrizzlePair pr = pairs[pi];
  const int L = a.h, W = a.w, HF = 2 * L * a.scale;
  float vy = 0.0f, vx = 0.0f, cpx = 1.0f;
  if (pr.me >= 0) {
    const int th = (L + a.tile - 1) / a.tile, tw = (W + a.tile - 1) / a.tile;
    int iy, ix;
    float fy, fx;
    bracket(y, th, a.tile, &iy, &fy);
    bracket(x, tw, a.tile, &ix, &fx);
    const int iy1 = min(iy + 1, th - 1), ix1 = min(ix + 1, tw - 1);
    const int o = a.tiles_off * pr.me;
    vy = interp_tiles(a.sdy + o, tw, iy, iy1, ix, ix1, fy, fx);
    vx = interp_tiles(a.sdx + o, tw, iy, iy1, ix, ix1, fy, fx);
    cpx = a.conf[o + min(y / a.tile, th - 1) * tw + min(x / a.tile, tw - 1)];
  }
  const int64_t plane = (int64_t)L * a.pitch;
  const float* Yk = a.Y + plane * pr.src;
  const float* Yt = a.Y + plane * pr.tgt;
  const float2* Ck = a.C + plane * pr.src;
  const float2* Ct = a.C + plane * pr.tgt;
  const int syi = clampi((int)lroundf((float)y - vy), 0, L - 1);
  const int sxi = clampi((int)lroundf((float)x - vx), 0, W - 1);
  const float sk = Yk[(int64_t)y * a.pitch + x];
  const float2 ck = Ck[(int64_t)y * a.pitch + x];
  const float dY = sk - Yt[(int64_t)syi * a.pitch + sxi];
  const float2 ct = Ct[(int64_t)syi * a.pitch + sxi];
  const float dr = ck.x - ct.x, di = ck.y - ct.y;
  const float d2 = dY * dY + (dr * dr + di * di);
  const float wgt = cpx * a.eps_b * a.eps_b / (d2 + a.eps_b * a.eps_b);
  const float yf = (2.0f * ((float)y + vy) + (float)a.parity[pr.src]) * (float)a.scale;
  const int xs = clampi((int)lroundf((float)x + vx), 0, W - 1);
  const int y0 = (int)floorf(yf);
  const float fyr = yf - (float)y0;
  const int64_t fp = (int64_t)HF * W;
  for (int off = 0; off < 2; ++off) {
    const int yt = clampi(y0 + off, 0, HF - 1);
    const float ww = wgt * (off == 0 ? (1.0f - fyr) : fyr);
    const int64_t q = (int64_t)yt * W + xs;
    atomicAdd(a.acc + q, ww * sk);
    atomicAdd(a.acc + fp + q, ww * ck.x);
    atomicAdd(a.acc + 2 * fp + q, ww * ck.y);
    atomicAdd(a.acc + 3 * fp + q, ww);
  }
}

// Coverage blend with the linearly interpolated plain weave of fields j0,
// j0 + 1 (sequence.cpp:385-419). One thread per fine sample.
__global__ void k_drizzle_resolve(DrizzleArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  const int L = a.h, W = a.w, HF = 2 * L * a.scale;
  if (x >= W || r >= HF) return;
  const int64_t plane = (int64_t)L * a.pitch;
  const int p0 = a.parity[a.j0], p1 = a.parity[a.j0 + 1];
  auto woven = [&](int row, float2* c) {
    // row 2 t + p1 from field j0 + 1 (written last), else 2 t + p0 from j0, else 0
    const int t = row >> 1, par = row & 1;
    const int64_t o = (int64_t)t * a.pitch + x;
    if (par == p1) {
      *c = a.C[plane * (a.j0 + 1) + o];
      return a.Y[plane * (a.j0 + 1) + o];
    }
    if (par == p0) {
      *c = a.C[plane * a.j0 + o];
      return a.Y[plane * a.j0 + o];
    }
    *c = make_float2(0.f, 0.f);
    return 0.0f;
  };
  const float fine = (float)r / (float)a.scale;
  const int f0 = clampi((int)floorf(fine), 0, 2 * L - 2);
  const float ff = fine - (float)f0;
  float2 c0, c1;
  const float y0v = woven(f0, &c0), y1v = woven(f0 + 1, &c1);
  const float baseY = y0v * (1.0f - ff) + y1v * ff;
  const float bcr = c0.x * (1.0f - ff) + c1.x * ff;
  const float bci = c0.y * (1.0f - ff) + c1.y * ff;
  const int64_t fp = (int64_t)HF * W, q = (int64_t)r * W + x;
  const float aw = a.acc[3 * fp + q];
  const float mix = aw / (aw + 0.35f);
  const float den = fmaxf(aw, 1e-9f);
  const float dzY = aw > 0.0f ? a.acc[q] / den : 0.0f;
  const float dcr = aw > 0.0f ? a.acc[fp + q] / den : 0.0f;
  const float dci = aw > 0.0f ? a.acc[2 * fp + q] / den : 0.0f;
  a.out_y[q] = mix * dzY + (1.0f - mix) * baseY;
  a.out_c[q] = make_float2(mix * dcr + (1.0f - mix) * bcr, mix * dci + (1.0f - mix) * bci);
}

void launch_drizzle(const DrizzlePair* d_pairs, int npairs, const DrizzleArgs& a, cudaStream_t st) {
  const int HF = 2 * a.h * a.scale;
  if (npairs > 0)
    k_drizzle_deposit<<<dim3((a.w + 127) / 128, a.h, npairs), 128, 0, st>>>(d_pairs, npairs, a);
  k_drizzle_resolve<<<dim3((a.w + 127) / 128, HF), 128, 0, st>>>(a);
}

void launch_vec_snap(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                     int max_w, const MeArgs& a, const float* dy, const float* dx, float* sdy,
                     float* sdx, cudaStream_t st) {
  if (npairs <= 0) return;
  const int nt = ((max_h + a.tile - 1) / a.tile) * ((max_w + a.tile - 1) / a.tile);
  k_vec_snap<<<dim3((nt + 63) / 64, npairs), 64, 0, st>>>(d_fields, d_pairs, npairs, a, dy, dx,
                                                          sdy, sdx);
}

}  // namespace hvdg
