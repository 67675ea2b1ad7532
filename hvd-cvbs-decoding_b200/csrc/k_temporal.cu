// k_temporal.cu -- per-window calibration and neighbour-term assembly of the
// 3-D (temporal) field decode.
//
// Reference: DecodeFieldWindowWithInits (hvd-core/src/engine/sequence.cpp):
//   * noise self-calibration, EstimateNoiseIre (engine/ntsc_geometry.cpp:49-71)
//     -> temporal_eps / nr_eps (sequence.cpp:437-449);
//   * the odd-offset half-line envelope gate (sequence.cpp:797-932, 1000-1026):
//     vertical gradient / second-difference envelopes of the current (Y, chi),
//     row-smoothed, median noise floor, per-pixel extremum factor;
//   * MotionCompensatePrev (engine/temporal.cpp:258-287): integer warp of the
//     neighbour's raw composite and carrier, confidence upsample, and the
//     carrier delta dc = c - c_w the solver's data term uses
//     (variational.cpp:255-267).
// Compiled without FMA contraction, like the motion kernels, so the float
// arithmetic follows the reference's order.
#include <cuda_runtime.h>

#include "hvdg_common.cuh"
#include "k_temporal.h"

namespace hvdg {

// ---- EstimateNoiseIre: one CTA (1024 threads) per field ---------------------
__global__ void __launch_bounds__(1024) k_noise(const FieldDesc* __restrict__ fields,
                                                const float* __restrict__ S,
                                                float* __restrict__ scratch,
                                                const int64_t* __restrict__ scratch_off,
                                                float* __restrict__ sigma) {
  __shared__ unsigned hist[256];
  __shared__ unsigned bc[2];
  const FieldDesc f = fields[blockIdx.x];
  const int w = f.w, h = f.h;
  if (w <= 8 || h <= 0) {
    if (threadIdx.x == 0) sigma[blockIdx.x] = 0.0f;
    return;
  }
  const int nx = w - 8;
  const int n = h * nx;
  float* d = scratch + scratch_off[blockIdx.x];
  const float* s = S + f.px_off;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int y = i / nx, x = i % nx;
    const float* r = s + (int64_t)y * f.pitch;
    d[i] = r[x] - 2.0f * r[x + 4] + r[x + 8];
  }
  __syncthreads();
  const float med = block_select_kth(d, n, n / 2, hist, bc);
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = fabsf(d[i] - med);
  __syncthreads();
  const float q = block_select_kth(d, n, n / 4, hist, bc);
  if (threadIdx.x == 0) sigma[blockIdx.x] = q / 0.3186f / sqrtf(6.0f);
}

// ---- envelope gate --------------------------------------------------------------
// (1) vertical one-sided gradient magnitude and second difference of (Y, chi)
__global__ void k_env_maps(const FieldDesc* __restrict__ fields, const int* __restrict__ list,
                           const float* __restrict__ Y, const float2* __restrict__ X,
                           float* __restrict__ gmag, float* __restrict__ lapmag) {
  const FieldDesc f = fields[list[blockIdx.z]];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int ym = y > 0 ? y - 1 : 0, yp = y + 1 < f.h ? y + 1 : f.h - 1;
  const float* Yf = Y + f.px_off;
  const float2* C = X + f.px_off;
  const int64_t o = (int64_t)y * f.pitch + x, om = (int64_t)ym * f.pitch + x,
                op = (int64_t)yp * f.pitch + x;
  const float dyu = Yf[o] - Yf[om];
  const float dyd = Yf[op] - Yf[o];
  const float dcu = sqrtf(cnorm(csub(C[o], C[om])));
  const float dcd = sqrtf(cnorm(csub(C[op], C[o])));
  const float mu = dyu * dyu + dcu * dcu;
  const float md = dyd * dyd + dcd * dcd;
  gmag[f.px_off + o] = fmaxf(mu, md);
  const float ly = Yf[o] - 0.5f * (Yf[om] + Yf[op]);
  const float2 avg = cscale(cadd(C[om], C[op]), 0.5f);
  const float lc = sqrtf(cnorm(csub(C[o], avg)));
  lapmag[f.px_off + o] = ly * ly + lc * lc;
}

// (2) smooth_rows (sequence.cpp:860-889): sliding sum over [x-2, x+2] clipped
// to the row, sqrt(mean), both maps. The running sums: one warp per (field,
// 32-row band, map): lane l runs row l's in-order float running sum (the
// same additions and subtractions in column order); the band's samples
// arrive 32 columns (plus the window's 3 / 2 columns either side) at a time
// through shared memory, one coalesced row segment per load instruction, and
// the sums leave the same way. The tile's rows are 41 floats apart, so a
// lane's reads along its row hit a different bank from every other lane's.
// The means and square roots, off the chain, follow in k_env_sqrt.
__global__ void k_env_smooth(const FieldDesc* __restrict__ fields, const int* __restrict__ list,
                             const float* __restrict__ gmag, const float* __restrict__ lapmag,
                             float* __restrict__ vraw, float* __restrict__ traw) {
  __shared__ float tile[32][41];
  const FieldDesc f = fields[list[blockIdx.y]];
  const int y0 = blockIdx.x * 32;
  if (y0 >= f.h) return;
  const int lane = threadIdx.x & 31;
  const int rows = min(32, f.h - y0);
  const bool live = lane < rows;
  const int ww = f.w;
  const int m = blockIdx.z;
  const float* src = (m == 0 ? gmag : lapmag) + f.px_off + (int64_t)y0 * f.pitch;
  float* out = (m == 0 ? vraw : traw) + f.px_off + (int64_t)y0 * f.pitch;
  float acc = 0.0f;
  if (live)
    for (int x = 0; x < (ww < 3 ? ww : 3); ++x) acc += src[(int64_t)lane * f.pitch + x];
  for (int c0 = 0; c0 < ww; c0 += 32) {
    // columns c0 - 3 .. c0 + 34 of every row of the band
    {
      // all loads issued before the first store
      float v[32], e[32];
      const int col = c0 - 3 + lane, col2 = c0 + 29 + lane;  // second pass: lanes 0-5
      const bool in1 = col >= 0 && col < ww, in2 = lane < 6 && col2 < ww;
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        v[q] = in1 && q < rows ? src[(int64_t)q * f.pitch + col] : 0.0f;
        e[q] = in2 && q < rows ? src[(int64_t)q * f.pitch + col2] : 0.0f;
      }
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        tile[q][lane] = v[q];
        if (lane < 6) tile[q][32 + lane] = e[q];
      }
    }
    __syncwarp();
    const int mm = min(32, ww - c0);  // columns of this chunk
    // column j reads tile columns j and j + 5 and then holds its running
    // sum in column j (no later column reads it)
    for (int j = 0; j < mm; ++j) {
      const int x = c0 + j;
      if (x > 0) {
        if (x + 2 < ww) acc += tile[lane][j + 5];
        if (x - 3 >= 0) acc -= tile[lane][j];
      }
      tile[lane][j] = acc;
    }
    __syncwarp();
#pragma unroll 4
    for (int q = 0; q < rows; ++q)
      if (lane < mm) out[(int64_t)q * f.pitch + c0 + lane] = tile[q][lane];
    __syncwarp();
  }
}

// (2b) the running sums to sqrt(sum / taps), taps = |[x-2, x+2] clipped to
// the row|, both maps, one thread per pixel
__global__ void k_env_sqrt(const FieldDesc* __restrict__ fields, const int* __restrict__ list,
                           float* __restrict__ vraw, float* __restrict__ traw) {
  const FieldDesc f = fields[list[blockIdx.z]];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int lo = x - 2, hi = x + 2;
  const int n_taps = (hi < f.w - 1 ? hi : f.w - 1) - (lo > 0 ? lo : 0) + 1;
  const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
  vraw[o] = sqrtf(vraw[o] / (float)n_taps);
  traw[o] = sqrtf(traw[o] / (float)n_taps);
}

// (3) median of every 7th envelope value (flat row-major index), per field
__global__ void __launch_bounds__(1024) k_env_floor(const FieldDesc* __restrict__ fields,
                                                    const int* __restrict__ list,
                                                    const float* __restrict__ vraw,
                                                    float* __restrict__ scratch,
                                                    const int64_t* __restrict__ scratch_off,
                                                    float* __restrict__ floor2) {
  __shared__ unsigned hist[256];
  __shared__ unsigned bc[2];
  const int fi = list[blockIdx.x];
  const FieldDesc f = fields[fi];
  const int64_t total = (int64_t)f.h * f.w;
  const int n = (int)((total + 6) / 7);
  float* smp = scratch + scratch_off[blockIdx.x];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int64_t flat = (int64_t)i * 7;
    const int y = (int)(flat / f.w), x = (int)(flat % f.w);
    smp[i] = vraw[f.px_off + (int64_t)y * f.pitch + x];
  }
  __syncthreads();
  // MedianOf (sequence.cpp:29-39): mean of the two middles for even n
  float med = 0.0f;
  if (n > 0) {
    med = block_select_kth(smp, n, n / 2, hist, bc);
    if (n % 2 == 0) {
      const float lo = block_select_kth(smp, n, n / 2 - 1, hist, bc);
      med = 0.5f * (med + lo);
    }
  }
  if (threadIdx.x == 0) floor2[blockIdx.x] = 2.25f * med * med;
}

// (4) floored envelope, extremum factor, final odd-offset gate
//     gate = max(floor_max * (1 - t^2), e2 / (e2 + b^2))
__global__ void k_env_gate(const FieldDesc* __restrict__ fields, const int* __restrict__ list,
                           const float* __restrict__ vraw, const float* __restrict__ traw,
                           const float* __restrict__ floor2, float e2, float floor_max,
                           float* __restrict__ gate) {
  const FieldDesc f = fields[list[blockIdx.z]];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
  const float v = vraw[o];
  const float g = sqrtf(fmaxf(0.0f, v * v - floor2[blockIdx.z]));
  const float t = g > 1e-6f ? fminf(fmaxf(traw[o] / g, 0.0f), 1.0f) : 0.0f;
  const float lapsm = 1.0f - t * t;
  const float floor_i = floor_max * lapsm;
  gate[o] = fmaxf(floor_i, e2 / (e2 + g * g));
}

// ---- neighbour planes -----------------------------------------------------------
// For each pair (ref = neighbour k, cur = field j) and pixel of j:
//   S_w = S_k[sy][sx], c_w = c_k(sy, sx)   (WarpByTiles / WarpByTilesComplex)
//   plane = (S_w - S_j, Re dc, Im dc, conf [* odd gate]),  dc = c_j - c_w
__global__ void k_nbr_assemble(const FieldDesc* __restrict__ fields,
                               const NbrPair* __restrict__ pairs, const float* __restrict__ S,
                               const float4* __restrict__ line_phasor,
                               const float2* __restrict__ col_phasor,
                               const int2* __restrict__ src_idx, const float* __restrict__ conf_px,
                               const int64_t* __restrict__ pix_off, const float* __restrict__ gate,
                               float4* __restrict__ nbr) {
  const NbrPair pr = pairs[blockIdx.z];
  const FieldDesc fj = fields[pr.cur];
  const FieldDesc fk = fields[pr.ref];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= fj.w || y >= fj.h) return;
  const int64_t o = (int64_t)y * fj.pitch + x;
  const int2 si = src_idx[pix_off[blockIdx.z] + o];
  const float sw = S[fk.px_off + (int64_t)si.x * fk.pitch + si.y];
  const float4 Lk = line_phasor[fk.line_off + si.x];
  const float2 cw = carrier(make_float2(Lk.x, Lk.y), col_phasor[fk.col_off + si.y], Lk.z);
  const float4 Lj = line_phasor[fj.line_off + y];
  const float2 cj = carrier(make_float2(Lj.x, Lj.y), col_phasor[fj.col_off + x], Lj.z);
  const float2 dc = csub(cj, cw);
  float cf = conf_px[pix_off[blockIdx.z] + o];
  if (pr.odd) cf *= gate[fj.px_off + o];
  nbr[fj.nbr_off + (int64_t)pr.slot * fj.plane_px + o] =
      make_float4(sw - S[fj.px_off + o], dc.x, dc.y, cf);
}

// ---- adaptive temporal strength (sequence.cpp:526-646) ----------------------
// Same-parity pair (j, j + stride): at y = 2, 5, 8, ... < h - 2 and x = 4, 8,
// ... with x + 7 < w, the 4-sample means of the two fields; where they agree
// within nr_eps, the triangle-7 demodulation of each field by its carrier and
// e = |d_j - d_k|^2 / 4. The float operations are the reference's, one by
// one and in its order (this translation unit is compiled without FMA
// contraction), so every skip decision and every e is the reference
// restatement's. E holds e (or -1 where skipped) per pair, row, column.
__global__ void k_amb_terms(const FieldDesc* __restrict__ fields, int stride, int nyi, int nx,
                            const float* __restrict__ S, const float4* __restrict__ lineph,
                            const float2* __restrict__ colph, float nr_eps,
                            double* __restrict__ E) {
  const int xi = blockIdx.x * blockDim.x + threadIdx.x;
  const int yi = blockIdx.y, j = blockIdx.z;
  if (xi >= nx) return;
  const FieldDesc fj = fields[j], fk = fields[j + stride];
  const int y = 2 + 3 * yi, x = 4 + 4 * xi;
  const float* Sj = S + fj.px_off + (int64_t)y * fj.pitch;
  const float* Sk = S + fk.px_off + (int64_t)y * fk.pitch;
  double e = -1.0;
  float mj = 0.f, mk = 0.f;
  for (int q = 0; q < 4; ++q) {
    mj += Sj[x + q];
    mk += Sk[x + q];
  }
  if (!(fabsf(mj - mk) * 0.25f > nr_eps)) {
    const float kW[7] = {1.f, 2.f, 3.f, 4.f, 3.f, 2.f, 1.f};
    auto demod = [&](const FieldDesc& f, const float* Sf) {
      const float4 L = lineph[f.line_off + y];
      float dr = 0.f, di = 0.f;
      for (int q = 0; q < 7; ++q) {
        const float sv = kW[q] * Sf[x + q];
        const float2 c = carrier(make_float2(L.x, L.y), colph[f.col_off + x + q], L.z);
        dr += sv * c.x;
        di += -sv * c.y;
      }
      return make_float2(dr * (1.0f / 16.0f), di * (1.0f / 16.0f));
    };
    const float2 dj = demod(fj, Sj), dk = demod(fk, Sk);
    const float er = dj.x - dk.x, ei = dj.y - dk.y;
    e = 0.25 * (double)(er * er + ei * ei);
  }
  E[((int64_t)j * nyi + yi) * nx + xi] = e;
}

// One warp per pair: the band sums in row order (bands of 8 rows, one lane
// each), the p95 of the band means over bands of >= 8 terms (or the mean of
// all terms, summed in row order, when no band has 8), its square root.
constexpr int kAmbMaxBands = 64;
__global__ void __launch_bounds__(32) k_amb_pairs(int nyi, int nx, const double* __restrict__ E,
                                                  float* __restrict__ amb, int* __restrict__ ok) {
  const int j = blockIdx.x, lane = threadIdx.x;
  const double* Ej = E + (int64_t)j * nyi * nx;
  const int nbands = min((nyi + 7) / 8, kAmbMaxBands);
  __shared__ double bacc[kAmbMaxBands];
  __shared__ int bn[kAmbMaxBands];
  for (int b = lane; b < nbands; b += 32) {
    double a = 0.0;
    int n = 0;
    for (int yi = 8 * b; yi < min(8 * b + 8, nyi); ++yi) {
      const double* r = Ej + (int64_t)yi * nx;
      int xi = 0;
      // 16 terms' loads in flight, then their additions in column order
      for (; xi + 16 <= nx; xi += 16) {
        double v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = r[xi + q];
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (v[q] >= 0.0) {
            a += v[q];
            ++n;
          }
      }
      for (; xi < nx; ++xi)
        if (r[xi] >= 0.0) {
          a += r[xi];
          ++n;
        }
    }
    bacc[b] = a;
    bn[b] = n;
  }
  __syncwarp();
  if (lane != 0) return;
  int ntot = 0;
  for (int b = 0; b < nbands; ++b) ntot += bn[b];
  float a = 0.f;
  if (ntot > 0) {
    float brms[kAmbMaxBands];
    int nb = 0;
    for (int b = 0; b < nbands; ++b)
      if (bn[b] >= 8) brms[nb++] = (float)(bacc[b] / (double)bn[b]);
    if (nb > 0) {
      const int k95 = min(nb - 1, (int)(0.95 * (double)nb));
      float v = brms[0];
      for (int i = 0; i < nb; ++i) {
        int less = 0, eq = 0;
        for (int t = 0; t < nb; ++t) {
          less += brms[t] < brms[i];
          eq += brms[t] == brms[i];
        }
        if (less <= k95 && k95 < less + eq) v = brms[i];
      }
      a = sqrtf(v);
    } else {
      double acc = 0.0;
      for (int64_t i = 0; i < (int64_t)nyi * nx; ++i)
        if (Ej[i] >= 0.0) acc += Ej[i];
      a = sqrtf((float)(acc / (double)ntot));
    }
  }
  amb[j] = a;
  ok[j] = ntot > 0;
}

void launch_amb_pairs(const FieldDesc* d_fields, int npairs, int stride, int nyi, int nx,
                      const float* S, const float4* lineph, const float2* colph, float nr_eps,
                      double* E, float* amb, int* ok, cudaStream_t st) {
  if (npairs <= 0 || nyi <= 0 || nx <= 0) return;
  k_amb_terms<<<dim3((nx + 127) / 128, nyi, npairs), 128, 0, st>>>(d_fields, stride, nyi, nx, S,
                                                                   lineph, colph, nr_eps, E);
  k_amb_pairs<<<npairs, 32, 0, st>>>(nyi, nx, E, amb, ok);
}

void launch_noise(const FieldDesc* d_fields, int nf, const float* S, float* scratch,
                  const int64_t* scratch_off, float* sigma, cudaStream_t st) {
  if (nf > 0) k_noise<<<nf, 1024, 0, st>>>(d_fields, S, scratch, scratch_off, sigma);
}

void launch_envelope(const FieldDesc* d_fields, const int* d_list, int n, int max_h, int max_w,
                     const float* Y, const float2* X, const EnvBuffers& e, float e2,
                     float floor_max, cudaStream_t st) {
  if (n <= 0) return;
  k_env_maps<<<dim3((max_w + 127) / 128, max_h, n), 128, 0, st>>>(d_fields, d_list, Y, X, e.gmag,
                                                                   e.lapmag);
  k_env_smooth<<<dim3((max_h + 31) / 32, n, 2), 32, 0, st>>>(d_fields, d_list, e.gmag, e.lapmag,
                                                             e.vraw, e.traw);
  k_env_sqrt<<<dim3((max_w + 127) / 128, max_h, n), 128, 0, st>>>(d_fields, d_list, e.vraw,
                                                                   e.traw);
  k_env_floor<<<n, 1024, 0, st>>>(d_fields, d_list, e.vraw, e.scratch, e.scratch_off, e.floor2);
  k_env_gate<<<dim3((max_w + 127) / 128, max_h, n), 128, 0, st>>>(
      d_fields, d_list, e.vraw, e.traw, e.floor2, e2, floor_max, e.gate);
}

void launch_nbr_assemble(const FieldDesc* d_fields, const NbrPair* d_pairs, int npairs, int max_h,
                         int max_w, const float* S, const float4* line_phasor,
                         const float2* col_phasor, const int2* src_idx, const float* conf_px,
                         const int64_t* pix_off, const float* gate, float4* nbr,
                         cudaStream_t st) {
  if (npairs <= 0) return;
  k_nbr_assemble<<<dim3((max_w + 127) / 128, max_h, npairs), 128, 0, st>>>(
      d_fields, d_pairs, S, line_phasor, col_phasor, src_idx, conf_px, pix_off, gate, nbr);
}

}  // namespace hvdg
