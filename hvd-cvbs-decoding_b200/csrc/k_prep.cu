// k_prep.cu -- field preparation: level conversion + active crop, burst
// lock-in (kernel a), burst amplitude (ACC), carrier phasor tables.
//
// Reference: PrepareFieldObs (hvd-core/src/engine/sequence.cpp:229-268),
// BurstLockin / BurstLockinPhase / BurstLockinPhasePal / BurstAmplitudeIre
// (engine/lockin.cpp:103-417), SampleToIre (engine/ntsc_geometry.h:301-304),
// ApplyChromaPhase (ntsc_geometry.h:341-352).
//
// One CTA per field for the lock-in: the per-line quadrature demodulation is
// a warp-shuffle reduction over the burst window accumulated in FP64; the
// per-field trajectory smoothing (two tridiagonal solves over <= 1024 lines)
// runs as a parallel cyclic reduction over the CTA.
#include <cuda_runtime.h>
#include <math_constants.h>

#include "hvdg_common.cuh"
#include "k_prep.h"
#include "per_device.h"

namespace hvdg {

__device__ __forceinline__ float sample_ire(const PrepDesc& p, int64_t idx) {
  float s;
  if (p.sample_type == 1) {
    s = (float)__ldg(reinterpret_cast<const uint16_t*>(p.samples) + idx);
  } else if (p.sample_type == 2) {
    s = (float)__ldg(reinterpret_cast<const int16_t*>(p.samples) + idx);
  } else {
    return __ldg(reinterpret_cast<const float*>(p.samples) + idx);
  }
  // (s - blanking) / ((white - blanking) / 100): same float operations as
  // SampleToIre / CodesPerIre.
  return __fdiv_rn(__fsub_rn(s, p.blank), p.codes_per_ire);
}

// exp(-i w0 x) in FP64; exact quadrants when w0 == pi/2.
__device__ __forceinline__ double2 lo_phasor(const PrepDesc& p, int x) {
  if (p.quadrant) {
    switch (x & 3) {
      case 0: return make_double2(1.0, 0.0);
      case 1: return make_double2(0.0, -1.0);
      case 2: return make_double2(-1.0, 0.0);
      default: return make_double2(0.0, 1.0);
    }
  }
  double s, c;
  sincos(p.w0 * (double)x, &s, &c);
  return make_double2(c, -s);
}

__device__ __forceinline__ double wrap_pi(double a) { return atan2(sin(a), cos(a)); }

// k-th smallest (0-based) among v[0..n) (doubles in shared memory), exact,
// by rank counting; all threads call; result broadcast through *out.
__device__ void block_rank_select(const double* v, int n, int k, double* out) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double vi = v[i];
    int less = 0, eq = 0;
    for (int j = 0; j < n; ++j) {
      const double vj = v[j];
      less += vj < vi;
      eq += vj == vi;
    }
    if (less <= k && k < less + eq) *out = vi;  // every writer writes the same value
  }
  __syncthreads();
}

// (diag(a) + lam L) x = a d, L the path-graph Laplacian (the end lines have
// one neighbour): TridiagSmooth (lockin.cpp:65-99), which sweeps it
// serially (Thomas). Here by parallel cyclic reduction: every step
// eliminates the neighbours at distance s from each equation at once, so
// after ceil(log2 n) steps each equation holds its own unknown alone. The
// system is symmetric and diagonally dominant (a >= 0, lam > 0), where the
// reduction is stable; the answer differs from the serial sweep by FP64
// rounding only. All threads of the CTA call it. Scratch: two buffers each
// of the lower, diagonal, upper and right-hand-side coefficients.
struct TriScratch {
  double* lo[2];
  double* di[2];
  double* up[2];
  double* rh[2];
};

__device__ void tridiag_smooth(const double* d, const double* a, int n, double lam, double* x,
                               TriScratch t) {
  if (n <= 1) {
    if (n == 1 && threadIdx.x == 0) x[0] = a[0] > 0.0 ? d[0] : 0.0;
    __syncthreads();
    return;
  }
  double *lo = t.lo[0], *di = t.di[0], *up = t.up[0], *rh = t.rh[0];
  double *lo2 = t.lo[1], *di2 = t.di[1], *up2 = t.up[1], *rh2 = t.rh[1];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    lo[i] = i > 0 ? -lam : 0.0;
    up[i] = i < n - 1 ? -lam : 0.0;
    di[i] = a[i] + 2.0 * lam - ((i == 0 || i == n - 1) ? lam : 0.0);
    rh[i] = a[i] * d[i];
  }
  __syncthreads();
  for (int s = 1; s < n; s <<= 1) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int im = i - s, ip = i + s;
      double b = di[i], r = rh[i], l = 0.0, u = 0.0;
      if (im >= 0) {
        const double k1 = lo[i] / di[im];
        b -= up[im] * k1;
        r -= rh[im] * k1;
        l = -lo[im] * k1;
      }
      if (ip < n) {
        const double k2 = up[i] / di[ip];
        b -= lo[ip] * k2;
        r -= rh[ip] * k2;
        u = -up[ip] * k2;
      }
      lo2[i] = l;
      di2[i] = b;
      up2[i] = u;
      rh2[i] = r;
    }
    __syncthreads();
    double* tmp;
    tmp = lo; lo = lo2; lo2 = tmp;
    tmp = di; di = di2; di2 = tmp;
    tmp = up; up = up2; up2 = tmp;
    tmp = rh; rh = rh2; rh2 = tmp;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = rh[i] / di[i];
  __syncthreads();
}

// One CTA per field. blockDim = 256.
__global__ void __launch_bounds__(256) k_burst_lockin(const PrepDesc* __restrict__ descs,
                                                      LockinOut out) {
  const PrepDesc p = descs[blockIdx.x];
  const int h = p.fh;
  extern __shared__ double lk_smem[];
  double* zr = lk_smem;
  double* zi = zr + kMaxLines;
  double* amp = zi + kMaxLines;
  double* d = amp + kMaxLines;
  double* a = d + kMaxLines;
  double* x = a + kMaxLines;
  double* model = x + kMaxLines;
  double* tc = model + kMaxLines;
  double* tdd = tc + kMaxLines;
  double* gbuf = tdd + kMaxLines;
  double* e0 = gbuf + kMaxLines;
  double* e1 = e0 + kMaxLines;
  signed char* good = reinterpret_cast<signed char*>(e1 + kMaxLines);
  signed char* sw = good + kMaxLines;
  __shared__ double s_amax, s_med, s_score[2];
  __shared__ double s_wmax[32];
  __shared__ int s_fg, s_ngood;
  // the smoother's scratch: arrays free once the weights a[] are formed
  const TriScratch tri{{zr, zi}, {amp, tc}, {tdd, gbuf}, {e0, e1}};

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int x0 = p.bx0, x1 = p.bx1, n = max(0, x1 - x0);
  // ---- per-line lock-in: z = mean((seg - mean) * exp(-i w0 x)) -------------
  for (int y = warp; y < h; y += nwarps) {
    double sum = 0.0;
    for (int xx = x0 + lane; xx < x1; xx += 32) sum += (double)sample_ire(p, (int64_t)y * p.fw + xx);
    sum = warp_allsum(sum);
    const double mean = n > 0 ? sum / n : 0.0;
    double ar = 0.0, ai = 0.0;
    for (int xx = x0 + lane; xx < x1; xx += 32) {
      const double v = (double)sample_ire(p, (int64_t)y * p.fw + xx) - mean;
      const double2 ph = lo_phasor(p, xx);
      ar += v * ph.x;
      ai += v * ph.y;
    }
    ar = warp_allsum(ar);
    ai = warp_allsum(ai);
    if (lane == 0) {
      zr[y] = n > 0 ? ar / n : 0.0;
      zi[y] = n > 0 ? ai / n : 0.0;
      amp[y] = sqrt(zr[y] * zr[y] + zi[y] * zi[y]);
    }
  }
  __syncthreads();
  // good lines: amplitude above 20 % of the field's maximum
  {
    double m = 0.0;
    for (int y = threadIdx.x; y < h; y += blockDim.x) m = fmax(m, amp[y]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) s_wmax[warp] = m;
    if (threadIdx.x == 0) {
      s_fg = h;
      s_ngood = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = 0.0;
      for (int w = 0; w < nwarps; ++w) mm = fmax(mm, s_wmax[w]);
      s_amax = mm;
    }
    __syncthreads();
    const double thr = s_amax > 0.0 ? s_amax * 0.2 : 1.0;
    for (int y = threadIdx.x; y < h; y += blockDim.x) {
      good[y] = amp[y] > thr;
      if (good[y]) {
        atomicMin(&s_fg, y);
        // the median below is a rank selection: the order of gbuf is free
        gbuf[atomicAdd(&s_ngood, 1)] = amp[y];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_fg == h) s_fg = -1;
    __syncthreads();
  }
  const int fg = s_fg;
  const double adv = p.adv;
  const double hpi = 0.5 * CUDART_PI;
  const double qpi = 0.25 * CUDART_PI;
  double* theta = model;  // reuse: final theta is written over model at the end

  if (fg < 0) {
    // No burst anywhere: NTSC keeps the raw angles (lockin.cpp:211); PAL uses
    // the model phase with alternating parity (lockin.cpp:348-355).
    for (int y = threadIdx.x; y < h; y += blockDim.x) {
      if (p.vswitch_family) {
        x[y] = adv * y;
        sw[y] = (y % 2 == 0) ? 1 : -1;
      } else {
        x[y] = atan2(zi[y], zr[y]) - hpi;
        sw[y] = 1;
      }
    }
    __syncthreads();
  } else {
    if (!p.vswitch_family) {
      // NTSC (lockin.cpp:198-228)
      const double th_fg = atan2(zi[fg], zr[fg]) - hpi;
      for (int y = threadIdx.x; y < h; y += blockDim.x) {
        const double th = atan2(zi[y], zr[y]) - hpi;
        model[y] = th_fg + adv * (double)(y - fg);
        d[y] = wrap_pi(th - model[y]);
        sw[y] = 1;
      }
    } else {
      // PAL family: two parity hypotheses (lockin.cpp:360-397)
      const double a_fg = atan2(zi[fg], zr[fg]);
      for (int hyp = 0; hyp < 2; ++hyp) {
        const double s_ref = hyp == 0 ? 1.0 : -1.0;
        const double theta_ref = a_fg - hpi + s_ref * qpi;
        double acc = 0.0;
        for (int y = threadIdx.x; y < h; y += blockDim.x) {
          if (!good[y]) continue;
          const double m = theta_ref + adv * (double)(y - fg);
          const bool same = ((y - fg) % 2) == 0;
          const double sy = same ? s_ref : -s_ref;
          const double dev = wrap_pi(atan2(zi[y], zr[y]) - (m + hpi - sy * qpi));
          acc += cos(dev) * amp[y];
        }
        acc = warp_allsum(acc);
        __shared__ double red[32];
        if (lane == 0) red[warp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
          double t = 0.0;
          for (int w = 0; w < nwarps; ++w) t += red[w];
          s_score[hyp] = t;
        }
        __syncthreads();
      }
      // hypothesis 0 wins ties (strict > against an initial -1e30)
      const double s_ref = (s_score[1] > s_score[0]) ? -1.0 : 1.0;
      const double theta_ref = a_fg - hpi + s_ref * qpi;
      for (int y = threadIdx.x; y < h; y += blockDim.x) {
        const double m = theta_ref + adv * (double)(y - fg);
        const bool same = ((y - fg) % 2) == 0;
        const double sy = same ? s_ref : -s_ref;
        model[y] = m;
        sw[y] = sy > 0 ? 1 : -1;
        const double theta_meas = atan2(zi[y], zr[y]) - hpi + sy * qpi;
        d[y] = wrap_pi(theta_meas - m);
      }
    }
    __syncthreads();
    // median good amplitude (upper median, lockin.cpp:85-90) + weights
    block_rank_select(gbuf, s_ngood, s_ngood / 2, &s_med);
    const double med = s_med + 1e-9;
    for (int y = threadIdx.x; y < h; y += blockDim.x)
      a[y] = good[y] ? fmin(fmax(amp[y] / med, 0.0), 2.0) : 0.0;
    __syncthreads();
    tridiag_smooth(d, a, h, 25.0, x, tri);
    // one Huber reweighting, then the final smooth
    for (int y = threadIdx.x; y < h; y += blockDim.x) {
      const double r = fabs(d[y] - x[y]);
      a[y] = a[y] * 0.15 / fmax(r, 0.15);
    }
    __syncthreads();
    tridiag_smooth(d, a, h, 25.0, x, tri);
    for (int y = threadIdx.x; y < h; y += blockDim.x) x[y] = model[y] + x[y];
    __syncthreads();
  }
  // x[] now holds theta. Chroma-phase trim (ApplyChromaPhase).
  for (int y = threadIdx.x; y < h; y += blockDim.x) {
    double th = x[y];
    if (p.chroma_phase_off != 0.0f) {
      const double off = (double)p.chroma_phase_off;
      th += (p.vswitch_family && sw[y] < 0) ? -off : off;
    }
    if (out.theta) out.theta[p.theta_off + y] = (float)th;
    if (out.theta64) out.theta64[p.theta_off + y] = th;
    if (out.vswitch) out.vswitch[p.theta_off + y] = sw[y];
    if (out.line_phasor && y >= p.fal && y < p.lal) {
      double s, c;
      sincos(th, &s, &c);
      out.line_phasor[p.line_off + (y - p.fal) * p.line_step] =
          make_float4((float)c, (float)s, sw[y] < 0 ? -1.0f : 1.0f, 0.0f);
    }
  }
  (void)theta;
}

// BurstAmplitudeIre (lockin.cpp:256-323). One CTA of kAmpThreads per
// field: a warp per line for the per-line envelope medians (a few fields per
// call, so the lines are spread over 32 warps), then the block selects.
constexpr int kAmpThreads = 1024;
__global__ void __launch_bounds__(kAmpThreads) k_burst_amplitude(const PrepDesc* __restrict__ descs,
                                                                 float* __restrict__ amp_out) {
  const PrepDesc p = descs[blockIdx.x];
  const int h = p.fh;
  const int x0 = p.bx0, x1 = p.bx1;
  __shared__ double per_line[kMaxLines];
  __shared__ double env[kAmpThreads / 32][64];
  __shared__ double s_m;
  __shared__ double good[kMaxLines];
  __shared__ int s_ng;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (x1 - x0 < 4) {
    if (threadIdx.x == 0) amp_out[blockIdx.x] = p.nominal_burst;
    return;
  }
  const int nenv = min(x1 - x0 - 3, 64);
  for (int y = warp; y < h; y += nwarps) {
    for (int s = lane; s < nenv; s += 32) {
      double ar = 0.0, ai = 0.0;
      for (int k = 0; k < 4; ++k) {
        const int xx = x0 + s + k;
        const double v = (double)sample_ire(p, (int64_t)y * p.fw + xx);
        const double2 ph = lo_phasor(p, xx);
        ar += v * ph.x;
        ai += v * ph.y;
      }
      env[warp][s] = 2.0 * sqrt(ar * ar + ai * ai) * 0.25;
    }
    __syncwarp();
    // upper median of env[warp][0..nenv) by rank counting within the warp
    const int kq = nenv / 2;
    for (int i = lane; i < nenv; i += 32) {
      const double vi = env[warp][i];
      int less = 0, eq = 0;
      for (int j = 0; j < nenv; ++j) {
        less += env[warp][j] < vi;
        eq += env[warp][j] == vi;
      }
      if (less <= kq && kq < less + eq) per_line[y] = vi;
    }
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x == 0) s_ng = 0;
  block_rank_select(per_line, h, h / 2, &s_m);
  // the lines above a quarter of the median, compacted in any order (the
  // rank select below does not depend on it)
  const double thr = 0.25 * s_m;
  for (int y = threadIdx.x; y < h; y += blockDim.x)
    if (per_line[y] > thr) good[atomicAdd(&s_ng, 1)] = per_line[y];
  __syncthreads();
  if (s_ng == 0) {
    if (threadIdx.x == 0) amp_out[blockIdx.x] = p.nominal_burst;
    return;
  }
  block_rank_select(good, s_ng, s_ng / 2, &s_m);
  if (threadIdx.x == 0) amp_out[blockIdx.x] = (float)s_m;
}

// Active crop + level conversion into the pitched S plane; zero fill of the
// pitch padding; non-finite detection. grid = (rows of all planes); row r
// copies source line rows[r].w of source field rows[r].z into row rows[r].y
// of plane rows[r].x (a field's own active picture, or one line of a woven
// frame).
__global__ void k_crop(const PrepDesc* __restrict__ descs, const int4* __restrict__ rows,
                       float* __restrict__ S, const int64_t* __restrict__ px_off,
                       const int* __restrict__ pitch, int* __restrict__ nonfinite) {
  const int4 rw = rows[blockIdx.x];
  const int f = rw.x;
  const PrepDesc p = descs[rw.z];
  const int w = p.a1 - p.a0;
  float* dst = S + px_off[f] + (int64_t)rw.y * pitch[f];
  const int64_t src = (int64_t)rw.w * p.fw + p.a0;
  for (int x = threadIdx.x; x < pitch[f]; x += blockDim.x) {
    float v = 0.0f;
    if (x < w) {
      v = sample_ire(p, src + x);
      if (!isfinite(v)) atomicOr(nonfinite, 1);
    }
    dst[x] = v;
  }
}

constexpr size_t kLockinSmem = 12 * kMaxLines * sizeof(double) + 2 * kMaxLines;

static void configure_prep_kernels_now() {
  cudaFuncSetAttribute(k_burst_lockin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kLockinSmem);
}

// The lock-in kernel's shared-memory opt-in, once per device.
void configure_prep_kernels() {
  static PerDeviceOnce once;
  once(configure_prep_kernels_now);
}

void launch_burst_lockin(const PrepDesc* d_descs, int n, LockinOut out, cudaStream_t st) {
  configure_prep_kernels();
  if (n > 0) k_burst_lockin<<<n, 256, kLockinSmem, st>>>(d_descs, out);
}
void launch_burst_amplitude(const PrepDesc* d_descs, int n, float* d_amp, cudaStream_t st) {
  if (n > 0) k_burst_amplitude<<<n, kAmpThreads, 0, st>>>(d_descs, d_amp);
}
void launch_crop(const PrepDesc* d_descs, const int4* d_rows, int total_rows, float* d_S,
                 const int64_t* d_px_off, const int* d_pitch, int* d_nonfinite, cudaStream_t st) {
  if (total_rows > 0)
    k_crop<<<total_rows, 256, 0, st>>>(d_descs, d_rows, d_S, d_px_off, d_pitch, d_nonfinite);
}

}  // namespace hvdg
