// k_frame.cu -- de-weave and re-weave of field-sequential int16 frames for
// the woven-frame decode (DecodeFrameBuffer / DecodeYcFrameBuffer,
// frame_bridge.cpp:168-377). Both are one pass over the frame: the split
// reads each source sample once and writes one float; the re-weave writes
// the four output planes of every flat line once. The float arithmetic of
// the level conversions and the requantisation is spelled out with
// round-to-nearest intrinsics so no multiply-add is contracted: the codes
// land on the same side of every rounding boundary as the reference's.
#include <cuda_runtime.h>

#include <algorithm>

#include "hvdg_common.cuh"
#include "k_frame.h"

namespace hvdg {

// SplitFrameFields (frame_bridge.cpp:61-99): field 1 = flat lines [0, f1),
// field 2 = flat lines [f1, fh), lines past field 2's end filled with the
// centre level; ire = (s - centre) / codes_per_ire (SampleToIre,
// ntsc_geometry.h:225-228; the C channel's (c - chroma_dc) / scale,
// frame_bridge.cpp:293-301). Lines are read through FrameLineOffset, so
// PAL's non-orthogonal lines stay registered.
// Slot 0 of a frame takes the block the field order puts on the even woven
// rows, so the weave itself needs no per-frame decision.
__global__ void __launch_bounds__(256) k_frame_split(FrameSplitArgs a) {
  const int row = blockIdx.x;  // (2 t + slot) * f1 + y
  const int q = row / a.f1, y = row - q * a.f1;
  const int t = q >> 1;
  const int swap = a.order == 2 ? (a.vote[t] < 0) : a.order;
  const int k = (q & 1) ^ swap;
  const int flat = k == 0 ? y : a.f1 + y;
  const bool valid = k == 0 ? (y < a.f1) : (flat < a.fh);
  const int16_t* src = a.frames + (int64_t)t * a.frame_stride + (valid ? a.line_off[flat] : 0);
  float* dst = a.fields + (int64_t)q * a.field_stride + (int64_t)y * a.fw;
  for (int x = threadIdx.x; x < a.fw; x += blockDim.x) {
    const float s = valid ? (float)src[x] : a.center;
    dst[x] = __fdiv_rn(__fsub_rn(s, a.center), a.codes_per_ire);
  }
}

// DetectFieldParity on the split fields, read straight from the int16 frame
// with the split's conversion: over field lines r (r0 step ystep) and
// columns x (a0 step 16), b / ac / au / ad = the 4-sample means at x of
// block 2 line r and block 1 lines r, r - 1, r + 1; ep = mean |b - (ac +
// ad) / 2|, em = mean |b - (ac + au) / 2|; undecided when the larger is
// <= 1e-9 or they differ by < 2 % of it, else +1 when ep < em.
//
// The terms are float, computed with the same rounded operations as the
// host's restatement. The host adds them in FP64 in loop order; here the
// `blocks` CTAs of a frame add contiguous slices of them in parallel, and
// the frame's last CTA to finish adds the slices' sums in slice order. Both
// sums of n non-negative terms are within (n - 1) u / (1 - (n - 1) u) of
// the exact one (u = 2^-53, any summation order), so when the parallel
// means sit further than that from every threshold of the decision the
// host's sums decide the same way. Otherwise that CTA re-adds the terms in
// the host's order (kVoteChunk at a time through shared memory, one thread
// adding) and decides on those sums: the decision is the host's in every
// case.
constexpr int kVoteChunk = 2048;
constexpr int kVoteThreads = 256;

__global__ void __launch_bounds__(kVoteThreads) k_frame_vote(FrameVoteArgs a) {
  __shared__ float tp[kVoteChunk], tm[kVoteChunk];
  __shared__ double wsum[2][kVoteThreads / 32];
  __shared__ int role;  // 0: done, 1: decided by the slice sums, 2: re-add in order
  const int t = blockIdx.x / a.blocks, blk = blockIdx.x - t * a.blocks;
  const int16_t* frame = a.frames + (int64_t)t * a.frame_stride;
  const int nt = a.rows * a.cols;
  auto lp = [&](int k, int row, int x) {
    const int flat = k == 0 ? row : a.f1 + row;
    const bool valid = k == 0 ? row < a.f1 : flat < a.fh;
    const int16_t* src = frame + (valid ? a.line_off[flat] + x : 0);
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float s = valid ? (float)src[j] : a.blank;
      const float v = __fdiv_rn(__fsub_rn(s, a.blank), a.codes_per_ire);
      acc = j == 0 ? v : __fadd_rn(acc, v);
    }
    return __fmul_rn(0.25f, acc);
  };
  auto terms = [&](int i, float& p, float& m) {
    const int r = a.r0 + (i / a.cols) * a.ystep;
    const int x = a.a0 + (i % a.cols) * 16;
    const float b = lp(1, r, x), ac = lp(0, r, x), au = lp(0, r - 1, x), ad = lp(0, r + 1, x);
    p = fabsf(__fsub_rn(b, __fmul_rn(0.5f, __fadd_rn(ac, ad))));
    m = fabsf(__fsub_rn(b, __fmul_rn(0.5f, __fadd_rn(ac, au))));
  };
  // means that decide: +1 / -1 / 0
  auto decide = [](double ep, double em) {
    const double lo = fmin(ep, em), hi = fmax(ep, em);
    if (hi <= 1e-9 || __ddiv_rn(__dsub_rn(hi, lo), hi) < 0.02) return 0;
    return ep < em ? 1 : -1;
  };
  // this CTA's slice
  const int per = (nt + a.blocks - 1) / a.blocks;
  const int i0 = blk * per, i1 = min(nt, i0 + per);
  double sp = 0.0, sm = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    float p, m;
    terms(i, p, m);
    sp += (double)p;
    sm += (double)m;
  }
  sp = warp_sum(sp);
  sm = warp_sum(sm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    wsum[0][warp] = sp;
    wsum[1][warp] = sm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bp = 0.0, bm = 0.0;
    for (int w = 0; w < kVoteThreads / 32; ++w) {
      bp += wsum[0][w];
      bm += wsum[1][w];
    }
    a.partial[2 * blockIdx.x] = bp;
    a.partial[2 * blockIdx.x + 1] = bm;
    __threadfence();
    role = atomicAdd(a.arrive + t, 1) == a.blocks - 1 ? 1 : 0;
    if (role) {
      __threadfence();
      double ep = 0.0, em = 0.0;
      for (int k = 0; k < a.blocks; ++k) {
        ep += __ldcg(a.partial + 2 * (t * a.blocks + k));
        em += __ldcg(a.partial + 2 * (t * a.blocks + k) + 1);
      }
      if (nt > 0) {
        ep /= (double)nt;
        em /= (double)nt;
        // relative distance of either sum (after the mean's division) from
        // the exact value, doubled for the two summation orders, with room
        const double tol = 8.0 * ((double)nt + 2.0) * 1.1102230246251565e-16;
        const double lo = fmin(ep, em), hi = fmax(ep, em);
        const bool near_floor = fabs(hi - 1e-9) <= tol * hi;
        const bool near_ratio = hi > 0.0 && fabs((hi - lo) / hi - 0.02) <= 4.0 * tol;
        if (near_floor || near_ratio) role = 2;
        else a.vote[t] = decide(ep, em);
      } else {
        a.vote[t] = 0;
      }
    }
  }
  __syncthreads();
  if (role != 2) return;
  double ep = 0.0, em = 0.0;
  for (int base = 0; base < nt; base += kVoteChunk) {
    const int m = min(kVoteChunk, nt - base);
    for (int j = threadIdx.x; j < m; j += blockDim.x) terms(base + j, tp[j], tm[j]);
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int j = 0; j < m; ++j) {
        ep = __dadd_rn(ep, (double)tp[j]);
        em = __dadd_rn(em, (double)tm[j]);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    a.vote[t] = decide(__ddiv_rn(ep, (double)nt), __ddiv_rn(em, (double)nt));
}

__device__ __forceinline__ int16_t clamp_u10(float v) {  // ClampU10, frame_bridge.cpp:25-28
  const long r = lroundf(v);
  return (int16_t)(r < 0 ? 0 : (r > 1023 ? 1023 : r));
}
__device__ __forceinline__ int16_t clamp_s10(float v) {  // ClampS10, frame_bridge.cpp:36-39
  const long r = lroundf(v);
  return (int16_t)(r < -1023 ? -1023 : (r > 1023 ? 1023 : r));
}

// One CTA per (frame, flat line). Outside the active picture: luma = the
// pass-through source line, chroma / u / v = 0. Inside: woven row
// r = 2 (field_line - fal) + field, with field 0 = flat lines < f1 (the
// re-weave always puts even woven rows on field-1 lines, whichever field the
// weave put there).
__global__ void __launch_bounds__(256) k_frame_out(FrameOutArgs a) {
  const int t = blockIdx.x / a.fh;
  const int line = blockIdx.x - t * a.fh;
  const int64_t o = ((int64_t)t * a.fh + line) * a.fw;
  const int16_t* src = a.passthrough + (int64_t)t * a.frame_stride + a.line_off[line];
  const int field = line < a.f1 ? 0 : 1;
  const int fl = line - field * a.f1;
  const int r = 2 * (fl - a.fal) + field;
  const bool active = fl >= a.fal && r < a.h;
  // ACC gain of this frame (AccGain(0.5 (a_top + a_bot), nominal),
  // colour.cpp:24-27; 1 without ACC), times chroma_gain
  float gain = a.chroma_gain;
  if (a.acc) {
    const float m = __fmul_rn(0.5f, __fadd_rn(a.amp[2 * t], a.amp[2 * t + 1]));
    const float acc = fminf(fmaxf(__fdiv_rn(a.nominal_burst, fmaxf(m, 1.0f)), 0.5f), 2.0f);
    gain = __fmul_rn(a.chroma_gain, acc);
  }
  const int64_t po = (int64_t)t * a.plane_stride + (int64_t)r * a.pitch;
  const float4 L = active ? __ldg(a.line_phasor + (int64_t)t * a.h + r) : make_float4(0, 0, 0, 0);
  for (int x = threadIdx.x; x < a.fw; x += blockDim.x) {
    int16_t yv = src[x], cv = 0;
    double uv = 0.0, vv = 0.0;
    const int c = x - a.a0;
    if (active && c >= 0 && c < a.w) {
      const float2 chi = a.mono ? make_float2(0.f, 0.f) : a.chi[po + c];
      float chroma;
      if (a.yc) {
        const float2 car = carrier(make_float2(L.x, L.y), __ldg(a.col_phasor + c), L.z);
        chroma = __fsub_rn(__fmul_rn(chi.x, car.x), __fmul_rn(chi.y, car.y));
      } else {
        const float luma = a.mono ? a.S[po + c] : a.Y[po + c];
        chroma = __fsub_rn(a.S[po + c], luma);
        yv = clamp_u10(__fadd_rn(a.blank, __fmul_rn(luma, a.scale)));
      }
      cv = clamp_s10(__fmul_rn(chroma, a.scale));
      vv = __dmul_rn(__dmul_rn((double)gain, (double)chi.x), (double)a.scale);
      uv = __dmul_rn(__dmul_rn((double)gain, (double)(-chi.y)), (double)a.scale);
    }
    a.luma[o + x] = yv;
    a.chroma[o + x] = cv;
    a.u[o + x] = uv;
    a.v[o + x] = vv;
  }
}

void launch_frame_split(const FrameSplitArgs& a, int n_frames, cudaStream_t st) {
  const int rows = 2 * n_frames * a.f1;
  if (rows > 0) k_frame_split<<<rows, 256, 0, st>>>(a);
}

int frame_vote_blocks(int terms) {
  return std::max(1, std::min(64, (terms + kVoteThreads - 1) / kVoteThreads));
}

void launch_frame_vote(const FrameVoteArgs& a, int n_frames, cudaStream_t st) {
  if (n_frames <= 0) return;
  cudaMemsetAsync(a.arrive, 0, sizeof(int) * n_frames, st);
  k_frame_vote<<<n_frames * a.blocks, kVoteThreads, 0, st>>>(a);
}

void launch_frame_out(const FrameOutArgs& a, int n_frames, cudaStream_t st) {
  const int rows = n_frames * a.fh;
  if (rows > 0) k_frame_out<<<rows, 256, 0, st>>>(a);
}

}  // namespace hvdg
