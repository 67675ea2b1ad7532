// k_frame.cu -- de-weave and re-weave of field-sequential int16 frames for
// the woven-frame decode (DecodeFrameBuffer / DecodeYcFrameBuffer,
// frame_bridge.cpp:168-377). Both are one pass over the frame: the split
// reads each source sample once and writes one float; the re-weave writes
// the four output planes of every flat line once. The float arithmetic of
// the level conversions and the requantisation is spelled out with
// round-to-nearest intrinsics so no multiply-add is contracted: the codes
// land on the same side of every rounding boundary as the reference's.
#include <cuda_runtime.h>

#include "hvdg_common.cuh"
#include "k_frame.h"

namespace hvdg {

// SplitFrameFields (frame_bridge.cpp:61-99): field 1 = flat lines [0, f1),
// field 2 = flat lines [f1, fh), lines past field 2's end filled with the
// centre level; ire = (s - centre) / codes_per_ire (SampleToIre,
// ntsc_geometry.h:225-228; the C channel's (c - chroma_dc) / scale,
// frame_bridge.cpp:293-301). Lines are read through FrameLineOffset, so
// PAL's non-orthogonal lines stay registered.
__global__ void __launch_bounds__(256) k_frame_split(FrameSplitArgs a) {
  const int row = blockIdx.x;  // (2 t + k) * f1 + y
  const int q = row / a.f1, y = row - q * a.f1;
  const int t = q >> 1, k = q & 1;
  const int flat = k == 0 ? y : a.f1 + y;
  const bool valid = k == 0 ? (y < a.f1) : (flat < a.fh);
  const int16_t* src = a.frames + (int64_t)t * a.frame_stride + (valid ? a.line_off[flat] : 0);
  float* dst = a.fields + (int64_t)q * a.field_stride + (int64_t)y * a.fw;
  for (int x = threadIdx.x; x < a.fw; x += blockDim.x) {
    const float s = valid ? (float)src[x] : a.center;
    dst[x] = __fdiv_rn(__fsub_rn(s, a.center), a.codes_per_ire);
  }
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

void launch_frame_out(const FrameOutArgs& a, int n_frames, cudaStream_t st) {
  const int rows = n_frames * a.fh;
  if (rows > 0) k_frame_out<<<rows, 256, 0, st>>>(a);
}

}  // namespace hvdg
