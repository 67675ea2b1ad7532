// k_temporal.h -- launchers of the window calibration and neighbour-term
// kernels (k_temporal.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hvdg_internal.h"

namespace hvdg {

// One neighbour term of field `cur`: the motion-compensated field `ref`.
struct NbrPair {
  int ref, cur;
  int slot;  // neighbour plane index of field `cur`
  int odd;   // odd temporal offset (opposite parity): apply the envelope gate
};

struct EnvBuffers {
  float *gmag, *lapmag, *vraw, *traw, *gate;  // planes (field layout)
  float* scratch;                             // per listed field sample buffer
  const int64_t* scratch_off;
  float* floor2;                              // per listed field
};

// Adaptive-strength ambiguity (sequence.cpp:526-646) of the same-parity
// pairs (j, j + stride), j < npairs: per pair the square root of the p95 band
// mean of the demodulation differences (amb), and whether any term was kept
// (ok). E: npairs x nyi x nx doubles of scratch; nyi rows y = 2, 5, ... < h - 2,
// nx columns x = 4, 8, ... with x + 7 < w.
void launch_amb_pairs(const FieldDesc* d_fields, int npairs, int stride, int nyi, int nx,
                      const float* S, const float4* lineph, const float2* colph, float nr_eps,
                      double* E, float* amb, int* ok, cudaStream_t st);
void launch_noise(const FieldDesc* d_fields, int nf, const float* S, float* scratch,
                  const int64_t* scratch_off, float* sigma, cudaStream_t st);
void launch_envelope(const FieldDesc* d_fields, const int* d_list, int n, int max_h, int max_w,
                     const float* Y, const float2* X, const EnvBuffers& e, float e2,
                     float floor_max, cudaStream_t st);
void launch_nbr_assemble(const FieldDesc* d_fields, const NbrPair* d_pairs, int npairs, int max_h,
                         int max_w, const float* S, const float4* line_phasor,
                         const float2* col_phasor, const int2* src_idx, const float* conf_px,
                         const int64_t* pix_off, const float* gate, float4* nbr,
                         cudaStream_t st);

}  // namespace hvdg
