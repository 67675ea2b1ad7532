// k_adjoint.h -- kernels of the decode adjoint (gradients of a loss on the
// decoded Y / chi with respect to the field samples and the regulariser
// scalars). No reference counterpart: the reference has no adjoint.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hvdg {

// One field's active planes (row pitch `pitch`) and carrier tables.
struct AdjGeom {
  int h, w, pitch;
  int hp, pad;                // init rows incl. the reflect pad
  const float4* line_phasor;  // active lines (cos, sin, sign, 0)
  const float2* col_phasor;   // active columns
};

struct AdjScalars {
  float eps, eps_c, k;        // charbonnier_eps, chroma_eps, structure_coupling
  float mu_h, mu_v;           // chroma prior weights (mu_h = lambda_c * aniso)
  float aniso;                // d mu_h / d lambda_c (mu_v = lambda_c)
};

// Per-outer planes of the backward pass.
struct AdjOuter {
  const float* S;             // active composite
  const float2* lam;          // H^-1 (sigma chibar), scaled by 1 / sigma below
  float inv_sigma;
  const float2* chi1;         // chi_{o+1}
  const float2* chi0;         // chi_o
  const float4* W;            // the forward's weights at chi_o
  float2* P;                  // (wx Dx r, wy Dy r), r = Re(lambda c)
  float2* GB;                 // (gbar_x, gbar_y): cotangents of Dx Yc_o, Dy Yc_o
  float2* A1;                 // 2 mbar_x Dx chi_o
  float2* A2;                 // 2 mbar_y Dy chi_o
  double* partials;           // per block: lambda_c, eps, eps_c, k
};

constexpr int kAdjBlock = 256;
int adj_blocks(const AdjGeom& g);

// chibar -= ybar conj(c), sbar = ybar (the output luma Y = S - Re[chi c]).
void launch_adj_output(const AdjGeom& g, const float* ybar, float* sbar, float2* chibar,
                       cudaStream_t st);
// per-block sums of |chibar|^2 (fixed order) -> partials[blocks]
void launch_adj_norm(const AdjGeom& g, const float2* chibar, double* partials, cudaStream_t st);
// B = -sigma chibar
void launch_adj_rhs(const AdjGeom& g, const float2* chibar, float sigma, float2* B,
                    cudaStream_t st);
// the per-outer backward step: pass A (pointwise cotangents + scalar
// partials), the fixed-order scalar reduction into acc[4], pass B (sbar +=,
// chibar = cotangent of chi_o)
void launch_adj_outer(const AdjGeom& g, const AdjScalars& sc, const AdjOuter& o, double* acc,
                      float* sbar, float2* chibar, cudaStream_t st);

// HolographicInit adjoint, pointwise / stencil parts.
struct AdjInit {
  const float* S;
  const float2* chi1;         // the two filtered variants (forward)
  const float2* chi2;
  const float2* chi0bar;      // cotangent of chi0
  float2* a;                  // (|Dx y1| + |Dy y1|, ... y2) then box-blurred in place -> E
  float2* tmp;                // box scratch
  float2* ebar;               // cotangents of E (then box-blurred -> abar)
  float2* cb1;                // chi0bar w1 / W
  float2* cb2;
  float2* adj_in;             // 2 x hp x pitch: the filter-pass inputs (pad rows zero)
};
void launch_adj_init_pointwise(const AdjGeom& g, const AdjInit& a, float* sbar, cudaStream_t st);
// sbar += Re(fold(u1 + u2) c), fold = transpose of the reflect-101 row pad
void launch_adj_fold(const AdjGeom& g, const float2* adj_out, float* sbar, cudaStream_t st);
// samples_bar (fh x fw, dense) = sbar / codes_per_ire on the active window, 0 elsewhere
void launch_adj_samples(const AdjGeom& g, const float* sbar, float inv_cpi, int fh, int fw,
                        int fal, int a0, float* samples_bar, cudaStream_t st);

}  // namespace hvdg
