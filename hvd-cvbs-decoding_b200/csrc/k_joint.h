// k_joint.h -- the anchored pass of the 3-D window: reference synthesis
// (SynthReference, hvd-core/src/engine/sequence.cpp:52-150) and the joint
// Y / chi IRLS + CG solve (VariationalRefineJoint, variational.cpp:558-891).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hvdg_internal.h"

namespace hvdg {

// Per-field CG control of the joint solve.
struct JointCtl {
  double gg, gg0;
  float alpha, beta;
  int pending, sel, done, iters;
};

constexpr int kJointMaxNbr = 8;

struct JointArgs {
  const FieldDesc* fields;     // batch descriptors (geometry, budget, mu, nbr planes)
  const int* flist;            // fields of this colour
  int nfl;
  int bx, by;                  // grid tiles per field (partials per field = bx * by)
  const float* S;
  const float4* line_phasor;
  const float2* col_phasor;
  const float4* nbr;           // (S_w - S, Re dc, Im dc, conf) per neighbour slot
  float nu, eps_t;             // temporal strength / robust scale
  const float* Ya;             // anchor luma / chroma / weight (per field planes)
  const float2* Ca;
  const float* Wa;
  float nu_a;
  float eps, eps_c, k;         // Charbonnier scales, structure coupling
  float4* X;                   // (Y, Re chi, Im chi, 0)
  float4* G[2];
  float4* D[2];
  float4* Q[2];
  float4* W;                   // (wx, wy, mu_h wcx, mu_v wcy), prior-scaled
  float4* W2;                  // (mu_d wd1, mu_d wd2, -, -), prior-scaled: the oriented
                               // chroma prior, when diag is set
  int diag;                    // the fields carry the oriented prior (mu_d > 0)
  float4* M0;                  // (m00, m01, m02, m11)
  float4* M1;                  // (m12, m22, b0, b1)
  float* M2;                   // b2
  double* partials;            // per field, per block: 5 values
  JointCtl* ctl;               // per batch field
};

// x = (Y, chi) from the planes; per-field control reset.
void launch_joint_load(const JointArgs& a, const float* Y, const float2* chi, int max_h, int max_w,
                       cudaStream_t st);
// one IRLS outer: weights, data matrix, gradient, then n_inner fused CG sweeps
void launch_joint_outer(const JointArgs& a, int n_inner, int max_h, int max_w, cudaStream_t st);
// the planes from x: Y (free, or S - Re[chi c] with output_fidelity) and chi
void launch_joint_store(const JointArgs& a, float* Y, float2* chi, bool output_fidelity,
                        int max_h, int max_w, cudaStream_t st);
// output fidelity (sequence.cpp:1102-1114): Y = S - Re[chi c] for the fields
// of a.flist
void launch_output_fidelity(const JointArgs& a, float* Y, const float2* chi, int max_h, int max_w,
                            cudaStream_t st);

// SynthReference: Geman-McClure motion-compensated blend of the decoded
// neighbours within nr_radius (bilinear warps with the half-line parity
// row offset), composite-domain confidence of the blend.
struct AnchorPair {
  int pair;                    // index into the colour's pair tables
  int k;                       // neighbour field
  float row_off;               // (p_j - p_k) / 2
};
struct AnchorGroup {
  int field;                   // j
  int count;
  AnchorPair p[kJointMaxNbr];
};
struct AnchorArgs {
  const FieldDesc* fields;
  const AnchorGroup* groups;
  int ngroups;
  int tile, tiles_off;         // per-pair tile arrays
  const float* snap_dy;        // VectorsPerPixel tiles (3x3-median snapped)
  const float* snap_dx;
  const float* conf_px;        // UpsampleConfidence per pair (pix_off)
  const int64_t* pix_off;
  const float* Y;              // current luma / chi states (batch planes)
  const float2* chi;
  const float* S;
  const float4* line_phasor;
  const float2* col_phasor;
  float eps_b;                 // nr_eps
  float* Ya;                   // outputs (batch planes)
  float2* Ca;
  float* Wa;
  float* resid;                // scratch plane (batch)
};
void launch_anchor(const AnchorArgs& a, int max_h, int max_w, cudaStream_t st);

// PsiClosedForm (sequence.cpp:160-227): per pixel, the weighted normal
// equations of the field's own observation and its motion-compensated
// neighbours (an N-step phase-shifting set) solved in closed form, blended
// with the current chi by the neighbours' total confidence. Overwrites chi
// of the fields in a.flist that have neighbour planes.
void launch_psi_init(const JointArgs& a, float2* chi, int max_h, int max_w, cudaStream_t st);

}  // namespace hvdg
