// k_solver.h -- launcher of the persistent IRLS + CG kernel (k_solver.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hvdg_internal.h"

namespace hvdg {

constexpr int kSolverThreads = 256;
// Units of a field arrive in groups of kGroupUnits consecutive units: the
// last unit of a group sums the group's partials, the last group the field's.
constexpr int kGroupShift = 5;
constexpr int kGroupUnits = 1 << kGroupShift;
enum PhaseKind { kPhaseR = 0, kPhaseG = 1, kPhaseI = 2, kPhaseF = 3 };

struct SolverArgs {
  const FieldDesc* fields;
  FieldCtl* ctl;
  const Unit* units;
  int unit_base;                // this launch processes units[unit_base, unit_base + n_units)
  int n_units;                  // units per phase (fields of this launch)
  int n_phases;                 // max phases over fields
  unsigned long long* queue;    // work counter (zeroed before launch)
  int* done_phase;              // per field, -1 before launch
  int* arrive;                  // per field, 0 before launch (arrived unit groups)
  double* partials;             // per unit x 5
  int* garrive;                 // per unit group (slot unit_begin + group), 0 before launch
  double* gpartials;            // per unit group x 5 (same slots)
  int* err;                     // set on a bounded-wait timeout
  long long phase_wait_limit;   // polls of a field's phase flag before giving up (err)
  const float* S;
  float2* X[2];                 // chi (double-buffered; final chi in X[0])
  float2* G[2];
  float2* D[2];
  float2* Q[2];
  float4* W;                    // (wx, wy, wcx, wcy)
  float2* W2;                   // (wd1, wd2) oriented-prior weights; null when no field
                                // of the launch has diag_prior > 0
  float* Y;                     // output-fidelity luma
  float4* M;                    // neighbour 2x2 data term (m11, m12, m22, -)
  float2* B;                    // neighbour constant term
  const float4* nbr;            // neighbour planes (S_w - S, Re dc, Im dc, conf)
  const float4* line_phasor;
  const float2* col_phasor;
};

int solver_max_blocks_per_sm(bool diag = false);
cudaError_t launch_solver(const SolverArgs& args, int grid, cudaStream_t st);

}  // namespace hvdg
