// k_prep.h -- launchers of the field-preparation kernels (k_prep.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hvdg {

// Per-field description of the raw samples and the geometry the lock-in
// and crop kernels need.
struct PrepDesc {
  const void* samples;     // device pointer, fh x fw
  int sample_type;         // hvdg_sample_type
  int quadrant;            // 1 => w0 == pi/2 exactly (standard subcarrier)
  float blank;             // blanking level (codes)
  float codes_per_ire;     // (white - blanking) / 100
  int fh, fw;
  int bx0, bx1;            // burst window
  int fal, lal;            // active lines [fal, lal)
  int a0, a1;              // active samples [a0, a1)
  int vswitch_family;      // PAL / PAL-M
  float nominal_burst;     // FieldGeometry::nominal_burst_ire
  double w0;               // phase per sample
  double adv;              // line advance
  float chroma_phase_off;  // -chroma_phase_deg * pi / 180 (float, as the reference)
  int theta_off;           // offset of this field in the full-field per-line outputs
  int line_off;            // line-phasor index of this field's first ACTIVE line
  int line_step;           // index step per active line (1; 2 in a woven frame)
};

struct LockinOut {
  float* theta;          // optional, full-field theta (float)
  double* theta64;       // optional, full-field theta (double)
  signed char* vswitch;  // optional, full-field V-switch senses
  float4* line_phasor;   // optional, active lines: (cos, sin, sign, 0)
};

void configure_prep_kernels();
void launch_burst_lockin(const PrepDesc* d_descs, int n, LockinOut out, cudaStream_t st);
void launch_burst_amplitude(const PrepDesc* d_descs, int n, float* d_amp, cudaStream_t st);
// rows: per S row (plane, plane row, source field, source line)
void launch_crop(const PrepDesc* d_descs, const int4* d_rows, int total_rows, float* d_S,
                 const int64_t* d_px_off, const int* d_pitch, int* d_nonfinite, cudaStream_t st);

}  // namespace hvdg
