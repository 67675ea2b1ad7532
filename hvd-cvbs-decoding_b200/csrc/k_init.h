// k_init.h -- launchers of the holographic-init and aniso kernels (k_init.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hvdg_internal.h"

namespace hvdg {

struct InitArgs {
  const FieldDesc* fields;
  const GeomDesc* geoms;
  const float* S;              // active composite planes
  const float4* line_phasor;   // per active line (cos, sin, sign, 0)
  const float2* col_phasor;    // per geometry column exp(i w0 (a0 + x))
  const float2* khat;          // kernel spectra (row / column, 2 variants each)
  const float2* tw_row;        // exp(-2 pi i k / kRowFft)
  const float2* tw_col;        // exp(-2 pi i k / kColFft) (the wide columns use tw_row)
  const float2* tw_long = nullptr;  // exp(-2 pi i k / kFftLong)
  int long_rows = 0;           // some geometry of the batch has row_m == kFftLong
  int long_cols = 0;           // some geometry of the batch has col_m == kFftLong
  float2* rowbuf;              // row-filtered variants: per field 2 x hp x pitch
  const int64_t* rowbuf_off;   // per field offset into rowbuf (float2)
  float2* chi1;                // variant outputs (pitched like the planes)
  float2* chi2;
  float2* chi0;                // blended init chi0
  float* Y;                    // init luma Y0
  const int* prow_field;       // padded row -> field
  const int* prow_first;       // field -> first padded row index
  const int* cgrp_field;       // column group -> field
  const int* cgrp_first;       // field -> first column group
  const int* btile_field;      // blend tile -> field
  const int* btile_first;      // field -> first blend tile
  // Adjoint mode (both non-null): the rows pass filters the two variant
  // planes of adj_in (per field at rowbuf_off, 2 x hp x pitch, pad rows
  // included) instead of the demodulated composite, and the columns pass
  // writes all hp filtered rows of each variant to adj_out (same layout)
  // instead of the cropped chi1 / chi2. The filters are real and even, so
  // this applies the adjoint of the forward crop (the x2 included).
  const float2* adj_in = nullptr;
  float2* adj_out = nullptr;
  // Symmetry variant (holographic_init.cpp:265-306), when chi3 is set: the
  // exact hp x w 2-D DFT of the padded demodulated field (Bluestein rows /
  // columns through rowbuf, which is free once the column pass is done),
  // the certified spectrum, its inverse cropped into chi3, blended as the
  // third variant.
  float2* chi3 = nullptr;
};

void configure_init_kernels();
void launch_init(const InitArgs& a, int total_prows, int total_cgroups, int total_btiles,
                 cudaStream_t st);
// Adjoint of the two row / column filter passes (rows, then columns; no blend).
void launch_init_filter_adjoint(const InitArgs& a, int total_prows, int total_cgroups,
                                cudaStream_t st);
void launch_aniso(FieldDesc* d_fields, int n_fields, const float2* chi0, cudaStream_t st);
int aniso_max_samples();
// columns per CTA of the column pass for a geometry with column length col_m
int init_col_group(int col_m);
int init_blend_tile();

}  // namespace hvdg
