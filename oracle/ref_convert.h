// ref_convert.h -- TEST INFRASTRUCTURE (oracle): the product's C-ABI structs
// (include/hvdg.h) converted to the reference engine's types, and float
// planes to / from the reference's Plane / ComplexPlane. Shared by the C
// entry points over the reference engine (ref_capi.cpp) and over the B200
// shim (shim_capi.cpp).
#pragma once

#include <algorithm>
#include <cstring>

#include "hvdg.h"
#include "engine/engine.h"
#include "engine/ntsc_geometry.h"
#include "frame_bridge.h"

namespace refconv {

inline hvd::FieldGeometry ToGeom(const hvdg_geometry& g) {
  hvd::FieldGeometry o;
  o.field_width = g.field_width;
  o.field_height = g.field_height;
  o.active_video_start = g.active_video_start;
  o.active_video_end = g.active_video_end;
  o.colour_burst_start = g.colour_burst_start;
  o.colour_burst_end = g.colour_burst_end;
  o.first_active_field_line = g.first_active_field_line;
  o.last_active_field_line = g.last_active_field_line;
  o.sample_rate = g.sample_rate;
  o.standard = g.standard == HVDG_STD_PAL     ? hvd::VideoStandard::kPal
               : g.standard == HVDG_STD_PAL_M ? hvd::VideoStandard::kPalM
                                              : hvd::VideoStandard::kNtsc;
  o.subcarrier_hz = g.subcarrier_hz;
  return o;
}

inline hvd::HvdConfig ToCfg(const hvdg_config& c) {
  hvd::HvdConfig o;
  o.lambda_c = c.lambda_c;
  o.chroma_aniso = c.chroma_aniso;
  o.charbonnier_eps = c.charbonnier_eps;
  o.chroma_eps = c.chroma_eps;
  o.structure_coupling = c.structure_coupling;
  o.diag_prior = c.diag_prior;
  o.cg_iterations = c.cg_iterations;
  o.irls_outer = c.irls_outer;
  o.cg_tol = c.cg_tol;
  o.fast = c.fast != 0;
  o.parallel_across_fields = c.parallel_across_fields != 0;
  o.symmetry_variant = c.symmetry_variant != 0;
  o.acc = c.acc != 0;
  o.chroma_gain = c.chroma_gain;
  o.monochrome = c.monochrome != 0;
  o.chroma_phase_deg = c.chroma_phase_deg;
  o.field_order = c.field_order;
  o.temporal_strength = c.temporal_strength;
  o.bidirectional = c.bidirectional != 0;
  o.passes = c.passes;
  o.temporal_eps = c.temporal_eps;
  o.nr_anchor = c.nr_anchor;
  o.nr_eps = c.nr_eps;
  o.nr_radius = c.nr_radius;
  o.mc_tile = c.mc_tile;
  o.mc_search = c.mc_search;
  o.trajectory_fit = c.trajectory_fit != 0;
  o.extended_temporal = c.extended_temporal != 0;
  o.coherence_gate = c.coherence_gate;
  o.odd_gate_floor = c.odd_gate_floor;
  o.output_fidelity = c.output_fidelity != 0;
  o.psi_init = c.psi_init != 0;
  o.selective_3d = c.selective_3d != 0;
  o.selective_max_area = c.selective_max_area;
  return o;
}

inline hvd::FrameParams ToFp(const hvdg_frame_params& f) {
  hvd::FrameParams o;
  o.standard = f.standard == HVDG_STD_PAL     ? hvd::VideoStandard::kPal
               : f.standard == HVDG_STD_PAL_M ? hvd::VideoStandard::kPalM
                                              : hvd::VideoStandard::kNtsc;
  o.frame_width = f.frame_width;
  o.frame_height = f.frame_height;
  o.field1_lines = f.field1_lines;
  o.active_video_start = f.active_video_start;
  o.active_video_end = f.active_video_end;
  o.colour_burst_start = f.colour_burst_start;
  o.colour_burst_end = f.colour_burst_end;
  o.first_active_frame_line = f.first_active_frame_line;
  o.last_active_frame_line = f.last_active_frame_line;
  o.black_level = f.black_level;
  o.white_level = f.white_level;
  o.blanking_level = f.blanking_level;
  o.chroma_dc = f.chroma_dc;
  o.sample_rate = f.sample_rate;
  o.subcarrier_hz = f.subcarrier_hz;
  o.extra_sample_line_count =
      std::min<int>(f.extra_sample_line_count, hvd::FrameParams::kMaxExtraSampleLines);
  for (int i = 0; i < o.extra_sample_line_count; ++i)
    o.extra_sample_lines[i] = f.extra_sample_lines[i];
  return o;
}

inline hvd::Plane PlaneFrom(const float* p, int h, int w) {
  hvd::Plane o(h, w);
  std::memcpy(o.data(), p, sizeof(float) * static_cast<size_t>(h) * w);
  return o;
}

inline hvd::ComplexPlane CPlaneFrom(const float* p, int h, int w) {
  hvd::ComplexPlane o(h, w);
  std::memcpy(o.data(), p, sizeof(float) * 2 * static_cast<size_t>(h) * w);
  return o;
}

inline void PlaneTo(const hvd::Plane& a, float* p) {
  std::memcpy(p, a.data(), sizeof(float) * a.size());
}
inline void CPlaneTo(const hvd::ComplexPlane& a, float* p) {
  std::memcpy(p, a.data(), sizeof(float) * 2 * a.size());
}

}  // namespace refconv
