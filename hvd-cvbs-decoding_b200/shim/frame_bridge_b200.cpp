// frame_bridge_b200.cpp -- hvd-core's frame-bridge decode entry points
// re-implemented on the B200 library's C ABI (include/hvdg.h):
//
//   hvd::DecodeFrameSequenceWindow  (frame_bridge.h:196-199)
//   hvd::DecodeFrameBuffer          (frame_bridge.h:149-150, 205-206)
//   hvd::DecodeYcFrameBuffer        (frame_bridge.h:223-228)
//
// Same signatures, same results (to the rounding the library's parity tests
// state), same failure convention: an empty vector / a default YcFrameS16
// where the reference returns one. Built inside the hvd-core tree in place
// of those four functions of frame_bridge.cpp (its other helpers stay), the
// decode-orc plugin links unchanged. Each host thread gets one library
// context (device arena, stream, graph cache), created on its first decode
// and destroyed when the thread exits. HVDG_DEVICE selects the CUDA device
// (default 0).
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "frame_bridge.h"
#include "hvdg.h"

namespace hvd {
namespace {

// The library context of the calling thread. An HvdEngine must not be used
// by two threads at once (frame_bridge.h:137-140), so the engines one thread
// uses run one after another and can share that thread's context. Keying
// contexts on the engine instead would keep one alive per engine for the
// life of the process: the stage builds a fresh engine per export worker and
// per preview trigger (hvd_chroma_decoder_stage.cpp:991, 1115, 1166), and
// each context holds a device arena and page-locked staging. The context
// is destroyed when its thread exits.
struct ThreadContext {
  hvdg_ctx* ctx = nullptr;
  ~ThreadContext() {
    if (ctx) hvdg_destroy(ctx);
  }
};

hvdg_ctx* ContextFor(const HvdEngine* /*engine*/) {
  thread_local ThreadContext tc;
  if (!tc.ctx) {
    const char* dev = std::getenv("HVDG_DEVICE");
    hvdg_ctx* ctx = nullptr;
    if (hvdg_create(dev ? std::atoi(dev) : 0, &ctx) != HVDG_OK) return nullptr;
    tc.ctx = ctx;
  }
  return tc.ctx;
}

int32_t ToHvdg(VideoStandard s) {
  return s == VideoStandard::kPal ? HVDG_STD_PAL
                                  : (s == VideoStandard::kPalM ? HVDG_STD_PAL_M : HVDG_STD_NTSC);
}

hvdg_frame_params ToHvdg(const FrameParams& f) {
  hvdg_frame_params o{};
  o.standard = ToHvdg(f.standard);
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
  o.extra_sample_line_count = f.extra_sample_line_count;
  for (int i = 0; i < f.extra_sample_line_count && i < HVDG_MAX_EXTRA_SAMPLE_LINES; ++i)
    o.extra_sample_lines[i] = f.extra_sample_lines[i];
  return o;
}

hvdg_config ToHvdg(const HvdConfig& c) {
  hvdg_config o;
  hvdg_config_default(&o);
  o.lambda_c = c.lambda_c;
  o.chroma_aniso = c.chroma_aniso;
  o.charbonnier_eps = c.charbonnier_eps;
  o.chroma_eps = c.chroma_eps;
  o.structure_coupling = c.structure_coupling;
  o.diag_prior = c.diag_prior;
  o.cg_iterations = c.cg_iterations;
  o.irls_outer = c.irls_outer;
  o.cg_tol = c.cg_tol;
  o.fast = c.fast ? 1 : 0;
  o.parallel_across_fields = c.parallel_across_fields ? 1 : 0;
  o.symmetry_variant = c.symmetry_variant ? 1 : 0;
  o.acc = c.acc ? 1 : 0;
  o.chroma_gain = c.chroma_gain;
  o.monochrome = c.monochrome ? 1 : 0;
  o.chroma_phase_deg = c.chroma_phase_deg;
  o.field_order = c.field_order;
  o.temporal_strength = c.temporal_strength;
  o.bidirectional = c.bidirectional ? 1 : 0;
  o.passes = c.passes;
  o.temporal_eps = c.temporal_eps;
  o.nr_anchor = c.nr_anchor;
  o.nr_eps = c.nr_eps;
  o.nr_radius = c.nr_radius;
  o.mc_tile = c.mc_tile;
  o.mc_search = c.mc_search;
  o.trajectory_fit = c.trajectory_fit ? 1 : 0;
  o.extended_temporal = c.extended_temporal ? 1 : 0;
  o.coherence_gate = c.coherence_gate;
  o.odd_gate_floor = c.odd_gate_floor;
  o.output_fidelity = c.output_fidelity ? 1 : 0;
  o.psi_init = c.psi_init ? 1 : 0;
  o.selective_3d = c.selective_3d ? 1 : 0;
  o.selective_max_area = c.selective_max_area;
  return o;
}

// A YcFrameS16 with its four planes allocated, and the C view of them.
YcFrameS16 Allocated(const FrameParams& fp, hvdg_yc_frame* view) {
  YcFrameS16 f;
  f.width = fp.frame_width;
  f.height = fp.frame_height;
  f.chroma_dc = fp.chroma_dc;
  const size_t n = static_cast<size_t>(fp.frame_width) * fp.frame_height;
  f.luma.assign(n, 0);
  f.chroma.assign(n, 0);
  f.u_plane.assign(n, 0.0);
  f.v_plane.assign(n, 0.0);
  *view = hvdg_yc_frame{f.luma.data(), f.chroma.data(), f.u_plane.data(), f.v_plane.data()};
  return f;
}

}  // namespace

std::vector<YcFrameS16> DecodeFrameSequenceWindow(const std::vector<const int16_t*>& frames,
                                                  int core_begin, int core_end,
                                                  const FrameParams& fp, const HvdConfig& cfg,
                                                  HvdEngine& engine, int64_t base_frame_id) {
  const int n = static_cast<int>(frames.size());
  if (n == 0 || core_begin < 0 || core_end > n || core_begin >= core_end) return {};
  hvdg_ctx* ctx = ContextFor(&engine);
  if (!ctx) return {};
  hvdg_set_debug_dir(ctx, cfg.debug_dir.empty() ? nullptr : cfg.debug_dir.c_str());
  std::vector<YcFrameS16> out;
  std::vector<hvdg_yc_frame> views(core_end - core_begin);
  for (int t = core_begin; t < core_end; ++t) out.push_back(Allocated(fp, &views[t - core_begin]));
  // views point into the vectors now owned by `out` (moved, not copied)
  for (int t = 0; t < core_end - core_begin; ++t)
    views[t] = hvdg_yc_frame{out[t].luma.data(), out[t].chroma.data(), out[t].u_plane.data(),
                             out[t].v_plane.data()};
  const hvdg_frame_params p = ToHvdg(fp);
  const hvdg_config c = ToHvdg(cfg);
  if (hvdg_decode_frame_sequence_window_at(ctx, frames.data(), n, core_begin, core_end,
                                           base_frame_id, &p, &c, views.data(),
                                           nullptr) != HVDG_OK)
    return {};
  return out;
}

YcFrameS16 DecodeFrameBuffer(const int16_t* frame, const FrameParams& fp, const HvdConfig& cfg,
                             HvdEngine& engine) {
  hvdg_ctx* ctx = ContextFor(&engine);
  if (!ctx || !frame) return YcFrameS16{};
  hvdg_yc_frame view;
  YcFrameS16 out = Allocated(fp, &view);
  const hvdg_frame_params p = ToHvdg(fp);
  const hvdg_config c = ToHvdg(cfg);
  if (hvdg_decode_frame_buffer(ctx, frame, &p, &c, &view) != HVDG_OK) return YcFrameS16{};
  return out;
}

YcFrameS16 DecodeFrameBuffer(const int16_t* frame, const FrameParams& fp, const HvdConfig& cfg) {
  HvdEngine engine;
  return DecodeFrameBuffer(frame, fp, cfg, engine);
}

YcFrameS16 DecodeYcFrameBuffer(const int16_t* luma, const int16_t* chroma, const FrameParams& fp,
                               const HvdConfig& cfg, HvdEngine& engine) {
  hvdg_ctx* ctx = ContextFor(&engine);
  if (!ctx || !luma || !chroma) return YcFrameS16{};
  hvdg_yc_frame view;
  YcFrameS16 out = Allocated(fp, &view);
  const hvdg_frame_params p = ToHvdg(fp);
  const hvdg_config c = ToHvdg(cfg);
  if (hvdg_decode_yc_frame_buffer(ctx, luma, chroma, &p, &c, &view) != HVDG_OK) return YcFrameS16{};
  return out;
}

YcFrameS16 DecodeYcFrameBuffer(const int16_t* luma, const int16_t* chroma, const FrameParams& fp,
                               const HvdConfig& cfg) {
  HvdEngine engine;
  return DecodeYcFrameBuffer(luma, chroma, fp, cfg, engine);
}

}  // namespace hvd
