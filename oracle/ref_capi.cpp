// ref_capi.cpp -- TEST INFRASTRUCTURE (oracle), never shipped or measured
// as the product. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline legs load the library this file is linked into.
//
// A plain C ABI over the UNMODIFIED reference engine (hvd-core/src, compiled
// from its own sources by oracle/Makefile) so the reference's own C++ path
// can be called from Python (ctypes) as the parity checker and timed as the
// CPU baseline. Each function names the reference entry point it forwards to.
// Structs are the product's C-ABI structs (include/hvdg.h), converted to the
// reference's types here.

#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "hvdg.h"
#include "engine/colour.h"
#include "engine/engine.h"
#include "engine/holographic_init.h"
#include "engine/lockin.h"
#include "engine/motion.h"
#include "engine/ntsc_geometry.h"
#include "engine/sequence.h"
#include "engine/temporal.h"
#include "engine/variational.h"
#include "frame_bridge.h"
#include "ref_convert.h"

using namespace refconv;

extern "C" {

int hvdref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// BurstLockinPhase (lockin.cpp:169) / BurstLockinPhasePal (lockin.cpp:325).
int hvdref_burst_lockin(const float* field, const hvdg_geometry* g, float* theta,
                        int8_t* vswitch) {
  const hvd::FieldGeometry geo = ToGeom(*g);
  const hvd::Plane f = PlaneFrom(field, geo.field_height, geo.field_width);
  if (geo.uses_vswitch()) {
    const hvd::PalBurstLockin r = hvd::BurstLockinPhasePal(f, geo);
    std::copy(r.theta.begin(), r.theta.end(), theta);
    if (vswitch) std::copy(r.vswitch.begin(), r.vswitch.end(), vswitch);
  } else {
    const std::vector<float> t = hvd::BurstLockinPhase(f, geo);
    std::copy(t.begin(), t.end(), theta);
    if (vswitch) std::fill(vswitch, vswitch + t.size(), int8_t{1});
  }
  return 0;
}

// BurstAmplitudeIre (lockin.cpp:256).
float hvdref_burst_amplitude(const float* field, const hvdg_geometry* g) {
  const hvd::FieldGeometry geo = ToGeom(*g);
  return hvd::BurstAmplitudeIre(PlaneFrom(field, geo.field_height, geo.field_width), geo);
}

// TridiagSmooth (lockin.cpp:133).
void hvdref_tridiag_smooth(const float* d, const float* a, int n, float lam, float* x) {
  const std::vector<float> dv(d, d + n), av(a, a + n);
  const std::vector<float> r = hvd::TridiagSmooth(dv, av, lam);
  std::copy(r.begin(), r.end(), x);
}

// MakeCarrier / MakeCarrierPal (ntsc_geometry.cpp:392/438), active lines.
void hvdref_make_carrier(const float* theta_active, const int8_t* vswitch_active,
                         int lines, const hvdg_geometry* g, float* carrier_ri) {
  const hvd::FieldGeometry geo = ToGeom(*g);
  const std::vector<float> th(theta_active, theta_active + lines);
  hvd::ComplexPlane c;
  if (geo.uses_vswitch()) {
    const std::vector<int8_t> sw(vswitch_active, vswitch_active + lines);
    c = hvd::MakeCarrierPal(th, sw, geo);
  } else {
    c = hvd::MakeCarrier(th, geo);
  }
  CPlaneTo(c, carrier_ri);
}

// PrepareFieldObs (sequence.cpp:229): field IRE -> active S + carrier.
int hvdref_prepare_field(const float* field, const hvdg_geometry* g,
                         const hvdg_config* cfg, int parity, float* s_active,
                         float* carrier_ri) {
  const hvd::FieldGeometry geo = ToGeom(*g);
  hvd::FieldInput fi;
  fi.samples = PlaneFrom(field, geo.field_height, geo.field_width);
  fi.is_first_field = parity == 0;
  const hvd::FieldObs obs = hvd::PrepareFieldObs(fi, geo, ToCfg(*cfg), parity);
  PlaneTo(obs.s, s_active);
  CPlaneTo(obs.carrier, carrier_ri);
  return 0;
}

// HolographicInit (holographic_init.cpp:427).
int hvdref_holographic_init(const float* s, const float* carrier_ri, int h, int w,
                            const hvdg_geometry* g, const hvdg_config* cfg,
                            float* y0, float* chi0) {
  hvd::Fft2d fft;
  const hvd::HoloInit r =
      hvd::HolographicInit(PlaneFrom(s, h, w), CPlaneFrom(carrier_ri, h, w),
                           ToGeom(*g), ToCfg(*cfg), &fft);
  PlaneTo(r.luma, y0);
  CPlaneTo(r.chroma, chi0);
  return 0;
}

// VariationalRefine (variational.cpp:198). `is_pal` sets HvdConfig::is_pal
// exactly as DecodeFieldWindowWithInits does (sequence.cpp:438).
int hvdref_variational_refine(const float* s, const float* carrier_ri,
                              const float* chi0_ri, int h, int w,
                              const hvdg_config* cfg, int is_pal, int n_nbr,
                              const float* const* nbr_s,
                              const float* const* nbr_carrier_ri,
                              const float* const* nbr_conf, float* y, float* chi) {
  hvd::HvdConfig c = ToCfg(*cfg);
  c.is_pal = is_pal != 0;
  std::vector<hvd::NeighborTerm> nb;
  for (int j = 0; j < n_nbr; ++j) {
    nb.push_back(hvd::NeighborTerm{PlaneFrom(nbr_s[j], h, w),
                                   CPlaneFrom(nbr_carrier_ri[j], h, w),
                                   PlaneFrom(nbr_conf[j], h, w)});
  }
  const hvd::RefineResult r = hvd::VariationalRefine(
      PlaneFrom(s, h, w), CPlaneFrom(carrier_ri, h, w), CPlaneFrom(chi0_ri, h, w), c, nb);
  PlaneTo(r.luma, y);
  CPlaneTo(r.chroma, chi);
  return 0;
}

// EstimateMotion (motion.cpp:397).
int hvdref_estimate_motion(const float* y_ref, const float* y_cur, int h, int w,
                           int tile, int search, float* dy, float* dx, float* conf) {
  const hvd::MotionField m =
      hvd::EstimateMotion(PlaneFrom(y_ref, h, w), PlaneFrom(y_cur, h, w), tile, search);
  PlaneTo(m.dy, dy);
  PlaneTo(m.dx, dx);
  PlaneTo(m.confidence, conf);
  return 0;
}

// VerifyMotion (motion.cpp:490-530): predictions pdy / pdx per tile.
int hvdref_verify_motion(const float* y_ref, const float* y_cur, int h, int w, int tile,
                         const float* pdy, const float* pdx, float* dy, float* dx, float* conf) {
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const hvd::MotionField m =
      hvd::VerifyMotion(PlaneFrom(y_ref, h, w), PlaneFrom(y_cur, h, w), PlaneFrom(pdy, th, tw),
                        PlaneFrom(pdx, th, tw), tile);
  PlaneTo(m.dy, dy);
  PlaneTo(m.dx, dx);
  PlaneTo(m.confidence, conf);
  return 0;
}

// BoxBlur (motion.cpp:391), in place.
void hvdref_box_blur(float* a, int h, int w, int r) {
  const hvd::Plane o = hvd::BoxBlur(PlaneFrom(a, h, w), r);
  PlaneTo(o, a);
}

// VectorsPerPixel (temporal.cpp:45).
void hvdref_vectors_per_pixel(const float* mdy, const float* mdx, int th, int tw,
                              int tile, int out_h, int out_w, float* dy, float* dx) {
  const hvd::PerPixelMotion v = hvd::VectorsPerPixel(
      PlaneFrom(mdy, th, tw), PlaneFrom(mdx, th, tw), tile, out_h, out_w);
  PlaneTo(v.dy, dy);
  PlaneTo(v.dx, dx);
}

// UpsampleConfidence / UpsampleConfidenceFast (temporal.cpp:227/245).
void hvdref_upsample_confidence(const float* conf, int th, int tw, int tile,
                                int out_h, int out_w, int fast, float* out) {
  const hvd::Plane c = PlaneFrom(conf, th, tw);
  const hvd::Plane o = fast ? hvd::UpsampleConfidenceFast(c, tile, out_h, out_w)
                            : hvd::UpsampleConfidence(c, tile, out_h, out_w);
  PlaneTo(o, out);
}

// EstimateNoiseIre (ntsc_geometry.cpp:49).
float hvdref_estimate_noise(const float* s, int h, int w) {
  return hvd::EstimateNoiseIre(PlaneFrom(s, h, w));
}

// PrepareFieldObs x n + DecodeFieldWindow (sequence.cpp:229-281): one
// window, one geometry. y_out[j]: active h x w; chi_out[j]: h x w x 2.
int hvdref_decode_field_window(const float* const* fields, const int* parities,
                               int nf, const hvdg_geometry* g,
                               const hvdg_config* cfg, float* const* y_out,
                               float* const* chi_out, float* diag5) {
  const hvd::FieldGeometry geo = ToGeom(*g);
  const hvd::HvdConfig c = ToCfg(*cfg);
  std::vector<hvd::FieldObs> obs(nf);
  for (int j = 0; j < nf; ++j) {
    hvd::FieldInput fi;
    fi.samples = PlaneFrom(fields[j], geo.field_height, geo.field_width);
    fi.is_first_field = parities[j] == 0;
    obs[j] = hvd::PrepareFieldObs(fi, geo, c, parities[j]);
  }
  hvd::HvdEngine engine;
  hvd::SequenceDiagnostics diag;
  const std::vector<hvd::DecodedField> dec = engine.DecodeSequenceWindow(obs, geo, c, &diag);
  for (int j = 0; j < nf; ++j) {
    PlaneTo(dec[j].luma, y_out[j]);
    CPlaneTo(dec[j].chroma, chi_out[j]);
  }
  if (diag5) {
    diag5[0] = diag.resolved_strength;
    diag5[1] = diag.ambiguity_ire;
    diag5[2] = diag.sigma_ire;
    diag5[3] = diag.temporal_eps;
    diag5[4] = diag.nr_eps;
  }
  return 0;
}

// Independent 2-D fields of mixed geometry / budget: the reference's
// per-field path (PrepareFieldObs + a one-field DecodeFieldWindow, i.e. the
// 2-D stride-1 sweep of sequence.cpp:1076-1084), OpenMP across fields as
// parallel_across_fields does. cfgs[j] carries each field's budget.
int hvdref_decode_fields(const float* const* fields, const int* parities, int nf,
                         const hvdg_geometry* const* geos,
                         const hvdg_config* const* cfgs, float* const* y_out,
                         float* const* chi_out, int across_fields) {
  auto one = [&](int j) {
    const hvd::FieldGeometry geo = ToGeom(*geos[j]);
    const hvd::HvdConfig c = ToCfg(*cfgs[j]);
    hvd::FieldInput fi;
    fi.samples = PlaneFrom(fields[j], geo.field_height, geo.field_width);
    fi.is_first_field = parities[j] == 0;
    std::vector<hvd::FieldObs> obs(1);
    obs[0] = hvd::PrepareFieldObs(fi, geo, c, parities[j]);
    hvd::Fft2d fft;
    const std::vector<hvd::DecodedField> dec =
        hvd::DecodeFieldWindow(obs, geo, c, &fft, nullptr);
    PlaneTo(dec[0].luma, y_out[j]);
    CPlaneTo(dec[0].chroma, chi_out[j]);
  };
  if (across_fields) {
#pragma omp parallel for schedule(dynamic)
    for (int j = 0; j < nf; ++j) one(j);
  } else {
    for (int j = 0; j < nf; ++j) one(j);
  }
  return 0;
}

// hvd::DecodeFrameSequenceWindow (frame_bridge.cpp:722). Outputs are
// (core_end - core_begin) frames of fw*fh each; returns the number of
// frames produced (0 where the reference returns an empty vector).
int hvdref_decode_frame_sequence_window(const int16_t* const* frames, int nframes,
                                        int core_begin, int core_end,
                                        const hvdg_frame_params* fp,
                                        const hvdg_config* cfg, int16_t* const* luma,
                                        int16_t* const* chroma, double* const* u,
                                        double* const* v) {
  const std::vector<const int16_t*> fr(frames, frames + nframes);
  hvd::HvdEngine engine;
  const std::vector<hvd::YcFrameS16> out = hvd::DecodeFrameSequenceWindow(
      fr, core_begin, core_end, ToFp(*fp), ToCfg(*cfg), engine, 0);
  for (size_t t = 0; t < out.size(); ++t) {
    std::copy(out[t].luma.begin(), out[t].luma.end(), luma[t]);
    std::copy(out[t].chroma.begin(), out[t].chroma.end(), chroma[t]);
    std::copy(out[t].u_plane.begin(), out[t].u_plane.end(), u[t]);
    std::copy(out[t].v_plane.begin(), out[t].v_plane.end(), v[t]);
  }
  return static_cast<int>(out.size());
}

static void CopyYc(const hvd::YcFrameS16& o, int16_t* luma, int16_t* chroma, double* u,
                   double* v) {
  std::copy(o.luma.begin(), o.luma.end(), luma);
  std::copy(o.chroma.begin(), o.chroma.end(), chroma);
  std::copy(o.u_plane.begin(), o.u_plane.end(), u);
  std::copy(o.v_plane.begin(), o.v_plane.end(), v);
}

// hvd::DecodeFrameBuffer (frame_bridge.cpp:161): the frame-weave decode of
// one composite frame; fw*fh outputs.
void hvdref_decode_frame_buffer(const int16_t* frame, const hvdg_frame_params* fp,
                                const hvdg_config* cfg, int16_t* luma, int16_t* chroma,
                                double* u, double* v) {
  hvd::HvdEngine engine;
  CopyYc(hvd::DecodeFrameBuffer(frame, ToFp(*fp), ToCfg(*cfg), engine), luma, chroma, u, v);
}

// hvd::DecodeYcFrameBuffer (frame_bridge.cpp:263): Y/C-native input.
void hvdref_decode_yc_frame_buffer(const int16_t* luma_in, const int16_t* chroma_in,
                                   const hvdg_frame_params* fp, const hvdg_config* cfg,
                                   int16_t* luma, int16_t* chroma, double* u, double* v) {
  hvd::HvdEngine engine;
  CopyYc(hvd::DecodeYcFrameBuffer(luma_in, chroma_in, ToFp(*fp), ToCfg(*cfg), engine), luma,
         chroma, u, v);
}

// DrizzleFrame (sequence.cpp:283): fields luma (h x w) / chroma (h x w x 2);
// outputs (2 h scale) x w.
void hvdref_drizzle_frame(const float* const* luma, const float* const* chroma,
                          const int* parities, int n, int j0, int h, int w,
                          const hvdg_config* cfg, int scale, float* out_luma, float* out_chroma) {
  std::vector<hvd::Plane> Ys;
  std::vector<hvd::ComplexPlane> Cs;
  for (int i = 0; i < n; ++i) {
    Ys.push_back(PlaneFrom(luma[i], h, w));
    Cs.push_back(CPlaneFrom(chroma[i], h, w));
  }
  const std::vector<int> par(parities, parities + n);
  const hvd::DrizzleResult r = hvd::DrizzleFrame(j0, Ys, Cs, par, ToCfg(*cfg), scale);
  PlaneTo(r.luma, out_luma);
  CPlaneTo(r.chroma, out_chroma);
}

// The same with HvdConfig::debug_dir and base_frame_id set (the diagnostic
// maps, frame_bridge.cpp:807-865).
int hvdref_decode_frame_sequence_window_debug(const int16_t* const* frames, int nframes,
                                              int core_begin, int core_end,
                                              const hvdg_frame_params* fp, const hvdg_config* cfg,
                                              const char* debug_dir, int64_t base_frame_id,
                                              int16_t* const* luma, int16_t* const* chroma,
                                              double* const* u, double* const* v) {
  const std::vector<const int16_t*> fr(frames, frames + nframes);
  hvd::HvdEngine engine;
  hvd::HvdConfig c = ToCfg(*cfg);
  c.debug_dir = debug_dir ? debug_dir : "";
  const std::vector<hvd::YcFrameS16> out = hvd::DecodeFrameSequenceWindow(
      fr, core_begin, core_end, ToFp(*fp), c, engine, base_frame_id);
  for (size_t t = 0; t < out.size(); ++t) CopyYc(out[t], luma[t], chroma[t], u[t], v[t]);
  return static_cast<int>(out.size());
}

// SplitFrameFields (frame_bridge.cpp:61): block-1 / block-2 fields in IRE.
void hvdref_split_frame_fields(const int16_t* frame, const hvdg_frame_params* fp,
                               float* top, float* bottom) {
  hvd::FieldInput a, b;
  hvd::SplitFrameFields(frame, ToFp(*fp), &a, &b, false);
  PlaneTo(a.samples, top);
  PlaneTo(b.samples, bottom);
}

// DetectFieldParity (frame_bridge.cpp:102).
int hvdref_detect_field_parity(const float* block1, const float* block2,
                               const hvdg_frame_params* fp) {
  const hvd::FrameParams f = ToFp(*fp);
  hvd::FieldInput a, b;
  a.samples = PlaneFrom(block1, f.field1_lines, f.frame_width);
  b.samples = PlaneFrom(block2, f.field1_lines, f.frame_width);
  return hvd::DetectFieldParity(a, b, f);
}

// Fft2d Forward / Inverse (the oracle FFT above; fft2d.h:30-33).
void hvdref_fft2d(const float* in_ri, int h, int w, int inverse, float* out_ri) {
  hvd::Fft2d f;
  const hvd::ComplexPlane in = CPlaneFrom(in_ri, h, w);
  CPlaneTo(inverse ? f.Inverse(in) : f.Forward(in), out_ri);
}

}  // extern "C"
