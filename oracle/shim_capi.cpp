// shim_capi.cpp -- TEST INFRASTRUCTURE (oracle): C entry points into the
// B200 shim (hvd-cvbs-decoding_b200/shim/frame_bridge_b200.cpp), i.e. the
// reference's own C++ frame-bridge signatures served by the B200 library,
// so the tests can drive the shim exactly as the decode-orc plugin would and
// compare it with the reference engine (ref_capi.cpp) and with the library's
// direct C ABI.
#include <cstdint>
#include <thread>
#include <vector>

#include "ref_convert.h"

using namespace refconv;

namespace {
void CopyOut(const hvd::YcFrameS16& o, int16_t* luma, int16_t* chroma, double* u, double* v) {
  std::copy(o.luma.begin(), o.luma.end(), luma);
  std::copy(o.chroma.begin(), o.chroma.end(), chroma);
  std::copy(o.u_plane.begin(), o.u_plane.end(), u);
  std::copy(o.v_plane.begin(), o.v_plane.end(), v);
}
}  // namespace

extern "C" {

// hvd::DecodeFrameSequenceWindow through the shim; returns the frame count.
int hvdshim_decode_frame_sequence_window(const int16_t* const* frames, int nframes,
                                         int core_begin, int core_end,
                                         const hvdg_frame_params* fp, const hvdg_config* cfg,
                                         int16_t* const* luma, int16_t* const* chroma,
                                         double* const* u, double* const* v) {
  static hvd::HvdEngine engine;  // one context, reused across calls (as the plugin keeps its engine)
  const std::vector<const int16_t*> fr(frames, frames + nframes);
  const std::vector<hvd::YcFrameS16> out = hvd::DecodeFrameSequenceWindow(
      fr, core_begin, core_end, ToFp(*fp), ToCfg(*cfg), engine, 0);
  for (size_t t = 0; t < out.size(); ++t) CopyOut(out[t], luma[t], chroma[t], u[t], v[t]);
  return static_cast<int>(out.size());
}

// hvd::DecodeFrameBuffer / DecodeYcFrameBuffer through the shim; returns 1
// when a frame came back (0: the reference's empty-result failure).
int hvdshim_decode_frame_buffer(const int16_t* frame, const hvdg_frame_params* fp,
                                const hvdg_config* cfg, int16_t* luma, int16_t* chroma,
                                double* u, double* v) {
  const hvd::YcFrameS16 o = hvd::DecodeFrameBuffer(frame, ToFp(*fp), ToCfg(*cfg));
  if (o.luma.empty()) return 0;
  CopyOut(o, luma, chroma, u, v);
  return 1;
}

int hvdshim_decode_yc_frame_buffer(const int16_t* luma_in, const int16_t* chroma_in,
                                   const hvdg_frame_params* fp, const hvdg_config* cfg,
                                   int16_t* luma, int16_t* chroma, double* u, double* v) {
  const hvd::YcFrameS16 o = hvd::DecodeYcFrameBuffer(luma_in, chroma_in, ToFp(*fp), ToCfg(*cfg));
  if (o.luma.empty()) return 0;
  CopyOut(o, luma, chroma, u, v);
  return 1;
}

// The stage's export pattern: `n_threads` worker threads one after another,
// each with its own fresh HvdEngine, decoding `frame` through
// hvd::DecodeFrameBuffer(..., engine) and exiting; returns how many decodes
// came back non-empty. Used to check that worker threads leave no device
// memory behind.
int hvdshim_decode_frame_buffer_workers(const int16_t* frame, const hvdg_frame_params* fp,
                                        const hvdg_config* cfg, int n_threads) {
  int ok = 0;
  for (int t = 0; t < n_threads; ++t) {
    std::thread worker([&] {
      hvd::HvdEngine engine;
      const hvd::YcFrameS16 o = hvd::DecodeFrameBuffer(frame, ToFp(*fp), ToCfg(*cfg), engine);
      if (!o.luma.empty()) ++ok;
    });
    worker.join();
  }
  return ok;
}

}  // extern "C"
