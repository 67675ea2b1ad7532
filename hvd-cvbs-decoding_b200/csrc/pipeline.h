// pipeline.h -- internal to the library: the context, the batch layout and
// the host pipeline stages shared by the C-ABI translation units
// (pipeline.cu: tables, planning, staging, the 2-D batch; window3d.cu: the
// 3-D field window; frames.cu: the frame bridges; host_misc.cu: kernel-level
// entry helpers and the adjoint driver; api.cu: the C ABI itself).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "hvdg.h"
#include "hvdg_internal.h"
#include "hvdg_host.h"
#include "k_adjoint.h"
#include "k_frame.h"
#include "k_init.h"
#include "k_joint.h"
#include "k_motion.h"
#include "k_temporal.h"
#include "k_prep.h"
#include "k_solver.h"

using hvdg::FieldCtl;
using hvdg::FieldDesc;
using hvdg::GeomDesc;
using hvdg::Unit;

namespace hvdg_pipe {

constexpr double kPi = 3.14159265358979323846;
using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// Geometry helpers (mirror FieldGeometry, ntsc_geometry.h:142-267)
// ---------------------------------------------------------------------------
// fn(i) for every i in [0, n), spread over up to 16 host threads (the
// calling one included) for the per-frame / per-pair host loops of the
// frame bridge; returns when all are done. Each i must write only its own
// outputs, so the results do not depend on the thread count.
template <typename F>
void parallel_for(int n, F&& fn) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::min(n, std::min(hw, 16));
  if (nt <= 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int> next{0};
  auto work = [&]() {
    for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) fn(i);
  };
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for (int k = 1; k < nt; ++k) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
}

inline bool uses_vswitch(const hvdg_geometry& g) {
  return g.standard == HVDG_STD_PAL || g.standard == HVDG_STD_PAL_M;
}
inline int last_active_line(const hvdg_geometry& g) {
  return g.last_active_field_line != 0 ? g.last_active_field_line : g.field_height;
}
inline double phase_per_sample(const hvdg_geometry& g) {
  if (g.subcarrier_hz <= 0.0) return 0.5 * kPi;
  return 2.0 * kPi * g.subcarrier_hz / g.sample_rate;
}
inline double line_advance(const hvdg_geometry& g) {
  if (g.subcarrier_hz <= 0.0) {
    if (g.standard == HVDG_STD_PAL) return 2.0 * kPi * 0.7516;
    if (g.standard == HVDG_STD_PAL_M) return 0.5 * kPi;
    return kPi;
  }
  const double cycles = g.subcarrier_hz * (double)g.field_width / g.sample_rate;
  return 2.0 * kPi * (cycles - std::floor(cycles));
}
inline float nominal_burst(const hvdg_geometry& g) {
  return g.standard == HVDG_STD_PAL ? 21.43f : 20.0f;
}

struct GeomTables {
  int w, h, hp, pad;
  int row_m;                     // row convolution length (kRowFft or kFftLong)
  int col_m;                     // column convolution length (kColFft, kColFftWide or kFftLong)
  std::vector<float2> khat_row;  // 2 * row_m
  std::vector<float2> khat_col;  // 2 * col_m
  std::vector<float2> col_phasor;
  // symmetry variant (built on first use): row chirp (w) | row chirp-filter
  // spectrum (row_m) | column chirp (hp) | column filter spectrum (col_m) |
  // gx (w) | gy (hp), the last two in .x
  bool sym_ready = false;
  std::vector<float2> sym;
};

using GeomKey = std::tuple<int, int, int, int, int, int, double, double>;

}  // namespace hvdg_pipe

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct hvdg_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[6] = {};
  std::string last_error;
  int batched = 1;
  int band_rows = 0;
  int ctas_per_sm = 0;
  long long phase_wait_limit = hvdg::kSpinLimit;  // solver phase-flag polls (~0.5 us each)
  hvdg::DeviceArena arena;
  hvdg::PinnedArena pinned;
  std::map<hvdg_pipe::GeomKey, hvdg_pipe::GeomTables> geoms;
  // arena generation: bumped whenever a call rewrites the arena's tables
  uint64_t epoch = 0;
  // CUDA-graph cache of the batched device-resident decode (one entry)
  int use_graphs = 1;
  cudaGraphExec_t gexec = nullptr;
  std::string gsig;
  uint64_t gepoch = 0;
  int* flags_host = nullptr;     // pinned, 4 ints
  void* ctl_host = nullptr;      // pinned FieldCtl[ctl_host_n]
  int ctl_host_n = 0;
  int gn = 0;                    // fields of the cached graph
  std::vector<int64_t> g_pix;    // per-field active px of the cached graph
  std::vector<int> g_outer;      // per-field IRLS outers of the cached graph
  // autotuner: batch signature -> (band rows, CTAs per SM)
  int autotune = 1;
  std::map<std::string, std::pair<int, int>> tune;
  // diagnostic maps of the sequence frame bridge (empty: off)
  std::string debug_dir;
  // asynchronous device-resident decodes: ordering against the caller's
  // stream, completion, and the result of a call that awaits hvdg_wait
  cudaEvent_t ev_in = nullptr, ev_done = nullptr;
  bool pending = false;           // a replay is in flight, hvdg_wait reads its flags
  bool settled = false;           // pending_status / pending_diag hold a finished call
  hvdg_status pending_status = HVDG_OK;
  hvdg_diag pending_diag{};
  bool pending_want_diag = false;
};

namespace hvdg_pipe {

// tile count limit of one integer-SAD confidence pass (its doubles live in shared memory)
constexpr int kSadMaxTiles = 6144;

// ---------------------------------------------------------------------------
// Batch planning
// ---------------------------------------------------------------------------
// One solve plane: a field's active picture, or a woven frame's.
struct FieldPlan {
  const hvdg_geometry* g;
  int h, w, pitch, fh, fw;
  int64_t px_off;
  int line_off, geom_slot;
  int hp;
  int64_t rowbuf_off;
};

// One source field of the lock-in / crop kernels (one per plane, or two per
// woven plane): its raw samples in the arena and its full-field per-line
// outputs.
struct PrepPlan {
  int fh, fw;
  int theta_off;
  int64_t raw_off, raw_bytes;
};

struct Layout {
  // byte offsets into the arena
  size_t o_raw, o_prep, o_fields, o_geoms, o_ctl, o_units, o_partials, o_done, o_arrive,
      o_flags, o_queue, o_lineph, o_theta, o_theta64, o_vsw, o_colph, o_khat, o_twr, o_twc,
      o_twl, o_S, o_Y, o_X0, o_X1, o_G0, o_G1, o_D0, o_D1, o_Q0, o_Q1, o_W, o_rowbuf, o_itab,
      o_amp;
  size_t o_W2 = 0;   // (wd1, wd2) plane, only when a field has the oriented prior
  size_t o_gpart = 0, o_garrive = 0;  // solver unit-group partials and arrival counters
  bool has_diag = false;
  size_t total;
  int64_t total_px, total_rowbuf;
  int total_lines, total_theta, total_units, total_prows, total_cgroups, total_btiles;
  int ncol, nkhat;
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Batch {
  std::vector<FieldPlan> fp;
  std::vector<PrepPlan> pp;
  std::vector<hvdg::PrepDesc> prep;
  std::vector<FieldDesc> fields;
  std::vector<GeomDesc> geoms;
  std::vector<const GeomTables*> gtabs;
  std::vector<int> gcol_off;
  std::vector<Unit> units;
  std::vector<int> itab;  // prow_field | prow_first | cgrp_field | cgrp_first | btile_field | btile_first
  int it_prow_field, it_prow_first, it_cgrp_field, it_cgrp_first, it_btile_field, it_btile_first;
  std::vector<int64_t> rowbuf_offs;
  std::vector<int4> crop_rows;  // per S row: (plane, row, source field, source line)
  std::vector<int64_t> px_offs;
  std::vector<int> pitches;
  // per field: the solver writes luma / chroma straight to the caller's
  // buffers (FieldDesc out_y / out_c), so no copy follows
  std::vector<char> direct_y, direct_c;
  Layout L;
  int max_phases = 0;
};

inline int elem_size(int sample_type) { return sample_type == HVDG_SAMPLES_F32_IRE ? 4 : 2; }

template <typename T>
T* at(hvdg_ctx* ctx, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(ctx->arena.base) + off);
}

struct RunOpts {
  bool device_io = false;  // samples / outputs are device pointers
  bool do_lockin = true;   // false: line phasors from theta_in / vswitch_in
  bool do_init = true;     // false: chi0 from chi0_in
  bool do_solve = true;    // false: outputs are the init (Y0, chi0)
  const float* s_in = nullptr;       // active S (dense h x w), replaces the crop
  const float* theta_in = nullptr;   // active-line theta
  const int8_t* vswitch_in = nullptr;
  const float* chi0_in = nullptr;    // dense h x w x 2
  float* amp_out = nullptr;          // optional per-field BurstAmplitudeIre (host)
  bool tables_only = false;          // stage_upload without the per-call reset
  int band_rows = -1;                // solver band height override (-1: context setting)
  int ctas_per_sm = -1;              // solver CTAs per SM override (-1: context setting)
  bool async = false;                // graph replay left in flight (hvdg_wait completes it)
  // the call's outputs: where the solver can reach them (device buffers, or
  // page-locked host buffers), its final phase writes them directly
  const hvdg_field_out* out_direct = nullptr;
  // woven frames: `in` holds two source fields per plane (plan_batch); their
  // F32 IRE samples are written into the arena's raw slots on the device
  const hvdg_geometry* weave_geom = nullptr;
};

// A batch uploaded to the arena: layout, table offsets, launch count.
struct Staged {
  Batch b;
  size_t it_itab = 0, it_crop = 0, it_pitch = 0, it_pxoff = 0, it_rbo = 0;
  size_t extra = 0;  // offset of the caller's extra region (after the batch layout)
  int launches = 0;
};

// ---------------------------------------------------------------------------
// Selective 3-D (DecodeWindowSelective, frame_bridge.cpp:490-718): a
// full-window 2-D decode, the Y/C-ambiguous boxes of its first field
// (AmbiguousBoxes, frame_bridge.cpp:402-580), the full 3-D window decode of
// each box, feather-blended in. A box's FieldObs crop (CropObs,
// frame_bridge.cpp:582-593) is the same field seen through a narrower active
// window -- S and the carrier of the crop are the crop of the field's, and
// the decode reads the geometry only for those and the sample rate -- so a
// box decodes as the window under a cropped geometry.
// ---------------------------------------------------------------------------
struct SelBox {
  int fy0 = 0, fy1 = 0, x0 = 0, x1 = 0;  // field coordinates inside the active picture
  bool valid = false;                     // an invalid single box: run full 3-D
};

hvdg_status check_plane(int w, int h, bool vsw);
hvdg_status check_geometry(const hvdg_geometry* g);
double fftfreq(int i, int n, double d);
std::vector<cd> kernel_spectrum(const std::vector<double>& mask, int M, double scale);
GeomTables make_geom_tables(const hvdg_geometry& g);
void host_fft(std::vector<cd>& a);
void bluestein_tables(int N, int M, std::vector<float2>* out);
void make_sym_tables(GeomTables& t, const hvdg_geometry& g);
GeomKey geom_key(const hvdg_geometry& g);
std::vector<float2> twiddles(int M);
int auto_band_rows_hw(hvdg_ctx* ctx, const std::vector<std::pair<int, int>>& hw);
int auto_band_rows(hvdg_ctx* ctx, const std::vector<FieldPlan>& fp);
hvdg_status plan_batch(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                       int band_rows, Batch& b, const hvdg_geometry* weave_geom = nullptr);
void mark(hvdg_ctx* ctx, int i);
float elapsed(hvdg_ctx* ctx, int a, int b);
void stage_reset(hvdg_ctx* ctx, const Staged& S);
hvdg_status stage_upload(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                         const RunOpts& opt, size_t extra_bytes, Staged& S);
hvdg::InitArgs init_args(hvdg_ctx* ctx, const Staged& S);
hvdg_status stage_prepare(hvdg_ctx* ctx, Staged& S, const RunOpts& opt);
hvdg::SolverArgs solver_args(hvdg_ctx* ctx, const Staged& S);
int solver_grid(hvdg_ctx* ctx, int n_units, int ctas_override = -1);
hvdg_status stage_finish(hvdg_ctx* ctx, Staged& S, hvdg_field_out* out, const RunOpts& opt,
                         hvdg_diag* diag);
hvdg_status run_batch_once(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                           hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt_in);
std::string batch_signature(const hvdg_field_in* in, int n, const hvdg_config* cfg);
hvdg_status run_batch_graph(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                            hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt);
hvdg_status graph_result(hvdg_ctx* ctx, hvdg_diag* diag);
hvdg_status run_batch(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                      hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt_in);
hvdg_status validate_fields(const hvdg_field_in* fields, int n, const hvdg_config* cfg,
                            hvdg_field_out* out);
float median_mean(std::vector<float> v);
float strength_from_pairs(const std::vector<float>& pair_amb, const std::vector<int>& pair_ok,
                          float nr_eps, float* amb_out);
hvdg_status decode_window_3d(hvdg_ctx* ctx, const hvdg_field_in* in, int nf,
                             const hvdg_config* cfg_in, hvdg_field_out* out, hvdg_diag* diag,
                             const RunOpts& opt);
hvdg_status decode_window_impl(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                               const hvdg_config* cfg, hvdg_field_out* out, hvdg_diag* diag,
                               const RunOpts& opt = RunOpts());
int64_t frame_line_offset(const hvdg_frame_params& fp, int line);
hvdg_geometry geometry_from_params(const hvdg_frame_params& fp);
void split_frame_fields(const int16_t* frame, const hvdg_frame_params& fp, float* top,
                        float* bottom);
int detect_field_parity(const float* b1, const float* b2, const hvdg_frame_params& fp,
                        const hvdg_geometry& g);
hvdg::FrameVoteArgs vote_grid(const hvdg_frame_params& P, const hvdg_geometry& g);
hvdg_status detect_field_parity_frames(hvdg_ctx* ctx, const int16_t* const* frames, int n,
                                       const hvdg_frame_params* fp, int32_t* votes);
std::vector<SelBox> ambiguous_boxes(const float* Y, const float* chi_ri, int h, int w,
                                    float max_area);
hvdg_status decode_selective_boxes(hvdg_ctx* ctx, const std::vector<hvdg_field_in>& fi,
                                   const hvdg_geometry& g, const hvdg_config* cfg,
                                   const std::vector<float*>& Yd,
                                   const std::vector<float*>& Cd);
void write_debug_maps(const std::string& dir, int64_t base_frame_id, int core_begin, int core_end,
                      bool f1_bottom, const hvdg_diag& d, float acc_gain,
                      const std::vector<float*>& Y,
                      const std::vector<std::vector<float2>>& car, const std::vector<int>& parity,
                      int lines, int aw);
int16_t clamp_u10(float v);
int16_t clamp_s10(float v);
hvdg_status lockin_one(hvdg_ctx* ctx, const float* field_ire, const hvdg_geometry* g, float* theta,
                       int8_t* vswitch, float* amp);
hvdg_status estimate_motion_sad(hvdg_ctx* ctx, const float* y_ref, const float* y_cur, int h,
                                int w, int block, int range, float* dy, float* dx,
                                float* confidence);
hvdg_status decode_adjoint_field(hvdg_ctx* ctx, const hvdg_field_in& fi, const hvdg_config& cfg,
                                 const float* y_bar, const float* chi_bar, float* samples_bar,
                                 double* scalar_bar, int adj_iters, hvdg_field_out* out,
                                 hvdg_diag* diag);
hvdg_status decode_woven_frames(hvdg_ctx* ctx, const int16_t* const* chroma,
                                const int16_t* const* luma, int n, const hvdg_frame_params* fp,
                                const hvdg_config* cfg, hvdg_yc_frame* out, hvdg_diag* diag,
                                bool yc);

}  // namespace hvdg_pipe
