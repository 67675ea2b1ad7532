// api.cu -- the C ABI (include/hvdg.h): context, device arena, batch
// planning, host-side tables, and the decode pipelines.
//
// Host orchestration replaces hvd-core's HvdEngine / DecodeFieldWindow
// driver (hvd-core/src/engine/engine.cpp:133-137,
// hvd-core/src/engine/sequence.cpp:229-281, 423-1116): instead of one OpenMP
// solve per field, a batch of fields is laid out in one device arena and
// every stage runs as one launch over all fields.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
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

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Geometry helpers (mirror FieldGeometry, ntsc_geometry.h:142-267)
// ---------------------------------------------------------------------------
bool uses_vswitch(const hvdg_geometry& g) {
  return g.standard == HVDG_STD_PAL || g.standard == HVDG_STD_PAL_M;
}
int last_active_line(const hvdg_geometry& g) {
  return g.last_active_field_line != 0 ? g.last_active_field_line : g.field_height;
}
double phase_per_sample(const hvdg_geometry& g) {
  if (g.subcarrier_hz <= 0.0) return 0.5 * kPi;
  return 2.0 * kPi * g.subcarrier_hz / g.sample_rate;
}
double line_advance(const hvdg_geometry& g) {
  if (g.subcarrier_hz <= 0.0) {
    if (g.standard == HVDG_STD_PAL) return 2.0 * kPi * 0.7516;
    if (g.standard == HVDG_STD_PAL_M) return 0.5 * kPi;
    return kPi;
  }
  const double cycles = g.subcarrier_hz * (double)g.field_width / g.sample_rate;
  return 2.0 * kPi * (cycles - std::floor(cycles));
}
float nominal_burst(const hvdg_geometry& g) {
  return g.standard == HVDG_STD_PAL ? 21.43f : 20.0f;
}

// Device-path limits of one solve plane of w x h (documented in
// include/hvdg.h): the row / column cyclic-convolution lengths of the init
// and the auto-aniso sample buffer.
hvdg_status check_plane(int w, int h, bool vsw, int col_max) {
  const int pad = std::min(hvdg::kInitPad, h - 1);
  if (2 * w - 1 > hvdg::kRowFft || 2 * (h + 2 * pad) - 1 > col_max) return HVDG_ERR_UNSUPPORTED;
  const int group = vsw ? 4 : 2;
  const int64_t n = (int64_t)((h / group) / 2) * ((w + 1) / 3);
  if (n > hvdg::aniso_max_samples()) return HVDG_ERR_UNSUPPORTED;
  return HVDG_OK;
}

hvdg_status check_geometry(const hvdg_geometry* g) {
  if (!g) return HVDG_ERR_BAD_ARGUMENT;
  if (g->standard < 0 || g->standard > 2) return HVDG_ERR_BAD_ARGUMENT;
  const int lal = last_active_line(*g);
  if (g->field_width < 1 || g->field_height < 1) return HVDG_ERR_BAD_GEOMETRY;
  if (g->active_video_start < 0 || g->active_video_end > g->field_width ||
      g->active_video_end - g->active_video_start < 2)
    return HVDG_ERR_BAD_GEOMETRY;
  if (g->first_active_field_line < 0 || lal > g->field_height ||
      lal - g->first_active_field_line < 2)
    return HVDG_ERR_BAD_GEOMETRY;
  if (g->colour_burst_start < 0 || g->colour_burst_end > g->field_width ||
      g->colour_burst_end < g->colour_burst_start)
    return HVDG_ERR_BAD_GEOMETRY;
  if (!(g->sample_rate > 0.0)) return HVDG_ERR_BAD_GEOMETRY;
  // device-path limits (documented in include/hvdg.h)
  if (g->field_height > hvdg::kMaxLines) return HVDG_ERR_UNSUPPORTED;
  const int w = g->active_video_end - g->active_video_start;
  const int h = lal - g->first_active_field_line;
  const hvdg_status st = check_plane(w, h, uses_vswitch(*g), hvdg::kColFft);
  if (st != HVDG_OK) return st;
  if (g->colour_burst_end - g->colour_burst_start > 64 + 3) return HVDG_ERR_UNSUPPORTED;
  return HVDG_OK;
}

// ---------------------------------------------------------------------------
// Host-side init tables (double precision, cached per geometry).
// ---------------------------------------------------------------------------
using cd = std::complex<double>;

// numpy.fft.fftfreq(n, d) (holographic_init.cpp:20-30)
double fftfreq(int i, int n, double d) {
  const int half = (n % 2 == 0) ? n / 2 : (n + 1) / 2;
  const int k = i < half ? i : i - n;
  return k / (n * d);
}

// Spectrum (length M, scaled by `scale` / M) of the circular kernel
// k = IDFT_n(mask), embedded for a cyclic convolution of length M >= 2n - 1.
std::vector<cd> kernel_spectrum(const std::vector<double>& mask, int M, double scale) {
  const int n = (int)mask.size();
  std::vector<cd> k(n);
  std::vector<cd> twn(n);
  for (int j = 0; j < n; ++j) twn[j] = cd(std::cos(2 * kPi * j / n), std::sin(2 * kPi * j / n));
  for (int j = 0; j < n; ++j) {
    cd acc = 0.0;
    for (int q = 0; q < n; ++q) acc += mask[q] * twn[(int64_t)j * q % n];
    k[j] = acc / (double)n;
  }
  std::vector<cd> emb(M, cd(0, 0));
  for (int j = -(n - 1); j <= n - 1; ++j) emb[((j % M) + M) % M] = k[((j % n) + n) % n];
  std::vector<cd> twm(M);
  for (int j = 0; j < M; ++j) twm[j] = cd(std::cos(2 * kPi * j / M), -std::sin(2 * kPi * j / M));
  std::vector<cd> out(M);
  for (int m = 0; m < M; ++m) {
    cd acc = 0.0;
    for (int j = 0; j < M; ++j) {
      if (emb[j] == cd(0, 0)) continue;
      acc += emb[j] * twm[(int64_t)j * m % M];
    }
    out[m] = acc * (scale / M);
  }
  return out;
}

struct GeomTables {
  int w, h, hp, pad;
  int col_m;                     // column convolution length (kColFft or kColFftWide)
  std::vector<float2> khat_row;  // 2 * kRowFft
  std::vector<float2> khat_col;  // 2 * col_m
  std::vector<float2> col_phasor;
  // symmetry variant (built on first use): row chirp (w) | row chirp-filter
  // spectrum (kRowFft) | column chirp (hp) | column filter spectrum (col_m) |
  // gx (w) | gy (hp), the last two in .x
  bool sym_ready = false;
  std::vector<float2> sym;
};

// The two crop variants of HolographicInit (holographic_init.cpp:236).
const double kVariants[2][2] = {{0.8, 120.0}, {1.8, 30.0}};

GeomTables make_geom_tables(const hvdg_geometry& g) {
  GeomTables t;
  t.w = g.active_video_end - g.active_video_start;
  t.h = last_active_line(g) - g.first_active_field_line;
  t.pad = std::min(hvdg::kInitPad, t.h > 1 ? t.h - 1 : 0);
  t.hp = t.h + 2 * t.pad;
  t.col_m = 2 * t.hp - 1 <= hvdg::kColFft ? hvdg::kColFft : hvdg::kColFftWide;
  for (int v = 0; v < 2; ++v) {
    std::vector<double> gx(t.w), gy(t.hp);
    const double cx = kVariants[v][0] * 1.0e6;
    const double cy = kVariants[v][1] / (2.0 * t.h);  // against the REAL height
    for (int i = 0; i < t.w; ++i) {
      const double r = fftfreq(i, t.w, 1.0 / g.sample_rate) / cx;
      gx[i] = std::exp(-0.5 * r * r);
    }
    for (int i = 0; i < t.hp; ++i) {
      const double r = fftfreq(i, t.hp, 1.0) / cy;
      gy[i] = std::exp(-0.5 * r * r);
    }
    for (const cd& c : kernel_spectrum(gx, hvdg::kRowFft, 1.0))
      t.khat_row.push_back(make_float2((float)c.real(), (float)c.imag()));
    // x2 of the init (holographic_init.cpp:247-251) folded into the column pass
    for (const cd& c : kernel_spectrum(gy, t.col_m, 2.0))
      t.khat_col.push_back(make_float2((float)c.real(), (float)c.imag()));
  }
  const double w0 = phase_per_sample(g);
  const bool quad = g.subcarrier_hz <= 0.0;
  for (int x = 0; x < t.w; ++x) {
    const int s = g.active_video_start + x;
    if (quad) {
      static const float2 q[4] = {{1.f, 0.f}, {0.f, 1.f}, {-1.f, 0.f}, {0.f, -1.f}};
      t.col_phasor.push_back(q[s & 3]);
    } else {
      t.col_phasor.push_back(make_float2((float)std::cos(w0 * s), (float)std::sin(w0 * s)));
    }
  }
  return t;
}

// In-place radix-2 DFT of a power-of-two length, exp(-2 pi i jk / n), double.
void host_fft(std::vector<cd>& a) {
  const int n = (int)a.size();
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; ++k) {
        const double ang = -2.0 * kPi * k / len;
        const cd u = a[i + k], v = a[i + k + len / 2] * cd(std::cos(ang), std::sin(ang));
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

// Bluestein tables of an exact-length DFT of length N through a cyclic
// convolution of length M: chirp c[n] = exp(-i pi n^2 / N) and the spectrum
// of the filter conj(c) wrapped to length M, divided by M.
void bluestein_tables(int N, int M, std::vector<float2>* out) {
  std::vector<cd> c(N);
  for (int k = 0; k < N; ++k) {
    const int64_t kk = (int64_t)k * k % (2LL * N);  // exact reduction of the phase
    c[k] = cd(std::cos(kPi * (double)kk / N), -std::sin(kPi * (double)kk / N));
  }
  for (int k = 0; k < N; ++k) out->push_back(make_float2((float)c[k].real(), (float)c[k].imag()));
  std::vector<cd> h(M, cd(0, 0));
  for (int k = 0; k < N; ++k) {
    h[k] = std::conj(c[k]);
    if (k) h[M - k] = std::conj(c[k]);
  }
  host_fft(h);
  for (int m = 0; m < M; ++m)
    out->push_back(make_float2((float)(h[m].real() / M), (float)(h[m].imag() / M)));
}

// The symmetry variant's tables (holographic_init.cpp:265-306). Its crop
// {1.3 MHz, 60 c/ph} multiplies the spectrum directly, so gx / gy are
// evaluated as GaussianLpf does (holographic_init.cpp:16-56): float
// frequencies, float cutoffs, float exp.
void make_sym_tables(GeomTables& t, const hvdg_geometry& g) {
  t.sym.clear();
  bluestein_tables(t.w, hvdg::kRowFft, &t.sym);
  bluestein_tables(t.hp, t.col_m, &t.sym);
  auto freq = [](int i, int n, double d) {
    const double inv = 1.0 / ((double)n * d);
    const int half = (n % 2 == 0) ? n / 2 : (n + 1) / 2;
    return (float)((i < half ? i : i - n) * inv);
  };
  const float cx = 1.3f * 1.0e6f;
  const float cy = 60.0f / (2.0f * (float)t.h);
  for (int x = 0; x < t.w; ++x) {
    const float r = freq(x, t.w, 1.0 / g.sample_rate) / cx;
    t.sym.push_back(make_float2(std::exp(-0.5f * r * r), 0.f));
  }
  for (int y = 0; y < t.hp; ++y) {
    const float r = freq(y, t.hp, 1.0) / cy;
    t.sym.push_back(make_float2(std::exp(-0.5f * r * r), 0.f));
  }
  t.sym_ready = true;
}

using GeomKey = std::tuple<int, int, int, int, int, int, double, double>;
GeomKey geom_key(const hvdg_geometry& g) {
  return GeomKey(g.active_video_start, g.active_video_end, g.first_active_field_line,
                 last_active_line(g), g.standard, g.field_width, g.sample_rate, g.subcarrier_hz);
}

std::vector<float2> twiddles(int M) {
  std::vector<float2> t(M);
  for (int k = 0; k < M; ++k) {
    const double a = -2.0 * kPi * k / M;
    t[k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  return t;
}

}  // namespace

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
  hvdg::DeviceArena arena;
  hvdg::PinnedArena pinned;
  std::map<GeomKey, GeomTables> geoms;
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

namespace hvdg {

// Init tables of one geometry (the same tables run_batch uploads), for
// translation units that launch the init kernels on their own memory.
void init_tables_for(const hvdg_geometry& g, std::vector<float2>* khat_row_col,
                     std::vector<float2>* col_phasor, std::vector<float2>* tw_row,
                     std::vector<float2>* tw_col, int* hp, int* pad) {
  const GeomTables t = make_geom_tables(g);
  khat_row_col->assign(t.khat_row.begin(), t.khat_row.end());
  khat_row_col->insert(khat_row_col->end(), t.khat_col.begin(), t.khat_col.end());
  *col_phasor = t.col_phasor;
  *tw_row = twiddles(kRowFft);
  *tw_col = twiddles(kColFft);
  *hp = t.hp;
  *pad = t.pad;
}

hvdg_status cuda_fail(hvdg_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HVDG_OK;
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  ctx->last_error = buf;
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? HVDG_ERR_OUT_OF_MEMORY : HVDG_ERR_CUDA;
}

hvdg_status DeviceArena::reserve(size_t bytes, cudaStream_t st) {
  if (bytes <= capacity) return HVDG_OK;
  if (base) {
    // work queued on the context stream may still read the old arena
    cudaStreamSynchronize(st);
    cudaFree(base);
  }
  base = nullptr;
  capacity = 0;
  const size_t want = bytes + bytes / 8;
  if (cudaMalloc(&base, want) != cudaSuccess) {
    cudaGetLastError();
    return HVDG_ERR_OUT_OF_MEMORY;
  }
  // zeroed on the context stream: the stream is non-blocking, so a
  // legacy-stream memset would race the uploads and kernels queued after it
  if (cudaMemsetAsync(base, 0, want, st) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(base);
    base = nullptr;
    return HVDG_ERR_CUDA;
  }
  capacity = want;
  return HVDG_OK;
}
DeviceArena::~DeviceArena() {
  if (base) cudaFree(base);
}
hvdg_status PinnedArena::reserve(size_t bytes) {
  if (bytes <= capacity) return HVDG_OK;
  if (base) cudaFreeHost(base);
  base = nullptr;
  capacity = 0;
  if (cudaMallocHost(&base, bytes) != cudaSuccess) {
    cudaGetLastError();
    return HVDG_ERR_OUT_OF_MEMORY;
  }
  capacity = bytes;
  return HVDG_OK;
}
PinnedArena::~PinnedArena() {
  if (base) cudaFreeHost(base);
}

}  // namespace hvdg

namespace {

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
      o_S, o_Y, o_X0, o_X1, o_G0, o_G1, o_D0, o_D1, o_Q0, o_Q1, o_W, o_rowbuf, o_itab, o_amp;
  size_t total;
  int64_t total_px, total_rowbuf;
  int total_lines, total_theta, total_units, total_prows, total_cgroups, total_btiles;
  int ncol, nkhat;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

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

int elem_size(int sample_type) { return sample_type == HVDG_SAMPLES_F32_IRE ? 4 : 2; }

// Solver band height when none is set: the tallest band (fewest halo rows)
// that still gives every resident warp a unit of the fields solved
// together; small batches (one field, one colour of a 3-D window) get short
// bands, so a phase is not bound by one warp walking 32 rows.
int auto_band_rows_hw(hvdg_ctx* ctx, const std::vector<std::pair<int, int>>& hw) {
  const int warps = ctx->sm_count * std::max(1, hvdg::solver_max_blocks_per_sm()) *
                    (hvdg::kSolverThreads / 32);
  static const int cand[] = {32, 24, 16, 12, 8, 6, 4};
  for (int band : cand) {
    int64_t units = 0;
    for (const auto& p : hw)
      units += (int64_t)((p.second + hvdg::kStrip - 1) / hvdg::kStrip) * ((p.first + band - 1) / band);
    if (units >= warps) return band;
  }
  return 4;
}

int auto_band_rows(hvdg_ctx* ctx, const std::vector<FieldPlan>& fp) {
  std::vector<std::pair<int, int>> hw;
  for (const FieldPlan& p : fp) hw.emplace_back(p.h, p.w);
  return auto_band_rows_hw(ctx, hw);
}

// Plan a batch. Normally every entry of `in` is one plane. With
// `weave_geom` set, `in` holds 2 m source fields, two per woven frame
// (WeaveAndBuildCarrier, engine.cpp:53-126): the field whose parity is 0
// lands on the even rows of its frame's plane, the other on the odd rows,
// and the planes take the geometry *weave_geom (the woven active picture:
// no blanking, 2 x active lines). The source fields are F32 IRE planes
// written on the device (the caller's split), so no raw upload is planned
// for them beyond their f32 slots.
hvdg_status plan_batch(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                       int band_rows, Batch& b, const hvdg_geometry* weave_geom = nullptr) {
  b = Batch();
  std::map<GeomKey, int> slot;
  int64_t px = 0, rawb = 0, rowb = 0;
  int lines = 0, theta = 0;
  if (weave_geom && (n % 2) != 0) return HVDG_ERR_BAD_ARGUMENT;
  const int m = weave_geom ? n / 2 : n;
  for (int k = 0; k < n; ++k) {
    const hvdg_geometry& g = *in[k].geometry;
    PrepPlan q;
    q.fh = g.field_height;
    q.fw = g.field_width;
    q.theta_off = theta;
    theta += q.fh;
    q.raw_bytes = (int64_t)q.fh * q.fw * elem_size(in[k].sample_type);
    q.raw_off = rawb;
    rawb += align_up(q.raw_bytes, 256);
    b.pp.push_back(q);
  }
  for (int i = 0; i < m; ++i) {
    const hvdg_geometry* gp = weave_geom ? weave_geom : in[i].geometry;
    const hvdg_geometry& g = *gp;
    const GeomKey key = geom_key(g);
    auto it = ctx->geoms.find(key);
    if (it == ctx->geoms.end()) it = ctx->geoms.emplace(key, make_geom_tables(g)).first;
    if (cfg->symmetry_variant && !it->second.sym_ready) make_sym_tables(it->second, g);
    int gs;
    auto sit = slot.find(key);
    if (sit == slot.end()) {
      gs = (int)b.gtabs.size();
      slot.emplace(key, gs);
      b.gtabs.push_back(&it->second);
    } else {
      gs = sit->second;
    }
    FieldPlan p;
    p.g = gp;
    p.fh = g.field_height;
    p.fw = g.field_width;
    p.h = last_active_line(g) - g.first_active_field_line;
    p.w = g.active_video_end - g.active_video_start;
    p.pitch = (p.w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
    p.px_off = px;
    px += (int64_t)p.h * p.pitch;
    p.line_off = lines;
    lines += p.h;
    p.geom_slot = gs;
    p.hp = it->second.hp;
    p.rowbuf_off = rowb;
    rowb += 2LL * p.hp * p.pitch;
    b.fp.push_back(p);
  }
  // geometry descriptors + packed tables
  int ncol = 0, nkhat = 0;
  for (size_t s = 0; s < b.gtabs.size(); ++s) {
    const GeomTables& t = *b.gtabs[s];
    GeomDesc gd;
    gd.w = t.w;
    gd.h = t.h;
    gd.hp = t.hp;
    gd.pad = t.pad;
    gd.khat_row_off = nkhat;
    nkhat += 2 * hvdg::kRowFft;
    gd.khat_col_off = nkhat;
    gd.col_m = t.col_m;
    nkhat += 2 * t.col_m;
    gd.sym_row_chirp = gd.sym_row_hhat = gd.sym_col_chirp = gd.sym_col_hhat = -1;
    gd.sym_gx = gd.sym_gy = -1;
    if (cfg->symmetry_variant) {
      gd.sym_row_chirp = nkhat;
      gd.sym_row_hhat = gd.sym_row_chirp + t.w;
      gd.sym_col_chirp = gd.sym_row_hhat + hvdg::kRowFft;
      gd.sym_col_hhat = gd.sym_col_chirp + t.hp;
      gd.sym_gx = gd.sym_col_hhat + t.col_m;
      gd.sym_gy = gd.sym_gx + t.w;
      nkhat += (int)t.sym.size();
    }
    b.geoms.push_back(gd);
    b.gcol_off.push_back(ncol);
    ncol += t.w;
  }
  // per-field descriptors, units
  const int band = band_rows > 0 ? band_rows : auto_band_rows(ctx, b.fp);
  for (int i = 0; i < m; ++i) {
    const FieldPlan& p = b.fp[i];
    const hvdg_geometry& g = *p.g;
    const hvdg_field_in& fi = in[weave_geom ? 2 * i : i];
    FieldDesc f;
    std::memset(&f, 0, sizeof(f));
    f.h = p.h;
    f.w = p.w;
    f.pitch = p.pitch;
    f.fh = p.fh;
    f.fw = p.fw;
    f.px_off = p.px_off;
    f.line_off = p.line_off;
    f.col_off = b.gcol_off[p.geom_slot];
    f.geom = p.geom_slot;
    f.is_pal = uses_vswitch(g) ? 1 : 0;
    // solver budget (variational.cpp:224-230)
    const int outer_cfg = fi.irls_outer > 0 ? fi.irls_outer : cfg->irls_outer;
    const int cg_cfg = fi.cg_iterations >= 0 ? fi.cg_iterations : cfg->cg_iterations;
    f.n_outer = std::max(1, outer_cfg);
    const int cg_total = cfg->fast ? cg_cfg * 2 / 3 : cg_cfg;
    f.n_inner = std::max(1, cg_total / f.n_outer);
    f.cg_tol = cfg->cg_tol > 0.0f ? cfg->cg_tol : (cfg->fast ? 0.10f : 0.02f);
    f.eps = cfg->charbonnier_eps;
    f.eps_c = cfg->chroma_eps;
    f.k_coupling = cfg->structure_coupling;
    f.lambda_c = cfg->lambda_c;
    f.aniso_cfg = cfg->chroma_aniso;
    f.mu_h = cfg->lambda_c;
    f.mu_v = cfg->lambda_c;
    f.plane_px = (int64_t)p.h * p.pitch;
    f.unit_begin = (int)b.units.size();
    for (int x0 = 0; x0 < p.w; x0 += hvdg::kStrip)
      for (int y0 = 0; y0 < p.h; y0 += band) b.units.push_back(Unit{i, x0, y0, std::min(p.h, y0 + band)});
    f.unit_count = (int)b.units.size() - f.unit_begin;
    f.n_phases = f.n_outer * (2 + f.n_inner) + 1;
    b.max_phases = std::max(b.max_phases, f.n_phases);
    b.fields.push_back(f);

    b.px_offs.push_back(p.px_off);
    b.pitches.push_back(p.pitch);
    b.rowbuf_offs.push_back(p.rowbuf_off);
  }
  // source-field descriptors and the crop rows
  for (int k = 0; k < n; ++k) {
    const hvdg_geometry& g = *in[k].geometry;
    const PrepPlan& q = b.pp[k];
    const int plane = weave_geom ? k / 2 : k;
    const FieldPlan& p = b.fp[plane];
    // woven: this field's active line y lands on plane row 2 y + row0
    const int row0 = weave_geom ? (in[k].parity == 0 ? 0 : 1) : 0;
    const int step = weave_geom ? 2 : 1;
    hvdg::PrepDesc pd;
    std::memset(&pd, 0, sizeof(pd));
    pd.sample_type = in[k].sample_type;
    pd.quadrant = g.subcarrier_hz <= 0.0 ? 1 : 0;
    pd.blank = in[k].blanking_level;
    pd.codes_per_ire = (in[k].white_level - in[k].blanking_level) / 100.0f;
    pd.fh = q.fh;
    pd.fw = q.fw;
    pd.bx0 = g.colour_burst_start;
    pd.bx1 = g.colour_burst_end;
    pd.fal = g.first_active_field_line;
    pd.lal = last_active_line(g);
    pd.a0 = g.active_video_start;
    pd.a1 = g.active_video_end;
    pd.vswitch_family = uses_vswitch(g) ? 1 : 0;
    pd.nominal_burst = nominal_burst(g);
    pd.w0 = phase_per_sample(g);
    pd.adv = line_advance(g);
    pd.chroma_phase_off = -cfg->chroma_phase_deg * 3.14159265358979323846f / 180.0f;
    pd.theta_off = q.theta_off;
    pd.line_off = p.line_off + row0;
    pd.line_step = step;
    b.prep.push_back(pd);
    const int lines_k = pd.lal - pd.fal;
    for (int y = 0; y < lines_k; ++y)
      b.crop_rows.push_back(make_int4(plane, row0 + step * y, k, pd.fal + y));
  }
  // init tables
  std::vector<int> prow_field, prow_first, cgrp_field, cgrp_first, btile_field, btile_first;
  const int bt = hvdg::init_blend_tile();
  for (int i = 0; i < m; ++i) {
    const FieldPlan& p = b.fp[i];
    const int cg = hvdg::init_col_group(b.gtabs[p.geom_slot]->col_m);
    prow_first.push_back((int)prow_field.size());
    for (int y = 0; y < p.hp; ++y) prow_field.push_back(i);
    cgrp_first.push_back((int)cgrp_field.size());
    for (int x = 0; x < p.w; x += cg) cgrp_field.push_back(i);
    btile_first.push_back((int)btile_field.size());
    const int nt = ((p.h + bt - 1) / bt) * ((p.w + bt - 1) / bt);
    for (int t = 0; t < nt; ++t) btile_field.push_back(i);
  }
  auto append = [&](const std::vector<int>& v) {
    const int off = (int)b.itab.size();
    b.itab.insert(b.itab.end(), v.begin(), v.end());
    return off;
  };
  b.it_prow_field = append(prow_field);
  b.it_prow_first = append(prow_first);
  b.it_cgrp_field = append(cgrp_field);
  b.it_cgrp_first = append(cgrp_first);
  b.it_btile_field = append(btile_field);
  b.it_btile_first = append(btile_first);
  // crop tables appended to itab too
  Layout& L = b.L;
  L.total_px = px;
  L.total_rowbuf = rowb;
  L.total_lines = lines;
  L.total_theta = theta;
  L.total_units = (int)b.units.size();
  L.total_prows = (int)prow_field.size();
  L.total_cgroups = (int)cgrp_field.size();
  L.total_btiles = (int)btile_field.size();
  L.ncol = ncol;
  L.nkhat = nkhat;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align_up(o + bytes, 256);
    return r;
  };
  L.o_raw = take(rawb);
  L.o_prep = take(sizeof(hvdg::PrepDesc) * n);
  L.o_fields = take(sizeof(FieldDesc) * m);
  L.o_geoms = take(sizeof(GeomDesc) * b.geoms.size());
  L.o_ctl = take(sizeof(FieldCtl) * m);
  L.o_units = take(sizeof(Unit) * b.units.size());
  L.o_partials = take(sizeof(double) * 5 * b.units.size());
  L.o_done = take(sizeof(int) * m);
  L.o_arrive = take(sizeof(int) * m);
  L.o_flags = take(sizeof(int) * 4);
  L.o_queue = take(sizeof(unsigned long long));
  L.o_lineph = take(sizeof(float4) * lines);
  L.o_theta = take(sizeof(float) * theta);
  L.o_theta64 = take(sizeof(double) * theta);
  L.o_vsw = take(theta);
  L.o_colph = take(sizeof(float2) * ncol);
  L.o_khat = take(sizeof(float2) * nkhat);
  L.o_twr = take(sizeof(float2) * hvdg::kRowFft);
  L.o_twc = take(sizeof(float2) * hvdg::kColFft);
  L.o_amp = take(sizeof(float) * n);
  // index tables: itab | pitches | crop rows (int4) | px_offs (int64) | rowbuf offs (int64)
  L.o_itab = take(sizeof(int) * (b.itab.size() + b.pitches.size()) + sizeof(int4) * b.crop_rows.size() +
                  sizeof(int64_t) * (b.px_offs.size() + b.rowbuf_offs.size()) + 64);
  L.o_S = take(sizeof(float) * px);
  L.o_Y = take(sizeof(float) * px);
  L.o_X0 = take(sizeof(float2) * px);
  L.o_X1 = take(sizeof(float2) * px);
  L.o_G0 = take(sizeof(float2) * px);
  L.o_G1 = take(sizeof(float2) * px);
  L.o_D0 = take(sizeof(float2) * px);
  L.o_D1 = take(sizeof(float2) * px);
  L.o_Q0 = take(sizeof(float2) * px);
  L.o_Q1 = take(sizeof(float2) * px);
  L.o_W = take(sizeof(float4) * px);
  L.o_rowbuf = take(sizeof(float2) * rowb);
  L.total = o;
  return HVDG_OK;
}

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

// Timing marks on the context stream. Inside a stream capture a record has
// to become a graph node (cudaEventRecordExternal), or replays never record
// the event and the elapsed times would be stale.
void mark(hvdg_ctx* ctx, int i) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cs);
  if (cs == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(ctx->ev[i], ctx->stream, cudaEventRecordExternal);
  else
    cudaEventRecord(ctx->ev[i], ctx->stream);
}

// Milliseconds between two marks (0 when either was not recorded).
float elapsed(hvdg_ctx* ctx, int a, int b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]) != cudaSuccess) {
    cudaGetLastError();
    ms = 0.f;
  }
  return ms;
}

// Per-call device state reset (solver control, flags, work queue) and the
// start event; stream-ordered, so it can live inside a captured graph.
void stage_reset(hvdg_ctx* ctx, const Staged& S) {
  const Layout& L = S.b.L;
  const int n = (int)S.b.fp.size();
  cudaStream_t s = ctx->stream;
  mark(ctx, 0);
  cudaMemsetAsync(at<char>(ctx, L.o_ctl), 0, sizeof(FieldCtl) * n, s);
  cudaMemsetAsync(at<char>(ctx, L.o_arrive), 0, sizeof(int) * n, s);
  cudaMemsetAsync(at<char>(ctx, L.o_done), 0xff, sizeof(int) * n, s);
  cudaMemsetAsync(at<char>(ctx, L.o_flags), 0, sizeof(int) * 4, s);
  cudaMemsetAsync(at<char>(ctx, L.o_queue), 0, sizeof(unsigned long long), s);
}

// Plan the batch, reserve the arena (+ `extra_bytes` for the caller), upload
// the tables and raw samples, reset the solver control state.
hvdg_status stage_upload(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                         const RunOpts& opt, size_t extra_bytes, Staged& S) {
  Batch& b = S.b;
  // drop a stale non-sticky error left by an earlier, already reported call,
  // so the launch checks below see only this call's launches
  cudaGetLastError();
  hvdg_status st = plan_batch(ctx, in, n, cfg, opt.band_rows >= 0 ? opt.band_rows : ctx->band_rows, b,
                              opt.weave_geom);
  if (st != HVDG_OK) return st;
  const Layout& L = b.L;
  const int m = (int)b.fp.size();
  S.extra = align_up(L.total, 256);
  st = ctx->arena.reserve(S.extra + extra_bytes, ctx->stream);
  if (st != HVDG_OK) {
    ctx->last_error = "device arena allocation failed";
    return st;
  }
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  std::vector<char> host(L.o_S - L.o_prep, 0);
  auto put = [&](size_t off, const void* src, size_t bytes) {
    if (bytes) std::memcpy(host.data() + (off - L.o_prep), src, bytes);
  };
  for (int k = 0; k < n; ++k) {
    b.prep[k].samples = (opt.device_io && !opt.weave_geom)
                            ? in[k].samples
                            : (const void*)(at<char>(ctx, L.o_raw) + b.pp[k].raw_off);
  }
  b.direct_y.assign(m, 0);
  b.direct_c.assign(m, 0);
  if (opt.out_direct && opt.do_solve && !opt.weave_geom) {
    // a buffer the kernel can address: device memory (device_io) or
    // page-locked host memory mapped into the device's address space
    auto reach = [&](void* p) -> void* {
      if (!p) return nullptr;
      if (opt.device_io) return p;
      cudaPointerAttributes pa;
      if (cudaPointerGetAttributes(&pa, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
      return pa.type == cudaMemoryTypeHost ? pa.devicePointer : nullptr;
    };
    for (int i = 0; i < m; ++i) {
      b.fields[i].out_y = static_cast<float*>(reach(opt.out_direct[i].luma));
      b.fields[i].out_c = static_cast<float2*>(reach(opt.out_direct[i].chroma));
      b.direct_y[i] = b.fields[i].out_y != nullptr;
      b.direct_c[i] = b.fields[i].out_c != nullptr;
    }
  }
  put(L.o_prep, b.prep.data(), sizeof(hvdg::PrepDesc) * n);
  put(L.o_fields, b.fields.data(), sizeof(FieldDesc) * m);
  put(L.o_geoms, b.geoms.data(), sizeof(GeomDesc) * b.geoms.size());
  put(L.o_units, b.units.data(), sizeof(Unit) * b.units.size());
  {
    std::vector<int> done(m, -1);
    put(L.o_done, done.data(), sizeof(int) * m);
  }
  {
    std::vector<float2> col, kh;
    for (size_t g = 0; g < b.gtabs.size(); ++g) {
      col.insert(col.end(), b.gtabs[g]->col_phasor.begin(), b.gtabs[g]->col_phasor.end());
      kh.insert(kh.end(), b.gtabs[g]->khat_row.begin(), b.gtabs[g]->khat_row.end());
      kh.insert(kh.end(), b.gtabs[g]->khat_col.begin(), b.gtabs[g]->khat_col.end());
      if (b.geoms[g].sym_row_chirp >= 0)
        kh.insert(kh.end(), b.gtabs[g]->sym.begin(), b.gtabs[g]->sym.end());
    }
    put(L.o_colph, col.data(), sizeof(float2) * col.size());
    put(L.o_khat, kh.data(), sizeof(float2) * kh.size());
    static const std::vector<float2> twr = twiddles(hvdg::kRowFft), twc = twiddles(hvdg::kColFft);
    put(L.o_twr, twr.data(), sizeof(float2) * twr.size());
    put(L.o_twc, twc.data(), sizeof(float2) * twc.size());
  }
  size_t it = L.o_itab;
  S.it_itab = it;
  put(it, b.itab.data(), sizeof(int) * b.itab.size());
  it += sizeof(int) * b.itab.size();
  S.it_pitch = it;
  put(it, b.pitches.data(), sizeof(int) * b.pitches.size());
  it += sizeof(int) * b.pitches.size();
  it = align_up(it, 16);
  S.it_crop = it;
  put(it, b.crop_rows.data(), sizeof(int4) * b.crop_rows.size());
  it += sizeof(int4) * b.crop_rows.size();
  S.it_pxoff = it;
  put(it, b.px_offs.data(), sizeof(int64_t) * b.px_offs.size());
  it += sizeof(int64_t) * b.px_offs.size();
  S.it_rbo = it;
  put(it, b.rowbuf_offs.data(), sizeof(int64_t) * b.rowbuf_offs.size());

  if (!opt.device_io && opt.do_lockin && !opt.weave_geom) {
    for (int i = 0; i < n; ++i) {
      e = cudaMemcpyAsync(at<char>(ctx, L.o_raw) + b.pp[i].raw_off, in[i].samples,
                          (size_t)b.pp[i].raw_bytes, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D samples");
    }
  }
  e = cudaMemcpyAsync(at<char>(ctx, L.o_prep), host.data(), host.size(), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D tables");
  ctx->epoch += 1;
  if (!opt.tables_only) stage_reset(ctx, S);
  return HVDG_OK;
}

// Holographic-init kernel arguments for a staged batch (variants chi1 / chi2
// land in G0 / D0, the blend in X0 and Y).
hvdg::InitArgs init_args(hvdg_ctx* ctx, const Staged& S) {
  const Batch& b = S.b;
  const Layout& L = b.L;
  hvdg::InitArgs ia;
  ia.fields = at<FieldDesc>(ctx, L.o_fields);
  ia.geoms = at<GeomDesc>(ctx, L.o_geoms);
  ia.S = at<float>(ctx, L.o_S);
  ia.line_phasor = at<float4>(ctx, L.o_lineph);
  ia.col_phasor = at<float2>(ctx, L.o_colph);
  ia.khat = at<float2>(ctx, L.o_khat);
  ia.tw_row = at<float2>(ctx, L.o_twr);
  ia.tw_col = at<float2>(ctx, L.o_twc);
  ia.rowbuf = at<float2>(ctx, L.o_rowbuf);
  ia.rowbuf_off = at<int64_t>(ctx, S.it_rbo);
  ia.chi1 = at<float2>(ctx, L.o_G0);
  ia.chi2 = at<float2>(ctx, L.o_D0);
  ia.chi0 = at<float2>(ctx, L.o_X0);
  ia.Y = at<float>(ctx, L.o_Y);
  // the symmetry variant's output: Q0 (the solver's planes are free during the init)
  ia.chi3 = (!b.geoms.empty() && b.geoms[0].sym_row_chirp >= 0) ? at<float2>(ctx, L.o_Q0) : nullptr;
  const int* itb = at<int>(ctx, S.it_itab);
  ia.prow_field = itb + b.it_prow_field;
  ia.prow_first = itb + b.it_prow_first;
  ia.cgrp_field = itb + b.it_cgrp_field;
  ia.cgrp_first = itb + b.it_cgrp_first;
  ia.btile_field = itb + b.it_btile_field;
  ia.btile_first = itb + b.it_btile_first;
  return ia;
}

// Lock-in (or caller phases), crop (or caller S), caller chi0, holographic init.
hvdg_status stage_prepare(hvdg_ctx* ctx, Staged& S, const RunOpts& opt) {
  const Batch& b = S.b;
  const Layout& L = b.L;
  const int n = (int)b.prep.size();  // source fields
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  mark(ctx, 1);
  hvdg::LockinOut lo;
  lo.theta = at<float>(ctx, L.o_theta);
  lo.theta64 = nullptr;
  lo.vswitch = at<signed char>(ctx, L.o_vsw);
  lo.line_phasor = at<float4>(ctx, L.o_lineph);
  std::vector<float4> lph_host;
  if (opt.do_lockin) {
    hvdg::launch_burst_lockin(at<hvdg::PrepDesc>(ctx, L.o_prep), n, lo, s);
    S.launches += 1;
    if (opt.amp_out) {
      hvdg::launch_burst_amplitude(at<hvdg::PrepDesc>(ctx, L.o_prep), n, at<float>(ctx, L.o_amp), s);
      e = cudaMemcpyAsync(opt.amp_out, at<float>(ctx, L.o_amp), sizeof(float) * n,
                          cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "copy burst amplitudes");
      S.launches += 1;
    }
  } else {
    // caller-supplied active-line phases (one field): exp(i theta) in FP64
    const FieldPlan& p = b.fp[0];
    lph_host.resize(p.h);
    for (int y = 0; y < p.h; ++y) {
      const double th = (double)opt.theta_in[y];
      const bool sw = uses_vswitch(*p.g) && opt.vswitch_in && opt.vswitch_in[y] < 0;
      lph_host[y] = make_float4((float)std::cos(th), (float)std::sin(th), sw ? -1.f : 1.f, 0.f);
    }
    e = cudaMemcpyAsync(at<float4>(ctx, L.o_lineph), lph_host.data(), sizeof(float4) * p.h,
                        cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D line phasors");
    // the host copy must outlive the async copy
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D line phasors");
  }
  if (opt.s_in) {
    const FieldPlan& p = b.fp[0];
    e = cudaMemcpy2DAsync(at<float>(ctx, L.o_S) + p.px_off, sizeof(float) * p.pitch, opt.s_in,
                          sizeof(float) * p.w, sizeof(float) * p.w, p.h, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D S");
  } else {
    hvdg::launch_crop(at<hvdg::PrepDesc>(ctx, L.o_prep), at<int4>(ctx, S.it_crop),
                      (int)b.crop_rows.size(), at<float>(ctx, L.o_S), at<int64_t>(ctx, S.it_pxoff),
                      at<int>(ctx, S.it_pitch), at<int>(ctx, L.o_flags) + 1, s);
    S.launches += 1;
  }
  if (opt.chi0_in) {
    const FieldPlan& p = b.fp[0];
    e = cudaMemcpy2DAsync(at<float2>(ctx, L.o_X0) + p.px_off, sizeof(float2) * p.pitch, opt.chi0_in,
                          sizeof(float2) * p.w, sizeof(float2) * p.w, p.h, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D chi0");
  }
  if (opt.do_init) {
    const hvdg::InitArgs ia = init_args(ctx, S);
    hvdg::launch_init(ia, L.total_prows, L.total_cgroups, L.total_btiles, s);
    S.launches += 3;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "prepare / init launch");
  return HVDG_OK;
}

hvdg::SolverArgs solver_args(hvdg_ctx* ctx, const Staged& S) {
  const Layout& L = S.b.L;
  hvdg::SolverArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.fields = at<FieldDesc>(ctx, L.o_fields);
  sa.ctl = at<FieldCtl>(ctx, L.o_ctl);
  sa.units = at<Unit>(ctx, L.o_units);
  sa.unit_base = 0;
  sa.n_units = L.total_units;
  sa.n_phases = S.b.max_phases;
  sa.queue = at<unsigned long long>(ctx, L.o_queue);
  sa.done_phase = at<int>(ctx, L.o_done);
  sa.arrive = at<int>(ctx, L.o_arrive);
  sa.partials = at<double>(ctx, L.o_partials);
  sa.err = at<int>(ctx, L.o_flags);
  sa.S = at<float>(ctx, L.o_S);
  sa.X[0] = at<float2>(ctx, L.o_X0);
  sa.X[1] = at<float2>(ctx, L.o_X1);
  sa.G[0] = at<float2>(ctx, L.o_G0);
  sa.G[1] = at<float2>(ctx, L.o_G1);
  sa.D[0] = at<float2>(ctx, L.o_D0);
  sa.D[1] = at<float2>(ctx, L.o_D1);
  sa.Q[0] = at<float2>(ctx, L.o_Q0);
  sa.Q[1] = at<float2>(ctx, L.o_Q1);
  sa.W = at<float4>(ctx, L.o_W);
  sa.Y = at<float>(ctx, L.o_Y);
  sa.line_phasor = at<float4>(ctx, L.o_lineph);
  sa.col_phasor = at<float2>(ctx, L.o_colph);
  return sa;
}

int solver_grid(hvdg_ctx* ctx, int n_units, int ctas_override = -1) {
  const int want = ctas_override >= 0 ? ctas_override : ctx->ctas_per_sm;
  const int maxb = std::max(1, hvdg::solver_max_blocks_per_sm());
  const int per_sm = want > 0 ? std::min(want, maxb) : maxb;
  const int grid = ctx->sm_count * per_sm;
  // never more warps than the first phase can use
  return std::max(1, std::min(grid, (n_units + (hvdg::kSolverThreads / 32) - 1) /
                                        (hvdg::kSolverThreads / 32)));
}

// Copy the outputs, read the flags, synchronise, fill the diagnostics.
hvdg_status stage_finish(hvdg_ctx* ctx, Staged& S, hvdg_field_out* out, const RunOpts& opt,
                         hvdg_diag* diag) {
  const Batch& b = S.b;
  const Layout& L = b.L;
  const int n = (int)b.fp.size();
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  const cudaMemcpyKind kind = opt.device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (int i = 0; i < n; ++i) {
    const FieldPlan& p = b.fp[i];
    if (out[i].luma && !b.direct_y[i]) {
      e = cudaMemcpy2DAsync(out[i].luma, sizeof(float) * p.w, at<float>(ctx, L.o_Y) + p.px_off,
                            sizeof(float) * p.pitch, sizeof(float) * p.w, p.h, kind, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "copy luma");
    }
    if (out[i].chroma && !b.direct_c[i]) {
      e = cudaMemcpy2DAsync(out[i].chroma, sizeof(float2) * p.w, at<float2>(ctx, L.o_X0) + p.px_off,
                            sizeof(float2) * p.pitch, sizeof(float2) * p.w, p.h, kind, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "copy chroma");
    }
    // per-field phases (planes that are fields: one source field each)
    const bool own = b.pp.size() == b.fp.size();
    if (out[i].theta && own) {
      e = cudaMemcpyAsync(out[i].theta, at<float>(ctx, L.o_theta) + b.pp[i].theta_off,
                          sizeof(float) * b.pp[i].fh, kind, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "copy theta");
    }
    if (out[i].vswitch && own) {
      e = cudaMemcpyAsync(out[i].vswitch, at<signed char>(ctx, L.o_vsw) + b.pp[i].theta_off,
                          b.pp[i].fh, kind, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "copy vswitch");
    }
  }
  int flags[4] = {0, 0, 0, 0};
  e = cudaMemcpyAsync(flags, at<int>(ctx, L.o_flags), sizeof(flags), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "copy flags");
  std::vector<FieldCtl> ctl(n);
  if (diag)
    cudaMemcpyAsync(ctl.data(), at<FieldCtl>(ctx, L.o_ctl), sizeof(FieldCtl) * n,
                    cudaMemcpyDeviceToHost, s);
  mark(ctx, 4);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "stream sync");
  if (diag) {
    diag->ms_total += elapsed(ctx, 0, 4);
    diag->ms_solver += elapsed(ctx, 2, 3);
    diag->ms_init += elapsed(ctx, 1, 2);
    for (int i = 0; i < n; ++i) {
      diag->cg_iterations_run += ctl[i].cg_iters;
      diag->solver_pixel_iters += (int64_t)ctl[i].cg_iters * b.fp[i].h * b.fp[i].w;
      diag->solver_pixel_outers += (int64_t)b.fields[i].n_outer * b.fp[i].h * b.fp[i].w;
    }
    diag->kernel_launches += S.launches;
  }
  if (flags[1]) {
    ctx->last_error = "non-finite input samples";
    return HVDG_ERR_NONFINITE_INPUT;
  }
  if (flags[0]) {
    ctx->last_error = "device-side bounded wait expired in the solver";
    return HVDG_ERR_DEVICE_TIMEOUT;
  }
  return HVDG_OK;
}

// The 2-D pipeline over one batch: lock-in, crop, init, aniso, solver.
hvdg_status run_batch_once(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                           hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt_in) {
  Staged S;
  RunOpts opt = opt_in;
  if (!opt.weave_geom) opt.out_direct = out;
  hvdg_status st = stage_upload(ctx, in, n, cfg, opt, 0, S);
  if (st != HVDG_OK) return st;
  st = stage_prepare(ctx, S, opt);
  if (st != HVDG_OK) return st;
  const Layout& L = S.b.L;
  cudaStream_t s = ctx->stream;
  if (opt.do_solve) {
    hvdg::launch_aniso(at<FieldDesc>(ctx, L.o_fields), (int)S.b.fp.size(), at<float2>(ctx, L.o_X0), s);
    S.launches += 1;
  }
  mark(ctx, 2);
  if (opt.do_solve) {
    const hvdg::SolverArgs sa = solver_args(ctx, S);
    const cudaError_t e =
        hvdg::launch_solver(sa, solver_grid(ctx, L.total_units, opt.ctas_per_sm), s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "solver launch");
    S.launches += 1;
  }
  mark(ctx, 3);
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) return hvdg::cuda_fail(ctx, le, "aniso / solver launch");
  return stage_finish(ctx, S, out, opt, diag);
}

// Batch signature for the tuning table: field shapes and solver budgets.
std::string batch_signature(const hvdg_field_in* in, int n, const hvdg_config* cfg) {
  std::string sig = std::to_string(n) + ":" + std::to_string(cfg->fast) + ":";
  for (int i = 0; i < n; ++i) {
    const hvdg_geometry& g = *in[i].geometry;
    const int outer = in[i].irls_outer > 0 ? in[i].irls_outer : cfg->irls_outer;
    const int cg = in[i].cg_iterations >= 0 ? in[i].cg_iterations : cfg->cg_iterations;
    sig += std::to_string(g.active_video_end - g.active_video_start) + "x" +
           std::to_string(last_active_line(g) - g.first_active_field_line) + "/" +
           std::to_string(outer) + "/" + std::to_string(cg) + ";";
  }
  return sig;
}

// Captured-graph replay of the batched device-resident decode. The tables
// are uploaded outside the graph; the graph holds the per-call resets, the
// kernels, the output copies and the flag read-back (into pinned memory).
hvdg_status graph_result(hvdg_ctx* ctx, hvdg_diag* diag);

hvdg_status run_batch_graph(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                            hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt) {
  std::string sig = batch_signature(in, n, cfg);
  // the effective tiling (a per-call override, else the context setting)
  const int band = opt.band_rows >= 0 ? opt.band_rows : ctx->band_rows;
  const int ctas = opt.ctas_per_sm >= 0 ? opt.ctas_per_sm : ctx->ctas_per_sm;
  sig += "|b" + std::to_string(band) + "c" + std::to_string(ctas);
  char buf[64];
  for (int i = 0; i < n; ++i) {
    std::snprintf(buf, sizeof(buf), "|%p,%p,%p,%p,%d,%d", in[i].samples, (void*)out[i].luma,
                  (void*)out[i].chroma, (void*)out[i].theta, in[i].sample_type, in[i].parity);
    sig += buf;
  }
  sig.append(reinterpret_cast<const char*>(cfg), sizeof(*cfg));
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  if (!(ctx->gexec && ctx->gsig == sig && ctx->gepoch == ctx->epoch)) {
    if (ctx->gexec) {
      cudaGraphExecDestroy(ctx->gexec);
      ctx->gexec = nullptr;
    }
    RunOpts o2 = opt;
    o2.tables_only = true;
    o2.out_direct = out;
    Staged S;
    hvdg_status st = stage_upload(ctx, in, n, cfg, o2, 0, S);
    if (st != HVDG_OK) return st;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "table upload");
    if (ctx->ctl_host_n < n) {
      if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
      ctx->ctl_host = nullptr;
      ctx->ctl_host_n = 0;
      if (cudaMallocHost(&ctx->ctl_host, sizeof(FieldCtl) * n) != cudaSuccess) {
        cudaGetLastError();
        return HVDG_ERR_OUT_OF_MEMORY;
      }
      ctx->ctl_host_n = n;
    }
    const Layout& L = S.b.L;
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "begin capture");
    stage_reset(ctx, S);
    st = stage_prepare(ctx, S, o2);
    if (st == HVDG_OK) {
      hvdg::launch_aniso(at<FieldDesc>(ctx, L.o_fields), n, at<float2>(ctx, L.o_X0), s);
      mark(ctx, 2);
      const hvdg::SolverArgs sa = solver_args(ctx, S);
      e = hvdg::launch_solver(sa, solver_grid(ctx, L.total_units, opt.ctas_per_sm), s);
      if (e != cudaSuccess) st = hvdg::cuda_fail(ctx, e, "solver launch");
      mark(ctx, 3);
    }
    for (int i = 0; i < n && st == HVDG_OK; ++i) {
      const FieldPlan& p = S.b.fp[i];
      if (out[i].luma && !S.b.direct_y[i])
        cudaMemcpy2DAsync(out[i].luma, sizeof(float) * p.w, at<float>(ctx, L.o_Y) + p.px_off,
                          sizeof(float) * p.pitch, sizeof(float) * p.w, p.h,
                          cudaMemcpyDeviceToDevice, s);
      if (out[i].chroma && !S.b.direct_c[i])
        cudaMemcpy2DAsync(out[i].chroma, sizeof(float2) * p.w, at<float2>(ctx, L.o_X0) + p.px_off,
                          sizeof(float2) * p.pitch, sizeof(float2) * p.w, p.h,
                          cudaMemcpyDeviceToDevice, s);
      if (out[i].theta)
        cudaMemcpyAsync(out[i].theta, at<float>(ctx, L.o_theta) + S.b.pp[i].theta_off,
                        sizeof(float) * S.b.pp[i].fh, cudaMemcpyDeviceToDevice, s);
      if (out[i].vswitch)
        cudaMemcpyAsync(out[i].vswitch, at<signed char>(ctx, L.o_vsw) + S.b.pp[i].theta_off,
                        S.b.pp[i].fh, cudaMemcpyDeviceToDevice, s);
    }
    cudaMemcpyAsync(ctx->flags_host, at<int>(ctx, L.o_flags), sizeof(int) * 4,
                    cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ctx->ctl_host, at<FieldCtl>(ctx, L.o_ctl), sizeof(FieldCtl) * n,
                    cudaMemcpyDeviceToHost, s);
    mark(ctx, 4);
    e = cudaStreamEndCapture(s, &graph);
    if (st != HVDG_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "end capture");
    e = cudaGraphInstantiate(&ctx->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      ctx->gexec = nullptr;
      return hvdg::cuda_fail(ctx, e, "graph instantiate");
    }
    ctx->gsig = sig;
    ctx->gepoch = ctx->epoch;
    ctx->gn = n;
    ctx->g_pix.assign(n, 0);
    ctx->g_outer.assign(n, 0);
    for (int i = 0; i < n; ++i) {
      ctx->g_pix[i] = (int64_t)S.b.fp[i].h * S.b.fp[i].w;
      ctx->g_outer[i] = S.b.fields[i].n_outer;
    }
  }
  e = cudaGraphLaunch(ctx->gexec, s);
  if (opt.async) {
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_done, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "graph launch");
    ctx->pending = true;
    return HVDG_OK;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "graph launch");
  return graph_result(ctx, diag);
}

// Diagnostics and status of the last replay of the cached graph (after it
// completed): timing marks, CG counts, the device flags.
hvdg_status graph_result(hvdg_ctx* ctx, hvdg_diag* diag) {
  if (diag) {
    diag->ms_total += elapsed(ctx, 0, 4);
    diag->ms_solver += elapsed(ctx, 2, 3);
    diag->ms_init += elapsed(ctx, 1, 2);
    const FieldCtl* ctl = static_cast<const FieldCtl*>(ctx->ctl_host);
    for (int i = 0; i < ctx->gn; ++i) {
      diag->cg_iterations_run += ctl[i].cg_iters;
      diag->solver_pixel_iters += (int64_t)ctl[i].cg_iters * ctx->g_pix[i];
      diag->solver_pixel_outers += (int64_t)ctx->g_outer[i] * ctx->g_pix[i];
    }
    diag->kernel_launches += 7;
  }
  if (ctx->flags_host[1]) {
    ctx->last_error = "non-finite input samples";
    return HVDG_ERR_NONFINITE_INPUT;
  }
  if (ctx->flags_host[0]) {
    ctx->last_error = "device-side bounded wait expired in the solver";
    return HVDG_ERR_DEVICE_TIMEOUT;
  }
  return HVDG_OK;
}

// Batched decode: autotune the solver tiling once per batch signature (band
// height x CTAs per SM, timed on the solver's own events), then run -- as a
// replayed CUDA graph when the buffers are device-resident.
hvdg_status run_batch(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                      hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt_in) {
  RunOpts opt = opt_in;
  if (opt.do_solve && opt.do_init && opt.do_lockin && !opt.amp_out && ctx->autotune &&
      ctx->band_rows == 0 && ctx->ctas_per_sm == 0 && n >= 8) {
    const std::string sig = batch_signature(in, n, cfg);
    auto it = ctx->tune.find(sig);
    if (it == ctx->tune.end()) {
      static const int cand[][2] = {{32, 0}, {16, 0}, {64, 0}, {24, 0}};
      float best = 1e30f;
      std::pair<int, int> pick(32, 0);
      for (const auto& c : cand) {
        RunOpts o = opt;
        o.band_rows = c[0];
        o.ctas_per_sm = c[1];
        hvdg_diag d;
        std::memset(&d, 0, sizeof(d));
        const hvdg_status st = run_batch_once(ctx, in, n, cfg, out, &d, o);
        if (st != HVDG_OK) return st;
        if (d.ms_solver < best) {
          best = d.ms_solver;
          pick = std::make_pair(c[0], c[1]);
        }
      }
      it = ctx->tune.emplace(sig, pick).first;
    }
    opt.band_rows = it->second.first;
    opt.ctas_per_sm = it->second.second;
  }
  if (opt.device_io && ctx->use_graphs && ctx->flags_host && opt.do_solve && opt.do_init &&
      opt.do_lockin && !opt.amp_out && !opt.s_in && !opt.chi0_in) {
    const hvdg_status st = run_batch_graph(ctx, in, n, cfg, out, diag, opt);
    if (st != HVDG_ERR_CUDA || ctx->gexec) return st;
    // capture / instantiation refused on this driver: fall back to direct
    // launches for the rest of this context's life
    cudaGetLastError();
    ctx->use_graphs = 0;
  }
  return run_batch_once(ctx, in, n, cfg, out, diag, opt);
}

hvdg_status validate_fields(const hvdg_field_in* fields, int n, const hvdg_config* cfg,
                            hvdg_field_out* out) {
  if (n < 0 || (n > 0 && (!fields || !out)) || !cfg) return HVDG_ERR_BAD_ARGUMENT;
  if (cfg->diag_prior > 0.0f) return HVDG_ERR_UNSUPPORTED;
  for (int i = 0; i < n; ++i) {
    if (!fields[i].samples || !fields[i].geometry) return HVDG_ERR_BAD_ARGUMENT;
    if (fields[i].sample_type < 0 || fields[i].sample_type > 2) return HVDG_ERR_BAD_ARGUMENT;
    if (fields[i].sample_type != HVDG_SAMPLES_F32_IRE &&
        !(fields[i].white_level != fields[i].blanking_level))
      return HVDG_ERR_BAD_ARGUMENT;
    const hvdg_status s = check_geometry(fields[i].geometry);
    if (s != HVDG_OK) return s;
  }
  return HVDG_OK;
}

float median_mean(std::vector<float> v) {
  // MedianOf (sequence.cpp:29-39): mean of the two middles for even n
  if (v.empty()) return 0.0f;
  const size_t k = v.size() / 2;
  std::nth_element(v.begin(), v.begin() + k, v.end());
  float m = v[k];
  if (v.size() % 2 == 0) {
    std::nth_element(v.begin(), v.begin() + k - 1, v.begin() + k);
    m = 0.5f * (m + v[k - 1]);
  }
  return m;
}

// Adaptive temporal strength (sequence.cpp:526-646): same-parity pair
// ambiguity from a triangle-7 demodulation of S by each field's carrier,
// per horizontal band, p95 of bands, median over pairs, noise-floor removal.
float adaptive_strength(const std::vector<std::vector<float>>& Sh,
                        const std::vector<std::vector<float4>>& Lh, const std::vector<float2>& P,
                        int h, int w, int stride, float nr_eps, float* amb_out) {
  static const float kW[7] = {1.f, 2.f, 3.f, 4.f, 3.f, 2.f, 1.f};
  const int nf = (int)Sh.size();
  auto car = [&](int f, int y, int x) {
    const float4 L = Lh[f][y];
    const float2 c = make_float2(L.x * P[x].x - L.y * P[x].y, L.x * P[x].y + L.y * P[x].x);
    return L.z < 0.f ? make_float2(-c.x, c.y) : c;
  };
  std::vector<float> ambs;
  for (int j = 0; j + stride < nf; ++j) {
    const int k = j + stride;
    std::vector<double> band_acc;
    std::vector<long> band_n;
    double acc = 0.0;
    long n = 0;
    int yi = 0;
    for (int y = 2; y < h - 2; y += 3, ++yi) {
      const int band = yi / 8;
      if (band >= (int)band_acc.size()) {
        band_acc.push_back(0.0);
        band_n.push_back(0);
      }
      for (int x = 4; x + 7 < w; x += 4) {
        float mj = 0.f, mk = 0.f;
        for (int q = 0; q < 4; ++q) {
          mj += Sh[j][(size_t)y * w + x + q];
          mk += Sh[k][(size_t)y * w + x + q];
        }
        if (std::fabs(mj - mk) * 0.25f > nr_eps) continue;
        auto demod = [&](int f) {
          float dr = 0.f, di = 0.f;
          for (int q = 0; q < 7; ++q) {
            const float sv = kW[q] * Sh[f][(size_t)y * w + x + q];
            const float2 c = car(f, y, x + q);
            dr += sv * c.x;
            di += -sv * c.y;
          }
          return make_float2(dr * (1.0f / 16.0f), di * (1.0f / 16.0f));
        };
        const float2 dj = demod(j), dk = demod(k);
        const float er = dj.x - dk.x, ei = dj.y - dk.y;
        const double e = 0.25 * (double)(er * er + ei * ei);
        acc += e;
        ++n;
        band_acc[band] += e;
        ++band_n[band];
      }
    }
    if (n > 0) {
      std::vector<float> brms;
      for (size_t b = 0; b < band_acc.size(); ++b)
        if (band_n[b] >= 8) brms.push_back((float)(band_acc[b] / band_n[b]));
      if (!brms.empty()) {
        const size_t k95 = std::min(brms.size() - 1, (size_t)(0.95 * brms.size()));
        std::nth_element(brms.begin(), brms.begin() + k95, brms.end());
        ambs.push_back(std::sqrt(brms[k95]));
      } else {
        ambs.push_back(std::sqrt((float)(acc / n)));
      }
    }
  }
  float amb = median_mean(ambs);
  const float sigma_d = nr_eps > 0.0f ? nr_eps / 3.0f : 1.0f;
  const float noise_floor = sigma_d * 0.29f;
  amb = std::sqrt(std::max(0.0f, amb * amb - noise_floor * noise_floor));
  if (amb_out) *amb_out = amb;
  return std::min(std::max(0.5f * amb - 0.05f, 0.0f), 1.5f);
}

// DecodeFieldWindowWithInits (sequence.cpp:423-1116) for one window of one
// geometry, temporal terms included: noise self-calibration, adaptive
// strength, coloured Gauss-Seidel sweep (or the sequential sweep in slow
// mode); per colour, motion estimation on the current luma state, warps,
// confidence upsampling, the odd-offset envelope gate and the neighbour
// planes, then the solver over that colour's fields.
hvdg_status decode_window_3d(hvdg_ctx* ctx, const hvdg_field_in* in, int nf,
                             const hvdg_config* cfg_in, hvdg_field_out* out, hvdg_diag* diag,
                             const RunOpts& opt) {
  hvdg_config cfg = *cfg_in;
  const hvdg_geometry& g = *in[0].geometry;
  const bool pal = uses_vswitch(g);
  std::vector<int> offs;
  if (cfg.extended_temporal) {
    offs = pal ? (cfg.bidirectional ? std::vector<int>{-4, -3, -2, -1, 1, 2, 3, 4}
                                    : std::vector<int>{-4, -3, -2, -1})
               : (cfg.bidirectional ? std::vector<int>{-3, -2, -1, 1, 2, 3}
                                    : std::vector<int>{-3, -2, -1});
  } else {
    offs = cfg.bidirectional ? std::vector<int>{-2, -1, 1, 2} : std::vector<int>{-2, -1};
  }
  if (pal) {
    if (cfg.coherence_gate == 0.6f) cfg.coherence_gate = 1.0f;
    if (cfg.nr_radius == 2) cfg.nr_radius = 4;
  }
  // ---- solver band height: set by the fields solved together (one colour
  // of the sweep: every field alone in the slow temporal sweep) ----
  RunOpts o3 = opt;
  if (o3.band_rows < 0 && ctx->band_rows <= 0) {
    const bool temporal = cfg.temporal_strength > 0.0f && cfg.cg_iterations > 0;
    int colour = nf;
    if ((cfg.fast || !temporal) && cfg.parallel_across_fields) {
      int max_off = 0;
      for (int o : offs) max_off = std::max(max_off, std::abs(o));
      const int reach = std::max(max_off, cfg.nr_anchor > 0.0f ? cfg.nr_radius : 0);
      const int stride = temporal ? reach + 1 : 1;
      colour = (nf + stride - 1) / stride;
    } else if (temporal) {
      colour = 1;
    }
    const int hh = last_active_line(g) - g.first_active_field_line;
    const int ww = g.active_video_end - g.active_video_start;
    o3.band_rows = auto_band_rows_hw(ctx, std::vector<std::pair<int, int>>(colour, {hh, ww}));
  }
  // ---- layout: batch + 3-D regions ----
  Batch plan;
  hvdg_status st = plan_batch(ctx, in, nf, &cfg, o3.band_rows >= 0 ? o3.band_rows : ctx->band_rows,
                              plan);
  if (st != HVDG_OK) return st;
  const int h = plan.fp[0].h, w = plan.fp[0].w, pitch = plan.fp[0].pitch;
  const int64_t plane = (int64_t)h * pitch;
  const int nofs = (int)offs.size();
  // me_mode 1: integer-SAD blocks (me_block, +-me_range); else the reference's
  // float-SSD pyramid on mc_tile tiles (+-mc_search)
  const bool sad_me = cfg.me_mode == 1;
  const int tile = sad_me ? cfg.me_block : cfg.mc_tile;
  const int search = sad_me ? cfg.me_range : cfg.mc_search;
  if (tile < 1 || search < 0 || tile > 1024 || search > 64) return HVDG_ERR_BAD_ARGUMENT;
  if (cfg.me_mode < 0 || cfg.me_mode > 1) return HVDG_ERR_BAD_ARGUMENT;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile, nt = th * tw;
  if (sad_me && (tile > hvdg::sad_max_block() || search > hvdg::sad_max_range() ||
                 nt > kSadMaxTiles)) {
    ctx->last_error = "integer-SAD motion: block, range or tile count above the supported maximum";
    return HVDG_ERR_UNSUPPORTED;
  }
  const int ct = std::max(4, tile / 4);
  const int nct = std::max(1, ((h / 4 + ct - 1) / ct) * ((w / 4 + ct - 1) / ct));
  const int dpitch = pitch / 4;
  const int64_t dplane = (int64_t)(h / 4 + 1) * dpitch;
  const int max_pairs = nf * nofs;
  size_t xo = 0;
  auto take = [&](size_t bytes) {
    const size_t r = xo;
    xo = align_up(xo + bytes, 256);
    return r;
  };
  const size_t x_M = take(sizeof(float4) * plane * nf);
  const size_t x_B = take(sizeof(float2) * plane * nf);
  const size_t x_nbr = take(sizeof(float4) * plane * nf * nofs);
  const size_t x_tmp = take(sizeof(float) * plane * nf);
  const size_t x_blur = take(sizeof(float) * plane * nf);
  const size_t x_dec = take(sizeof(float) * dplane * nf);
  const size_t x_cdy = take(sizeof(float) * nct * max_pairs);
  const size_t x_cdx = take(sizeof(float) * nct * max_pairs);
  size_t x_t[13];
  for (int i = 0; i < 13; ++i) x_t[i] = take(sizeof(float) * nt * max_pairs);
  size_t x_sd[4] = {0, 0, 0, 0};  // integer-SAD tile statistics (doubles)
  if (sad_me)
    for (int i = 0; i < 4; ++i) x_sd[i] = take(sizeof(double) * nt * max_pairs);
  const size_t x_src = take(sizeof(int2) * plane * max_pairs);
  const size_t x_cpx = take(sizeof(float) * plane * max_pairs);
  const size_t x_ctmp = take(sizeof(float) * plane * max_pairs);
  // fast-mode motion cache (pass-0 motion reused by later passes,
  // sequence.cpp:674-692): dy, dx, conf per window pair slot
  const size_t x_mcache = take(sizeof(float) * 3 * (size_t)nt * max_pairs);
  // coherence gate: 4 channel planes per pair of the largest colour + scratch
  const bool gate_cfg = cfg.coherence_gate > 0.0f;
  const int64_t coh_stride = gate_cfg ? plane * max_pairs : 0;
  const size_t x_coh = take(sizeof(float) * 4 * (size_t)coh_stride);
  // anchored pass (passes > 1, nr_anchor > 0): pre-snap motion, the anchor's
  // own per-pixel vectors and confidences, the anchor planes and the joint
  // solver's planes
  const bool anchor_on = cfg.temporal_strength > 0.0f && cfg.cg_iterations > 0 &&
                         std::max(1, cfg.passes) > 1 && cfg.nr_anchor > 0.0f && nf > 1;
  const size_t AP = anchor_on ? 1 : 0;
  const size_t x_pre = take(sizeof(float) * 3 * (size_t)nt * max_pairs * AP);
  const size_t x_asnap = take(sizeof(float) * 4 * (size_t)nt * max_pairs * AP);
  const size_t x_asrc = take(sizeof(int2) * plane * max_pairs * AP);
  const size_t x_acpx = take(sizeof(float) * plane * max_pairs * AP);
  const size_t x_actmp = take(sizeof(float) * plane * max_pairs * AP);
  const size_t x_ya = take(sizeof(float) * plane * nf * AP);
  const size_t x_caa = take(sizeof(float2) * plane * nf * AP);
  const size_t x_wa = take(sizeof(float) * plane * nf * AP);
  const size_t x_res = take(sizeof(float) * plane * nf * AP);
  const size_t x_jp = take(sizeof(float4) * 10 * plane * nf * AP);
  const size_t x_jm2 = take(sizeof(float) * plane * nf * AP);
  const int jbx = (w + 31) / 32, jby = (h + 7) / 8;
  const size_t x_jpart = take(sizeof(double) * 5 * (size_t)jbx * jby * nf * AP);
  const size_t x_jctl = take(sizeof(hvdg::JointCtl) * nf + sizeof(hvdg::AnchorGroup) * nf +
                             sizeof(int) * nf + 256);
  const size_t x_ctab = take(sizeof(hvdg::TrajGroup) * 2 * nf + sizeof(hvdg::TrajPair) * max_pairs +
                             sizeof(int) * 2 * max_pairs + 256);
  size_t x_env[5];
  for (int i = 0; i < 5; ++i) x_env[i] = take(sizeof(float) * plane * nf);
  const size_t env_samples = ((size_t)h * w + 6) / 7;
  const size_t x_escr = take(sizeof(float) * env_samples * nf);
  const size_t x_nscr = take(sizeof(float) * (size_t)h * std::max(1, w - 8) * nf);
  const size_t x_small = take(sizeof(float) * 4 * nf + sizeof(int64_t) * (3 * nf + max_pairs) +
                              sizeof(int) * nf + sizeof(hvdg::MeField) * nf +
                              sizeof(hvdg::MePair) * max_pairs +
                              sizeof(hvdg::NbrPair) * max_pairs + 1024);
  Staged S;
  st = stage_upload(ctx, in, nf, &cfg, o3, xo, S);
  if (st != HVDG_OK) return st;
  Batch& b = S.b;
  const Layout& L = b.L;
  auto X = [&](size_t off) { return S.extra + off; };
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  st = stage_prepare(ctx, S, opt);
  if (st != HVDG_OK) return st;

  // ---- small device tables ----
  char* small = at<char>(ctx, X(x_small));
  float* d_sigma = reinterpret_cast<float*>(small);
  float* d_floor2 = d_sigma + nf;
  int64_t* d_nscr_off = reinterpret_cast<int64_t*>(align_up((size_t)(d_floor2 + nf), 8));
  int64_t* d_escr_off = d_nscr_off + nf;
  int64_t* d_pix_off = d_escr_off + nf;
  int* d_list = reinterpret_cast<int*>(d_pix_off + max_pairs);
  hvdg::MeField* d_mf = reinterpret_cast<hvdg::MeField*>(align_up((size_t)(d_list + nf), 16));
  hvdg::MePair* d_mp = reinterpret_cast<hvdg::MePair*>(d_mf + nf);
  hvdg::NbrPair* d_np = reinterpret_cast<hvdg::NbrPair*>(d_mp + max_pairs);
  std::vector<int64_t> nscr_off(nf), escr_off(nf), pix_off(max_pairs);
  std::vector<hvdg::MeField> mf(nf);
  for (int j = 0; j < nf; ++j) {
    nscr_off[j] = (int64_t)j * h * std::max(1, w - 8);
    escr_off[j] = (int64_t)j * env_samples;
    mf[j].h = h;
    mf[j].w = w;
    mf[j].pitch = pitch;
    mf[j].dpitch = dpitch;
    mf[j].y_off = b.fp[j].px_off;
    mf[j].t_off = b.fp[j].px_off;
    mf[j].b_off = b.fp[j].px_off;
    mf[j].d_off = (int64_t)j * dplane;
  }
  for (int p = 0; p < max_pairs; ++p) pix_off[p] = (int64_t)p * plane;
  e = cudaMemcpyAsync(d_nscr_off, nscr_off.data(), sizeof(int64_t) * nf, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_pix_off, pix_off.data(), sizeof(int64_t) * max_pairs, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_mf, mf.data(), sizeof(hvdg::MeField) * nf, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D window tables");

  // ---- noise self-calibration (sequence.cpp:437-449) ----
  hvdg::launch_noise(at<FieldDesc>(ctx, L.o_fields), nf, at<float>(ctx, L.o_S),
                     at<float>(ctx, X(x_nscr)), d_nscr_off, d_sigma, s);
  std::vector<float> sig(nf);
  e = cudaMemcpyAsync(sig.data(), d_sigma, sizeof(float) * nf, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "noise estimate");
  const float sigma = median_mean(sig);
  if (cfg.temporal_eps <= 0.0f) cfg.temporal_eps = std::min(std::max(7.0f * sigma, 4.0f), 20.0f);
  if (cfg.nr_eps <= 0.0f) cfg.nr_eps = std::min(std::max(3.0f * sigma, 3.0f), 12.0f);
  float amb = 0.0f;
  const int amb_stride = pal ? 4 : 2;
  if (cfg.temporal_strength == 0.0f && cfg.cg_iterations > 0 && nf > amb_stride) {
    std::vector<std::vector<float>> Sh(nf, std::vector<float>((size_t)h * w));
    std::vector<std::vector<float4>> Lh(nf, std::vector<float4>(h));
    for (int j = 0; j < nf; ++j) {
      e = cudaMemcpy2DAsync(Sh[j].data(), sizeof(float) * w, at<float>(ctx, L.o_S) + b.fp[j].px_off,
                            sizeof(float) * pitch, sizeof(float) * w, h, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(Lh[j].data(), at<float4>(ctx, L.o_lineph) + b.fp[j].line_off,
                            sizeof(float4) * h, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "D2H window state");
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "D2H window state");
    cfg.temporal_strength = adaptive_strength(Sh, Lh, b.gtabs[0]->col_phasor, h, w, amb_stride,
                                              cfg.nr_eps, &amb);
  }
  if (cfg.temporal_strength < 0.0f) cfg.temporal_strength = 0.0f;
  if (diag) {
    diag->sigma_ire = sigma;
    diag->ambiguity_ire = amb;
    diag->resolved_strength = std::max(0.0f, cfg.temporal_strength);
    diag->temporal_eps = cfg.temporal_eps;
    diag->nr_eps = cfg.nr_eps;
  }
  const bool has_temporal = cfg.temporal_strength > 0.0f && cfg.cg_iterations > 0;
  const int n_passes = has_temporal ? std::max(1, cfg.passes) : 1;
  if (has_temporal) {
    const bool anchor = n_passes > 1 && cfg.nr_anchor > 0.0f && nf > 1;
    bool gate_any = false;
    for (int pass = 0; pass < n_passes; ++pass)
      if (cfg.coherence_gate > 0.0f && !(cfg.fast && pass == 0)) gate_any = true;
    (void)gate_any;
    if (nofs > hvdg::kTrajMaxPairs) return HVDG_ERR_UNSUPPORTED;
    if (anchor) {
      // the anchor reuses the neighbour pairs' motion: every offset within
      // nr_radius must be a neighbour offset
      for (int o = -cfg.nr_radius; o <= cfg.nr_radius; ++o) {
        if (o == 0) continue;
        if (std::find(offs.begin(), offs.end(), o) == offs.end()) {
          ctx->last_error = "anchored pass: nr_radius reaches offsets outside the temporal set";
          return HVDG_ERR_UNSUPPORTED;
        }
      }
      if (2 * cfg.nr_radius > hvdg::kJointMaxNbr) return HVDG_ERR_UNSUPPORTED;
    }
  }
  // ---- colours (sequence.cpp:1052-1099) ----
  std::vector<std::vector<int>> colors;
  if ((cfg.fast || !has_temporal) && cfg.parallel_across_fields) {
    int max_off = 0;
    for (int o : offs) max_off = std::max(max_off, std::abs(o));
    const int reach = std::max(max_off, cfg.nr_anchor > 0.0f ? cfg.nr_radius : 0);
    const int stride = has_temporal ? reach + 1 : 1;
    for (int c = 0; c < stride; ++c) {
      std::vector<int> col;
      for (int j = c; j < nf; j += stride) col.push_back(j);
      if (!col.empty()) colors.push_back(col);
    }
  } else if (!has_temporal) {
    std::vector<int> all;
    for (int j = 0; j < nf; ++j) all.push_back(j);
    colors.push_back(all);
  } else {
    for (int j = 0; j < nf; ++j) colors.push_back({j});
  }
  // units regrouped by colour (each field's units stay contiguous)
  std::vector<Unit> cunits;
  std::vector<int> cbegin, ccount, cphases;
  for (const auto& col : colors) {
    cbegin.push_back((int)cunits.size());
    int ph = 0;
    for (int j : col) {
      FieldDesc& f = b.fields[j];
      const int ub = (int)cunits.size();
      for (int u = 0; u < f.unit_count; ++u) cunits.push_back(b.units[f.unit_begin + u]);
      f.unit_begin = ub;
      ph = std::max(ph, f.n_phases);
    }
    ccount.push_back((int)cunits.size() - cbegin.back());
    cphases.push_back(ph);
  }
  // neighbour planes per field (slot per valid offset)
  for (int j = 0; j < nf; ++j) {
    FieldDesc& f = b.fields[j];
    f.nu = has_temporal ? cfg.temporal_strength : 0.0f;
    f.eps_t = cfg.temporal_eps;
    f.nbr_off = (int64_t)j * nofs * plane;
    f.plane_px = plane;
    f.n_nbr = 0;
    f.has_nbr = 0;
  }
  e = cudaMemcpyAsync(at<Unit>(ctx, L.o_units), cunits.data(), sizeof(Unit) * cunits.size(),
                      cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D units");
  hvdg::SolverArgs sa = solver_args(ctx, S);
  sa.M = at<float4>(ctx, X(x_M));
  sa.B = at<float2>(ctx, X(x_B));
  sa.nbr = at<float4>(ctx, X(x_nbr));
  hvdg::MeArgs ma;
  ma.tile = tile;
  ma.search = search;
  ma.coarse_off = nct;
  ma.tiles_off = nt;
  hvdg::MeBuffers mb;
  mb.luma = at<float>(ctx, L.o_Y);
  mb.tmp = at<float>(ctx, X(x_tmp));
  mb.blur = at<float>(ctx, X(x_blur));
  mb.dec = at<float>(ctx, X(x_dec));
  mb.cdy = at<float>(ctx, X(x_cdy));
  mb.cdx = at<float>(ctx, X(x_cdx));
  mb.mdy = at<float>(ctx, X(x_t[0]));
  mb.mdx = at<float>(ctx, X(x_t[1]));
  mb.sdy = at<float>(ctx, X(x_t[2]));
  mb.sdx = at<float>(ctx, X(x_t[3]));
  mb.best = at<float>(ctx, X(x_t[4]));
  mb.dy = at<float>(ctx, X(x_t[5]));
  mb.dx = at<float>(ctx, X(x_t[6]));
  mb.conf = at<float>(ctx, X(x_t[7]));
  hvdg::SadArgs sad_a;
  sad_a.block = tile;
  sad_a.range = search;
  sad_a.tiles_off = nt;
  hvdg::SadBuffers sad_b;
  sad_b.luma = mb.luma;
  sad_b.vsum = reinterpret_cast<int*>(mb.tmp);
  sad_b.qblur = reinterpret_cast<int*>(mb.blur);
  sad_b.mdy = mb.mdy;
  sad_b.mdx = mb.mdx;
  sad_b.sdy = mb.sdy;
  sad_b.sdx = mb.sdx;
  sad_b.dy = mb.dy;
  sad_b.dx = mb.dx;
  sad_b.conf = mb.conf;
  sad_b.bestv = sad_me ? at<double>(ctx, X(x_sd[0])) : nullptr;
  sad_b.s1 = sad_me ? at<double>(ctx, X(x_sd[1])) : nullptr;
  sad_b.s2 = sad_me ? at<double>(ctx, X(x_sd[2])) : nullptr;
  sad_b.npx = sad_me ? at<double>(ctx, X(x_sd[3])) : nullptr;
  hvdg::VecBuffers vb;
  vb.dy = mb.dy;
  vb.dx = mb.dx;
  vb.conf = mb.conf;
  vb.snap_dy = at<float>(ctx, X(x_t[8]));
  vb.snap_dx = at<float>(ctx, X(x_t[9]));
  vb.c2 = at<float>(ctx, X(x_t[10]));
  vb.c2_snap = at<float>(ctx, X(x_t[11]));
  vb.c2_snap2 = at<float>(ctx, X(x_t[12]));
  vb.src_idx = at<int2>(ctx, X(x_src));
  vb.pix_off = d_pix_off;
  vb.conf_tmp = at<float>(ctx, X(x_ctmp));
  vb.conf_px = at<float>(ctx, X(x_cpx));
  hvdg::EnvBuffers eb;
  eb.gmag = at<float>(ctx, X(x_env[0]));
  eb.lapmag = at<float>(ctx, X(x_env[1]));
  eb.vraw = at<float>(ctx, X(x_env[2]));
  eb.traw = at<float>(ctx, X(x_env[3]));
  eb.gate = at<float>(ctx, X(x_env[4]));
  eb.scratch = at<float>(ctx, X(x_escr));
  eb.scratch_off = d_escr_off;
  eb.floor2 = d_floor2;
  const float e2 = cfg.temporal_eps * cfg.temporal_eps;
  const float floor_max = std::min(std::max(cfg.odd_gate_floor, 0.0f), 1.0f);
  mark(ctx, 2);
  for (int pass = 0; pass < n_passes; ++pass) {
    for (size_t ci = 0; ci < colors.size(); ++ci) {
      const std::vector<int>& col = colors[ci];
      std::vector<hvdg::MePair> mp;
      std::vector<hvdg::NbrPair> np;
      std::vector<int> env_list;
      std::vector<int64_t> env_off;
      // pairs: the fully searched ones first, then (fast mode with the
      // trajectory fit, float motion) the predicted + verified ones
      // (sequence.cpp:699-763)
      std::vector<hvdg::TrajPair> tp;
      std::vector<hvdg::TrajGroup> groups, searched;
      std::vector<int> grp, gid;
      int n_full = 0;
      if (has_temporal) {
        struct P {
          int k, j, slot, odd, g, o, oi;
        };
        std::vector<P> full, pred;
        const bool predict = cfg.fast && cfg.trajectory_fit && !sad_me;
        for (int gi = 0; gi < (int)col.size(); ++gi) {
          const int j = col[gi];
          int slot = 0;
          bool any_odd = false;
          for (int oi = 0; oi < nofs; ++oi) {
            const int o = offs[oi];
            const int k = j + o;
            if (k < 0 || k >= nf) continue;
            const bool is_full = !predict || o == -1 || o == 1 || o == 2;
            (is_full ? full : pred).push_back(P{k, j, slot++, (o & 1) != 0 ? 1 : 0, gi, o, oi});
            any_odd = any_odd || (o & 1) != 0;
          }
          b.fields[j].n_nbr = slot;
          b.fields[j].has_nbr = slot > 0 ? 1 : 0;
          if (!slot) b.fields[j].nu = 0.0f;
          if (any_odd) {
            env_list.push_back(j);
            env_off.push_back(escr_off[j]);
          }
        }
        groups.assign(col.size(), hvdg::TrajGroup{});
        searched.assign(col.size(), hvdg::TrajGroup{});
        for (auto& G : groups) G.count = 0;
        for (auto& G : searched) G.count = 0;
        n_full = (int)full.size();
        for (int pass_list = 0; pass_list < 2; ++pass_list) {
          for (const P& q : pass_list == 0 ? full : pred) {
            const int pi = (int)mp.size();
            mp.push_back(hvdg::MePair{q.k, q.j});
            np.push_back(hvdg::NbrPair{q.k, q.j, q.slot, q.odd});
            tp.push_back(hvdg::TrajPair{q.o, (float)(in[q.k].parity - in[q.j].parity) / 2.0f});
            gid.push_back(q.j * nofs + q.oi);
            groups[q.g].pair[groups[q.g].count++] = pi;
            if (pass_list == 0) searched[q.g].pair[searched[q.g].count++] = pi;
            else grp.push_back(q.g);
          }
        }
      }
      e = cudaMemcpyAsync(at<FieldDesc>(ctx, L.o_fields), b.fields.data(), sizeof(FieldDesc) * nf,
                          cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D fields");
      const int npairs = (int)mp.size();
      if (npairs > 0) {
        e = cudaMemcpyAsync(d_mp, mp.data(), sizeof(hvdg::MePair) * npairs, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_np, np.data(), sizeof(hvdg::NbrPair) * npairs, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D pairs");
        // small tables of this colour
        char* ct = at<char>(ctx, X(x_ctab));
        hvdg::TrajGroup* d_groups = reinterpret_cast<hvdg::TrajGroup*>(ct);
        hvdg::TrajGroup* d_searched = d_groups + nf;
        hvdg::TrajPair* d_tp = reinterpret_cast<hvdg::TrajPair*>(d_searched + nf);
        int* d_grp = reinterpret_cast<int*>(d_tp + max_pairs);
        int* d_gid = d_grp + max_pairs;
        e = cudaMemcpyAsync(d_groups, groups.data(), sizeof(hvdg::TrajGroup) * groups.size(),
                            cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_searched, searched.data(), sizeof(hvdg::TrajGroup) * searched.size(),
                              cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_tp, tp.data(), sizeof(hvdg::TrajPair) * tp.size(),
                              cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && !grp.empty())
          e = cudaMemcpyAsync(d_grp, grp.data(), sizeof(int) * grp.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_gid, gid.data(), sizeof(int) * gid.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D trajectory tables");
        float* mcache = at<float>(ctx, X(x_mcache));
        const int64_t mc_stride = (int64_t)nt * max_pairs;
        const bool joint_pass = anchor_on && pass >= 1;
        if (cfg.fast && pass > 0) {
          // fast mode: every pair's motion comes from pass 0 (cached before
          // the consensus snap, which is re-applied: same inputs, same result)
          hvdg::launch_motion_cache(d_gid, npairs, nt, nt, mb.dy, mb.dx, mb.conf, mcache, mc_stride,
                                    false, s);
        } else {
          if (sad_me)
            hvdg::launch_motion_sad(d_mf, nf, h, w, d_mp, n_full, sad_a, sad_b, s);
          else
            hvdg::launch_motion(d_mf, nf, h, w, d_mp, n_full, ma, mb, s);
          const int npred = npairs - n_full;
          if (npred > 0) {
            const int64_t ofs = (int64_t)n_full * nt;
            hvdg::launch_traj_verify(d_mf, d_mp, n_full, npred, d_grp, d_searched, d_tp, mb.blur, h,
                                     w, ma, mb.dy, mb.dx, mb.mdy, mb.mdx, mb.sdy, mb.sdx, mb.best,
                                     s);
            hvdg::launch_me_confidence(d_mf, d_mp + n_full, npred, h, w, ma, mb.blur, mb.mdy + ofs,
                                       mb.mdx + ofs, mb.sdy + ofs, mb.sdx + ofs, mb.best + ofs,
                                       mb.dy + ofs, mb.dx + ofs, mb.conf + ofs, s);
            S.launches += 2;
          }
          if (cfg.fast && n_passes > 1)
            hvdg::launch_motion_cache(d_gid, npairs, nt, nt, mb.dy, mb.dx, mb.conf, mcache,
                                      mc_stride, true, s);
        }
        if (joint_pass) {
          // the anchor blends with the pairwise motion as estimated (before
          // the consensus snap), sequence.cpp:70-102
          float* pre = at<float>(ctx, X(x_pre));
          const size_t tb = sizeof(float) * (size_t)nt * npairs;
          e = cudaMemcpyAsync(pre, mb.dy, tb, cudaMemcpyDeviceToDevice, s);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(pre + (size_t)nt * max_pairs, mb.dx, tb, cudaMemcpyDeviceToDevice, s);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(pre + 2 * (size_t)nt * max_pairs, mb.conf, tb,
                                cudaMemcpyDeviceToDevice, s);
          if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "anchor motion copy");
        }
        if (cfg.trajectory_fit && npairs >= 2) {
          hvdg::launch_traj_snap(d_mf, d_mp, d_groups, (int)groups.size(), d_tp, h, w, tile, nt,
                                 mb.dy, mb.dx, mb.conf, s);
          S.launches += 1;
        }
        vb.conf_bytes = sizeof(float) * plane * npairs;
        hvdg::launch_vectors(d_mf, d_mp, npairs, h, w, ma, vb, cfg.fast != 0, s);
        S.launches += 8;
        if (gate_cfg && !(cfg.fast && pass == 0)) {
          // coherence gate against the current chi of both fields
          hvdg::CohBuffers cb;
          cb.chi = at<float2>(ctx, L.o_X0);
          cb.snap_dy = vb.snap_dy;
          cb.snap_dx = vb.snap_dx;
          cb.terms = at<float>(ctx, X(x_coh));
          cb.tmp = vb.conf_tmp;
          cb.conf_px = vb.conf_px;
          cb.pix_off = d_pix_off;
          cb.chan_stride = coh_stride;
          hvdg::launch_coherence_gate(d_mf, d_mp, npairs, h, w, ma, cb, cfg.coherence_gate, s);
          S.launches += 10;
        }
        if (!env_list.empty()) {
          e = cudaMemcpyAsync(d_list, env_list.data(), sizeof(int) * env_list.size(),
                              cudaMemcpyHostToDevice, s);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_escr_off, env_off.data(), sizeof(int64_t) * env_off.size(),
                                cudaMemcpyHostToDevice, s);
          if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D env list");
          hvdg::launch_envelope(at<FieldDesc>(ctx, L.o_fields), d_list, (int)env_list.size(), h, w,
                                at<float>(ctx, L.o_Y), at<float2>(ctx, L.o_X0), eb, e2, floor_max,
                                s);
          S.launches += 4;
        }
        hvdg::launch_nbr_assemble(at<FieldDesc>(ctx, L.o_fields), d_np, npairs, h, w,
                                  at<float>(ctx, L.o_S), at<float4>(ctx, L.o_lineph),
                                  at<float2>(ctx, L.o_colph), vb.src_idx, vb.conf_px, d_pix_off,
                                  eb.gate, at<float4>(ctx, X(x_nbr)), s);
        S.launches += 1;
      }
      // solver state reset for this colour, aniso at the current chi
      cudaMemsetAsync(at<char>(ctx, L.o_ctl), 0, sizeof(FieldCtl) * nf, s);
      cudaMemsetAsync(at<char>(ctx, L.o_arrive), 0, sizeof(int) * nf, s);
      cudaMemsetAsync(at<char>(ctx, L.o_done), 0xff, sizeof(int) * nf, s);
      cudaMemsetAsync(at<char>(ctx, L.o_queue), 0, sizeof(unsigned long long), s);
      if (pass == 0 && cfg.psi_init && has_temporal) {
        // PsiClosedForm init of the colour's fields that have neighbours
        // (sequence.cpp:1033-1035), before the anisotropy is resolved
        char* jc = at<char>(ctx, X(x_jctl));
        int* d_fl = reinterpret_cast<int*>(reinterpret_cast<hvdg::AnchorGroup*>(
                        reinterpret_cast<hvdg::JointCtl*>(jc) + nf) + nf);
        e = cudaMemcpyAsync(d_fl, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D psi field list");
        hvdg::JointArgs pj;
        std::memset(&pj, 0, sizeof(pj));
        pj.fields = at<FieldDesc>(ctx, L.o_fields);
        pj.flist = d_fl;
        pj.nfl = (int)col.size();
        pj.S = at<float>(ctx, L.o_S);
        pj.line_phasor = at<float4>(ctx, L.o_lineph);
        pj.col_phasor = at<float2>(ctx, L.o_colph);
        pj.nbr = at<float4>(ctx, X(x_nbr));
        hvdg::launch_psi_init(pj, at<float2>(ctx, L.o_X0), h, w, s);
        S.launches += 1;
      }
      hvdg::launch_aniso(at<FieldDesc>(ctx, L.o_fields), nf, at<float2>(ctx, L.o_X0), s);
      if (anchor_on && pass >= 1) {
        // ---- anchored pass: SynthReference + VariationalRefineJoint ----
        char* jc = at<char>(ctx, X(x_jctl));
        hvdg::JointCtl* d_jctl = reinterpret_cast<hvdg::JointCtl*>(jc);
        hvdg::AnchorGroup* d_ag = reinterpret_cast<hvdg::AnchorGroup*>(d_jctl + nf);
        int* d_fl = reinterpret_cast<int*>(d_ag + nf);
        std::vector<hvdg::AnchorGroup> ag;
        for (int j : col) {
          hvdg::AnchorGroup G{};
          G.field = j;
          G.count = 0;
          for (size_t pi = 0; pi < mp.size(); ++pi) {
            if (mp[pi].cur != j) continue;
            const int k = mp[pi].ref;
            if (std::abs(k - j) > cfg.nr_radius) continue;
            G.p[G.count++] = hvdg::AnchorPair{(int)pi, k,
                                              (float)(in[j].parity - in[k].parity) / 2.0f};
          }
          ag.push_back(G);
        }
        e = cudaMemcpyAsync(d_ag, ag.data(), sizeof(hvdg::AnchorGroup) * ag.size(),
                            cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_fl, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D anchor tables");
        // the anchor's per-pixel vectors / confidences (VectorsPerPixel and
        // the slow UpsampleConfidence of the pre-snap motion)
        float* pre = at<float>(ctx, X(x_pre));
        float* asn = at<float>(ctx, X(x_asnap));
        hvdg::VecBuffers va = vb;
        va.dy = pre;
        va.dx = pre + (size_t)nt * max_pairs;
        va.conf = pre + 2 * (size_t)nt * max_pairs;
        va.snap_dy = asn;
        va.snap_dx = asn + (size_t)nt * max_pairs;
        va.c2 = asn + 2 * (size_t)nt * max_pairs;
        va.c2_snap = asn + 3 * (size_t)nt * max_pairs;
        va.c2_snap2 = va.c2_snap;
        va.src_idx = at<int2>(ctx, X(x_asrc));
        va.conf_px = at<float>(ctx, X(x_acpx));
        va.conf_tmp = at<float>(ctx, X(x_actmp));
        const int npairs_c = (int)mp.size();
        va.conf_bytes = sizeof(float) * plane * npairs_c;
        if (npairs_c > 0) hvdg::launch_vectors(d_mf, d_mp, npairs_c, h, w, ma, va, false, s);
        hvdg::AnchorArgs aa;
        aa.fields = at<FieldDesc>(ctx, L.o_fields);
        aa.groups = d_ag;
        aa.ngroups = (int)ag.size();
        aa.tile = tile;
        aa.tiles_off = nt;
        aa.snap_dy = va.snap_dy;
        aa.snap_dx = va.snap_dx;
        aa.conf_px = va.conf_px;
        aa.pix_off = d_pix_off;
        aa.Y = at<float>(ctx, L.o_Y);
        aa.chi = at<float2>(ctx, L.o_X0);
        aa.S = at<float>(ctx, L.o_S);
        aa.line_phasor = at<float4>(ctx, L.o_lineph);
        aa.col_phasor = at<float2>(ctx, L.o_colph);
        aa.eps_b = cfg.nr_eps;
        aa.Ya = at<float>(ctx, X(x_ya));
        aa.Ca = at<float2>(ctx, X(x_caa));
        aa.Wa = at<float>(ctx, X(x_wa));
        aa.resid = at<float>(ctx, X(x_res));
        hvdg::launch_anchor(aa, h, w, s);
        hvdg::JointArgs ja;
        ja.fields = at<FieldDesc>(ctx, L.o_fields);
        ja.flist = d_fl;
        ja.nfl = (int)col.size();
        ja.bx = jbx;
        ja.by = jby;
        ja.S = at<float>(ctx, L.o_S);
        ja.line_phasor = at<float4>(ctx, L.o_lineph);
        ja.col_phasor = at<float2>(ctx, L.o_colph);
        ja.nbr = at<float4>(ctx, X(x_nbr));
        ja.nu = cfg.temporal_strength;
        ja.eps_t = cfg.temporal_eps;
        ja.Ya = aa.Ya;
        ja.Ca = aa.Ca;
        ja.Wa = aa.Wa;
        ja.nu_a = cfg.nr_anchor;
        ja.eps = cfg.charbonnier_eps;
        ja.eps_c = cfg.chroma_eps;
        ja.k = cfg.structure_coupling;
        float4* jp = at<float4>(ctx, X(x_jp));
        const int64_t bp = plane * nf;
        ja.X = jp;
        ja.G[0] = jp + bp;
        ja.G[1] = jp + 2 * bp;
        ja.D[0] = jp + 3 * bp;
        ja.D[1] = jp + 4 * bp;
        ja.Q[0] = jp + 5 * bp;
        ja.Q[1] = jp + 6 * bp;
        ja.W = jp + 7 * bp;
        ja.M0 = jp + 8 * bp;
        ja.M1 = jp + 9 * bp;
        ja.M2 = at<float>(ctx, X(x_jm2));
        ja.partials = at<double>(ctx, X(x_jpart));
        ja.ctl = d_jctl;
        const FieldDesc& f0 = b.fields[col[0]];
        hvdg::launch_joint_load(ja, at<float>(ctx, L.o_Y), at<float2>(ctx, L.o_X0), h, w, s);
        for (int o = 0; o < f0.n_outer; ++o) hvdg::launch_joint_outer(ja, f0.n_inner, h, w, s);
        hvdg::launch_joint_store(ja, at<float>(ctx, L.o_Y), at<float2>(ctx, L.o_X0), false, h, w, s);
        e = cudaGetLastError();
        if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "anchored pass launch");
        S.launches += 6 + f0.n_outer * (6 + 2 * f0.n_inner);
      } else {
        sa.unit_base = cbegin[ci];
        sa.n_units = ccount[ci];
        sa.n_phases = cphases[ci];
        e = hvdg::launch_solver(sa, solver_grid(ctx, ccount[ci]), s);
        if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "solver launch");
        S.launches += 2;
      }
      // the solved fields' luma / chi now replace their init state (Ys[j], chis[j])
    }
  }
  if (anchor_on && cfg.output_fidelity) {
    // the anchored pass leaves Y free; the output reverts to data fidelity
    std::vector<int> all(nf);
    for (int j = 0; j < nf; ++j) all[j] = j;
    int* d_fl = reinterpret_cast<int*>(reinterpret_cast<hvdg::AnchorGroup*>(
                    reinterpret_cast<hvdg::JointCtl*>(at<char>(ctx, X(x_jctl))) + nf) + nf);
    e = cudaMemcpyAsync(d_fl, all.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D field list");
    hvdg::JointArgs ja;
    std::memset(&ja, 0, sizeof(ja));
    ja.fields = at<FieldDesc>(ctx, L.o_fields);
    ja.flist = d_fl;
    ja.nfl = nf;
    ja.S = at<float>(ctx, L.o_S);
    ja.line_phasor = at<float4>(ctx, L.o_lineph);
    ja.col_phasor = at<float2>(ctx, L.o_colph);
    hvdg::launch_output_fidelity(ja, at<float>(ctx, L.o_Y), at<float2>(ctx, L.o_X0), h, w, s);
  }
  mark(ctx, 3);
  return stage_finish(ctx, S, out, opt, diag);
}

// DecodeFieldWindow (sequence.cpp:270-281, 423-1116) over one window of one
// geometry. With the temporal terms off every field is independent (the
// stride-1 sweep, sequence.cpp:1076-1084) and the window is one batch.
hvdg_status decode_window_impl(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                               const hvdg_config* cfg, hvdg_field_out* out, hvdg_diag* diag,
                               const RunOpts& opt = RunOpts()) {
  const hvdg_geometry& g = *fields[0].geometry;
  const int amb_stride = uses_vswitch(g) ? 4 : 2;
  const bool scan = cfg->temporal_strength == 0.0f && cfg->cg_iterations > 0 && n > amb_stride;
  cudaSetDevice(ctx->device);
  if (diag) std::memset(diag, 0, sizeof(*diag));
  if (n > 1 && (scan || cfg->temporal_strength > 0.0f))
    return decode_window_3d(ctx, fields, n, cfg, out, diag, opt);
  if (ctx->batched || opt.amp_out) return run_batch(ctx, fields, n, cfg, out, diag, opt);
  for (int i = 0; i < n; ++i) {
    const hvdg_status st = run_batch(ctx, fields + i, 1, cfg, out + i, diag, opt);
    if (st != HVDG_OK) return st;
  }
  return HVDG_OK;
}

// ---------------------------------------------------------------------------
// Frame bridge (hvd-core/src/frame_bridge.cpp): de-weave, field-order vote,
// weave + 10-bit requantisation, on the host around the device window decode.
// ---------------------------------------------------------------------------
int64_t frame_line_offset(const hvdg_frame_params& fp, int line) {
  // FrameLineOffset (frame_bridge.h:106-112)
  int64_t off = (int64_t)line * fp.frame_width;
  for (int i = 0; i < fp.extra_sample_line_count && i < HVDG_MAX_EXTRA_SAMPLE_LINES; ++i)
    if (fp.extra_sample_lines[i] < line) ++off;
  return off;
}

hvdg_geometry geometry_from_params(const hvdg_frame_params& fp) {
  // FieldGeometryFromParams (frame_bridge.cpp:43-59)
  hvdg_geometry g;
  std::memset(&g, 0, sizeof(g));
  g.field_width = fp.frame_width;
  g.field_height = fp.field1_lines;
  g.active_video_start = fp.active_video_start;
  g.active_video_end = fp.active_video_end;
  g.colour_burst_start = fp.colour_burst_start;
  g.colour_burst_end = fp.colour_burst_end;
  g.first_active_field_line = fp.first_active_frame_line / 2;
  g.last_active_field_line = fp.last_active_frame_line != 0 ? fp.last_active_frame_line / 2 : 0;
  g.sample_rate = fp.sample_rate;
  g.subcarrier_hz = fp.subcarrier_hz;
  g.standard = fp.standard;
  return g;
}

// SplitFrameFields (frame_bridge.cpp:61-99): block 1 / block 2 in IRE.
void split_frame_fields(const int16_t* frame, const hvdg_frame_params& fp, float* top,
                        float* bottom) {
  const int fw = fp.frame_width, fh = fp.frame_height, f1 = fp.field1_lines, f2 = fh - f1;
  const float cpi = (fp.white_level - fp.blanking_level) / 100.0f;
  for (int y = 0; y < f1; ++y) {
    const int64_t ot = frame_line_offset(fp, y);
    const int64_t ob = frame_line_offset(fp, f1 + y);
    for (int x = 0; x < fw; ++x) {
      const float st = (y < f1) ? (float)frame[ot + x] : fp.blanking_level;
      const float sb = (y < f2) ? (float)frame[ob + x] : fp.blanking_level;
      top[(size_t)y * fw + x] = (st - fp.blanking_level) / cpi;
      bottom[(size_t)y * fw + x] = (sb - fp.blanking_level) / cpi;
    }
  }
}

// DetectFieldParity (frame_bridge.cpp:102-149) over a sampler
// ire(block, field_line, x) of the two de-woven fields in IRE.
template <typename Ire>
int detect_field_parity_t(Ire ire, const hvdg_frame_params& fp, const hvdg_geometry& g) {
  const int fal = g.first_active_field_line, lal = last_active_line(g);
  const int a0 = fp.active_video_start, a1 = fp.active_video_end;
  const int lines = lal - fal, width = a1 - a0;
  if (lines < 8 || width < 32) return 0;
  const int ystep = std::max(1, lines / 120);
  double ep = 0.0, em = 0.0;
  long n = 0;
  for (int r = fal + 1; r + 1 < lal; r += ystep) {
    for (int x = a0; x + 4 <= a1; x += 16) {
      auto lp = [&](int k, int row) {
        return 0.25f * (ire(k, row, x) + ire(k, row, x + 1) + ire(k, row, x + 2) + ire(k, row, x + 3));
      };
      const float b = lp(1, r), ac = lp(0, r), au = lp(0, r - 1), ad = lp(0, r + 1);
      ep += std::fabs(b - 0.5f * (ac + ad));
      em += std::fabs(b - 0.5f * (ac + au));
      ++n;
    }
  }
  if (n == 0) return 0;
  ep /= (double)n;
  em /= (double)n;
  const double lo = std::min(ep, em), hi = std::max(ep, em);
  if (hi <= 1e-9 || (hi - lo) / hi < 0.02) return 0;
  return ep < em ? +1 : -1;
}

int detect_field_parity(const float* b1, const float* b2, const hvdg_frame_params& fp,
                        const hvdg_geometry& g) {
  const int fw = fp.frame_width;
  return detect_field_parity_t(
      [&](int k, int row, int x) { return (k == 0 ? b1 : b2)[(size_t)row * fw + x]; }, fp, g);
}

// The same vote read straight from an int16 frame: each sample the vote
// touches is converted exactly as SplitFrameFields converts it.
int detect_field_parity_frame(const int16_t* frame, const hvdg_frame_params& fp,
                              const hvdg_geometry& g) {
  const int f1 = fp.field1_lines, fh = fp.frame_height;
  const float cpi = (fp.white_level - fp.blanking_level) / 100.0f;
  return detect_field_parity_t(
      [&](int k, int row, int x) {
        const int flat = k == 0 ? row : f1 + row;
        const bool valid = k == 0 ? row < f1 : flat < fh;
        const float s = valid ? (float)frame[frame_line_offset(fp, flat) + x] : fp.blanking_level;
        return (s - fp.blanking_level) / cpi;
      },
      fp, g);
}

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

// AmbiguousBoxes: tile score sqrt(luma HF energy x chroma-magnitude HF
// energy) over 16 x 16 tiles (HF = minus a count-normalised 8 x 8 box mean),
// tiles >= 4 x the median score, kept where >= 2 of their 8 neighbours are
// flagged and off the outer tile ring; row bands of >= 2 such tiles (at
// most 4, closest bands merged), per band one box per column run (gap <= 2,
// single tiles dropped) with a 16-row / 48-column halo. Empty: stay 2-D;
// one invalid box: no band but a median above 3 IRE^2, or the boxes cover
// more than max_area of the field.
std::vector<SelBox> ambiguous_boxes(const float* Y, const float* chi_ri, int h, int w,
                                    float max_area) {
  const int T = 16, HX = 48, HY = 16, K = T / 2;
  const int th = (h + T - 1) / T, tw = (w + T - 1) / T;
  const size_t np = (size_t)h * w;
  std::vector<float> ya(Y, Y + np), ca(np);
  for (size_t i = 0; i < np; ++i)
    ca[i] = std::abs(std::complex<float>(chi_ri[2 * i], chi_ri[2 * i + 1]));
  // count-normalised separable box mean over offsets [-K/2, K - K/2)
  auto box_mean = [&](const std::vector<float>& a) {
    std::vector<float> v(np), o(np);
    for (int x = 0; x < w; ++x)
      for (int y = 0; y < h; ++y) {
        float acc = 0.0f;
        int n = 0;
        for (int d = -K / 2; d < K - K / 2; ++d) {
          if (y + d < 0 || y + d >= h) continue;
          acc += a[(size_t)(y + d) * w + x];
          ++n;
        }
        v[(size_t)y * w + x] = acc / std::max(n, 1);
      }
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        float acc = 0.0f;
        int n = 0;
        for (int d = -K / 2; d < K - K / 2; ++d) {
          if (x + d < 0 || x + d >= w) continue;
          acc += v[(size_t)y * w + x + d];
          ++n;
        }
        o[(size_t)y * w + x] = acc / std::max(n, 1);
      }
    return o;
  };
  const std::vector<float> ly = box_mean(ya), lc = box_mean(ca);
  std::vector<double> ey((size_t)th * tw, 0.0), ec((size_t)th * tw, 0.0);
  std::vector<int> cnt((size_t)th * tw, 0);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t i = (size_t)y * w + x, t = (size_t)(y / T) * tw + x / T;
      const double dy = ya[i] - ly[i], dc = ca[i] - lc[i];
      ey[t] += dy * dy;
      ec[t] += dc * dc;
      ++cnt[t];
    }
  std::vector<float> score((size_t)th * tw);
  for (size_t t = 0; t < score.size(); ++t)
    score[t] = (float)std::sqrt((ey[t] / std::max(cnt[t], 1)) * (ec[t] / std::max(cnt[t], 1)));
  std::vector<float> srt = score;
  std::nth_element(srt.begin(), srt.begin() + srt.size() / 2, srt.end());
  const float med = srt[srt.size() / 2];
  const float thr = 4.0f * med;
  auto flag = [&](int ty, int tx) { return score[(size_t)ty * tw + tx] >= thr; };
  std::vector<char> dense((size_t)th * tw, 0);
  for (int ty = 1; ty + 1 < th; ++ty)
    for (int tx = 1; tx + 1 < tw; ++tx) {
      if (!flag(ty, tx)) continue;
      int nb = 0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
          if (dy || dx) nb += flag(ty + dy, tx + dx);
      dense[(size_t)ty * tw + tx] = nb >= 2;
    }
  std::vector<std::pair<int, int>> bands;
  for (int ty = 0; ty < th; ++ty) {
    int row_n = 0;
    for (int tx = 0; tx < tw; ++tx) row_n += dense[(size_t)ty * tw + tx];
    if (row_n < 2) continue;
    if (!bands.empty() && ty - bands.back().second <= 1)
      bands.back().second = ty;
    else
      bands.emplace_back(ty, ty);
  }
  std::vector<SelBox> boxes;
  if (bands.empty()) {
    if (med > 3.0f) boxes.push_back(SelBox{});
    return boxes;
  }
  while (bands.size() > 4) {  // merge the two closest neighbouring bands
    size_t bi = 0;
    int best = INT32_MAX;
    for (size_t i = 0; i + 1 < bands.size(); ++i) {
      const int gap = bands[i + 1].first - bands[i].second;
      if (gap < best) {
        best = gap;
        bi = i;
      }
    }
    bands[bi].second = bands[bi + 1].second;
    bands.erase(bands.begin() + (long)bi + 1);
  }
  for (const auto& bd : bands) {
    std::vector<char> col(tw, 0);
    for (int ty = bd.first; ty <= bd.second; ++ty)
      for (int tx = 0; tx < tw; ++tx) col[tx] |= dense[(size_t)ty * tw + tx];
    int y0 = std::max(0, bd.first * T - HY);
    y0 -= y0 % 2;  // keep the crop on the field's line parity
    const int y1 = std::min(h, (bd.second + 1) * T + HY);
    std::vector<std::pair<int, int>> runs;
    for (int tx = 0; tx < tw; ++tx) {
      if (!col[tx]) continue;
      if (!runs.empty() && tx - runs.back().second <= 2)
        runs.back().second = tx;
      else
        runs.emplace_back(tx, tx);
    }
    const size_t first = boxes.size();
    for (const auto& r : runs) {
      if (r.second - r.first < 1) continue;
      const int x0 = std::max(0, r.first * T - HX), x1 = std::min(w, (r.second + 1) * T + HX);
      if (boxes.size() > first && x0 <= boxes.back().x1) {
        boxes.back().x1 = x1;
      } else {
        SelBox b;
        b.fy0 = y0;
        b.fy1 = y1;
        b.x0 = x0;
        b.x1 = x1;
        b.valid = true;
        boxes.push_back(b);
      }
    }
  }
  double area = 0.0;
  for (const SelBox& b : boxes) area += (double)(b.fy1 - b.fy0) * (b.x1 - b.x0);
  if (area > (double)max_area * h * w) {
    boxes.clear();
    boxes.push_back(SelBox{});
  }
  return boxes;
}

// The 3-D part of DecodeWindowSelective on top of the 2-D decode already in
// Yd / Cd (h x w per field; Cd interleaved re, im).
hvdg_status decode_selective_boxes(hvdg_ctx* ctx, const std::vector<hvdg_field_in>& fi,
                                   const hvdg_geometry& g, const hvdg_config* cfg,
                                   std::vector<std::vector<float>>& Yd,
                                   std::vector<std::vector<float>>& Cd) {
  const int nf = (int)fi.size();
  const int h = last_active_line(g) - g.first_active_field_line;
  const int w = g.active_video_end - g.active_video_start;
  const std::vector<SelBox> boxes =
      ambiguous_boxes(Yd[0].data(), Cd[0].data(), h, w, cfg->selective_max_area);
  if (boxes.empty()) return HVDG_OK;
  std::vector<hvdg_field_out> fo(nf);
  if (!boxes[0].valid) {  // ambiguity everywhere: the full 3-D window
    for (int j = 0; j < nf; ++j) fo[j] = hvdg_field_out{Yd[j].data(), Cd[j].data(), nullptr, nullptr};
    return decode_window_impl(ctx, fi.data(), nf, cfg, fo.data(), nullptr);
  }
  for (const SelBox& b : boxes) {
    hvdg_geometry gb = g;
    gb.first_active_field_line = g.first_active_field_line + b.fy0;
    gb.last_active_field_line = g.first_active_field_line + b.fy1;
    gb.active_video_start = g.active_video_start + b.x0;
    gb.active_video_end = g.active_video_start + b.x1;
    const int bh = b.fy1 - b.fy0, bw = b.x1 - b.x0;
    std::vector<hvdg_field_in> fb = fi;
    std::vector<std::vector<float>> Y3(nf, std::vector<float>((size_t)bh * bw)),
        C3(nf, std::vector<float>((size_t)bh * bw * 2));
    for (int j = 0; j < nf; ++j) {
      fb[j].geometry = &gb;
      fo[j] = hvdg_field_out{Y3[j].data(), C3[j].data(), nullptr, nullptr};
    }
    const hvdg_status st = decode_window_impl(ctx, fb.data(), nf, cfg, fo.data(), nullptr);
    if (st != HVDG_OK) return st;
    // feather: linear ramps over min(16, bh / 3) rows and min(48, bw / 3) columns
    const int hy = std::min(16, bh / 3), hx = std::min(48, bw / 3);
    for (int j = 0; j < nf; ++j)
      for (int y = 0; y < bh; ++y) {
        float ry = 1.0f;
        if (y < hy)
          ry = (float)y / hy;
        else if (y >= bh - hy)
          ry = (float)(bh - 1 - y) / hy;
        for (int x = 0; x < bw; ++x) {
          float rx = 1.0f;
          if (x < hx)
            rx = (float)x / hx;
          else if (x >= bw - hx)
            rx = (float)(bw - 1 - x) / hx;
          const float m = ry * rx;
          const size_t o = (size_t)(b.fy0 + y) * w + b.x0 + x, q = (size_t)y * bw + x;
          Yd[j][o] = Yd[j][o] * (1.0f - m) + Y3[j][q] * m;
          Cd[j][2 * o] = Cd[j][2 * o] * (1.0f - m) + C3[j][2 * q] * m;
          Cd[j][2 * o + 1] = Cd[j][2 * o + 1] * (1.0f - m) + C3[j][2 * q + 1] * m;
        }
      }
  }
  return HVDG_OK;
}

// The sequence bridge's diagnostic maps (frame_bridge.cpp:807-865): one
// decision-log line per call appended to <dir>/diag.txt, and per core frame
// <dir>/rainbow_<id>.pgm, the woven map of residual chroma in the decoded
// luma: the triangle-7 demodulation of Y by the field's own carrier, summed
// with the same-parity field two ahead (or behind) -- static luma cancels
// between same-parity fields (the carrier has flipped), a correlated
// separation error survives; 0..8 IRE -> 0..255.
void write_debug_maps(const std::string& dir, int64_t base_frame_id, int core_begin, int core_end,
                      bool f1_bottom, const hvdg_diag& d, float acc_gain,
                      const std::vector<std::vector<float>>& Y,
                      const std::vector<std::vector<float2>>& car, const std::vector<int>& parity,
                      int lines, int aw) {
  if (FILE* log = std::fopen((dir + "/diag.txt").c_str(), "a")) {
    std::fprintf(log, "frames %lld..%lld: f1_bottom=%d sigma=%g amb=%g strength=%g eps_t=%g nr_eps=%g acc=%g\n",
                 (long long)(base_frame_id + core_begin), (long long)(base_frame_id + core_end - 1),
                 f1_bottom ? 1 : 0, d.sigma_ire, d.ambiguity_ire, d.resolved_strength,
                 d.temporal_eps, d.nr_eps, acc_gain);
    std::fclose(log);
  }
  static const float kW[7] = {1, 2, 3, 4, 3, 2, 1};
  const int nfields = (int)Y.size();
  for (int t = core_begin; t < core_end; ++t) {
    std::vector<uint8_t> img((size_t)2 * lines * aw, 0);
    for (int half = 0; half < 2; ++half) {
      const int j = 2 * t + half;
      const int j2 = (j + 2 < nfields) ? j + 2 : j - 2;
      const int p = parity[j];
      for (int r = 0; r < lines; ++r)
        for (int x = 0; x + 7 <= aw; ++x) {
          std::complex<float> dj(0.f, 0.f), dk(0.f, 0.f);
          for (int k = 0; k < 7; ++k) {
            const size_t o = (size_t)r * aw + x + k;
            dj += kW[k] * Y[j][o] * std::conj(std::complex<float>(car[j][o].x, car[j][o].y));
            if (j2 >= 0)
              dk += kW[k] * Y[j2][o] * std::conj(std::complex<float>(car[j2][o].x, car[j2][o].y));
          }
          const float e = (j2 >= 0) ? std::abs(dj + dk) / 32.0f : std::abs(dj) / 16.0f;
          const int v = std::min(std::max((int)(e * 32.0f), 0), 255);
          img[(size_t)(2 * r + p) * aw + x + 3] = (uint8_t)v;
        }
    }
    char name[64];
    std::snprintf(name, sizeof(name), "/rainbow_%06lld.pgm", (long long)(base_frame_id + t));
    if (FILE* f = std::fopen((dir + name).c_str(), "wb")) {
      std::fprintf(f, "P5\n%d %d\n255\n", aw, 2 * lines);
      std::fwrite(img.data(), 1, img.size(), f);
      std::fclose(f);
    }
  }
}

int16_t clamp_u10(float v) {
  const long r = std::lround(v);
  return (int16_t)std::min<long>(std::max<long>(r, 0), 1023);
}
int16_t clamp_s10(float v) {
  const long r = std::lround(v);
  return (int16_t)std::min<long>(std::max<long>(r, -1023), 1023);
}

// Lock-in / burst amplitude of one IRE field (kernel-level entry points).
hvdg_status lockin_one(hvdg_ctx* ctx, const float* field_ire, const hvdg_geometry* g, float* theta,
                       int8_t* vswitch, float* amp) {
  hvdg_status st = check_geometry(g);
  if (st != HVDG_OK) return st;
  cudaSetDevice(ctx->device);
  const size_t fbytes = sizeof(float) * g->field_width * g->field_height;
  const size_t o_field = 0;
  const size_t o_desc = align_up(fbytes, 256);
  const size_t o_theta = align_up(o_desc + sizeof(hvdg::PrepDesc), 256);
  const size_t o_vsw = align_up(o_theta + sizeof(float) * g->field_height, 256);
  const size_t o_amp = align_up(o_vsw + g->field_height, 256);
  const size_t o_lph = align_up(o_amp + sizeof(float), 256);
  const size_t total = align_up(o_lph + sizeof(float4) * g->field_height, 256);
  st = ctx->arena.reserve(total, ctx->stream);
  if (st != HVDG_OK) return st;
  ctx->epoch += 1;
  char* base = static_cast<char*>(ctx->arena.base);
  hvdg::PrepDesc pd;
  std::memset(&pd, 0, sizeof(pd));
  pd.samples = base + o_field;
  pd.sample_type = HVDG_SAMPLES_F32_IRE;
  pd.quadrant = g->subcarrier_hz <= 0.0 ? 1 : 0;
  pd.fh = g->field_height;
  pd.fw = g->field_width;
  pd.bx0 = g->colour_burst_start;
  pd.bx1 = g->colour_burst_end;
  pd.fal = g->first_active_field_line;
  pd.lal = last_active_line(*g);
  pd.a0 = g->active_video_start;
  pd.a1 = g->active_video_end;
  pd.vswitch_family = uses_vswitch(*g) ? 1 : 0;
  pd.nominal_burst = nominal_burst(*g);
  pd.w0 = phase_per_sample(*g);
  pd.adv = line_advance(*g);
  pd.line_step = 1;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(base + o_field, field_ire, fbytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D field");
  e = cudaMemcpyAsync(base + o_desc, &pd, sizeof(pd), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D desc");
  const hvdg::PrepDesc* dd = reinterpret_cast<const hvdg::PrepDesc*>(base + o_desc);
  if (theta) {
    hvdg::LockinOut lo;
    lo.theta = reinterpret_cast<float*>(base + o_theta);
    lo.theta64 = nullptr;
    lo.vswitch = reinterpret_cast<signed char*>(base + o_vsw);
    lo.line_phasor = reinterpret_cast<float4*>(base + o_lph);
    hvdg::launch_burst_lockin(dd, 1, lo, s);
    cudaMemcpyAsync(theta, base + o_theta, sizeof(float) * g->field_height, cudaMemcpyDeviceToHost, s);
    if (vswitch) cudaMemcpyAsync(vswitch, base + o_vsw, g->field_height, cudaMemcpyDeviceToHost, s);
  }
  if (amp) {
    hvdg::launch_burst_amplitude(dd, 1, reinterpret_cast<float*>(base + o_amp), s);
    cudaMemcpyAsync(amp, base + o_amp, sizeof(float), cudaMemcpyDeviceToHost, s);
  }
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "lock-in");
  return HVDG_OK;
}

// Integer-SAD motion estimation of one pair (me_mode 1): block x block
// tiles, exhaustive +-range; tile outputs like EstimateMotion's.
hvdg_status estimate_motion_sad(hvdg_ctx* ctx, const float* y_ref, const float* y_cur, int h,
                                int w, int block, int range, float* dy, float* dx,
                                float* confidence) {
  if (block > hvdg::sad_max_block() || range > hvdg::sad_max_range()) {
    ctx->last_error = "integer-SAD motion: block or range above the supported maximum";
    return HVDG_ERR_UNSUPPORTED;
  }
  const int th = (h + block - 1) / block, tw = (w + block - 1) / block, nt = th * tw;
  if (nt > kSadMaxTiles) {
    ctx->last_error = "integer-SAD motion: too many tiles for one confidence pass";
    return HVDG_ERR_UNSUPPORTED;
  }
  cudaSetDevice(ctx->device);
  const int pitch = (w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
  const size_t plane = (size_t)h * pitch;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align_up(o + bytes, 256);
    return r;
  };
  const size_t o_f = take(sizeof(hvdg::MeField) * 2);
  const size_t o_p = take(sizeof(hvdg::MePair));
  const size_t o_l = take(sizeof(float) * 2 * plane);
  const size_t o_v = take(sizeof(int) * 2 * plane);
  const size_t o_q = take(sizeof(int) * 2 * plane);
  size_t of[7], od[4];
  for (int i = 0; i < 7; ++i) of[i] = take(sizeof(float) * nt);
  for (int i = 0; i < 4; ++i) od[i] = take(sizeof(double) * nt);
  hvdg_status st = ctx->arena.reserve(o, ctx->stream);
  if (st != HVDG_OK) return st;
  ctx->epoch += 1;
  char* base = static_cast<char*>(ctx->arena.base);
  hvdg::MeField mf[2];
  for (int i = 0; i < 2; ++i) {
    std::memset(&mf[i], 0, sizeof(mf[i]));
    mf[i].h = h;
    mf[i].w = w;
    mf[i].pitch = pitch;
    mf[i].y_off = mf[i].t_off = mf[i].b_off = (int64_t)i * plane;
  }
  const hvdg::MePair pr{0, 1};
  cudaStream_t s = ctx->stream;
  cudaGetLastError();
  cudaError_t e = cudaMemcpyAsync(base + o_f, mf, sizeof(mf), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_p, &pr, sizeof(pr), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(base + o_l, sizeof(float) * pitch, y_ref, sizeof(float) * w,
                          sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(base + o_l + sizeof(float) * plane, sizeof(float) * pitch, y_cur,
                          sizeof(float) * w, sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D motion inputs");
  hvdg::SadArgs a;
  a.block = block;
  a.range = range;
  a.tiles_off = nt;
  hvdg::SadBuffers b;
  b.luma = reinterpret_cast<const float*>(base + o_l);
  b.vsum = reinterpret_cast<int*>(base + o_v);
  b.qblur = reinterpret_cast<int*>(base + o_q);
  b.mdy = reinterpret_cast<float*>(base + of[0]);
  b.mdx = reinterpret_cast<float*>(base + of[1]);
  b.sdy = reinterpret_cast<float*>(base + of[2]);
  b.sdx = reinterpret_cast<float*>(base + of[3]);
  b.dy = reinterpret_cast<float*>(base + of[4]);
  b.dx = reinterpret_cast<float*>(base + of[5]);
  b.conf = reinterpret_cast<float*>(base + of[6]);
  b.bestv = reinterpret_cast<double*>(base + od[0]);
  b.s1 = reinterpret_cast<double*>(base + od[1]);
  b.s2 = reinterpret_cast<double*>(base + od[2]);
  b.npx = reinterpret_cast<double*>(base + od[3]);
  hvdg::launch_motion_sad(reinterpret_cast<const hvdg::MeField*>(base + o_f), 2, h, w,
                          reinterpret_cast<const hvdg::MePair*>(base + o_p), 1, a, b, s);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, b.dy, sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, b.dx, sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(confidence, b.conf, sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "integer-SAD motion estimation");
  return HVDG_OK;
}

// Decode adjoint of one 2-D field (no reference counterpart): forward with
// the IRLS iterates checkpointed (one solver launch per outer, so chi_o and
// the weights W(chi_o) can be kept), then the reverse sweep over the outers
// (an adjoint CG solve per outer in the same persistent solver, weights
// frozen, right-hand side injected as a constant gradient term), then the
// HolographicInit adjoint and the crop / level transposes.
hvdg_status decode_adjoint_field(hvdg_ctx* ctx, const hvdg_field_in& fi, const hvdg_config& cfg,
                                 const float* y_bar, const float* chi_bar, float* samples_bar,
                                 double* scalar_bar, int adj_iters, hvdg_field_out* out,
                                 hvdg_diag* diag) {
  const hvdg_geometry& g = *fi.geometry;
  const int h = last_active_line(g) - g.first_active_field_line;
  const int w = g.active_video_end - g.active_video_start;
  const int pitch = (w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
  const int pad = std::min(hvdg::kInitPad, h - 1 > 0 ? h - 1 : 0);
  const int hp = h + 2 * pad;
  const int64_t plane = (int64_t)h * pitch;
  const int64_t rplane = (int64_t)hp * pitch;
  // the forward's budget, one outer per solver launch
  const int n_outer = std::max(1, fi.irls_outer > 0 ? fi.irls_outer : cfg.irls_outer);
  const int cg_cfg = fi.cg_iterations >= 0 ? fi.cg_iterations : cfg.cg_iterations;
  const int cg_total = cfg.fast ? cg_cfg * 2 / 3 : cg_cfg;
  const int n_inner = std::max(1, cg_total / n_outer);
  hvdg_config c1 = cfg;
  c1.irls_outer = 1;
  c1.cg_iterations = n_inner;
  c1.fast = 0;
  c1.cg_tol = cfg.cg_tol > 0.0f ? cfg.cg_tol : (cfg.fast ? 0.10f : 0.02f);
  hvdg_field_in f1 = fi;
  f1.irls_outer = 1;
  f1.cg_iterations = n_inner;
  hvdg::AdjGeom ag;
  ag.h = h;
  ag.w = w;
  ag.pitch = pitch;
  ag.hp = hp;
  ag.pad = pad;
  const int nb = hvdg::adj_blocks(ag);
  size_t xo = 0;
  auto take = [&](size_t bytes) {
    const size_t r = xo;
    xo = align_up(xo + bytes, 256);
    return r;
  };
  const size_t x_ck = take(sizeof(float2) * plane * (n_outer + 1));
  const size_t x_wk = take(sizeof(float4) * plane * n_outer);
  const size_t x_cv = take(sizeof(float2) * plane * 2);
  const size_t x_zero = take(sizeof(float) * plane);
  const size_t x_B = take(sizeof(float2) * plane);
  const size_t x_yb = take(sizeof(float) * plane);
  const size_t x_cb = take(sizeof(float2) * plane);
  const size_t x_sb = take(sizeof(float) * plane);
  const size_t x_pa = take(sizeof(float2) * plane * 4);
  const size_t x_ai = take(sizeof(float2) * plane * 5);
  const size_t x_ain = take(sizeof(float2) * rplane * 2);
  const size_t x_aout = take(sizeof(float2) * rplane * 2);
  const size_t x_part = take(sizeof(double) * 4 * nb);
  const size_t x_acc = take(sizeof(double) * 4);
  const size_t x_smp = take(sizeof(float) * (size_t)g.field_height * g.field_width);
  RunOpts opt;
  Staged S;
  hvdg_status st = stage_upload(ctx, &f1, 1, &c1, opt, xo, S);
  if (st != HVDG_OK) return st;
  const Layout& L = S.b.L;
  auto X = [&](size_t off) { return S.extra + off; };
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  st = stage_prepare(ctx, S, opt);
  if (st != HVDG_OK) return st;
  ag.line_phasor = at<float4>(ctx, L.o_lineph);
  ag.col_phasor = at<float2>(ctx, L.o_colph);
  float2* ck = at<float2>(ctx, X(x_ck));
  float4* wk = at<float4>(ctx, X(x_wk));
  float2* cv = at<float2>(ctx, X(x_cv));
  // init variants and chi_0 (before the solver reuses G0 / D0)
  e = cudaMemcpyAsync(cv, at<float2>(ctx, L.o_G0), sizeof(float2) * plane, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cv + plane, at<float2>(ctx, L.o_D0), sizeof(float2) * plane,
                        cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ck, at<float2>(ctx, L.o_X0), sizeof(float2) * plane, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint checkpoints");
  hvdg::launch_aniso(at<FieldDesc>(ctx, L.o_fields), 1, at<float2>(ctx, L.o_X0), s);
  // ---- forward, one outer per launch ----
  hvdg::SolverArgs sa = solver_args(ctx, S);
  const int grid = solver_grid(ctx, L.total_units);
  int cg_run = 0;
  for (int o = 0; o < n_outer; ++o) {
    stage_reset(ctx, S);
    e = hvdg::launch_solver(sa, grid, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint forward solver");
    e = cudaMemcpyAsync(ck + (o + 1) * plane, at<float2>(ctx, L.o_X0), sizeof(float2) * plane,
                        cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(wk + o * plane, at<float4>(ctx, L.o_W), sizeof(float4) * plane,
                          cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint checkpoints");
    FieldCtl ctl;
    int flags[4];
    e = cudaMemcpyAsync(&ctl, at<FieldCtl>(ctx, L.o_ctl), sizeof(ctl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(flags, at<int>(ctx, L.o_flags), sizeof(flags), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint forward");
    if (flags[1]) {
      ctx->last_error = "non-finite input samples";
      return HVDG_ERR_NONFINITE_INPUT;
    }
    if (flags[0]) {
      ctx->last_error = "device-side bounded wait expired in the solver";
      return HVDG_ERR_DEVICE_TIMEOUT;
    }
    cg_run += ctl.cg_iters;
  }
  if (out && (out->luma || out->chroma)) {
    if (out->luma)
      e = cudaMemcpy2DAsync(out->luma, sizeof(float) * w, at<float>(ctx, L.o_Y), sizeof(float) * pitch,
                            sizeof(float) * w, h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && out->chroma)
      e = cudaMemcpy2DAsync(out->chroma, sizeof(float2) * w, at<float2>(ctx, L.o_X0),
                            sizeof(float2) * pitch, sizeof(float2) * w, h, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint forward outputs");
  }
  // ---- reverse sweep ----
  FieldDesc fd;
  e = cudaMemcpyAsync(&fd, at<FieldDesc>(ctx, L.o_fields), sizeof(fd), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint field descriptor");
  hvdg::AdjScalars sc;
  sc.eps = cfg.charbonnier_eps;
  sc.eps_c = cfg.chroma_eps;
  sc.k = cfg.structure_coupling;
  sc.mu_h = fd.mu_h;
  sc.mu_v = fd.mu_v;
  sc.aniso = cfg.lambda_c != 0.0f ? fd.mu_h / cfg.lambda_c : 1.0f;
  FieldDesc fa = fd;
  fa.n_outer = 1;
  fa.n_inner = adj_iters;
  fa.n_phases = 2 + adj_iters + 1;
  fa.cg_tol = 1e-6f;
  fa.adj_flags = hvdg::kAdjFixedW | hvdg::kAdjExtB;
  fa.has_nbr = 0;
  float* zero = at<float>(ctx, X(x_zero));
  float2* B = at<float2>(ctx, X(x_B));
  float* yb = at<float>(ctx, X(x_yb));
  float2* cb = at<float2>(ctx, X(x_cb));
  float* sb = at<float>(ctx, X(x_sb));
  float2* pa = at<float2>(ctx, X(x_pa));
  double* part = at<double>(ctx, X(x_part));
  double* acc = at<double>(ctx, X(x_acc));
  e = cudaMemsetAsync(zero, 0, sizeof(float) * plane, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(yb, 0, sizeof(float) * plane, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(cb, 0, sizeof(float2) * plane, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(double) * 4, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(yb, sizeof(float) * pitch, y_bar, sizeof(float) * w, sizeof(float) * w, h,
                          cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(cb, sizeof(float2) * pitch, chi_bar, sizeof(float2) * w,
                          sizeof(float2) * w, h, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(at<FieldDesc>(ctx, L.o_fields), &fa, sizeof(fa), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint cotangents");
  hvdg::launch_adj_output(ag, yb, sb, cb, s);
  hvdg::SolverArgs sadj = sa;
  sadj.S = zero;
  sadj.B = B;
  sadj.n_phases = fa.n_phases;
  std::vector<double> np(nb);
  int adj_run = 0;
  for (int o = n_outer - 1; o >= 0; --o) {
    // scale the right-hand side to unit rms (the solver's absolute exit is
    // relative to the field size)
    hvdg::launch_adj_norm(ag, cb, part, s);
    e = cudaMemcpyAsync(np.data(), part, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint norm");
    double ss = 0.0;
    for (int i = 0; i < nb; ++i) ss += np[i];
    if (!(ss > 0.0)) {
      // zero cotangent: every contribution of this and earlier outers is zero
      break;
    }
    const float sigma = (float)(1.0 / std::sqrt(ss / ((double)h * w)));
    hvdg::launch_adj_rhs(ag, cb, sigma, B, s);
    e = cudaMemcpyAsync(at<float4>(ctx, L.o_W), wk + o * plane, sizeof(float4) * plane,
                        cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(at<float2>(ctx, L.o_X0), 0, sizeof(float2) * plane, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint solve setup");
    stage_reset(ctx, S);
    e = hvdg::launch_solver(sadj, grid, s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint solver");
    hvdg::AdjOuter ao;
    ao.S = at<float>(ctx, L.o_S);
    ao.lam = at<float2>(ctx, L.o_X0);
    ao.inv_sigma = 1.0f / sigma;
    ao.chi1 = ck + (o + 1) * plane;
    ao.chi0 = ck + o * plane;
    ao.W = wk + o * plane;
    ao.P = pa;
    ao.GB = pa + plane;
    ao.A1 = pa + 2 * plane;
    ao.A2 = pa + 3 * plane;
    ao.partials = part;
    hvdg::launch_adj_outer(ag, sc, ao, acc, sb, cb, s);
    FieldCtl ctl;
    int flags[4];
    e = cudaMemcpyAsync(&ctl, at<FieldCtl>(ctx, L.o_ctl), sizeof(ctl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(flags, at<int>(ctx, L.o_flags), sizeof(flags), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint outer");
    if (flags[0]) {
      ctx->last_error = "device-side bounded wait expired in the adjoint solver";
      return HVDG_ERR_DEVICE_TIMEOUT;
    }
    adj_run += ctl.cg_iters;
  }
  // ---- HolographicInit adjoint (chibar now holds the cotangent of chi_0) ----
  float2* ai = at<float2>(ctx, X(x_ai));
  float2* ain = at<float2>(ctx, X(x_ain));
  float2* aout = at<float2>(ctx, X(x_aout));
  hvdg::AdjInit ia;
  ia.S = at<float>(ctx, L.o_S);
  ia.chi1 = cv;
  ia.chi2 = cv + plane;
  ia.chi0bar = cb;
  ia.a = ai;
  ia.tmp = ai + plane;
  ia.ebar = ai + 2 * plane;
  ia.cb1 = ai + 3 * plane;
  ia.cb2 = ai + 4 * plane;
  ia.adj_in = ain;
  e = cudaMemsetAsync(ain, 0, sizeof(float2) * rplane * 2, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint init setup");
  hvdg::launch_adj_init_pointwise(ag, ia, sb, s);
  hvdg::InitArgs fa_init = init_args(ctx, S);
  fa_init.adj_in = ain;
  fa_init.adj_out = aout;
  hvdg::launch_init_filter_adjoint(fa_init, L.total_prows, L.total_cgroups, s);
  hvdg::launch_adj_fold(ag, aout, sb, s);
  const float cpi = fi.sample_type == HVDG_SAMPLES_F32_IRE
                        ? 1.0f
                        : (fi.white_level - fi.blanking_level) / 100.0f;
  float* smp = at<float>(ctx, X(x_smp));
  hvdg::launch_adj_samples(ag, sb, 1.0f / cpi, g.field_height, g.field_width,
                           g.first_active_field_line, g.active_video_start, smp, s);
  double accv[4];
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(samples_bar, smp, sizeof(float) * (size_t)g.field_height * g.field_width,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(accv, acc, sizeof(accv), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adjoint outputs");
  for (int i = 0; i < 4; ++i) scalar_bar[i] += accv[i];
  if (diag) {
    diag->cg_iterations_run += cg_run + adj_run;
    diag->kernel_launches += 8 + n_outer * 6 + 12;
  }
  return HVDG_OK;
}

// ---------------------------------------------------------------------------
// Woven-frame decode: DecodeFrameBuffer (frame_bridge.cpp:168-255, engine
// DecodeFrame engine.cpp:141-195) and DecodeYcFrameBuffer
// (frame_bridge.cpp:263-377, engine DecodeChromaOnly engine.cpp:197-237), n
// independent frames in one batch. On the device: de-weave of the int16
// frames (k_frame_split), per-field lock-in + burst amplitude, the weave of
// S and of the line phasors straight into the woven plane (crop rows and
// line_step), holographic init on the woven plane (column length 2048),
// then -- composite only -- aniso + IRLS / CG; re-weave and requantisation
// (k_frame_out). On the host: the field-order vote and the copies.
// `chroma` frames are the composite frames (yc = false) or the C channel
// (yc = true, with `luma` the Y channel passed through).
// ---------------------------------------------------------------------------
hvdg_status decode_woven_frames(hvdg_ctx* ctx, const int16_t* const* chroma,
                                const int16_t* const* luma, int n, const hvdg_frame_params* fp,
                                const hvdg_config* cfg, hvdg_yc_frame* out, hvdg_diag* diag,
                                bool yc) {
  if (!ctx || !fp || !cfg || n < 0 || (n > 0 && (!chroma || !out || (yc && !luma))))
    return HVDG_ERR_BAD_ARGUMENT;
  for (int t = 0; t < n; ++t) {
    if (!chroma[t] || (yc && !luma[t])) return HVDG_ERR_BAD_ARGUMENT;
    if (!out[t].luma || !out[t].chroma || !out[t].u_plane || !out[t].v_plane)
      return HVDG_ERR_BAD_ARGUMENT;
  }
  const hvdg_frame_params& P = *fp;
  if (P.frame_width < 1 || P.frame_height < 2 || P.field1_lines < 1 ||
      P.field1_lines > P.frame_height || !(P.white_level != P.blanking_level))
    return HVDG_ERR_BAD_GEOMETRY;
  const hvdg_geometry g = geometry_from_params(P);
  hvdg_status st = check_geometry(&g);
  if (st != HVDG_OK) return st;
  const int lines = last_active_line(g) - g.first_active_field_line;
  const int w = g.active_video_end - g.active_video_start;
  st = check_plane(w, 2 * lines, uses_vswitch(g), hvdg::kColFftWide);
  if (st != HVDG_OK) {
    ctx->last_error = "woven frame beyond the device-path limits";
    return st;
  }
  if (cfg->diag_prior > 0.0f) return HVDG_ERR_UNSUPPORTED;
  if (diag) std::memset(diag, 0, sizeof(*diag));
  if (n == 0) return HVDG_OK;
  cudaSetDevice(ctx->device);
  const int fw = P.frame_width, fh = P.frame_height, f1 = P.field1_lines;
  // the woven plane: no blanking, 2 x active lines, the field's columns
  hvdg_geometry gw = g;
  gw.field_height = 2 * lines;
  gw.first_active_field_line = 0;
  gw.last_active_field_line = 2 * lines;
  // field order per frame (ResolveField1IsBottom, frame_bridge.cpp:152-160;
  // the Y/C path resolves auto to the format convention, :283-287). The
  // field flagged first lands on the even woven rows (engine.cpp:55-57).
  std::vector<hvdg_field_in> fi(2 * (size_t)n);
  for (int t = 0; t < n; ++t) {
    bool f1_bottom = cfg->field_order == 2;
    if (!yc && cfg->field_order == 0) f1_bottom = detect_field_parity_frame(chroma[t], P, g) < 0;
    for (int k = 0; k < 2; ++k) {
      hvdg_field_in& f = fi[2 * t + k];
      std::memset(&f, 0, sizeof(f));
      f.samples = nullptr;
      f.sample_type = HVDG_SAMPLES_F32_IRE;
      f.parity = (k == 0) == !f1_bottom ? 0 : 1;
      f.geometry = &g;
      f.irls_outer = 0;
      f.cg_iterations = -1;
    }
  }
  RunOpts opt;
  opt.weave_geom = &gw;
  opt.do_solve = !yc && cfg->cg_iterations > 0 && !cfg->monochrome;
  // extra region: line offsets | source frames | pass-through luma | outputs
  const int64_t need = frame_line_offset(P, fh - 1) + fw;  // samples the reference reads
  const int64_t stride = (int64_t)align_up((size_t)need, 128);
  const size_t npx = (size_t)fw * fh;
  const size_t o_lines = 0;
  const size_t o_src = align_up(sizeof(int64_t) * fh, 256);
  const size_t o_pass = align_up(o_src + sizeof(int16_t) * stride * n, 256);
  const size_t o_ol = align_up(o_pass + (yc ? sizeof(int16_t) * stride * n : 0), 256);
  const size_t o_oc = align_up(o_ol + sizeof(int16_t) * npx * n, 256);
  const size_t o_ou = align_up(o_oc + sizeof(int16_t) * npx * n, 256);
  const size_t o_ov = align_up(o_ou + sizeof(double) * npx * n, 256);
  const size_t xbytes = align_up(o_ov + sizeof(double) * npx * n, 256);
  Staged S;
  st = stage_upload(ctx, fi.data(), 2 * n, cfg, opt, xbytes, S);
  if (st != HVDG_OK) return st;
  const Batch& b = S.b;
  const Layout& L = b.L;
  cudaStream_t s = ctx->stream;
  char* X = at<char>(ctx, S.extra);
  std::vector<int64_t> loff(fh);
  for (int y = 0; y < fh; ++y) loff[y] = frame_line_offset(P, y);
  cudaError_t e = cudaMemcpyAsync(X + o_lines, loff.data(), sizeof(int64_t) * fh,
                                  cudaMemcpyHostToDevice, s);
  for (int t = 0; t < n && e == cudaSuccess; ++t) {
    e = cudaMemcpyAsync(X + o_src + sizeof(int16_t) * stride * t, chroma[t], sizeof(int16_t) * need,
                        cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && yc)
      e = cudaMemcpyAsync(X + o_pass + sizeof(int16_t) * stride * t, luma[t],
                          sizeof(int16_t) * need, cudaMemcpyHostToDevice, s);
  }
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D frames");
  mark(ctx, 0);  // device time of the kernels: from the split to the re-weave
  const float cpi = (P.white_level - P.blanking_level) / 100.0f;
  hvdg::FrameSplitArgs sp;
  sp.frames = reinterpret_cast<const int16_t*>(X + o_src);
  sp.frame_stride = stride;
  sp.line_off = reinterpret_cast<const int64_t*>(X + o_lines);
  sp.fw = fw;
  sp.fh = fh;
  sp.f1 = f1;
  sp.center = yc ? P.chroma_dc : P.blanking_level;
  sp.codes_per_ire = cpi;
  sp.fields = at<float>(ctx, L.o_raw);
  sp.field_stride = (b.pp.size() > 1 ? b.pp[1].raw_off - b.pp[0].raw_off : 0) / (int64_t)sizeof(float);
  hvdg::launch_frame_split(sp, n, s);
  S.launches += 1;
  st = stage_prepare(ctx, S, opt);
  if (st != HVDG_OK) return st;
  hvdg::launch_burst_amplitude(at<hvdg::PrepDesc>(ctx, L.o_prep), 2 * n, at<float>(ctx, L.o_amp), s);
  S.launches += 1;
  if (opt.do_solve) {
    hvdg::launch_aniso(at<FieldDesc>(ctx, L.o_fields), n, at<float2>(ctx, L.o_X0), s);
    S.launches += 1;
  }
  mark(ctx, 2);
  if (opt.do_solve) {
    const hvdg::SolverArgs sa = solver_args(ctx, S);
    e = hvdg::launch_solver(sa, solver_grid(ctx, L.total_units, opt.ctas_per_sm), s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "solver launch");
    S.launches += 1;
  }
  mark(ctx, 3);
  const FieldPlan& p0 = b.fp[0];
  hvdg::FrameOutArgs fo;
  fo.Y = at<float>(ctx, L.o_Y);
  fo.chi = at<float2>(ctx, L.o_X0);
  fo.S = at<float>(ctx, L.o_S);
  fo.plane_stride = n > 1 ? b.fp[1].px_off - p0.px_off : 0;
  fo.pitch = p0.pitch;
  fo.h = p0.h;
  fo.w = p0.w;
  fo.line_phasor = at<float4>(ctx, L.o_lineph);
  fo.col_phasor = at<float2>(ctx, L.o_colph);
  fo.amp = at<float>(ctx, L.o_amp);
  fo.passthrough = reinterpret_cast<const int16_t*>(X + (yc ? o_pass : o_src));
  fo.frame_stride = stride;
  fo.line_off = reinterpret_cast<const int64_t*>(X + o_lines);
  fo.fw = fw;
  fo.fh = fh;
  fo.f1 = f1;
  fo.fal = g.first_active_field_line;
  fo.a0 = P.active_video_start;
  fo.blank = P.blanking_level;
  fo.scale = cpi;
  fo.chroma_gain = cfg->chroma_gain;
  fo.nominal_burst = nominal_burst(g);
  fo.acc = cfg->acc ? 1 : 0;
  fo.yc = yc ? 1 : 0;
  fo.mono = (!yc && cfg->monochrome) ? 1 : 0;
  fo.luma = reinterpret_cast<int16_t*>(X + o_ol);
  fo.chroma = reinterpret_cast<int16_t*>(X + o_oc);
  fo.u = reinterpret_cast<double*>(X + o_ou);
  fo.v = reinterpret_cast<double*>(X + o_ov);
  hvdg::launch_frame_out(fo, n, s);
  S.launches += 1;
  mark(ctx, 4);
  e = cudaGetLastError();
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "frame kernels");
  for (int t = 0; t < n && e == cudaSuccess; ++t) {
    e = cudaMemcpyAsync(out[t].luma, fo.luma + npx * t, sizeof(int16_t) * npx,
                        cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out[t].chroma, fo.chroma + npx * t, sizeof(int16_t) * npx,
                          cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out[t].u_plane, fo.u + npx * t, sizeof(double) * npx,
                          cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out[t].v_plane, fo.v + npx * t, sizeof(double) * npx,
                          cudaMemcpyDeviceToHost, s);
  }
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "D2H frames");
  int flags[4] = {0, 0, 0, 0};
  float amp01[2] = {0.f, 0.f};
  std::vector<FieldCtl> ctl(n);
  e = cudaMemcpyAsync(flags, at<int>(ctx, L.o_flags), sizeof(flags), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(amp01, at<float>(ctx, L.o_amp), sizeof(amp01), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && diag)
    e = cudaMemcpyAsync(ctl.data(), at<FieldCtl>(ctx, L.o_ctl), sizeof(FieldCtl) * n,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "frame decode sync");
  if (diag) {
    diag->ms_total = elapsed(ctx, 0, 4);
    diag->ms_solver = elapsed(ctx, 2, 3);
    diag->ms_init = elapsed(ctx, 1, 2);
    float acc = 1.0f;
    if (cfg->acc) {
      const float m = 0.5f * (amp01[0] + amp01[1]);
      acc = std::min(std::max(nominal_burst(g) / std::max(m, 1.0f), 0.5f), 2.0f);
    }
    diag->acc_gain = acc;
    for (int i = 0; i < n; ++i) {
      if (opt.do_solve) diag->cg_iterations_run += ctl[i].cg_iters;
      if (opt.do_solve) diag->solver_pixel_iters += (int64_t)ctl[i].cg_iters * b.fp[i].h * b.fp[i].w;
      if (opt.do_solve)
        diag->solver_pixel_outers += (int64_t)b.fields[i].n_outer * b.fp[i].h * b.fp[i].w;
    }
    diag->kernel_launches = S.launches;
  }
  if (flags[1]) {
    ctx->last_error = "non-finite input samples";
    return HVDG_ERR_NONFINITE_INPUT;
  }
  if (flags[0]) {
    ctx->last_error = "device-side bounded wait expired in the solver";
    return HVDG_ERR_DEVICE_TIMEOUT;
  }
  return HVDG_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

static void settle(hvdg_ctx* ctx);


int hvdg_abi_version(void) { return HVDG_ABI_VERSION; }

const char* hvdg_status_string(hvdg_status s) {
  switch (s) {
    case HVDG_OK: return "HVDG_OK";
    case HVDG_ERR_BAD_ARGUMENT: return "HVDG_ERR_BAD_ARGUMENT";
    case HVDG_ERR_BAD_GEOMETRY: return "HVDG_ERR_BAD_GEOMETRY";
    case HVDG_ERR_NONFINITE_INPUT: return "HVDG_ERR_NONFINITE_INPUT";
    case HVDG_ERR_DEVICE_TIMEOUT: return "HVDG_ERR_DEVICE_TIMEOUT";
    case HVDG_ERR_CUDA: return "HVDG_ERR_CUDA";
    case HVDG_ERR_OUT_OF_MEMORY: return "HVDG_ERR_OUT_OF_MEMORY";
    case HVDG_ERR_UNSUPPORTED: return "HVDG_ERR_UNSUPPORTED";
    case HVDG_ERR_NO_DEVICE: return "HVDG_ERR_NO_DEVICE";
  }
  return "HVDG_ERR_UNKNOWN";
}

void hvdg_config_default(hvdg_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->lambda_c = 1.0f;
  c->chroma_aniso = 0.0f;
  c->charbonnier_eps = 0.5f;
  c->chroma_eps = 1.0f;
  c->structure_coupling = 0.25f;
  c->diag_prior = 0.0f;
  c->cg_iterations = 2;
  c->irls_outer = 4;
  c->cg_tol = 0.0f;
  c->fast = 1;
  c->parallel_across_fields = 1;
  c->symmetry_variant = 0;
  c->acc = 1;
  c->chroma_gain = 1.0f;
  c->monochrome = 0;
  c->chroma_phase_deg = 0.0f;
  c->field_order = 0;
  c->temporal_strength = 0.0f;
  c->bidirectional = 1;
  c->passes = 2;
  c->temporal_eps = 0.0f;
  c->nr_anchor = 1.0f;
  c->nr_eps = 0.0f;
  c->nr_radius = 2;
  c->mc_tile = 32;
  c->mc_search = 16;
  c->trajectory_fit = 1;
  c->extended_temporal = 1;
  c->coherence_gate = 0.6f;
  c->odd_gate_floor = 0.35f;
  c->output_fidelity = 1;
  c->psi_init = 0;
  c->selective_3d = 0;
  c->selective_max_area = 0.45f;
  c->me_mode = 0;
  c->me_block = 16;
  c->me_range = 16;
}

void hvdg_geometry_default(int standard, hvdg_geometry* g) {
  if (!g) return;
  std::memset(g, 0, sizeof(*g));
  if (standard == HVDG_STD_PAL) {
    g->field_width = 1135;
    g->field_height = 313;
    g->active_video_start = 185;
    g->active_video_end = 1107;
    g->colour_burst_start = 98;
    g->colour_burst_end = 138;
    g->first_active_field_line = 22;
    g->sample_rate = 4.0 * 4433618.75;
  } else {
    g->field_width = 910;
    g->field_height = 263;
    g->active_video_start = 134;
    g->active_video_end = 894;
    g->colour_burst_start = 78;
    g->colour_burst_end = 110;
    g->first_active_field_line = 21;
    g->sample_rate = 4.0 * 315.0e6 / 88.0;
  }
  g->last_active_field_line = 0;
  g->standard = standard;
  g->subcarrier_hz = 0.0;
}

hvdg_status hvdg_create(int device, hvdg_ctx** out) {
  if (!out) return HVDG_ERR_BAD_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0 || device < 0 || device >= n) {
    cudaGetLastError();
    return HVDG_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
    cudaGetLastError();
    return HVDG_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return HVDG_ERR_NO_DEVICE;
  }
  hvdg_ctx* ctx = new hvdg_ctx();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    cudaGetLastError();
    return HVDG_ERR_CUDA;
  }
  for (auto& ev : ctx->ev) cudaEventCreate(&ev);
  cudaEventCreateWithFlags(&ctx->ev_in, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->ev_done, cudaEventDisableTiming);
  if (cudaMallocHost(&ctx->flags_host, sizeof(int) * 4) != cudaSuccess) {
    cudaGetLastError();
    ctx->flags_host = nullptr;
    ctx->use_graphs = 0;
  }
  // one-time kernel attributes, outside any stream capture
  hvdg::solver_max_blocks_per_sm();
  hvdg::configure_prep_kernels();
  hvdg::configure_init_kernels();
  *out = ctx;
  return HVDG_OK;
}

void hvdg_destroy(hvdg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  for (auto& ev : ctx->ev) cudaEventDestroy(ev);
  if (ctx->ev_in) cudaEventDestroy(ctx->ev_in);
  if (ctx->ev_done) cudaEventDestroy(ctx->ev_done);
  if (ctx->flags_host) cudaFreeHost(ctx->flags_host);
  if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* hvdg_last_error(const hvdg_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

hvdg_status hvdg_set_batching(hvdg_ctx* ctx, int batched) {
  settle(ctx);
  if (!ctx) return HVDG_ERR_BAD_ARGUMENT;
  ctx->batched = batched ? 1 : 0;
  return HVDG_OK;
}

hvdg_status hvdg_set_tuning(hvdg_ctx* ctx, int band_rows, int ctas_per_sm) {
  settle(ctx);
  if (!ctx || band_rows < 0 || ctas_per_sm < 0) return HVDG_ERR_BAD_ARGUMENT;
  ctx->band_rows = band_rows;
  ctx->ctas_per_sm = ctas_per_sm;
  return HVDG_OK;
}

// Complete an asynchronous call still in flight on the context (every entry
// point that uses the context stream or the arena does this first); its
// status and diagnostics wait for hvdg_wait.
static void settle(hvdg_ctx* ctx) {
  if (!ctx || !ctx->pending) return;
  ctx->pending = false;
  std::memset(&ctx->pending_diag, 0, sizeof(ctx->pending_diag));
  const cudaError_t e = cudaEventSynchronize(ctx->ev_done);
  ctx->pending_status = e != cudaSuccess ? hvdg::cuda_fail(ctx, e, "asynchronous decode")
                                         : graph_result(ctx, &ctx->pending_diag);
  ctx->settled = true;
}

static hvdg_status decode_fields_impl(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                                      const hvdg_config* cfg, hvdg_field_out* out,
                                      hvdg_diag* diag, bool device_io, bool async = false) {
  if (!ctx) return HVDG_ERR_BAD_ARGUMENT;
  settle(ctx);
  hvdg_status st = validate_fields(fields, n, cfg, out);
  if (st != HVDG_OK) return st;
  if (n == 0) return HVDG_OK;
  cudaSetDevice(ctx->device);
  if (diag) std::memset(diag, 0, sizeof(*diag));
  RunOpts opt;
  opt.device_io = device_io;
  opt.async = async;
  if (ctx->batched) return run_batch(ctx, fields, n, cfg, out, diag, opt);
  for (int i = 0; i < n; ++i) {
    st = run_batch(ctx, fields + i, 1, cfg, out + i, diag, opt);
    if (st != HVDG_OK) return st;
  }
  return HVDG_OK;
}

hvdg_status hvdg_decode_fields(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                               const hvdg_config* cfg, hvdg_field_out* out, hvdg_diag* diag) {
  return decode_fields_impl(ctx, fields, n, cfg, out, diag, false);
}

hvdg_status hvdg_decode_fields_device(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                                      const hvdg_config* cfg, hvdg_field_out* out,
                                      hvdg_diag* diag) {
  return decode_fields_impl(ctx, fields, n, cfg, out, diag, true);
}

hvdg_status hvdg_decode_fields_device_async(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                                            const hvdg_config* cfg, hvdg_field_out* out,
                                            void* stream) {
  if (!ctx) return HVDG_ERR_BAD_ARGUMENT;
  settle(ctx);
  ctx->settled = false;
  cudaSetDevice(ctx->device);
  cudaStream_t us = static_cast<cudaStream_t>(stream);
  if (us) {
    // the decode reads what the caller's stream wrote before this call
    cudaError_t e = cudaEventRecord(ctx->ev_in, us);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_in, 0);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "order after the caller's stream");
  }
  hvdg_diag d;
  const hvdg_status st = decode_fields_impl(ctx, fields, n, cfg, out, &d, true, true);
  if (st != HVDG_OK) return st;
  if (!ctx->pending) {
    // completed synchronously (first call of a batch shape, or no graphs)
    ctx->pending_status = st;
    ctx->pending_diag = d;
    ctx->settled = true;
    return HVDG_OK;
  }
  if (us) {
    const cudaError_t e = cudaStreamWaitEvent(us, ctx->ev_done, 0);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "order the caller's stream after");
  }
  return HVDG_OK;
}

hvdg_status hvdg_wait(hvdg_ctx* ctx, hvdg_diag* diag) {
  if (!ctx) return HVDG_ERR_BAD_ARGUMENT;
  settle(ctx);
  if (!ctx->settled) {
    if (diag) std::memset(diag, 0, sizeof(*diag));
    return HVDG_OK;
  }
  ctx->settled = false;
  if (diag) *diag = ctx->pending_diag;
  return ctx->pending_status;
}

hvdg_status hvdg_decode_field_window(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                                     const hvdg_config* cfg, hvdg_field_out* out,
                                     hvdg_diag* diag) {
  settle(ctx);
  if (!ctx || !cfg) return HVDG_ERR_BAD_ARGUMENT;
  hvdg_status st = validate_fields(fields, n, cfg, out);
  if (st != HVDG_OK) return st;
  if (n == 0) return HVDG_OK;
  for (int i = 1; i < n; ++i)
    if (geom_key(*fields[i].geometry) != geom_key(*fields[0].geometry)) return HVDG_ERR_BAD_GEOMETRY;
  return decode_window_impl(ctx, fields, n, cfg, out, diag);
}

hvdg_status hvdg_burst_lockin(hvdg_ctx* ctx, const float* field_ire, const hvdg_geometry* g,
                              float* theta, int8_t* vswitch) {
  settle(ctx);
  if (!ctx || !field_ire || !g || !theta) return HVDG_ERR_BAD_ARGUMENT;
  if (uses_vswitch(*g) && !vswitch) return HVDG_ERR_BAD_ARGUMENT;
  return lockin_one(ctx, field_ire, g, theta, vswitch, nullptr);
}

hvdg_status hvdg_burst_amplitude(hvdg_ctx* ctx, const float* field_ire, const hvdg_geometry* g,
                                 float* amplitude_ire) {
  settle(ctx);
  if (!ctx || !field_ire || !g || !amplitude_ire) return HVDG_ERR_BAD_ARGUMENT;
  return lockin_one(ctx, field_ire, g, nullptr, nullptr, amplitude_ire);
}

hvdg_status hvdg_estimate_motion(hvdg_ctx* ctx, const float* y_ref, const float* y_cur, int h,
                                 int w, int tile, int search, int me_mode, float* dy, float* dx,
                                 float* confidence) {
  settle(ctx);
  if (!ctx || !y_ref || !y_cur || !dy || !dx || !confidence || h < 1 || w < 1 || tile < 1 ||
      search < 0 || me_mode < 0 || me_mode > 1)
    return HVDG_ERR_BAD_ARGUMENT;
  if (me_mode == 1) return estimate_motion_sad(ctx, y_ref, y_cur, h, w, tile, search, dy, dx,
                                               confidence);
  if (4 * tile > 4096 || search > 64) return HVDG_ERR_UNSUPPORTED;
  cudaSetDevice(ctx->device);
  const int pitch = (w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
  const int dpitch = pitch / 4;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const int ct = std::max(4, tile / 4);
  const int cth = (h / 4 + ct - 1) / ct, ctw = (w / 4 + ct - 1) / ct;
  const size_t plane = (size_t)h * pitch;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align_up(o + bytes, 256);
    return r;
  };
  const size_t o_f = take(sizeof(hvdg::MeField) * 2);
  const size_t o_p = take(sizeof(hvdg::MePair));
  const size_t o_l = take(sizeof(float) * 2 * plane);
  const size_t o_t = take(sizeof(float) * 2 * plane);
  const size_t o_b = take(sizeof(float) * 2 * plane);
  const size_t o_d = take(sizeof(float) * 2 * (size_t)(h / 4 + 1) * dpitch);
  const size_t nct = (size_t)std::max(1, cth * ctw), nt = (size_t)th * tw;
  const size_t o_cdy = take(sizeof(float) * nct), o_cdx = take(sizeof(float) * nct);
  size_t ot[8];
  for (int i = 0; i < 8; ++i) ot[i] = take(sizeof(float) * nt);
  hvdg_status st = ctx->arena.reserve(o, ctx->stream);
  if (st != HVDG_OK) return st;
  ctx->epoch += 1;
  char* base = static_cast<char*>(ctx->arena.base);
  hvdg::MeField mf[2];
  for (int i = 0; i < 2; ++i) {
    mf[i].h = h;
    mf[i].w = w;
    mf[i].pitch = pitch;
    mf[i].dpitch = dpitch;
    mf[i].y_off = mf[i].t_off = mf[i].b_off = (int64_t)i * plane;
    mf[i].d_off = (int64_t)i * (h / 4 + 1) * dpitch;
  }
  hvdg::MePair pr{0, 1};
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(base + o_f, mf, sizeof(mf), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_p, &pr, sizeof(pr), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(base + o_l, sizeof(float) * pitch, y_ref, sizeof(float) * w,
                          sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(base + o_l + sizeof(float) * plane, sizeof(float) * pitch, y_cur,
                          sizeof(float) * w, sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D motion inputs");
  hvdg::MeArgs a;
  a.tile = tile;
  a.search = search;
  a.coarse_off = (int)nct;
  a.tiles_off = (int)nt;
  hvdg::MeBuffers mb;
  mb.luma = reinterpret_cast<const float*>(base + o_l);
  mb.tmp = reinterpret_cast<float*>(base + o_t);
  mb.blur = reinterpret_cast<float*>(base + o_b);
  mb.dec = reinterpret_cast<float*>(base + o_d);
  mb.cdy = reinterpret_cast<float*>(base + o_cdy);
  mb.cdx = reinterpret_cast<float*>(base + o_cdx);
  mb.mdy = reinterpret_cast<float*>(base + ot[0]);
  mb.mdx = reinterpret_cast<float*>(base + ot[1]);
  mb.sdy = reinterpret_cast<float*>(base + ot[2]);
  mb.sdx = reinterpret_cast<float*>(base + ot[3]);
  mb.best = reinterpret_cast<float*>(base + ot[4]);
  mb.dy = reinterpret_cast<float*>(base + ot[5]);
  mb.dx = reinterpret_cast<float*>(base + ot[6]);
  mb.conf = reinterpret_cast<float*>(base + ot[7]);
  hvdg::launch_motion(reinterpret_cast<const hvdg::MeField*>(base + o_f), 2, h, w,
                      reinterpret_cast<const hvdg::MePair*>(base + o_p), 1, a, mb, s);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, mb.dy, sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, mb.dx, sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(confidence, mb.conf, sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "motion estimation");
  return HVDG_OK;
}

hvdg_status hvdg_set_debug_dir(hvdg_ctx* ctx, const char* dir) {
  if (!ctx) return HVDG_ERR_BAD_ARGUMENT;
  ctx->debug_dir = dir ? dir : "";
  return HVDG_OK;
}

hvdg_status hvdg_decode_frame_sequence_window(hvdg_ctx* ctx, const int16_t* const* frames,
                                              int n_frames, int core_begin, int core_end,
                                              const hvdg_frame_params* fp, const hvdg_config* cfg,
                                              hvdg_yc_frame* out, hvdg_diag* diag) {
  return hvdg_decode_frame_sequence_window_at(ctx, frames, n_frames, core_begin, core_end, 0, fp,
                                              cfg, out, diag);
}

hvdg_status hvdg_decode_frame_sequence_window_at(hvdg_ctx* ctx, const int16_t* const* frames,
                                                 int n_frames, int core_begin, int core_end,
                                                 int64_t base_frame_id,
                                                 const hvdg_frame_params* fp,
                                                 const hvdg_config* cfg, hvdg_yc_frame* out,
                                                 hvdg_diag* diag) {
  settle(ctx);
  if (!ctx || !fp || !cfg) return HVDG_ERR_BAD_ARGUMENT;
  // the reference returns an empty vector for these windows (frame_bridge.cpp:728-731)
  if (n_frames <= 0 || !frames || core_begin < 0 || core_end > n_frames || core_begin >= core_end)
    return HVDG_ERR_BAD_ARGUMENT;
  if (!out) return HVDG_ERR_BAD_ARGUMENT;
  for (int t = 0; t < n_frames; ++t)
    if (!frames[t]) return HVDG_ERR_BAD_ARGUMENT;
  for (int t = 0; t < core_end - core_begin; ++t)
    if (!out[t].luma || !out[t].chroma || !out[t].u_plane || !out[t].v_plane)
      return HVDG_ERR_BAD_ARGUMENT;
  const hvdg_frame_params& P = *fp;
  if (P.frame_width < 1 || P.frame_height < 2 || P.field1_lines < 1 ||
      P.field1_lines > P.frame_height || !(P.white_level != P.blanking_level))
    return HVDG_ERR_BAD_GEOMETRY;
  const hvdg_geometry g = geometry_from_params(P);
  hvdg_status st = check_geometry(&g);
  if (st != HVDG_OK) return st;
  const int fw = P.frame_width, fh = P.frame_height, f1 = P.field1_lines;
  const float scale = (P.white_level - P.blanking_level) / 100.0f;
  // ---- de-weave + field-order vote ----
  const int nfield = 2 * n_frames;
  std::vector<std::vector<float>> ire(nfield, std::vector<float>((size_t)f1 * fw));
  for (int t = 0; t < n_frames; ++t)
    split_frame_fields(frames[t], P, ire[2 * t].data(), ire[2 * t + 1].data());
  bool f1_bottom = cfg->field_order == 2;
  if (cfg->field_order == 0) {
    int vote = 0;
    for (int t = 0; t < n_frames; ++t)
      vote += detect_field_parity(ire[2 * t].data(), ire[2 * t + 1].data(), P, g);
    f1_bottom = vote < 0;
  }
  const int p_first = f1_bottom ? 1 : 0;
  // ---- window decode (burst amplitudes measured on the same upload) ----
  const int h = last_active_line(g) - g.first_active_field_line;
  const int w = g.active_video_end - g.active_video_start;
  std::vector<hvdg_field_in> fi(nfield);
  std::vector<hvdg_field_out> fo(nfield);
  std::vector<std::vector<float>> Yd(nfield, std::vector<float>((size_t)h * w));
  std::vector<std::vector<float>> Cd(nfield, std::vector<float>((size_t)h * w * 2));
  std::vector<std::vector<float>> th(nfield, std::vector<float>(f1));
  std::vector<std::vector<int8_t>> vs(nfield, std::vector<int8_t>(f1));
  for (int j = 0; j < nfield; ++j) {
    std::memset(&fi[j], 0, sizeof(fi[j]));
    fi[j].samples = ire[j].data();
    fi[j].sample_type = HVDG_SAMPLES_F32_IRE;
    fi[j].parity = (j % 2 == 0) ? p_first : 1 - p_first;
    fi[j].geometry = &g;
    fi[j].irls_outer = 0;
    fi[j].cg_iterations = -1;
    fo[j].luma = Yd[j].data();
    fo[j].chroma = Cd[j].data();
    fo[j].theta = th[j].data();
    fo[j].vswitch = vs[j].data();
  }
  std::vector<float> amps(nfield, 0.0f);
  RunOpts opt;
  opt.amp_out = amps.data();
  hvdg_diag local;
  hvdg_diag* dg = diag ? diag : &local;
  if (cfg->selective_3d && cfg->cg_iterations > 0 && cfg->temporal_strength >= 0.0f) {
    // frame_bridge.cpp:800-802: the 2-D base, then the ambiguous boxes in 3-D
    hvdg_config c2d = *cfg;
    c2d.temporal_strength = -1.0f;
    st = decode_window_impl(ctx, fi.data(), nfield, &c2d, fo.data(), dg, opt);
    if (st != HVDG_OK) return st;
    st = decode_selective_boxes(ctx, fi, g, cfg, Yd, Cd);
  } else {
    st = decode_window_impl(ctx, fi.data(), nfield, cfg, fo.data(), dg, opt);
  }
  if (st != HVDG_OK) return st;
  float acc_gain = 1.0f;
  if (cfg->acc) {
    std::vector<float> a = amps;
    const size_t k = a.size() / 2;
    std::nth_element(a.begin(), a.begin() + k, a.end());
    acc_gain = std::min(std::max(nominal_burst(g) / std::max(a[k], 1.0f), 0.5f), 2.0f);
  }
  const float gain = cfg->chroma_gain * acc_gain;
  dg->acc_gain = acc_gain;
  // ---- weave core frames by true parity + 10-bit requantisation ----
  const int fal = g.first_active_field_line, a0 = P.active_video_start;
  const double w0 = phase_per_sample(g);
  const bool vsw = uses_vswitch(g);
  std::vector<float2> colp(w);
  for (int x = 0; x < w; ++x) {
    const int smp = g.active_video_start + x;
    if (g.subcarrier_hz <= 0.0) {
      static const float2 q[4] = {{1.f, 0.f}, {0.f, 1.f}, {-1.f, 0.f}, {0.f, -1.f}};
      colp[x] = q[smp & 3];
    } else {
      colp[x] = make_float2((float)std::cos(w0 * smp), (float)std::sin(w0 * smp));
    }
  }
  if (!ctx->debug_dir.empty()) {
    // diagnostic maps (frame_bridge.cpp:807-865): the per-call decision log
    // and, per core frame, the woven residual-chroma-in-luma map
    std::vector<std::vector<float2>> car(nfield);
    for (int j = 0; j < nfield; ++j) {
      car[j].resize((size_t)h * w);
      for (int y = 0; y < h; ++y) {
        const double thv = (double)th[j][fal + y];
        const float2 Lc = make_float2((float)std::cos(thv), (float)std::sin(thv));
        const bool sw = vsw && vs[j][fal + y] < 0;
        for (int x = 0; x < w; ++x) {
          float cr = Lc.x * colp[x].x - Lc.y * colp[x].y;
          const float ci = Lc.x * colp[x].y + Lc.y * colp[x].x;
          if (sw) cr = -cr;
          car[j][(size_t)y * w + x] = make_float2(cr, ci);
        }
      }
    }
    std::vector<int> parity(nfield);
    for (int j = 0; j < nfield; ++j) parity[j] = fi[j].parity;
    write_debug_maps(ctx->debug_dir, base_frame_id, core_begin, core_end, f1_bottom, *dg, acc_gain,
                     Yd, car, parity, h, w);
  }
  for (int t = core_begin; t < core_end; ++t) {
    hvdg_yc_frame& yc = out[t - core_begin];
    const size_t sz = (size_t)fw * fh;
    std::fill(yc.chroma, yc.chroma + sz, (int16_t)0);
    std::fill(yc.u_plane, yc.u_plane + sz, 0.0);
    std::fill(yc.v_plane, yc.v_plane + sz, 0.0);
    for (int line = 0; line < fh; ++line) {
      const int64_t src = frame_line_offset(P, line);
      std::copy(frames[t] + src, frames[t] + src + fw, yc.luma + (size_t)line * fw);
    }
    const int j0 = 2 * t, j1 = j0 + 1;
    int p0 = fi[j0].parity, p1 = fi[j1].parity;
    if (p0 == p1) {
      p0 = 0;
      p1 = 1;
    }
    for (int r = 0; r < 2 * h; ++r) {
      const bool row_even = (r % 2) == 0;
      const bool use_first = (r % 2) == p0;
      const int j = use_first ? j0 : j1;
      const int fl = r / 2;
      const int flat_line = row_even ? (fal + fl) : (f1 + fal + fl);
      if (flat_line < 0 || flat_line >= fh) continue;
      const double thv = (double)th[j][fal + fl];
      const float2 Lc = make_float2((float)std::cos(thv), (float)std::sin(thv));
      const bool sw = vsw && vs[j][fal + fl] < 0;
      for (int c = 0; c < w; ++c) {
        const int flat_col = a0 + c;
        if (flat_col < 0 || flat_col >= fw) continue;
        const size_t idx = (size_t)flat_line * fw + flat_col;
        const float y_ire = Yd[j][(size_t)fl * w + c];
        float cr = Cd[j][2 * ((size_t)fl * w + c)], ci = Cd[j][2 * ((size_t)fl * w + c) + 1];
        if (cfg->monochrome) {
          cr = 0.0f;
          ci = 0.0f;
        }
        float car_r = Lc.x * colp[c].x - Lc.y * colp[c].y;
        const float car_i = Lc.x * colp[c].y + Lc.y * colp[c].x;
        if (sw) car_r = -car_r;
        yc.luma[idx] = clamp_u10(P.blanking_level + y_ire * scale);
        yc.chroma[idx] = clamp_s10((cr * car_r - ci * car_i) * scale);
        yc.v_plane[idx] = gain * (double)cr * scale;
        yc.u_plane[idx] = gain * (double)(-ci) * scale;
      }
    }
  }
  return HVDG_OK;
}

hvdg_status hvdg_decode_frame_buffer(hvdg_ctx* ctx, const int16_t* frame,
                                     const hvdg_frame_params* fp, const hvdg_config* cfg,
                                     hvdg_yc_frame* out) {
  settle(ctx);
  if (!frame || !out) return HVDG_ERR_BAD_ARGUMENT;
  return decode_woven_frames(ctx, &frame, nullptr, 1, fp, cfg, out, nullptr, false);
}

hvdg_status hvdg_decode_frame_buffers(hvdg_ctx* ctx, const int16_t* const* frames, int n_frames,
                                      const hvdg_frame_params* fp, const hvdg_config* cfg,
                                      hvdg_yc_frame* out, hvdg_diag* diag) {
  settle(ctx);
  return decode_woven_frames(ctx, frames, nullptr, n_frames, fp, cfg, out, diag, false);
}

hvdg_status hvdg_decode_yc_frame_buffer(hvdg_ctx* ctx, const int16_t* luma, const int16_t* chroma,
                                        const hvdg_frame_params* fp, const hvdg_config* cfg,
                                        hvdg_yc_frame* out) {
  settle(ctx);
  if (!luma || !chroma || !out) return HVDG_ERR_BAD_ARGUMENT;
  return decode_woven_frames(ctx, &chroma, &luma, 1, fp, cfg, out, nullptr, true);
}

hvdg_status hvdg_decode_yc_frame_buffers(hvdg_ctx* ctx, const int16_t* const* luma,
                                         const int16_t* const* chroma, int n_frames,
                                         const hvdg_frame_params* fp, const hvdg_config* cfg,
                                         hvdg_yc_frame* out, hvdg_diag* diag) {
  settle(ctx);
  return decode_woven_frames(ctx, chroma, luma, n_frames, fp, cfg, out, diag, true);
}

hvdg_status hvdg_ambiguous_boxes(const float* luma, const float* chroma, int h, int w,
                                 float max_area, int32_t* boxes, int max_boxes, int* n_boxes) {
  if (!luma || !chroma || !n_boxes || h < 1 || w < 1 || max_boxes < 0 ||
      (max_boxes > 0 && !boxes))
    return HVDG_ERR_BAD_ARGUMENT;
  const std::vector<SelBox> b = ambiguous_boxes(luma, chroma, h, w, max_area);
  if (!b.empty() && !b[0].valid) {
    *n_boxes = -1;
    return HVDG_OK;
  }
  *n_boxes = (int)b.size();
  for (int i = 0; i < (int)b.size() && i < max_boxes; ++i) {
    boxes[4 * i + 0] = b[i].fy0;
    boxes[4 * i + 1] = b[i].fy1;
    boxes[4 * i + 2] = b[i].x0;
    boxes[4 * i + 3] = b[i].x1;
  }
  return HVDG_OK;
}

hvdg_status hvdg_drizzle_frame(hvdg_ctx* ctx, const float* const* luma, const float* const* chroma,
                               const int32_t* parities, int n, int j0, int h, int w,
                               const hvdg_config* cfg, int scale, float* out_luma,
                               float* out_chroma) {
  settle(ctx);
  if (!ctx || !luma || !chroma || !parities || !cfg || !out_luma || !out_chroma || n < 2 ||
      j0 < 0 || j0 + 1 >= n || h < 1 || w < 1 || scale < 1 || cfg->mc_tile < 1 ||
      cfg->mc_search < 0 || cfg->nr_radius < 0)
    return HVDG_ERR_BAD_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (!luma[i] || !chroma[i]) return HVDG_ERR_BAD_ARGUMENT;
  const int tile = cfg->mc_tile, search = cfg->mc_search;
  if (4 * tile > 4096 || search > 64) return HVDG_ERR_UNSUPPORTED;
  cudaSetDevice(ctx->device);
  // pairs (sequence.cpp:300-310): for each target jt in {j0, j0 + 1}, the
  // sources k within 2 nr_radius fields, the sibling skipped, the target
  // itself with zero motion and confidence 1
  std::vector<hvdg::MePair> mp;
  std::vector<hvdg::DrizzlePair> dp;
  for (int jt = j0; jt <= j0 + 1; ++jt)
    for (int k = std::max(0, j0 - 2 * cfg->nr_radius);
         k < std::min(n, j0 + 2 + 2 * cfg->nr_radius); ++k) {
      if ((k == j0 || k == j0 + 1) && k != jt) continue;
      hvdg::DrizzlePair d{k, jt, -1, 0};
      if (k != jt) {
        d.me = (int)mp.size();
        mp.push_back(hvdg::MePair{k, jt});
      }
      dp.push_back(d);
    }
  const int P = (int)mp.size();
  const int pitch = (w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
  const int dpitch = pitch / 4;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const int ct = std::max(4, tile / 4);
  const int cth = (h / 4 + ct - 1) / ct, ctw = (w / 4 + ct - 1) / ct;
  const size_t plane = (size_t)h * pitch;
  const int HF = 2 * h * scale;
  const size_t fine = (size_t)HF * w;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align_up(o + bytes, 256);
    return r;
  };
  const size_t o_f = take(sizeof(hvdg::MeField) * n);
  const size_t o_p = take(sizeof(hvdg::MePair) * std::max(P, 1));
  const size_t o_dp = take(sizeof(hvdg::DrizzlePair) * dp.size());
  const size_t o_par = take(sizeof(int) * n);
  const size_t o_l = take(sizeof(float) * n * plane);
  const size_t o_c = take(sizeof(float2) * n * plane);
  const size_t o_t = take(sizeof(float) * n * plane);
  const size_t o_b = take(sizeof(float) * n * plane);
  const size_t o_d = take(sizeof(float) * n * (size_t)(h / 4 + 1) * dpitch);
  const size_t nct = (size_t)std::max(1, cth * ctw), nt = (size_t)th * tw;
  const size_t o_cdy = take(sizeof(float) * nct * std::max(P, 1));
  const size_t o_cdx = take(sizeof(float) * nct * std::max(P, 1));
  size_t ot[10];
  for (int i = 0; i < 10; ++i) ot[i] = take(sizeof(float) * nt * std::max(P, 1));
  const size_t o_acc = take(sizeof(float) * 4 * fine);
  const size_t o_oy = take(sizeof(float) * fine);
  const size_t o_oc = take(sizeof(float2) * fine);
  hvdg_status st = ctx->arena.reserve(o, ctx->stream);
  if (st != HVDG_OK) return st;
  ctx->epoch += 1;
  cudaGetLastError();
  char* base = static_cast<char*>(ctx->arena.base);
  std::vector<hvdg::MeField> mf(n);
  for (int i = 0; i < n; ++i) {
    mf[i].h = h;
    mf[i].w = w;
    mf[i].pitch = pitch;
    mf[i].dpitch = dpitch;
    mf[i].y_off = mf[i].t_off = mf[i].b_off = (int64_t)i * plane;
    mf[i].d_off = (int64_t)i * (h / 4 + 1) * dpitch;
  }
  std::vector<int> par(parities, parities + n);
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(base + o_f, mf.data(), sizeof(hvdg::MeField) * n,
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && P > 0)
    e = cudaMemcpyAsync(base + o_p, mp.data(), sizeof(hvdg::MePair) * P, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + o_dp, dp.data(), sizeof(hvdg::DrizzlePair) * dp.size(),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + o_par, par.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = cudaMemcpy2DAsync(base + o_l + sizeof(float) * plane * i, sizeof(float) * pitch, luma[i],
                          sizeof(float) * w, sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(base + o_c + sizeof(float2) * plane * i, sizeof(float2) * pitch,
                            chroma[i], sizeof(float2) * w, sizeof(float2) * w, h,
                            cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(base + o_acc, 0, sizeof(float) * 4 * fine, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D drizzle inputs");
  hvdg::MeArgs a;
  a.tile = tile;
  a.search = search;
  a.coarse_off = (int)nct;
  a.tiles_off = (int)nt;
  hvdg::MeBuffers mb;
  mb.luma = reinterpret_cast<const float*>(base + o_l);
  mb.tmp = reinterpret_cast<float*>(base + o_t);
  mb.blur = reinterpret_cast<float*>(base + o_b);
  mb.dec = reinterpret_cast<float*>(base + o_d);
  mb.cdy = reinterpret_cast<float*>(base + o_cdy);
  mb.cdx = reinterpret_cast<float*>(base + o_cdx);
  mb.mdy = reinterpret_cast<float*>(base + ot[0]);
  mb.mdx = reinterpret_cast<float*>(base + ot[1]);
  mb.sdy = reinterpret_cast<float*>(base + ot[2]);
  mb.sdx = reinterpret_cast<float*>(base + ot[3]);
  mb.best = reinterpret_cast<float*>(base + ot[4]);
  mb.dy = reinterpret_cast<float*>(base + ot[5]);
  mb.dx = reinterpret_cast<float*>(base + ot[6]);
  mb.conf = reinterpret_cast<float*>(base + ot[7]);
  const hvdg::MeField* d_f = reinterpret_cast<const hvdg::MeField*>(base + o_f);
  const hvdg::MePair* d_p = reinterpret_cast<const hvdg::MePair*>(base + o_p);
  float* snap_dy = reinterpret_cast<float*>(base + ot[8]);
  float* snap_dx = reinterpret_cast<float*>(base + ot[9]);
  if (P > 0) {
    hvdg::launch_motion(d_f, n, h, w, d_p, P, a, mb, s);
    hvdg::launch_vec_snap(d_f, d_p, P, h, w, a, mb.dy, mb.dx, snap_dy, snap_dx, s);
  }
  hvdg::DrizzleArgs da;
  da.Y = mb.luma;
  da.C = reinterpret_cast<const float2*>(base + o_c);
  da.parity = reinterpret_cast<const int*>(base + o_par);
  da.h = h;
  da.w = w;
  da.pitch = pitch;
  da.tile = tile;
  da.sdy = snap_dy;
  da.sdx = snap_dx;
  da.conf = mb.conf;
  da.tiles_off = (int)nt;
  da.eps_b = cfg->nr_eps > 0.0f ? cfg->nr_eps : 3.0f;
  da.scale = scale;
  da.j0 = j0;
  da.acc = reinterpret_cast<float*>(base + o_acc);
  da.out_y = reinterpret_cast<float*>(base + o_oy);
  da.out_c = reinterpret_cast<float2*>(base + o_oc);
  hvdg::launch_drizzle(reinterpret_cast<const hvdg::DrizzlePair*>(base + o_dp), (int)dp.size(), da,
                       s);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out_luma, da.out_y, sizeof(float) * fine, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out_chroma, da.out_c, sizeof(float2) * fine, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "drizzle");
  return HVDG_OK;
}

hvdg_status hvdg_holographic_init(hvdg_ctx* ctx, const float* s, const float* theta_active,
                                  const int8_t* vswitch_active, const hvdg_geometry* g,
                                  const hvdg_config* cfg, float* luma0, float* chi0) {
  settle(ctx);
  if (!ctx || !s || !theta_active || !g || !cfg || !luma0 || !chi0) return HVDG_ERR_BAD_ARGUMENT;
  hvdg_status st = check_geometry(g);
  if (st != HVDG_OK) return st;
  if (uses_vswitch(*g) && !vswitch_active) return HVDG_ERR_BAD_ARGUMENT;
  cudaSetDevice(ctx->device);
  hvdg_field_in fi;
  std::memset(&fi, 0, sizeof(fi));
  fi.samples = s;
  fi.sample_type = HVDG_SAMPLES_F32_IRE;
  fi.geometry = g;
  fi.irls_outer = 0;
  fi.cg_iterations = -1;
  hvdg_field_out fo;
  std::memset(&fo, 0, sizeof(fo));
  fo.luma = luma0;
  fo.chroma = chi0;
  RunOpts opt;
  opt.do_lockin = false;
  opt.do_solve = false;
  opt.s_in = s;
  opt.theta_in = theta_active;
  opt.vswitch_in = vswitch_active;
  return run_batch(ctx, &fi, 1, cfg, &fo, nullptr, opt);
}

hvdg_status hvdg_variational_refine(hvdg_ctx* ctx, const float* s, const float* theta_active,
                                    const int8_t* vswitch_active, const float* chi0,
                                    const hvdg_geometry* g, const hvdg_config* cfg, float* luma,
                                    float* chi) {
  settle(ctx);
  if (!ctx || !s || !theta_active || !chi0 || !g || !cfg || !luma || !chi)
    return HVDG_ERR_BAD_ARGUMENT;
  hvdg_status st = check_geometry(g);
  if (st != HVDG_OK) return st;
  if (cfg->diag_prior > 0.0f) return HVDG_ERR_UNSUPPORTED;
  if (uses_vswitch(*g) && !vswitch_active) return HVDG_ERR_BAD_ARGUMENT;
  cudaSetDevice(ctx->device);
  hvdg_field_in fi;
  std::memset(&fi, 0, sizeof(fi));
  fi.samples = s;
  fi.sample_type = HVDG_SAMPLES_F32_IRE;
  fi.geometry = g;
  fi.irls_outer = 0;
  fi.cg_iterations = -1;
  hvdg_field_out fo;
  std::memset(&fo, 0, sizeof(fo));
  fo.luma = luma;
  fo.chroma = chi;
  RunOpts opt;
  opt.do_lockin = false;
  opt.do_init = false;
  opt.s_in = s;
  opt.theta_in = theta_active;
  opt.vswitch_in = vswitch_active;
  opt.chi0_in = chi0;
  return run_batch(ctx, &fi, 1, cfg, &fo, nullptr, opt);
}

hvdg_status hvdg_decode_fields_adjoint(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                                       const hvdg_config* cfg, const float* const* y_bar,
                                       const float* const* chi_bar, float* const* samples_bar,
                                       double* scalar_bar, int adjoint_cg_iterations,
                                       hvdg_field_out* out, hvdg_diag* diag) {
  settle(ctx);
  if (!ctx || !cfg || n < 0 || (n > 0 && (!fields || !y_bar || !chi_bar || !samples_bar)) ||
      !scalar_bar)
    return HVDG_ERR_BAD_ARGUMENT;
  if (cfg->temporal_strength >= 0.0f) {
    ctx->last_error = "the adjoint covers the 2-D decode (temporal_strength < 0)";
    return HVDG_ERR_UNSUPPORTED;
  }
  if (cfg->diag_prior > 0.0f || cfg->symmetry_variant) return HVDG_ERR_UNSUPPORTED;
  for (int i = 0; i < n; ++i) {
    if (!fields[i].samples || !fields[i].geometry || !y_bar[i] || !chi_bar[i] || !samples_bar[i])
      return HVDG_ERR_BAD_ARGUMENT;
    const hvdg_status st = check_geometry(fields[i].geometry);
    if (st != HVDG_OK) return st;
  }
  cudaSetDevice(ctx->device);
  const int iters = adjoint_cg_iterations > 0 ? adjoint_cg_iterations : 300;
  for (int i = 0; i < 4; ++i) scalar_bar[i] = 0.0;
  for (int i = 0; i < n; ++i) {
    const hvdg_status st = decode_adjoint_field(ctx, fields[i], *cfg, y_bar[i], chi_bar[i],
                                                samples_bar[i], scalar_bar, iters,
                                                out ? &out[i] : nullptr, diag);
    if (st != HVDG_OK) return st;
  }
  return HVDG_OK;
}

}  // extern "C"
