// noalloc.cu -- holographic initialisation that allocates no device memory.
//
// Some hosts of this library cannot call cudaMalloc: a plugin running inside
// an application that owns the CUDA allocator (or forbids allocation after
// start-up), or a real-time path where an allocation may stall or fail at
// the wrong moment. hvdg_holographic_init_noalloc serves them: it runs the
// same init kernels as hvdg_holographic_init, with all of their scratch
// (pitched planes, row-filter buffers, kernel spectra, index tables) carved
// out of one fixed, file-scope device array instead of a context arena.
//
// The array is HVDG_NOALLOC_SCRATCH_BYTES (32 MiB). It is part of the
// module, so every GPU that loads this library holds it until the process
// exits, whether or not the entry point is ever called. This entry runs the
// init's register transforms only (row convolution 2048 points: at most
// 1024 active samples; column convolution 1024 points: at most 480 active
// lines; larger fields, which the context path takes through its
// shared-memory transforms, are refused here); those fields need at most
// ~24 MiB of it (kWorstLayout below), so the array's size never limits a
// field this entry takes. Host code cannot use the symbol itself as
// a device address; the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it for the
// life of the process, so that first call should come before any stream
// capture, and a cudaDeviceReset of that device between calls is not
// supported (the module may load again at another address). The
// array keeps the last call's contents; every region a call reads is written
// by that call first (the padded composite plane is cleared explicitly).
// All calls share the one array, so calls whose work overlaps on the GPU
// (several host threads, or several streams) race on it: serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "hvdg.h"
#include "hvdg_host.h"
#include "hvdg_internal.h"
#include "k_init.h"

namespace {

constexpr size_t kScratchBytes = HVDG_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
hvdg_status scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return HVDG_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return HVDG_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return HVDG_OK;
}

constexpr size_t up(size_t x) { return (x + 255) / 256 * 256; }

// The layout below at the largest plane this entry accepts (w <= 1024
// active samples, h + 2 pad <= 512 padded lines), tables included: the
// scratch array holds every accepted field.
constexpr size_t kMaxW = hvdg::kRowFft / 2, kMaxHp = (hvdg::kColFft + 1) / 2;
constexpr size_t kWorstLayout =
    up(sizeof(hvdg::FieldDesc)) + up(sizeof(hvdg::GeomDesc)) + up(16 * kMaxHp) +
    up(8 * kMaxW) + up(8 * (2 * hvdg::kRowFft + hvdg::kColFft)) + up(8 * hvdg::kRowFft) +
    up(8 * hvdg::kColFft) + up(4 * (kMaxHp + 1 + kMaxW + 1 + kMaxHp * kMaxW + 1)) + up(8) +
    2 * up(4 * kMaxHp * kMaxW) + 3 * up(8 * kMaxHp * kMaxW) + up(8 * 2 * kMaxHp * kMaxW);
static_assert(kWorstLayout <= kScratchBytes, "scratch array smaller than the largest field");

}  // namespace

extern "C" hvdg_status hvdg_holographic_init_noalloc(const float* s, const float* theta_active,
                                                     const int8_t* vswitch_active,
                                                     const hvdg_geometry* g, float* luma0,
                                                     float* chi0) {
  using hvdg::FieldDesc;
  using hvdg::GeomDesc;
  if (!s || !theta_active || !g || !luma0 || !chi0) return HVDG_ERR_BAD_ARGUMENT;
  // the same checks (and statuses) as hvdg_holographic_init, then the
  // init's own convolution lengths
  const hvdg_status gst = hvdg::check_field_geometry(g);
  if (gst != HVDG_OK) return gst;
  const bool vsw = g->standard == HVDG_STD_PAL || g->standard == HVDG_STD_PAL_M;
  if (vsw && !vswitch_active) return HVDG_ERR_BAD_ARGUMENT;
  const int lal = g->last_active_field_line != 0 ? g->last_active_field_line : g->field_height;
  const int h = lal - g->first_active_field_line;
  const int w = g->active_video_end - g->active_video_start;
  const int pad0 = h - 1 < hvdg::kInitPad ? h - 1 : hvdg::kInitPad;
  if (2 * w - 1 > hvdg::kRowFft || 2 * (h + 2 * pad0) - 1 > hvdg::kColFft) return HVDG_ERR_UNSUPPORTED;

  std::vector<float2> khat, colph, twr, twc;
  int hp = 0, pad = 0;
  hvdg::init_tables_for(*g, &khat, &colph, &twr, &twc, &hp, &pad);
  const int pitch = (w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
  const int cgroup = hvdg::init_col_group(hvdg::kColFft), bt = hvdg::init_blend_tile();
  const int ngroups = (w + cgroup - 1) / cgroup;
  const int ntiles = ((h + bt - 1) / bt) * ((w + bt - 1) / bt);

  // ---- layout inside the static array ----
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = up(o + bytes);
    return r;
  };
  const size_t o_field = take(sizeof(FieldDesc));
  const size_t o_geom = take(sizeof(GeomDesc));
  const size_t o_lph = take(sizeof(float4) * h);
  const size_t o_colph = take(sizeof(float2) * colph.size());
  const size_t o_khat = take(sizeof(float2) * khat.size());
  const size_t o_twr = take(sizeof(float2) * twr.size());
  const size_t o_twc = take(sizeof(float2) * twc.size());
  const size_t n_itab = (size_t)hp + 1 + ngroups + 1 + ntiles + 1;
  const size_t o_itab = take(sizeof(int) * n_itab);
  const size_t o_rbo = take(sizeof(int64_t));
  const size_t o_S = take(sizeof(float) * h * pitch);
  const size_t o_Y = take(sizeof(float) * h * pitch);
  const size_t o_c0 = take(sizeof(float2) * h * pitch);
  const size_t o_c1 = take(sizeof(float2) * h * pitch);
  const size_t o_c2 = take(sizeof(float2) * h * pitch);
  const size_t o_row = take(sizeof(float2) * 2 * (size_t)hp * pitch);
  if (o > kWorstLayout) return HVDG_ERR_UNSUPPORTED;  // cannot happen after the checks above

  void* vbase = nullptr;
  hvdg_status st = scratch_address(&vbase);
  if (st != HVDG_OK) return st;
  char* base = static_cast<char*>(vbase);

  // ---- host-side tables ----
  FieldDesc f;
  std::memset(&f, 0, sizeof(f));
  f.h = h;
  f.w = w;
  f.pitch = pitch;
  f.fh = g->field_height;
  f.fw = g->field_width;
  f.is_pal = vsw ? 1 : 0;
  GeomDesc gd;
  gd.w = w;
  gd.h = h;
  gd.hp = hp;
  gd.pad = pad;
  gd.khat_row_off = 0;
  gd.khat_col_off = 2 * hvdg::kRowFft;
  gd.row_m = hvdg::kRowFft;
  gd.col_m = hvdg::kColFft;
  gd.sym_row_chirp = gd.sym_row_hhat = gd.sym_col_chirp = gd.sym_col_hhat = -1;
  gd.sym_gx = gd.sym_gy = -1;
  std::vector<float4> lph(h);
  for (int y = 0; y < h; ++y) {
    const double th = (double)theta_active[y];
    const bool sw = vsw && vswitch_active[y] < 0;
    lph[y] = make_float4((float)std::cos(th), (float)std::sin(th), sw ? -1.f : 1.f, 0.f);
  }
  std::vector<int> itab;
  for (int y = 0; y < hp; ++y) itab.push_back(0);
  itab.push_back(0);
  for (int x = 0; x < ngroups; ++x) itab.push_back(0);
  itab.push_back(0);
  for (int t = 0; t < ntiles; ++t) itab.push_back(0);
  itab.push_back(0);
  const int64_t rbo = 0;

  auto h2d = [&](size_t off, const void* src, size_t bytes) {
    return cudaMemcpy(base + off, src, bytes, cudaMemcpyHostToDevice);
  };
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = h2d(o_field, &f, sizeof(f));
  if (e == cudaSuccess) e = h2d(o_geom, &gd, sizeof(gd));
  if (e == cudaSuccess) e = h2d(o_lph, lph.data(), sizeof(float4) * h);
  if (e == cudaSuccess) e = h2d(o_colph, colph.data(), sizeof(float2) * colph.size());
  if (e == cudaSuccess) e = h2d(o_khat, khat.data(), sizeof(float2) * khat.size());
  if (e == cudaSuccess) e = h2d(o_twr, twr.data(), sizeof(float2) * twr.size());
  if (e == cudaSuccess) e = h2d(o_twc, twc.data(), sizeof(float2) * twc.size());
  if (e == cudaSuccess) e = h2d(o_itab, itab.data(), sizeof(int) * itab.size());
  if (e == cudaSuccess) e = h2d(o_rbo, &rbo, sizeof(rbo));
  // the composite plane starts at zero (pitch padding), then the field
  if (e == cudaSuccess) e = cudaMemset(base + o_S, 0, sizeof(float) * h * pitch);
  if (e == cudaSuccess)
    e = cudaMemcpy2D(base + o_S, sizeof(float) * pitch, s, sizeof(float) * w, sizeof(float) * w,
                     h, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? HVDG_ERR_OUT_OF_MEMORY : HVDG_ERR_CUDA;
  }

  hvdg::InitArgs ia;
  ia.fields = reinterpret_cast<const FieldDesc*>(base + o_field);
  ia.geoms = reinterpret_cast<const GeomDesc*>(base + o_geom);
  ia.S = reinterpret_cast<const float*>(base + o_S);
  ia.line_phasor = reinterpret_cast<const float4*>(base + o_lph);
  ia.col_phasor = reinterpret_cast<const float2*>(base + o_colph);
  ia.khat = reinterpret_cast<const float2*>(base + o_khat);
  ia.tw_row = reinterpret_cast<const float2*>(base + o_twr);
  ia.tw_col = reinterpret_cast<const float2*>(base + o_twc);
  ia.rowbuf = reinterpret_cast<float2*>(base + o_row);
  ia.rowbuf_off = reinterpret_cast<const int64_t*>(base + o_rbo);
  ia.chi1 = reinterpret_cast<float2*>(base + o_c1);
  ia.chi2 = reinterpret_cast<float2*>(base + o_c2);
  ia.chi0 = reinterpret_cast<float2*>(base + o_c0);
  ia.Y = reinterpret_cast<float*>(base + o_Y);
  const int* it = reinterpret_cast<const int*>(base + o_itab);
  ia.prow_field = it;
  ia.prow_first = it + hp;
  ia.cgrp_field = it + hp + 1;
  ia.cgrp_first = it + hp + 1 + ngroups;
  ia.btile_field = it + hp + 1 + ngroups + 1;
  ia.btile_first = it + hp + 1 + ngroups + 1 + ntiles;
  hvdg::launch_init(ia, hp, ngroups, ntiles, 0);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpy2D(chi0, sizeof(float2) * w, base + o_c0, sizeof(float2) * pitch,
                     sizeof(float2) * w, h, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy2D(luma0, sizeof(float) * w, base + o_Y, sizeof(float) * pitch,
                     sizeof(float) * w, h, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return HVDG_ERR_CUDA;
  }
  return HVDG_OK;
}
