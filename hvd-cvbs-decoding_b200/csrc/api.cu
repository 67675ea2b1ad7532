// api.cu -- the C ABI (include/hvdg.h): context lifetime, the entry points
// and their argument checks, asynchronous completion; the pipelines live in
// pipeline.cu, window3d.cu, frames.cu and host_misc.cu.
#include "pipeline.h"

using namespace hvdg_pipe;


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

hvdg_status hvdg_set_device_wait_limit(hvdg_ctx* ctx, int64_t polls) {
  settle(ctx);
  if (!ctx) return HVDG_ERR_BAD_ARGUMENT;
  ctx->phase_wait_limit = polls > 0 ? (long long)polls : hvdg::kSpinLimit;
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

hvdg_status hvdg_verify_motion(hvdg_ctx* ctx, const float* y_ref, const float* y_cur, int h,
                               int w, int tile, const float* pdy, const float* pdx, float* dy,
                               float* dx, float* confidence) {
  settle(ctx);
  if (!ctx || !y_ref || !y_cur || !pdy || !pdx || !dy || !dx || !confidence || h < 1 || w < 1 ||
      tile < 1)
    return HVDG_ERR_BAD_ARGUMENT;
  if (tile > 4096) return HVDG_ERR_UNSUPPORTED;
  cudaSetDevice(ctx->device);
  const int pitch = (w + hvdg::kStrip - 1) / hvdg::kStrip * hvdg::kStrip;
  const int th = (h + tile - 1) / tile, tw = (w + tile - 1) / tile;
  const size_t plane = (size_t)h * pitch, nt = (size_t)th * tw;
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
  size_t ot[10];
  for (int i = 0; i < 10; ++i) ot[i] = take(sizeof(float) * nt);
  hvdg_status st = ctx->arena.reserve(o, ctx->stream);
  if (st != HVDG_OK) return st;
  ctx->epoch += 1;
  char* base = static_cast<char*>(ctx->arena.base);
  hvdg::MeField mf[2];
  std::memset(mf, 0, sizeof(mf));
  for (int i = 0; i < 2; ++i) {
    mf[i].h = h;
    mf[i].w = w;
    mf[i].pitch = pitch;
    mf[i].dpitch = pitch / 4;
    mf[i].y_off = mf[i].t_off = mf[i].b_off = (int64_t)i * plane;
  }
  hvdg::MePair pr;  // plane 0 holds y_cur, plane 1 y_ref
  pr.ref = 1;
  pr.cur = 0;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(base + o_f, mf, sizeof(mf), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_p, &pr, sizeof(pr), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(base + o_l, sizeof(float) * pitch, y_cur, sizeof(float) * w,
                          sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(base + o_l + sizeof(float) * plane, sizeof(float) * pitch, y_ref,
                          sizeof(float) * w, sizeof(float) * w, h, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + ot[8], pdy, sizeof(float) * nt, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + ot[9], pdx, sizeof(float) * nt, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D verify inputs");
  hvdg::MeArgs a;
  std::memset(&a, 0, sizeof(a));
  a.tile = tile;
  a.search = 0;
  a.coarse_off = 1;
  a.tiles_off = (int)nt;
  hvdg::MeBuffers mb;
  std::memset(&mb, 0, sizeof(mb));
  mb.luma = reinterpret_cast<const float*>(base + o_l);
  mb.tmp = reinterpret_cast<float*>(base + o_t);
  mb.blur = reinterpret_cast<float*>(base + o_b);
  auto P = [&](int i) { return reinterpret_cast<float*>(base + ot[i]); };
  const hvdg::MeField* d_f = reinterpret_cast<const hvdg::MeField*>(base + o_f);
  const hvdg::MePair* d_p = reinterpret_cast<const hvdg::MePair*>(base + o_p);
  hvdg::launch_motion_blur(d_f, 2, h, w, mb, s);
  hvdg::launch_traj_verify(d_f, d_p, 0, 1, nullptr, nullptr, nullptr, mb.blur, h, w, a, nullptr,
                           nullptr, P(0), P(1), P(2), P(3), P(4), s, P(8), P(9));
  hvdg::launch_me_confidence(d_f, d_p, 1, h, w, a, mb.blur, P(0), P(1), P(2), P(3), P(4), P(5),
                             P(6), P(7), s);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, P(5), sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, P(6), sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(confidence, P(7), sizeof(float) * nt, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "motion verification");
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
  // host planes in the context's page-locked staging area (the window's
  // uploads and downloads then run at the link's rate); pageable when it
  // cannot grow
  const int h = last_active_line(g) - g.first_active_field_line;
  const int w = g.active_video_end - g.active_video_start;
  // each plane 256-byte aligned; after the planes, the fields' burst
  // amplitudes (a page-locked target keeps their copy asynchronous)
  const size_t n_ire = align_up((size_t)f1 * fw, 64), n_y = align_up((size_t)h * w, 64);
  const size_t staging = (size_t)nfield * (n_ire + 3 * n_y) + align_up((size_t)nfield, 64);
  std::vector<float> pageable;
  float* stage = nullptr;
  if (ctx->pinned.reserve(sizeof(float) * staging) == HVDG_OK) {
    stage = static_cast<float*>(ctx->pinned.base);
  } else {
    pageable.resize(staging);
    stage = pageable.data();
  }
  std::vector<float*> ire(nfield), Yd(nfield), Cd(nfield);
  for (int j = 0; j < nfield; ++j) {
    ire[j] = stage + (size_t)j * n_ire;
    Yd[j] = stage + (size_t)nfield * n_ire + (size_t)j * n_y;
    Cd[j] = stage + (size_t)nfield * (n_ire + n_y) + (size_t)j * 2 * n_y;
  }
  std::vector<int> votes(n_frames, 0);
  const bool auto_order = cfg->field_order == 0;
  parallel_for(n_frames, [&](int t) {
    split_frame_fields(frames[t], P, ire[2 * t], ire[2 * t + 1]);
    if (auto_order) votes[t] = detect_field_parity(ire[2 * t], ire[2 * t + 1], P, g);
  });
  bool f1_bottom = cfg->field_order == 2;
  if (auto_order) {
    int vote = 0;
    for (int t = 0; t < n_frames; ++t) vote += votes[t];
    f1_bottom = vote < 0;
  }
  const int p_first = f1_bottom ? 1 : 0;
  // ---- window decode (burst amplitudes measured on the same upload) ----
  std::vector<hvdg_field_in> fi(nfield);
  std::vector<hvdg_field_out> fo(nfield);
  std::vector<std::vector<float>> th(nfield, std::vector<float>(f1));
  std::vector<std::vector<int8_t>> vs(nfield, std::vector<int8_t>(f1));
  for (int j = 0; j < nfield; ++j) {
    std::memset(&fi[j], 0, sizeof(fi[j]));
    fi[j].samples = ire[j];
    fi[j].sample_type = HVDG_SAMPLES_F32_IRE;
    fi[j].parity = (j % 2 == 0) ? p_first : 1 - p_first;
    fi[j].geometry = &g;
    fi[j].irls_outer = 0;
    fi[j].cg_iterations = -1;
    fo[j].luma = Yd[j];
    fo[j].chroma = Cd[j];
    fo[j].theta = th[j].data();
    fo[j].vswitch = vs[j].data();
  }
  float* amps = stage + (size_t)nfield * (n_ire + 3 * n_y);
  std::fill(amps, amps + nfield, 0.0f);
  RunOpts opt;
  opt.amp_out = amps;
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
    std::vector<float> a(amps, amps + nfield);
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
  // each core frame in kWeaveBands bands of frame lines, the bands on the
  // host threads: the caller's output pages are first touched (and the
  // planes filled) by many threads at once
  constexpr int kWeaveBands = 8;
  parallel_for((core_end - core_begin) * kWeaveBands, [&](int task) {
    const int ti = task / kWeaveBands, band = task % kWeaveBands;
    const int t = core_begin + ti;
    hvdg_yc_frame& yc = out[ti];
    const int l0 = (int)((int64_t)fh * band / kWeaveBands);
    const int l1 = (int)((int64_t)fh * (band + 1) / kWeaveBands);
    const size_t b0 = (size_t)l0 * fw, b1 = (size_t)l1 * fw;
    std::fill(yc.chroma + b0, yc.chroma + b1, (int16_t)0);
    std::fill(yc.u_plane + b0, yc.u_plane + b1, 0.0);
    std::fill(yc.v_plane + b0, yc.v_plane + b1, 0.0);
    for (int line = l0; line < l1; ++line) {
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
      if (flat_line < l0 || flat_line >= l1) continue;
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
  });
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

hvdg_status hvdg_detect_field_parity(hvdg_ctx* ctx, const int16_t* const* frames, int n_frames,
                                     const hvdg_frame_params* fp, int32_t* votes) {
  settle(ctx);
  return detect_field_parity_frames(ctx, frames, n_frames, fp, votes);
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
