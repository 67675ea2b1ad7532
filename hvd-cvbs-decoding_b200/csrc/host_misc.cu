// host_misc.cu -- drivers behind the kernel-level entry points (lock-in of
// one field, integer-SAD motion of one pair) and the adjoint of the 2-D
// decode.
#include "pipeline.h"

namespace hvdg_pipe {

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

}  // namespace hvdg_pipe
