// window3d.cu -- the 3-D field window (DecodeFieldWindow with temporal
// terms, hvd-core/src/engine/sequence.cpp:423-1116): noise calibration,
// adaptive strength, motion, neighbour terms, colour-ordered solves, the
// anchored pass, on the batch staged by pipeline.cu.
#include "pipeline.h"

namespace hvdg_pipe {

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

// Adaptive temporal strength (sequence.cpp:526-646), the host's part: the
// median over the same-parity pairs of their ambiguities (measured on the
// device, k_amb_terms / k_amb_pairs), the noise floor removed, mapped to a
// strength.
float strength_from_pairs(const std::vector<float>& pair_amb, const std::vector<int>& pair_ok,
                          float nr_eps, float* amb_out) {
  std::vector<float> ambs;
  for (size_t j = 0; j < pair_amb.size(); ++j)
    if (pair_ok[j]) ambs.push_back(pair_amb[j]);
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
    // an automatic strength (0) is measured after the batch is planned; it
    // resolves above 0 on all but clean static content, so such a window is
    // planned for the temporal sweep too
    const int scan_stride = pal ? 4 : 2;
    const bool temporal =
        (cfg.temporal_strength > 0.0f || (cfg.temporal_strength == 0.0f && nf > scan_stride)) &&
        cfg.cg_iterations > 0;
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
  const size_t x_jp = take(sizeof(float4) * (cfg.diag_prior > 0.0f ? 11 : 10) * plane * nf * AP);
  const size_t x_jm2 = take(sizeof(float) * plane * nf * AP);
  const int jbx = (w + 31) / 32, jby = (h + 7) / 8;
  const size_t x_jpart = take(sizeof(double) * 5 * (size_t)jbx * jby * nf * AP);
  const size_t x_jctl = take(sizeof(hvdg::JointCtl) * nf + sizeof(hvdg::AnchorGroup) * nf +
                             sizeof(int) * nf + 256);
  const size_t x_ctab = take(sizeof(hvdg::TrajGroup) * 2 * nf + sizeof(hvdg::TrajPair) * max_pairs +
                             sizeof(int) * 2 * max_pairs + 256);
  size_t x_env[5];
  for (int i = 0; i < 5; ++i) x_env[i] = take(sizeof(float) * plane * nf);
  // adaptive strength: the demodulation terms of each same-parity pair at
  // rows 2, 5, ... < h - 2 and columns 4, 8, ... (x + 7 < w), and the pairs'
  // ambiguities
  const int amb_stride = pal ? 4 : 2;
  int amb_nyi = 0, amb_nx = 0;
  for (int y = 2; y < h - 2; y += 3) ++amb_nyi;
  for (int x = 4; x + 7 < w; x += 4) ++amb_nx;
  const int amb_pairs = std::max(0, nf - amb_stride);
  const size_t x_amb = take(sizeof(double) * (size_t)std::max(1, amb_pairs) * amb_nyi * amb_nx);
  const size_t x_ambo = take((sizeof(float) + sizeof(int)) * (size_t)std::max(1, amb_pairs) + 256);
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
  if (cfg.temporal_strength == 0.0f && cfg.cg_iterations > 0 && nf > amb_stride) {
    float* d_amb = at<float>(ctx, X(x_ambo));
    int* d_ambok = reinterpret_cast<int*>(align_up((size_t)(d_amb + amb_pairs), 16));
    hvdg::launch_amb_pairs(at<FieldDesc>(ctx, L.o_fields), amb_pairs, amb_stride, amb_nyi, amb_nx,
                           at<float>(ctx, L.o_S), at<float4>(ctx, L.o_lineph),
                           at<float2>(ctx, L.o_colph), cfg.nr_eps, at<double>(ctx, X(x_amb)),
                           d_amb, d_ambok, s);
    S.launches += 2;
    std::vector<float> pair_amb(amb_pairs);
    std::vector<int> pair_ok(amb_pairs);
    e = cudaMemcpyAsync(pair_amb.data(), d_amb, sizeof(float) * amb_pairs, cudaMemcpyDeviceToHost,
                        s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(pair_ok.data(), d_ambok, sizeof(int) * amb_pairs,
                          cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "adaptive strength");
    cfg.temporal_strength = strength_from_pairs(pair_amb, pair_ok, cfg.nr_eps, &amb);
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
          S.launches += 5;
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
      cudaMemsetAsync(at<char>(ctx, L.o_garrive), 0, sizeof(int) * L.total_units, s);
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
        ja.diag = cfg.diag_prior > 0.0f ? 1 : 0;
        ja.W2 = ja.diag ? jp + 10 * bp : nullptr;
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
                               const RunOpts& opt) {
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

}  // namespace hvdg_pipe
