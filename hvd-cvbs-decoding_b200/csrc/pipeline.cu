// pipeline.cu -- geometry checks and the per-geometry init tables (FP64 on
// the host, cached in the context), the device arena, batch planning, the
// staging of a batch into the arena (tables, samples, lock-in, crop, init)
// and the 2-D batch decode: one pass, a captured-graph replay, the tiling
// autotuner.
//
// Host orchestration replaces hvd-core's HvdEngine / DecodeFieldWindow
// driver (hvd-core/src/engine/engine.cpp:133-137,
// hvd-core/src/engine/sequence.cpp:229-281, 423-1116): instead of one OpenMP
// solve per field, a batch of fields is laid out in one device arena and
// every stage runs as one launch over all fields.
#include "pipeline.h"

namespace hvdg_pipe {

// Device-path limits of one solve plane of w x h (documented in
// include/hvdg.h): the longest row / column cyclic convolution of the init
// (kFftLong: up to 2048 active samples, 2048 padded lines) and the
// auto-aniso sample buffer.
hvdg_status check_plane(int w, int h, bool vsw) {
  const int pad = std::min(hvdg::kInitPad, h - 1);
  if (2 * w - 1 > hvdg::kFftLong || 2 * (h + 2 * pad) - 1 > hvdg::kFftLong)
    return HVDG_ERR_UNSUPPORTED;
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
  const hvdg_status st = check_plane(w, h, uses_vswitch(*g));
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

// The two crop variants of HolographicInit (holographic_init.cpp:236).
const double kVariants[2][2] = {{0.8, 120.0}, {1.8, 30.0}};

GeomTables make_geom_tables(const hvdg_geometry& g) {
  GeomTables t;
  t.w = g.active_video_end - g.active_video_start;
  t.h = last_active_line(g) - g.first_active_field_line;
  t.pad = std::min(hvdg::kInitPad, t.h > 1 ? t.h - 1 : 0);
  t.hp = t.h + 2 * t.pad;
  t.row_m = 2 * t.w - 1 <= hvdg::kRowFft ? hvdg::kRowFft : hvdg::kFftLong;
  t.col_m = 2 * t.hp - 1 <= hvdg::kColFft       ? hvdg::kColFft
            : 2 * t.hp - 1 <= hvdg::kColFftWide ? hvdg::kColFftWide
                                                : hvdg::kFftLong;
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
    for (const cd& c : kernel_spectrum(gx, t.row_m, 1.0))
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
  bluestein_tables(t.w, t.row_m, &t.sym);
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

// Solver band height when none is set: the tallest band (fewest halo rows)
// that still gives every resident warp a unit of the fields solved
// together; small batches (one field, one colour of a 3-D window) get short
// bands, so a phase is not bound by one warp walking 32 rows.
int auto_band_rows_hw(hvdg_ctx* ctx, const std::vector<std::pair<int, int>>& hw) {
  const int warps = ctx->sm_count * std::max(1, hvdg::solver_max_blocks_per_sm()) *
                    (hvdg::kSolverThreads / 32);
  // a lone field (or a few) never fills the resident warps; there a CG
  // phase costs a unit's fixed latency plus ~1 us per row, and 3-row bands
  // measured fastest (single NTSC field: 2-row 2.82, 3-row 2.29, 4-row
  // 2.44 ms of solver for 5 x 30)
  static const int cand[] = {32, 24, 16, 12, 8, 6, 4, 3};
  for (int band : cand) {
    int64_t units = 0;
    for (const auto& p : hw)
      units += (int64_t)((p.second + hvdg::kStrip - 1) / hvdg::kStrip) * ((p.first + band - 1) / band);
    if (units >= warps) return band;
  }
  return 3;
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
                       int band_rows, Batch& b, const hvdg_geometry* weave_geom) {
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
    gd.row_m = t.row_m;
    nkhat += 2 * t.row_m;
    gd.khat_col_off = nkhat;
    gd.col_m = t.col_m;
    nkhat += 2 * t.col_m;
    gd.sym_row_chirp = gd.sym_row_hhat = gd.sym_col_chirp = gd.sym_col_hhat = -1;
    gd.sym_gx = gd.sym_gy = -1;
    if (cfg->symmetry_variant) {
      gd.sym_row_chirp = nkhat;
      gd.sym_row_hhat = gd.sym_row_chirp + t.w;
      gd.sym_col_chirp = gd.sym_row_hhat + t.row_m;
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
    f.diag_prior = cfg->diag_prior > 0.0f ? cfg->diag_prior : 0.0f;
    f.mu_h = cfg->lambda_c;
    f.mu_v = cfg->lambda_c;
    f.mu_d = 0.0f;
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
  L.o_gpart = take(sizeof(double) * 5 * b.units.size());
  L.o_garrive = take(sizeof(int) * b.units.size());
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
  L.o_twl = take(sizeof(float2) * hvdg::kFftLong);
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
  L.has_diag = false;
  for (const FieldDesc& f : b.fields) L.has_diag |= f.diag_prior > 0.0f;
  L.o_W2 = L.has_diag ? take(sizeof(float2) * px) : 0;
  L.o_rowbuf = take(sizeof(float2) * rowb);
  L.total = o;
  return HVDG_OK;
}

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
  cudaMemsetAsync(at<char>(ctx, L.o_garrive), 0, sizeof(int) * L.total_units, s);
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
    static const std::vector<float2> twr = twiddles(hvdg::kRowFft), twc = twiddles(hvdg::kColFft),
                                     twl = twiddles(hvdg::kFftLong);
    put(L.o_twr, twr.data(), sizeof(float2) * twr.size());
    put(L.o_twc, twc.data(), sizeof(float2) * twc.size());
    put(L.o_twl, twl.data(), sizeof(float2) * twl.size());
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
  ia.tw_long = at<float2>(ctx, L.o_twl);
  for (const GeomDesc& gd : b.geoms) {
    ia.long_rows |= gd.row_m == hvdg::kFftLong;
    ia.long_cols |= gd.col_m == hvdg::kFftLong;
  }
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
  sa.garrive = at<int>(ctx, L.o_garrive);
  sa.gpartials = at<double>(ctx, L.o_gpart);
  sa.err = at<int>(ctx, L.o_flags);
  sa.phase_wait_limit = ctx->phase_wait_limit;
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
  sa.W2 = L.has_diag ? at<float2>(ctx, L.o_W2) : nullptr;
  sa.Y = at<float>(ctx, L.o_Y);
  sa.line_phasor = at<float4>(ctx, L.o_lineph);
  sa.col_phasor = at<float2>(ctx, L.o_colph);
  return sa;
}

int solver_grid(hvdg_ctx* ctx, int n_units, int ctas_override) {
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

hvdg_status run_batch_graph(hvdg_ctx* ctx, const hvdg_field_in* in, int n, const hvdg_config* cfg,
                            hvdg_field_out* out, hvdg_diag* diag, const RunOpts& opt) {
  std::string sig = batch_signature(in, n, cfg);
  // the effective tiling (a per-call override, else the context setting)
  const int band = opt.band_rows >= 0 ? opt.band_rows : ctx->band_rows;
  const int ctas = opt.ctas_per_sm >= 0 ? opt.ctas_per_sm : ctx->ctas_per_sm;
  sig += "|b" + std::to_string(band) + "c" + std::to_string(ctas) + "w" +
         std::to_string(ctx->phase_wait_limit);
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

}  // namespace hvdg_pipe

namespace hvdg {

using namespace hvdg_pipe;


hvdg_status check_field_geometry(const hvdg_geometry* g) { return check_geometry(g); }

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
