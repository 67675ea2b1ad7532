// frames.cu -- the frame bridges (hvd-core/src/frame_bridge.cpp): de-weave
// and field-order vote, the selective 3-D boxes, the diagnostic maps, and
// the woven-frame decode of DecodeFrameBuffer / DecodeYcFrameBuffer.
#include "pipeline.h"

namespace hvdg_pipe {

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
                                   const std::vector<float*>& Yd,
                                   const std::vector<float*>& Cd) {
  const int nf = (int)fi.size();
  const int h = last_active_line(g) - g.first_active_field_line;
  const int w = g.active_video_end - g.active_video_start;
  const std::vector<SelBox> boxes =
      ambiguous_boxes(Yd[0], Cd[0], h, w, cfg->selective_max_area);
  if (boxes.empty()) return HVDG_OK;
  std::vector<hvdg_field_out> fo(nf);
  if (!boxes[0].valid) {  // ambiguity everywhere: the full 3-D window
    for (int j = 0; j < nf; ++j) fo[j] = hvdg_field_out{Yd[j], Cd[j], nullptr, nullptr};
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
                      const std::vector<float*>& Y,
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

// The field-order vote's sample grid and levels (DetectFieldParity,
// frame_bridge.cpp:102-149; the host restatement detect_field_parity_t):
// field lines fal + 1, fal + 1 + ystep, ... below lal - 1, columns a0,
// a0 + 16, ... with 4 samples each. rows * cols == 0: no vote (0).
hvdg::FrameVoteArgs vote_grid(const hvdg_frame_params& P, const hvdg_geometry& g) {
  hvdg::FrameVoteArgs v;
  std::memset(&v, 0, sizeof(v));
  const int fal = g.first_active_field_line, lal = last_active_line(g);
  v.fh = P.frame_height;
  v.f1 = P.field1_lines;
  v.blank = P.blanking_level;
  v.codes_per_ire = (P.white_level - P.blanking_level) / 100.0f;
  v.r0 = fal + 1;
  v.ystep = std::max(1, (lal - fal) / 120);
  v.a0 = P.active_video_start;
  if (lal - fal >= 8 && P.active_video_end - P.active_video_start >= 32) {
    for (int r = fal + 1; r + 1 < lal; r += v.ystep) ++v.rows;
    for (int x = P.active_video_start; x + 4 <= P.active_video_end; x += 16) ++v.cols;
  }
  v.blocks = hvdg::frame_vote_blocks(v.rows * v.cols);
  return v;
}

// DetectFieldParity of n int16 frames on the device (k_frame_vote, the
// decode's own vote): +1 block 1 on top, -1 block 2 on top, 0 undecided.
hvdg_status detect_field_parity_frames(hvdg_ctx* ctx, const int16_t* const* frames, int n,
                                       const hvdg_frame_params* fp, int32_t* votes) {
  if (!ctx || !fp || n < 0 || (n > 0 && (!frames || !votes))) return HVDG_ERR_BAD_ARGUMENT;
  for (int t = 0; t < n; ++t)
    if (!frames[t]) return HVDG_ERR_BAD_ARGUMENT;
  const hvdg_frame_params& P = *fp;
  if (P.frame_width < 1 || P.frame_height < 2 || P.field1_lines < 1 ||
      P.field1_lines > P.frame_height || !(P.white_level != P.blanking_level))
    return HVDG_ERR_BAD_GEOMETRY;
  const hvdg_geometry g = geometry_from_params(P);
  hvdg_status st = check_geometry(&g);
  if (st != HVDG_OK) return st;
  if (n == 0) return HVDG_OK;
  hvdg::FrameVoteArgs va = vote_grid(P, g);
  if (va.rows * va.cols == 0) {
    for (int t = 0; t < n; ++t) votes[t] = 0;
    return HVDG_OK;
  }
  cudaSetDevice(ctx->device);
  const int fh = P.frame_height;
  const int64_t need = frame_line_offset(P, fh - 1) + P.frame_width;
  const int64_t stride = (int64_t)align_up((size_t)need, 128);
  const size_t o_lines = 0;
  const size_t o_src = align_up(sizeof(int64_t) * fh, 256);
  const size_t o_vote = align_up(o_src + sizeof(int16_t) * stride * n, 256);
  const size_t o_arrive = align_up(o_vote + sizeof(int) * n, 256);
  const size_t o_part = align_up(o_arrive + sizeof(int) * n, 256);
  const size_t total = align_up(o_part + sizeof(double) * 2 * va.blocks * n, 256);
  st = ctx->arena.reserve(total, ctx->stream);
  if (st != HVDG_OK) return st;
  ctx->epoch += 1;
  char* X = at<char>(ctx, 0);
  cudaStream_t s = ctx->stream;
  std::vector<int64_t> loff(fh);
  for (int y = 0; y < fh; ++y) loff[y] = frame_line_offset(P, y);
  cudaError_t e = cudaMemcpyAsync(X + o_lines, loff.data(), sizeof(int64_t) * fh,
                                  cudaMemcpyHostToDevice, s);
  for (int t = 0; t < n && e == cudaSuccess; ++t)
    e = cudaMemcpyAsync(X + o_src + sizeof(int16_t) * stride * t, frames[t],
                        sizeof(int16_t) * need, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "H2D frames");
  va.frames = reinterpret_cast<const int16_t*>(X + o_src);
  va.frame_stride = stride;
  va.line_off = reinterpret_cast<const int64_t*>(X + o_lines);
  va.vote = reinterpret_cast<int*>(X + o_vote);
  va.arrive = reinterpret_cast<int*>(X + o_arrive);
  va.partial = reinterpret_cast<double*>(X + o_part);
  hvdg::launch_frame_vote(va, n, s);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(votes, X + o_vote, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return hvdg::cuda_fail(ctx, e, "field-order vote");
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
  st = check_plane(w, 2 * lines, uses_vswitch(g));
  if (st != HVDG_OK) {
    ctx->last_error = "woven frame beyond the device-path limits";
    return st;
  }
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
  // field flagged first lands on the even woven rows (engine.cpp:55-57):
  // source slot 0 of a frame has parity 0 and the split fills it with the
  // block the order (or the device vote, k_frame_vote) puts on top.
  std::vector<hvdg_field_in> fi(2 * (size_t)n);
  for (int t = 0; t < n; ++t) {
    for (int k = 0; k < 2; ++k) {
      hvdg_field_in& f = fi[2 * t + k];
      std::memset(&f, 0, sizeof(f));
      f.samples = nullptr;
      f.sample_type = HVDG_SAMPLES_F32_IRE;
      f.parity = k;
      f.geometry = &g;
      f.irls_outer = 0;
      f.cg_iterations = -1;
    }
  }
  const hvdg::FrameVoteArgs vg = vote_grid(P, g);  // rows * cols == 0: undecided = top
  const bool device_vote = !yc && cfg->field_order == 0 && vg.rows * vg.cols > 0;
  const int split_order = device_vote ? 2 : (cfg->field_order == 2 ? 1 : 0);
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
  const size_t o_vote = align_up(o_ov + sizeof(double) * npx * n, 256);
  const size_t o_arrive = align_up(o_vote + sizeof(int) * n, 256);
  const size_t o_part = align_up(o_arrive + sizeof(int) * n, 256);
  const size_t xbytes = align_up(o_part + (device_vote ? sizeof(double) * 2 * vg.blocks * n : 0), 256);
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
  sp.order = split_order;
  sp.vote = reinterpret_cast<const int*>(X + o_vote);
  if (device_vote) {
    hvdg::FrameVoteArgs va = vg;
    va.frames = sp.frames;
    va.frame_stride = stride;
    va.line_off = sp.line_off;
    va.vote = reinterpret_cast<int*>(X + o_vote);
    va.arrive = reinterpret_cast<int*>(X + o_arrive);
    va.partial = reinterpret_cast<double*>(X + o_part);
    hvdg::launch_frame_vote(va, n, s);
    S.launches += 1;
  }
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

}  // namespace hvdg_pipe
