// k_init.cu -- holographic initialisation (kernel b) and the auto chroma
// anisotropy (variational.cpp:130-196).
//
// Reference: HolographicInit (hvd-core/src/engine/holographic_init.cpp:200-317):
// demodulate S by conj(carrier), reflect-101 pad 16 rows, 2-D FFT, two
// separable Gaussian sideband crops {0.8 MHz, 120 c/ph} and {1.8 MHz, 30 c/ph},
// inverse FFT, crop, x2, edge-energy blend w = 1 / (BoxBlur_3(|Dx Y|+|Dy Y|) + 0.5).
//
// Because each crop mask is separable (gy[y] * gx[x]) the 2-D
// "FFT -> mask -> inverse FFT" equals a circular convolution along rows with
// k_x = IDFT_w(gx) followed by one along columns with k_y = IDFT_hp(gy). Each
// circular convolution of length n runs as a cyclic convolution of
// power-of-two length M >= 2n - 1 (rows: 2048; columns: 1024, or 2048 for
// woven frames) with the kernel's FFT precomputed on the host: a four-step
// FFT held in registers (32 values per lane, one warp per 1024 points),
// mask multiply in registers, inverse FFT, write. Rows and columns past
// those lengths (up to 2048 samples / padded lines) run at M = 4096 through
// a shared-memory FFT (k_init_rows_long, k_init_cols_long).
//   k_init_rows : one warp pair per padded row -> both row-filtered variants
//   k_init_cols : one warp (pair) per column -> chi_1, chi_2 (x2 folded in)
//   k_init_blend: edge-energy blend -> chi0, Y0
#include <cuda_runtime.h>

#include <cmath>

#include "hvdg_common.cuh"
#include "k_init.h"
#include "per_device.h"

namespace hvdg {

// ---- Stockham autosort FFT (radix 4, one radix-2 stage when needed) --------
// Length M (power of two). `tw` = exp(-2 pi i k / M), k in [0, M). Threads
// [tid, nt) of the cooperating group call it together; `sync` separates the
// stages. Returns the buffer (a or b) holding the result.
template <int M, bool INV, typename Sync>
__device__ __forceinline__ float2* fft_stockham(float2* a, float2* b,
                                                const float2* __restrict__ tw, int tid,
                                                int nt, Sync sync) {
  float2* src = a;
  float2* dst = b;
#pragma unroll 1
  for (int Ns = 1; Ns < M;) {
    const int R = ((M / Ns) % 4 == 0) ? 4 : 2;
    const int nb = M / R;
    const int st = M / (Ns * R);
    if (R == 4) {
      for (int j = tid; j < nb; j += nt) {
        const int k = j & (Ns - 1);
        float2 v0 = src[j], v1 = src[j + nb], v2 = src[j + 2 * nb], v3 = src[j + 3 * nb];
        if (k) {
          float2 w1 = __ldg(tw + k * st), w2 = __ldg(tw + 2 * k * st), w3 = __ldg(tw + 3 * k * st);
          if (INV) {
            w1.y = -w1.y;
            w2.y = -w2.y;
            w3.y = -w3.y;
          }
          v1 = cmul(v1, w1);
          v2 = cmul(v2, w2);
          v3 = cmul(v3, w3);
        }
        const float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = csub(v1, v3);
        const float2 t3r = INV ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);
        const int base = (j / Ns) * Ns * 4 + k;
        dst[base] = cadd(t0, t2);
        dst[base + Ns] = cadd(t1, t3r);
        dst[base + 2 * Ns] = csub(t0, t2);
        dst[base + 3 * Ns] = csub(t1, t3r);
      }
    } else {
      for (int j = tid; j < nb; j += nt) {
        const int k = j & (Ns - 1);
        float2 v0 = src[j], v1 = src[j + nb];
        if (k) {
          float2 w1 = __ldg(tw + k * st);
          if (INV) w1.y = -w1.y;
          v1 = cmul(v1, w1);
        }
        const int base = (j / Ns) * Ns * 2 + k;
        dst[base] = cadd(v0, v1);
        dst[base + Ns] = csub(v0, v1);
      }
    }
    sync();
    float2* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};
struct WarpSync {
  __device__ void operator()() const { __syncwarp(); }
};

__device__ __forceinline__ int mirror_row(int y, int h) {
  // reflect-101 (holographic_init.cpp:126-131)
  if (h <= 1) return 0;
  const int period = 2 * h - 2;
  y = ((y % period) + period) % period;
  return y < h ? y : period - y;
}

__device__ __forceinline__ float2 carrier_at(const InitArgs& a, const FieldDesc& f, int y,
                                             int x) {
  const float4 L = __ldg(a.line_phasor + f.line_off + y);
  const float2 P = __ldg(a.col_phasor + f.col_off + x);
  return carrier(make_float2(L.x, L.y), P, L.z);
}

// ---- columns ---------------------------------------------------------------
// grid = (column groups over all fields); block = 128; dynamic smem ~32 KiB;
// up to 170 registers, 3 CTAs per SM. The column length M of a geometry is
// 1024 (field planes: 2 hp - 1 <= 1024; 4 columns per CTA, one warp each) or
// 2048 (woven frames, hp up to 1024; 2 columns per CTA, two warps each).
// Each column's cyclic convolution runs in registers (col_conv_reg): a
// column of 1024 is a 32 x 32 four-step FFT -- 32-point FFTs along each
// lane's 32 values, twiddles, a transpose through
// the column's shared-memory slot, 32-point FFTs again -- and the inverse
// mirrors it back to natural order; a column of 2048 adds one radix-2 step
// (decimation in time forward, in frequency inverse) between the two warps.
constexpr int kColThreads = 128;
constexpr int kColGroup = 4;
constexpr int kColGroupWide = 2;
// Columns sit kColPad float2 apart beyond their length, so the 4 columns
// of a row in the coalesced fill and write-back alternate between the two
// halves of the shared-memory banks (2-way instead of 4-way conflicts).
constexpr int kColPad = 8;
constexpr int kColSmem =
    (kColGroup * (kColFft + kColPad) > kColGroupWide * (kColFftWide + kColPad)
         ? kColGroup * (kColFft + kColPad)
         : kColGroupWide * (kColFftWide + kColPad)) *
    (int)sizeof(float2);

struct PairSync {  // the 64 threads of one wide column (named barrier 1 + pair)
  int id;
  __device__ void operator()() const { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }
};

__host__ __device__ constexpr int brev5(int i) {
  return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// exp(-2 pi i k / 32), k < 16, and exp(-2 pi i m / 64), m < 32: twiddles
// read as constant-bank operands (no registers); filled from the host
// (configure_init_kernels).
__constant__ float2 c_tw32[16];
__constant__ float2 c_tw64[32];

// Keeps the compiler from hoisting the loads that follow above this point:
// the register FFT holds 32 complex values per lane, and loads of all the
// twiddles or spectrum values ahead of their use would not fit beside them.
__device__ __forceinline__ void load_fence() { asm volatile("" ::: "memory"); }

// v[j] *= exp(-+2 pi i lane j / 1024), j = 1..31 (INV: conjugate), each
// twiddle the product of two table values, lane (8 a) and lane b.
template <bool INV>
__device__ __forceinline__ void twiddle1024(float2 (&v)[32], const float2* __restrict__ tw,
                                            int lane) {
  float2 wb[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) wb[b] = __ldg(tw + ((lane * b) & 1023));
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    load_fence();
    const float2 wa = __ldg(tw + ((8 * a * lane) & 1023));
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int j = 8 * a + b;
      if (j == 0) continue;
      float2 w = a == 0 ? wb[b] : (b == 0 ? wa : cmul(wa, wb[b]));
      if (INV) w.y = -w.y;
      v[j] = cmul(v[j], w);
    }
  }
}

// 32-point DFT of one lane's registers (radix-2 decimation in time, natural
// order in and out; INV: conjugate twiddles, unnormalised).
template <bool INV>
__device__ __forceinline__ void fft32_reg(float2 (&v)[32], const float2* __restrict__ tw1024) {
  (void)tw1024;
  float2 a[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) a[i] = v[brev5(i)];
#pragma unroll
  for (int len = 2; len <= 32; len <<= 1) {
    const int half = len >> 1;
#pragma unroll
    for (int k = 0; k < half; ++k) {
      float2 w = make_float2(1.f, 0.f);
      if (k) {
        w = c_tw32[k * (32 / len)];
        if (INV) w.y = -w.y;
      }
#pragma unroll
      for (int i = 0; i < 32; i += len) {
        const float2 t = k ? cmul(a[i + k + half], w) : a[i + k + half];
        const float2 u = a[i + k];
        a[i + k] = cadd(u, t);
        a[i + k + half] = csub(u, t);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = a[i];
}

// 1024-point DFT by one warp. In: lane l holds x[l + 32 k] in v[k]. Out:
// lane j holds X[j + 32 m] in v[m]. scr: 1024 float2 of this warp's shared
// memory (the transpose, XOR-swizzled so no access has bank conflicts).
__device__ __forceinline__ void fft1024_fwd(float2 (&v)[32], float2* scr,
                                            const float2* __restrict__ tw, int lane) {
  fft32_reg<false>(v, tw);
  twiddle1024<false>(v, tw, lane);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 32; ++j) scr[j * 32 + (lane ^ j)] = v[j];
  __syncwarp();
#pragma unroll
  for (int l = 0; l < 32; ++l) v[l] = scr[lane * 32 + (l ^ lane)];
  __syncwarp();
  fft32_reg<false>(v, tw);
}

// The inverse (unnormalised): in, lane j holds Y[j + 32 m] in v[m]; out,
// lane l holds y[l + 32 k] in v[k].
__device__ __forceinline__ void fft1024_inv(float2 (&v)[32], float2* scr,
                                            const float2* __restrict__ tw, int lane) {
  fft32_reg<true>(v, tw);
  twiddle1024<true>(v, tw, lane);
  __syncwarp();
#pragma unroll
  for (int l = 0; l < 32; ++l) scr[l * 32 + (lane ^ l)] = v[l];
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = scr[lane * 32 + (j ^ lane)];
  __syncwarp();
  fft32_reg<true>(v, tw);
}

struct NoSync {
  __device__ void operator()() const { __syncwarp(); }
};

// Forward DFT of length M (1024 or 2048) held in registers. In: v[k] =
// x[(lane + 32 k) S + sub], S = M / 1024. Out: v[m] = X[sub 1024 + lane +
// 32 m]. buf: the M float2 of shared memory of this column (or row), which
// no thread of it reads any more. M = 1024: one warp (sub 0). M = 2048: two
// warps (sub 0 / 1, paired by `sync`), each taking one parity of the samples.
template <int M, typename Sync>
__device__ __forceinline__ void fft_reg_fwd(float2 (&v)[32], float2* buf,
                                            const float2* __restrict__ tw1024,
                                            const float2* __restrict__ tw2048, int sub, int lane,
                                            Sync sync) {
  constexpr int S = M / 1024;
  float2* scr = buf + sub * 1024;
  fft1024_fwd(v, scr, tw1024, lane);  // E (sub 0) / O (sub 1) of the parities
  if (S == 2) {
    // X[q] = E[q] + W^q O[q], X[q + 1024] = E[q] - W^q O[q], W = exp(-2 pi i / 2048)
    if (sub == 1) {
      // W^(lane + 32 m) = W^lane exp(-2 pi i m / 64)
      const float2 wl = __ldg(tw2048 + lane);
#pragma unroll
      for (int m = 0; m < 32; ++m) v[m] = cmul(v[m], cmul(wl, c_tw64[m]));
    }
    sync();
#pragma unroll
    for (int m = 0; m < 32; ++m) scr[lane + 32 * m] = v[m];
    sync();
    const float2* other = buf + (1 - sub) * 1024;
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      const float2 o = other[lane + 32 * m];
      v[m] = sub == 0 ? cadd(v[m], o) : csub(o, v[m]);
    }
    sync();
  }
}

// The inverse (unnormalised), from fft_reg_fwd's output layout back to its
// input layout; same buf and pairing.
template <int M, typename Sync>
__device__ __forceinline__ void fft_reg_inv(float2 (&v)[32], float2* buf,
                                            const float2* __restrict__ tw1024,
                                            const float2* __restrict__ tw2048, int sub, int lane,
                                            Sync sync) {
  constexpr int S = M / 1024;
  float2* scr = buf + sub * 1024;
  if (S == 2) {
    // even outputs from Y[q] + Y[q + 1024], odd from (Y[q] - Y[q + 1024]) W^-q
#pragma unroll
    for (int m = 0; m < 32; ++m) scr[lane + 32 * m] = v[m];
    sync();
    const float2* other = buf + (1 - sub) * 1024;
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      const float2 o = other[lane + 32 * m];
      if (sub == 0) {
        v[m] = cadd(v[m], o);
      } else {
        float2 w = cmul(__ldg(tw2048 + lane), c_tw64[m]);
        w.y = -w.y;
        v[m] = cmul(csub(o, v[m]), w);
      }
    }
    sync();
  }
  fft1024_inv(v, scr, tw1024, lane);
}

// In-place cyclic convolution of one column in shared memory:
// buf[0, M / 2) <- IFFT_M(FFT_M(buf) * kh)[0, M / 2), kh the kernel
// spectrum (1/M folded in). The column's samples fill at most its first
// M / 2 entries (M >= 2 hp - 1), so the upper half is zero by construction:
// it is neither read nor written, and the zeros, known at compile time,
// prune the first radix-2 stage of the forward transform (and the unused
// half of the inverse's last stage).
template <int M, typename Sync>
__device__ __forceinline__ void col_conv_reg(float2* buf, const float2* __restrict__ kh,
                                             const float2* __restrict__ tw1024,
                                             const float2* __restrict__ tw2048, int sub, int lane,
                                             Sync sync) {
  constexpr int S = M / 1024;
  float2 v[32];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = buf[(lane + 32 * k) * S + sub];
#pragma unroll
  for (int k = 16; k < 32; ++k) v[k] = make_float2(0.f, 0.f);
  sync();
  fft_reg_fwd<M>(v, buf, tw1024, tw2048, sub, lane, sync);
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    if ((m & 7) == 0) load_fence();
    v[m] = cmul(v[m], __ldg(kh + sub * 1024 + lane + 32 * m));
  }
  fft_reg_inv<M>(v, buf, tw1024, tw2048, sub, lane, sync);
  sync();
#pragma unroll
  for (int k = 0; k < 16; ++k) buf[(lane + 32 * k) * S + sub] = v[k];
  sync();
}

template <int M, int G, typename Sync>
__device__ __forceinline__ void init_cols_body(const InitArgs& a, const FieldDesc& f,
                                               const GeomDesc& gd, int f_idx, int x0, int col,
                                               int sub, int lane, Sync sync) {
  extern __shared__ float2 sm_cols[];
  float2* buf = sm_cols + col * (M + kColPad);
  for (int v = 0; v < 2; ++v) {
    const float2* src = a.rowbuf + a.rowbuf_off[f_idx] + (int64_t)v * gd.hp * f.pitch;
    // cooperative coalesced load of rows [0, hp), zeros to M / 2 (the input
    // half of col_conv_reg): thread -> (row, column-in-group), all of a
    // thread's loads issued before its shared-memory stores
    constexpr int kPer = (M / 2) * G / kColThreads;
    static_assert((M / 2) * G % kColThreads == 0, "fill split");
    float2 val[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = threadIdx.x + j * kColThreads;
      const int row = i / G, c = i % G;
      val[j] = make_float2(0.f, 0.f);
      if (row < gd.hp && x0 + c < f.w) val[j] = src[(int64_t)row * f.pitch + x0 + c];
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = threadIdx.x + j * kColThreads;
      sm_cols[(i % G) * (M + kColPad) + i / G] = val[j];
    }
    __syncthreads();
    col_conv_reg<M>(buf, a.khat + gd.khat_col_off + v * M, a.tw_col, a.tw_row, sub, lane, sync);
    __syncthreads();
    if (a.adj_out) {
      // adjoint mode: every padded row (the transposed crop)
      float2* dst = a.adj_out + a.rowbuf_off[f_idx] + (int64_t)v * gd.hp * f.pitch;
      for (int i = threadIdx.x; i < gd.hp * G; i += blockDim.x) {
        const int y = i / G, c = i % G;
        if (x0 + c < f.w) dst[(int64_t)y * f.pitch + x0 + c] = sm_cols[c * (M + kColPad) + y];
      }
    } else {
      float2* dst = (v == 0 ? a.chi1 : a.chi2) + f.px_off;
      for (int i = threadIdx.x; i < f.h * G; i += blockDim.x) {
        const int y = i / G, c = i % G;
        if (x0 + c < f.w)
          dst[(int64_t)y * f.pitch + x0 + c] = sm_cols[c * (M + kColPad) + y + gd.pad];
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kColThreads, 3) k_init_cols(InitArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gidx = blockIdx.x;
  const int f_idx = a.cgrp_field[gidx];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.col_m == kFftLong) return;  // k_init_cols_long (uniform per CTA)
  if (gd.col_m == kColFftWide) {
    const int x0 = (gidx - a.cgrp_first[f_idx]) * kColGroupWide;
    const int pair = warp >> 1;
    init_cols_body<kColFftWide, kColGroupWide>(a, f, gd, f_idx, x0, pair, warp & 1, lane,
                                               PairSync{1 + pair});
  } else {
    const int x0 = (gidx - a.cgrp_first[f_idx]) * kColGroup;
    init_cols_body<kColFft, kColGroup>(a, f, gd, f_idx, x0, warp, 0, lane, NoSync());
  }
}

// ---- rows ------------------------------------------------------------------
// grid = ceil(total padded rows / 2); block = 128 (two rows, a warp pair
// each); dynamic smem 64 KiB (per row: the 2048-float2 slot of the register
// FFT and the row's spectrum); up to 170 registers, 3 CTAs per SM. A row's
// 2048-point DFT runs in registers like a wide column (fft_reg_fwd /
// fft_reg_inv): warp `sub` of the pair loads the samples of parity `sub`,
// already demodulated, straight from S. The spectrum is parked in shared
// memory, each thread re-reading only the values it wrote, and filtered by
// both variants' kernel spectra in turn; each result goes out through the
// slot as one coalesced row of the pitch. A row's samples fill at most the
// first half of the 2048 points (2 w - 1 <= 2048), so the upper half is a
// compile-time zero on the way in and is not stored on the way out.
constexpr int kRowThreads = 128;
constexpr int kRowsPerCta = kRowThreads / 64;
constexpr int kRowSmem = kRowsPerCta * 2 * kRowFft * (int)sizeof(float2);

__global__ void __launch_bounds__(kRowThreads, 3) k_init_rows(InitArgs a, int total_prows) {
  extern __shared__ float2 sm_rows[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = warp >> 1, sub = warp & 1, tp = threadIdx.x & 63;
  const int r = blockIdx.x * kRowsPerCta + pair;
  if (r >= total_prows) return;  // only pair barriers below
  const PairSync sync{1 + pair};
  float2* buf = sm_rows + pair * 2 * kRowFft;
  float2* spec = buf + kRowFft;
  const int f_idx = a.prow_field[r];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.row_m != kRowFft) return;  // k_init_rows_long (uniform per pair)
  const int yp = r - a.prow_first[f_idx];
  float2 v[32];
  // v[k] (natural order, x = 2 (lane + 32 k) + sub) -> out[0, pitch), zero
  // beyond the active width; leaves buf free.
  auto store_row = [&](float2* out) {
    sync();
#pragma unroll
    for (int k = 0; k < 16; ++k) buf[2 * (lane + 32 * k) + sub] = v[k];
    sync();
    for (int i = tp; i < f.pitch; i += 64) out[i] = i < f.w ? buf[i] : make_float2(0.f, 0.f);
    sync();
  };
  if (a.adj_in) {
    // adjoint mode: each variant filters its own input row
    for (int var = 0; var < 2; ++var) {
      const int64_t row = a.rowbuf_off[f_idx] + ((int64_t)var * gd.hp + yp) * f.pitch;
      const float2* in = a.adj_in + row;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int x = 2 * (lane + 32 * k) + sub;
        v[k] = x < f.w ? in[x] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int k = 16; k < 32; ++k) v[k] = make_float2(0.f, 0.f);
      fft_reg_fwd<kRowFft>(v, buf, a.tw_col, a.tw_row, sub, lane, sync);
      const float2* kh = a.khat + gd.khat_row_off + var * kRowFft + sub * 1024 + lane;
#pragma unroll
      for (int m = 0; m < 32; ++m) {
        if ((m & 7) == 0) load_fence();
        v[m] = cmul(v[m], __ldg(kh + 32 * m));
      }
      fft_reg_inv<kRowFft>(v, buf, a.tw_col, a.tw_row, sub, lane, sync);
      store_row(a.rowbuf + row);
    }
    return;
  }
  const int sy = mirror_row(yp - gd.pad, f.h);
  const float* S = a.S + f.px_off + (int64_t)sy * f.pitch;
  const float2* P = a.col_phasor + f.col_off;
  const float4 L = __ldg(a.line_phasor + f.line_off + sy);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if ((k & 7) == 0) load_fence();
    const int x = 2 * (lane + 32 * k) + sub;
    float2 val = make_float2(0.f, 0.f);
    if (x < f.w) {
      const float s = S[x];
      const float2 c = carrier(make_float2(L.x, L.y), __ldg(P + x), L.z);
      val = make_float2(s * c.x, -s * c.y);  // S * conj(c)
    }
    v[k] = val;
  }
#pragma unroll
  for (int k = 16; k < 32; ++k) v[k] = make_float2(0.f, 0.f);
  fft_reg_fwd<kRowFft>(v, buf, a.tw_col, a.tw_row, sub, lane, sync);
  float2* my_spec = spec + sub * 1024 + lane;
#pragma unroll
  for (int m = 0; m < 32; ++m) my_spec[32 * m] = v[m];
  for (int var = 0; var < 2; ++var) {
    const float2* kh = a.khat + gd.khat_row_off + var * kRowFft + sub * 1024 + lane;
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      if ((m & 7) == 0) load_fence();
      v[m] = cmul(my_spec[32 * m], __ldg(kh + 32 * m));
    }
    fft_reg_inv<kRowFft>(v, buf, a.tw_col, a.tw_row, sub, lane, sync);
    store_row(a.rowbuf + a.rowbuf_off[f_idx] + ((int64_t)var * gd.hp + yp) * f.pitch);
  }
}

// ---- symmetry variant (holographic_init.cpp:265-306) ------------------------
// The certification min(|D[k]|, |D[-k]|) / (|D[k]| + eps) is not separable,
// so this variant needs the exact hp x w 2-D DFT of the padded demodulated
// field. Each exact-length 1-D DFT runs as Bluestein's chirp-z transform
// (Bluestein 1970): with c[n] = exp(-i pi n^2 / N),
//   X[k] = c[k] sum_n (x[n] c[n]) conj(c[k - n]),
// a cyclic convolution of length M >= 2 N - 1 (rows row_m, columns col_m):
// FFT, multiply by hhat = FFT_M(conj(c), wrapped) / M, inverse FFT. The
// inverse 2-D DFT is conj(DFT(conj(X))) / (hp w): conjugate on the column
// pass's load and on the row pass's store. rowbuf (free once the column pass
// of the two crop variants is done) holds plane 0 = the spectrum and
// plane 1 = the certified spectrum, per field.

// mode 0: forward DFT of padded row yp of the demodulated field -> plane 0.
// mode 1: last pass of the inverse, rows [pad, pad + h) of plane 1 -> chi3,
//         x 2 / (hp w) (Fft2d::Inverse's 1 / (hp w), then the init's x2).
// grid = total padded rows; block 256; dynamic smem 2 x M float2. M is the
// geometry's row length (kRowFft, or kFftLong past 1024 active samples);
// each instantiation takes the rows of its own length.
template <int M>
__global__ void __launch_bounds__(256) k_sym_rows(InitArgs a, int mode) {
  extern __shared__ float2 sm_sym[];
  float2* P = sm_sym;
  float2* Q = P + M;
  const int r = blockIdx.x;
  const int f_idx = a.prow_field[r];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.row_m != M) return;  // uniform per CTA
  const float2* tw = M == kRowFft ? a.tw_row : a.tw_long;
  const int yp = r - a.prow_first[f_idx];
  if (mode == 1 && (yp < gd.pad || yp >= gd.pad + f.h)) return;  // uniform per CTA
  const float2* chirp = a.khat + gd.sym_row_chirp;
  const float2* hh = a.khat + gd.sym_row_hhat;
  float2* plane0 = a.rowbuf + a.rowbuf_off[f_idx];
  float2* plane1 = plane0 + (int64_t)gd.hp * f.pitch;
  if (mode == 0) {
    const int sy = mirror_row(yp - gd.pad, f.h);
    const float* S = a.S + f.px_off + (int64_t)sy * f.pitch;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      float2 v = make_float2(0.f, 0.f);
      if (i < f.w) {
        const float s = S[i];
        const float2 c = carrier_at(a, f, sy, i);
        v = cmul(make_float2(s * c.x, -s * c.y), __ldg(chirp + i));
      }
      P[i] = v;
    }
  } else {
    const float2* src = plane1 + (int64_t)yp * f.pitch;
    for (int i = threadIdx.x; i < M; i += blockDim.x)
      P[i] = i < f.w ? cmul(src[i], __ldg(chirp + i)) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* spec = fft_stockham<M, false>(P, Q, tw, threadIdx.x, blockDim.x, BlockSync());
  float2* oth = spec == P ? Q : P;
  for (int i = threadIdx.x; i < M; i += blockDim.x) oth[i] = cmul(spec[i], __ldg(hh + i));
  __syncthreads();
  float2* res = fft_stockham<M, true>(oth, spec, tw, threadIdx.x, blockDim.x, BlockSync());
  if (mode == 0) {
    float2* dst = plane0 + (int64_t)yp * f.pitch;
    for (int i = threadIdx.x; i < f.pitch; i += blockDim.x)
      dst[i] = i < f.w ? cmul(res[i], __ldg(chirp + i)) : make_float2(0.f, 0.f);
  } else {
    const float scale = 2.0f / ((float)gd.hp * (float)f.w);
    float2* dst = a.chi3 + f.px_off + (int64_t)(yp - gd.pad) * f.pitch;
    for (int i = threadIdx.x; i < f.pitch; i += blockDim.x) {
      float2 v = make_float2(0.f, 0.f);
      if (i < f.w) {
        const float2 X = cmul(res[i], __ldg(chirp + i));
        v = make_float2(X.x * scale, -X.y * scale);
      }
      dst[i] = v;
    }
  }
}

// Column DFTs in place. mode 0: forward on plane 0; mode 1: the conjugated
// input of the inverse, on plane 1 (the row pass conjugates the output).
// The chirps multiply on the way into and out of shared memory; the chirp
// filter's cyclic convolution is col_conv_reg.
template <int M, int G, typename Sync>
__device__ __forceinline__ void sym_cols_body(const InitArgs& a, const FieldDesc& f,
                                              const GeomDesc& gd, int f_idx, int x0, int col,
                                              int sub, int lane, Sync sync, int mode) {
  extern __shared__ float2 sm_cols[];
  const float2* chirp = a.khat + gd.sym_col_chirp;
  float2* plane = a.rowbuf + a.rowbuf_off[f_idx] + (mode ? (int64_t)gd.hp * f.pitch : 0);
  for (int i = threadIdx.x; i < (M / 2) * G; i += blockDim.x) {
    const int row = i / G, c = i % G;
    float2 v = make_float2(0.f, 0.f);
    if (row < gd.hp && x0 + c < f.w) {
      v = plane[(int64_t)row * f.pitch + x0 + c];
      if (mode) v.y = -v.y;
      v = cmul(v, __ldg(chirp + row));
    }
    sm_cols[c * (M + kColPad) + row] = v;
  }
  __syncthreads();
  col_conv_reg<M>(sm_cols + col * (M + kColPad), a.khat + gd.sym_col_hhat, a.tw_col, a.tw_row,
                  sub, lane, sync);
  __syncthreads();
  for (int i = threadIdx.x; i < gd.hp * G; i += blockDim.x) {
    const int row = i / G, c = i % G;
    if (x0 + c < f.w)
      plane[(int64_t)row * f.pitch + x0 + c] =
          cmul(sm_cols[c * (M + kColPad) + row], __ldg(chirp + row));
  }
}

__global__ void __launch_bounds__(kColThreads, 3) k_sym_cols(InitArgs a, int mode) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gidx = blockIdx.x;
  const int f_idx = a.cgrp_field[gidx];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.col_m == kFftLong) return;  // k_sym_cols_long (uniform per CTA)
  if (gd.col_m == kColFftWide) {
    const int x0 = (gidx - a.cgrp_first[f_idx]) * kColGroupWide;
    const int pair = warp >> 1;
    sym_cols_body<kColFftWide, kColGroupWide>(a, f, gd, f_idx, x0, pair, warp & 1, lane,
                                              PairSync{1 + pair}, mode);
  } else {
    const int x0 = (gidx - a.cgrp_first[f_idx]) * kColGroup;
    sym_cols_body<kColFft, kColGroup>(a, f, gd, f_idx, x0, warp, 0, lane, NoSync(), mode);
  }
}

// Certified spectrum (holographic_init.cpp:276-290): plane 1 = plane 0 x
// min(m, m_r) / (m + 1e-6) x gy[y] gx[x], m_r the magnitude at the point
// reflection ((hp - y) mod hp, (w - x) mod w). grid = total padded rows.
__global__ void __launch_bounds__(256) k_sym_certify(InitArgs a) {
  const int r = blockIdx.x;
  const int f_idx = a.prow_field[r];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  const int y = r - a.prow_first[f_idx];
  const int ry = (gd.hp - y) % gd.hp;
  const float2* plane0 = a.rowbuf + a.rowbuf_off[f_idx];
  float2* dst = a.rowbuf + a.rowbuf_off[f_idx] + (int64_t)(gd.hp + y) * f.pitch;
  const float2* row = plane0 + (int64_t)y * f.pitch;
  const float2* rrow = plane0 + (int64_t)ry * f.pitch;
  const float gy = __ldg(a.khat + gd.sym_gy + y).x;
  for (int x = threadIdx.x; x < f.pitch; x += blockDim.x) {
    float2 v = make_float2(0.f, 0.f);
    if (x < f.w) {
      const int rx = (f.w - x) % f.w;
      const float2 X = row[x];
      const float m = hypotf(X.x, X.y);
      const float2 R = rrow[rx];
      const float mr = hypotf(R.x, R.y);
      const float sym = fminf(m, mr) / (m + 1e-6f);
      const float k = gy * __ldg(a.khat + gd.sym_gx + x).x;
      v = make_float2(X.x * sym * k, X.y * sym * k);
    }
    dst[x] = v;
  }
}

// ---- long rows / columns (kFftLong) -----------------------------------------
// Planes past the register transforms' lengths (more than 1024 active
// samples, or more than 1024 padded lines) run their cyclic convolutions at
// length kFftLong = 4096 through the shared-memory Stockham FFT
// (fft_stockham: six radix-4 stages, a block barrier after each), one CTA of
// 256 threads per padded row or per column, with the same kernel spectra,
// layouts and outputs as the register kernels. These kernels run over the
// same padded-row / column-group grids and take only the rows / columns of
// geometries with the long length (the register kernels skip those); a long
// column geometry has one column per group.
constexpr int kLongThreads = 256;
constexpr int kLongColSmem = 2 * kFftLong * (int)sizeof(float2);  // ping-pong: 64 KiB
constexpr int kLongRowSmem = 3 * kFftLong * (int)sizeof(float2);  // + the row's spectrum

// P holds x (zero past the data, barrier taken) -> the cyclic convolution of
// x with the kernel whose spectrum (1/M folded in) is kh; returns the buffer
// (P or Q) holding it, barrier taken.
__device__ __forceinline__ float2* long_conv(float2* P, float2* Q, const float2* __restrict__ kh,
                                             const float2* __restrict__ tw) {
  float2* spec = fft_stockham<kFftLong, false>(P, Q, tw, threadIdx.x, blockDim.x, BlockSync());
  for (int i = threadIdx.x; i < kFftLong; i += blockDim.x) spec[i] = cmul(spec[i], __ldg(kh + i));
  __syncthreads();
  return fft_stockham<kFftLong, true>(spec, spec == P ? Q : P, tw, threadIdx.x, blockDim.x,
                                      BlockSync());
}

// grid = total padded rows; block 256; dynamic smem kLongRowSmem.
__global__ void __launch_bounds__(kLongThreads) k_init_rows_long(InitArgs a) {
  extern __shared__ float2 sm_long[];
  float2* P = sm_long;
  float2* Q = P + kFftLong;
  float2* spec = Q + kFftLong;
  const int r = blockIdx.x;
  const int f_idx = a.prow_field[r];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.row_m != kFftLong) return;  // uniform per CTA
  const int yp = r - a.prow_first[f_idx];
  const float2 z = make_float2(0.f, 0.f);
  // res -> out[0, pitch), zero beyond the active width; the barrier frees P / Q
  auto store_row = [&](const float2* res, float2* out) {
    for (int i = threadIdx.x; i < f.pitch; i += blockDim.x) out[i] = i < f.w ? res[i] : z;
    __syncthreads();
  };
  if (a.adj_in) {
    // adjoint mode: each variant filters its own input row
    for (int var = 0; var < 2; ++var) {
      const int64_t row = a.rowbuf_off[f_idx] + ((int64_t)var * gd.hp + yp) * f.pitch;
      const float2* in = a.adj_in + row;
      for (int i = threadIdx.x; i < kFftLong; i += blockDim.x) P[i] = i < f.w ? in[i] : z;
      __syncthreads();
      const float2* res =
          long_conv(P, Q, a.khat + gd.khat_row_off + var * kFftLong, a.tw_long);
      store_row(res, a.rowbuf + row);
    }
    return;
  }
  const int sy = mirror_row(yp - gd.pad, f.h);
  const float* S = a.S + f.px_off + (int64_t)sy * f.pitch;
  for (int i = threadIdx.x; i < kFftLong; i += blockDim.x) {
    float2 v = z;
    if (i < f.w) {
      const float s = S[i];
      const float2 c = carrier_at(a, f, sy, i);
      v = make_float2(s * c.x, -s * c.y);  // S * conj(c)
    }
    P[i] = v;
  }
  __syncthreads();
  const float2* X = fft_stockham<kFftLong, false>(P, Q, a.tw_long, threadIdx.x, blockDim.x,
                                                  BlockSync());
  for (int i = threadIdx.x; i < kFftLong; i += blockDim.x) spec[i] = X[i];
  __syncthreads();
  for (int var = 0; var < 2; ++var) {
    const float2* kh = a.khat + gd.khat_row_off + var * kFftLong;
    for (int i = threadIdx.x; i < kFftLong; i += blockDim.x) P[i] = cmul(spec[i], __ldg(kh + i));
    __syncthreads();
    const float2* res = fft_stockham<kFftLong, true>(P, Q, a.tw_long, threadIdx.x, blockDim.x,
                                                     BlockSync());
    store_row(res, a.rowbuf + a.rowbuf_off[f_idx] + ((int64_t)var * gd.hp + yp) * f.pitch);
  }
}

// grid = total column groups; block 256; dynamic smem kLongColSmem. Column
// x of a long geometry: rows [0, hp) of each row-filtered variant -> chi1 /
// chi2 rows [pad, pad + h) (adjoint mode: all hp rows into adj_out).
__global__ void __launch_bounds__(kLongThreads) k_init_cols_long(InitArgs a) {
  extern __shared__ float2 sm_long[];
  float2* P = sm_long;
  float2* Q = P + kFftLong;
  const int gidx = blockIdx.x;
  const int f_idx = a.cgrp_field[gidx];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.col_m != kFftLong) return;  // uniform per CTA
  const int x = gidx - a.cgrp_first[f_idx];
  for (int v = 0; v < 2; ++v) {
    const int64_t plane = a.rowbuf_off[f_idx] + (int64_t)v * gd.hp * f.pitch + x;
    const float2* src = a.rowbuf + plane;
    for (int i = threadIdx.x; i < kFftLong; i += blockDim.x)
      P[i] = i < gd.hp ? src[(int64_t)i * f.pitch] : make_float2(0.f, 0.f);
    __syncthreads();
    const float2* res = long_conv(P, Q, a.khat + gd.khat_col_off + v * kFftLong, a.tw_long);
    if (a.adj_out) {
      float2* dst = a.adj_out + plane;
      for (int y = threadIdx.x; y < gd.hp; y += blockDim.x) dst[(int64_t)y * f.pitch] = res[y];
    } else {
      float2* dst = (v == 0 ? a.chi1 : a.chi2) + f.px_off + x;
      for (int y = threadIdx.x; y < f.h; y += blockDim.x)
        dst[(int64_t)y * f.pitch] = res[y + gd.pad];
    }
    __syncthreads();
  }
}

// The symmetry variant's column DFTs of a long geometry (sym_cols_body at
// length kFftLong): grid = total column groups; block 256; smem kLongColSmem.
__global__ void __launch_bounds__(kLongThreads) k_sym_cols_long(InitArgs a, int mode) {
  extern __shared__ float2 sm_long[];
  float2* P = sm_long;
  float2* Q = P + kFftLong;
  const int gidx = blockIdx.x;
  const int f_idx = a.cgrp_field[gidx];
  const FieldDesc f = a.fields[f_idx];
  const GeomDesc gd = a.geoms[f.geom];
  if (gd.col_m != kFftLong) return;  // uniform per CTA
  const int x = gidx - a.cgrp_first[f_idx];
  const float2* chirp = a.khat + gd.sym_col_chirp;
  float2* plane = a.rowbuf + a.rowbuf_off[f_idx] + (mode ? (int64_t)gd.hp * f.pitch : 0) + x;
  for (int i = threadIdx.x; i < kFftLong; i += blockDim.x) {
    float2 v = make_float2(0.f, 0.f);
    if (i < gd.hp) {
      v = plane[(int64_t)i * f.pitch];
      if (mode) v.y = -v.y;
      v = cmul(v, __ldg(chirp + i));
    }
    P[i] = v;
  }
  __syncthreads();
  const float2* res = long_conv(P, Q, a.khat + gd.sym_col_hhat, a.tw_long);
  for (int i = threadIdx.x; i < gd.hp; i += blockDim.x)
    plane[(int64_t)i * f.pitch] = cmul(res[i], __ldg(chirp + i));
}

// ---- blend -----------------------------------------------------------------
// Edge-energy blend (holographic_init.cpp:240-316). 32 x 32 output tile per
// CTA; y_v on the tile + 4 halo (forward difference + box radius 3); the box
// blur is zero-padded at the field border with constant 1/7 normalisation.
constexpr int kBT = 32;
constexpr int kBH = kBT + 8;  // y_v tile incl. halo [-3, +4]
__global__ void __launch_bounds__(256) k_init_blend(InitArgs a) {
  const int f_idx = a.btile_field[blockIdx.x];
  const FieldDesc f = a.fields[f_idx];
  const int t = blockIdx.x - a.btile_first[f_idx];
  const int ntx = (f.w + kBT - 1) / kBT;
  const int ty0 = (t / ntx) * kBT, tx0 = (t % ntx) * kBT;
  __shared__ float yv[kBH][kBH + 1];
  __shared__ float ev[kBH][kBH + 1];
  __shared__ float vb[kBT][kBH + 1];
  __shared__ float wsum[kBT][kBT];
  __shared__ float2 num[kBT][kBT];
  const float* S = a.S + f.px_off;
  const int nv = a.chi3 ? 3 : 2;
  for (int v = 0; v < nv; ++v) {
    const float2* chi = (v == 0 ? a.chi1 : (v == 1 ? a.chi2 : a.chi3)) + f.px_off;
    // residual luma on [ty0-3, ty0+kBT+5) x [tx0-3, ...)
    for (int i = threadIdx.x; i < kBH * kBH; i += blockDim.x) {
      const int ly = i / kBH, lx = i % kBH;
      const int y = ty0 - 3 + ly, x = tx0 - 3 + lx;
      float val = 0.f;
      if (y >= 0 && y < f.h && x >= 0 && x < f.w) {
        const int64_t o = (int64_t)y * f.pitch + x;
        val = S[o] - re_mul(chi[o], carrier_at(a, f, y, x));
      }
      yv[ly][lx] = val;
    }
    __syncthreads();
    // e = |Dx y| + |Dy y| (forward, zero on the last column / row), zero
    // outside the field (the box blur's zero padding).
    for (int i = threadIdx.x; i < (kBH - 1) * (kBH - 1); i += blockDim.x) {
      const int ly = i / (kBH - 1), lx = i % (kBH - 1);
      const int y = ty0 - 3 + ly, x = tx0 - 3 + lx;
      float e = 0.f;
      if (y >= 0 && y < f.h && x >= 0 && x < f.w) {
        const float dx = (x + 1 < f.w) ? yv[ly][lx + 1] - yv[ly][lx] : 0.f;
        const float dy = (y + 1 < f.h) ? yv[ly + 1][lx] - yv[ly][lx] : 0.f;
        e = fabsf(dx) + fabsf(dy);
      }
      ev[ly][lx] = e;
    }
    __syncthreads();
    // vertical box (rows of the tile, all halo columns)
    for (int i = threadIdx.x; i < kBT * (kBT + 6); i += blockDim.x) {
      const int ly = i / (kBT + 6), lx = i % (kBT + 6);
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < 7; ++k) acc += ev[ly + k][lx];
      vb[ly][lx] = acc * (1.0f / 7.0f);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kBT * kBT; i += blockDim.x) {
      const int ly = i / kBT, lx = i % kBT;
      const int y = ty0 + ly, x = tx0 + lx;
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < 7; ++k) acc += vb[ly][lx + k];
      const float E = acc * (1.0f / 7.0f);
      const float wt = 1.0f / (E + 0.5f);
      float2 cv = make_float2(0.f, 0.f);
      if (y < f.h && x < f.w) cv = chi[(int64_t)y * f.pitch + x];
      if (v == 0) {
        num[ly][lx] = cscale(cv, wt);
        wsum[ly][lx] = wt;
      } else {
        num[ly][lx] = cadd(num[ly][lx], cscale(cv, wt));
        wsum[ly][lx] += wt;
      }
    }
    __syncthreads();
  }
  float2* X = a.chi0 + f.px_off;
  float* Y = a.Y + f.px_off;
  for (int i = threadIdx.x; i < kBT * kBT; i += blockDim.x) {
    const int ly = i / kBT, lx = i % kBT;
    const int y = ty0 + ly, x = tx0 + lx;
    if (y < f.h && x < f.w) {
      const float2 c0 = make_float2(num[ly][lx].x / wsum[ly][lx], num[ly][lx].y / wsum[ly][lx]);
      const int64_t o = (int64_t)y * f.pitch + x;
      X[o] = c0;
      Y[o] = S[o] - re_mul(c0, carrier_at(a, f, y, x));
    }
  }
}

// ---- auto chroma anisotropy (variational.cpp:130-196) ----------------------
// Two CTAs (1024 threads) per field, one per axis: p98 of |delta| of 2-line
// (NTSC) / 4-line (PAL) group averages, sampled at odd group rows and every
// 3rd column, horizontal (axis 0) or vertical (axis 1) neighbour, exact k-th
// element by radix select. The field's second CTA to finish maps the ratio
// of the two to the split and writes mu_h, mu_v, mu_d.
constexpr int kAnisoMax = 49152;
__global__ void __launch_bounds__(1024) k_aniso(FieldDesc* fields, const float2* __restrict__ chi0) {
  extern __shared__ float sm_an[];
  __shared__ unsigned hist[256];
  __shared__ unsigned bc[2];
  __shared__ int last;
  FieldDesc& f = fields[blockIdx.x];
  const int axis = blockIdx.y;
  if (!(f.aniso_cfg > 0.0f)) {
    const int group = f.is_pal ? 4 : 2;
    const int Hh = f.h / group;
    const int nt = Hh / 2;                // t = 1, 3, 5, ... < Hh
    const int nx = (f.w - 1 + 2) / 3;     // x = 1, 4, 7, ... < w
    int n = nt * nx;
    if (n > kAnisoMax) n = kAnisoMax;     // geometry guard (the host rejects larger)
    const float2* c = chi0 + f.px_off;
    const float inv = 1.0f / (float)group;
    // kAnisoBatch samples per thread and pass, all their loads issued before
    // the first sum (one L2 round trip per batch, not per sample)
    constexpr int kAnisoBatch = 4;
    for (int i0 = threadIdx.x; i0 < n; i0 += kAnisoBatch * blockDim.x) {
      float2 pv[kAnisoBatch][4], qv[kAnisoBatch][4];
#pragma unroll
      for (int b = 0; b < kAnisoBatch; ++b) {
        const int i = i0 + b * blockDim.x;
        const int ti = i / nx, xi = i % nx;
        const int tt = 1 + 2 * ti, x = 1 + 3 * xi;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          pv[b][k] = qv[b][k] = make_float2(0.f, 0.f);
          if (i < n && k < group) {
            pv[b][k] = c[(int64_t)(group * tt + k) * f.pitch + x];
            qv[b][k] = axis == 0 ? c[(int64_t)(group * tt + k) * f.pitch + x - 1]
                                 : c[(int64_t)(group * (tt - 1) + k) * f.pitch + x];
          }
        }
      }
#pragma unroll
      for (int b = 0; b < kAnisoBatch; ++b) {
        const int i = i0 + b * blockDim.x;
        float2 p = make_float2(0.f, 0.f), q = p;
        // the same order of additions as one sample at a time: k = 0, 1, ...
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (k < group) {
            p = cadd(p, pv[b][k]);
            q = cadd(q, qv[b][k]);
          }
        }
        if (i < n) sm_an[i] = sqrtf(cnorm(csub(cscale(p, inv), cscale(q, inv))));
      }
    }
    __syncthreads();
    const float p98 = n > 0 ? block_select_kth(sm_an, n, n - 1 - n / 50, hist, bc) : 0.f;
    if (threadIdx.x == 0) f.aniso_p98[axis] = p98;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    // two arrivals per run (the counter is not reset between graph replays)
    last = (atomicAdd(&f.aniso_arrive, 1) & 1) == 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  float aniso = f.aniso_cfg;
  if (!(aniso > 0.0f)) {
    const float p0 = __ldcg(&f.aniso_p98[0]), p1 = __ldcg(&f.aniso_p98[1]);
    const float r = p1 / fmaxf(p0, 1e-6f);
    if (f.is_pal)
      aniso = fminf(fmaxf(0.7f + 0.9f * (r - 1.3f), 0.55f), 1.0f);
    else
      aniso = fminf(fmaxf(0.5f + 1.1f * (r - 1.3f), 0.5f), 1.0f);
  }
  // the oriented prior's weight, and the renormalisation that keeps the
  // total chroma prior mass (variational.cpp:207-219)
  const float mu_d = f.lambda_c * f.diag_prior * 0.5f;
  const float tot0 = f.lambda_c * (1.0f + aniso);
  const float scale = mu_d > 0.0f ? tot0 / (tot0 + 2.0f * mu_d) : 1.0f;
  f.mu_h = (f.lambda_c * aniso) * scale;
  f.mu_v = f.lambda_c * scale;
  f.mu_d = mu_d > 0.0f ? mu_d * scale : 0.0f;
}

constexpr int kAnisoSmem = kAnisoMax * (int)sizeof(float);

static void configure_init_kernels_now() {
  float2 tw32[16];
  for (int k = 0; k < 16; ++k) {
    const double a = -2.0 * 3.14159265358979323846 * k / 32.0;
    tw32[k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  cudaMemcpyToSymbol(c_tw32, tw32, sizeof(tw32));
  float2 tw64[32];
  for (int m = 0; m < 32; ++m) {
    const double a = -2.0 * 3.14159265358979323846 * m / 64.0;
    tw64[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  cudaMemcpyToSymbol(c_tw64, tw64, sizeof(tw64));
  cudaFuncSetAttribute(k_init_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, kRowSmem);
  cudaFuncSetAttribute(k_init_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, kColSmem);
  cudaFuncSetAttribute(k_sym_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, kColSmem);
  cudaFuncSetAttribute(k_sym_rows<kFftLong>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kLongColSmem);
  cudaFuncSetAttribute(k_init_rows_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kLongRowSmem);
  cudaFuncSetAttribute(k_init_cols_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kLongColSmem);
  cudaFuncSetAttribute(k_sym_cols_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kLongColSmem);
  cudaFuncSetAttribute(k_aniso, cudaFuncAttributeMaxDynamicSharedMemorySize, kAnisoSmem);
}

// Kernel attributes and the twiddle constants, once per device.
void configure_init_kernels() {
  static PerDeviceOnce once;
  once(configure_init_kernels_now);
}

// The row and column filter passes: the register kernels, then (when the
// batch holds a long geometry) the shared-memory ones over the same grids.
static void launch_filter_passes(const InitArgs& a, int total_prows, int total_cgroups,
                                 cudaStream_t st) {
  if (total_prows > 0) {
    k_init_rows<<<(total_prows + kRowsPerCta - 1) / kRowsPerCta, kRowThreads, kRowSmem, st>>>(
        a, total_prows);
    if (a.long_rows) k_init_rows_long<<<total_prows, kLongThreads, kLongRowSmem, st>>>(a);
  }
  if (total_cgroups > 0) {
    k_init_cols<<<total_cgroups, kColThreads, kColSmem, st>>>(a);
    if (a.long_cols) k_init_cols_long<<<total_cgroups, kLongThreads, kLongColSmem, st>>>(a);
  }
}

void launch_init(const InitArgs& a, int total_prows, int total_cgroups, int total_btiles,
                 cudaStream_t st) {
  configure_init_kernels();
  launch_filter_passes(a, total_prows, total_cgroups, st);
  if (a.chi3 && total_prows > 0 && total_cgroups > 0) {
    const int sym_smem = 2 * kRowFft * sizeof(float2);
    auto sym_rows = [&](int mode) {
      k_sym_rows<kRowFft><<<total_prows, 256, sym_smem, st>>>(a, mode);
      if (a.long_rows) k_sym_rows<kFftLong><<<total_prows, 256, kLongColSmem, st>>>(a, mode);
    };
    auto sym_cols = [&](int mode) {
      k_sym_cols<<<total_cgroups, kColThreads, kColSmem, st>>>(a, mode);
      if (a.long_cols) k_sym_cols_long<<<total_cgroups, kLongThreads, kLongColSmem, st>>>(a, mode);
    };
    sym_rows(0);
    sym_cols(0);
    k_sym_certify<<<total_prows, 256, 0, st>>>(a);
    sym_cols(1);
    sym_rows(1);
  }
  if (total_btiles > 0) k_init_blend<<<total_btiles, 256, 0, st>>>(a);
}

void launch_init_filter_adjoint(const InitArgs& a, int total_prows, int total_cgroups,
                                cudaStream_t st) {
  configure_init_kernels();
  launch_filter_passes(a, total_prows, total_cgroups, st);
}

void launch_aniso(FieldDesc* d_fields, int n_fields, const float2* chi0, cudaStream_t st) {
  const int smem = kAnisoSmem;
  configure_init_kernels();
  if (n_fields > 0) k_aniso<<<dim3(n_fields, 2), 1024, smem, st>>>(d_fields, chi0);
}

int aniso_max_samples() { return kAnisoMax; }
int init_col_group(int col_m) {
  return col_m == kFftLong ? 1 : col_m == kColFftWide ? kColGroupWide : kColGroup;
}
int init_blend_tile() { return kBT; }

}  // namespace hvdg
