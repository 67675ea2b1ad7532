// k_adjoint.cu -- pointwise / stencil kernels of the decode adjoint.
//
// No reference counterpart (the reference has no adjoint). The forward being
// differentiated is VariationalRefine (hvd-core/src/engine/variational.cpp:
// 198-556: lagged-diffusivity weights :406-433, gradient :286-347) preceded
// by HolographicInit (holographic_init.cpp:200-317) and followed by the
// output luma Y = S - Re[chi c] (sequence.cpp:1102-1114).
//
// Per IRLS outer o (implicit function: chi_{o+1} minimises the quadratic
// with the weights W(chi_o) frozen), given lambda = H^-1 chibar_{o+1} from
// the solver run in adjoint mode, and r = Re(lambda c):
//   Sbar   += 2 [DxT(wx Dx r) + DyT(wy Dy r)]                (dg/dS)
//   mubar  = -2 sum wc* Re(conj(D* lambda) D* chi_{o+1})     (dg/dmu)
//   Wbar   = 2 D*Yc_{o+1} D*r (luma), -2 mu* Re(..) (chroma) (dg/dW)
// and the chain through W(chi_o; eps, eps_c, k):
//   gbar_x = Wbar_x (-wx gx / (gx^2 + eps^2)) + Wbar_cx (-wcx k gx / Rx),
//   mbar_x = Wbar_cx (-wcx / (2 Rx)),  Rx = |Dx chi_o|^2 + k gx^2 + eps_c^2,
//   Ycbar  = DxT(gbar_x) + DyT(gbar_y);   Sbar += Ycbar;
//   chibar_o = -Ycbar conj(c) + DxT(2 mbar_x Dx chi_o) + DyT(2 mbar_y Dy chi_o).
// The scalar partials are reduced per block and then in a fixed order.
#include <cuda_runtime.h>

#include "hvdg_common.cuh"
#include "k_adjoint.h"

namespace hvdg {

namespace {

constexpr int kBX = 32, kBY = 8;

__device__ __forceinline__ float2 car(const AdjGeom& g, int y, int x) {
  const float4 L = __ldg(g.line_phasor + y);
  return carrier(make_float2(L.x, L.y), __ldg(g.col_phasor + x), L.z);
}

__device__ __forceinline__ float2 cmulf(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// DxT / DyT of a complex plane at (y, x) (gradients.h:61-101): a[x-1] - a[x]
// with the missing terms dropped at the borders.
__device__ __forceinline__ float2 dxt_c(const float2* a, int64_t o, int x, int w) {
  const float2 z = make_float2(0.f, 0.f);
  const float2 l = x > 0 ? a[o - 1] : z, r = x < w - 1 ? a[o] : z;
  return make_float2(l.x - r.x, l.y - r.y);
}
__device__ __forceinline__ float2 dyt_c(const float2* a, int64_t o, int y, int h, int pitch) {
  const float2 z = make_float2(0.f, 0.f);
  const float2 u = y > 0 ? a[o - pitch] : z, d = y < h - 1 ? a[o] : z;
  return make_float2(u.x - d.x, u.y - d.y);
}

// fixed-order block reduction of N doubles; thread 0 holds the result
template <int N>
__device__ void block_sum(double (&v)[N], double* sh /* N * warps */) {
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  const int nw = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < N; ++i) sh[warp * N + i] = v[i];
  __syncthreads();
  if (warp == 0 && lane == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double s = 0.0;
      for (int j = 0; j < nw; ++j) s += sh[j * N + i];
      v[i] = s;
    }
  }
}

__global__ void k_adj_output(AdjGeom g, const float* __restrict__ ybar, float* __restrict__ sbar,
                             float2* __restrict__ chib) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  const int64_t o = (int64_t)y * g.pitch + x;
  const float yb = ybar[o];
  const float2 c = car(g, y, x);
  sbar[o] = yb;
  float2 v = chib[o];
  v.x -= yb * c.x;   // - ybar conj(c)
  v.y += yb * c.y;
  chib[o] = v;
}

__global__ void k_adj_norm(AdjGeom g, const float2* __restrict__ chib, double* __restrict__ part) {
  __shared__ double sh[kBX * kBY / 32];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  double v[1] = {0.0};
  if (x < g.w && y < g.h) {
    const float2 a = chib[(int64_t)y * g.pitch + x];
    v[0] = (double)a.x * a.x + (double)a.y * a.y;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = v[0];
}

__global__ void k_adj_rhs(AdjGeom g, const float2* __restrict__ chib, float sigma,
                          float2* __restrict__ B) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  const int64_t o = (int64_t)y * g.pitch + x;
  const float2 a = chib[o];
  B[o] = make_float2(-sigma * a.x, -sigma * a.y);
}

__global__ void k_adj_pass_a(AdjGeom g, AdjScalars sc, AdjOuter p) {
  __shared__ double sh[4 * kBX * kBY / 32];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  double part[4] = {0.0, 0.0, 0.0, 0.0};
  if (x < g.w && y < g.h) {
    const int64_t o = (int64_t)y * g.pitch + x;
    const bool hx = x + 1 < g.w, hy = y + 1 < g.h;
    const float2 z = make_float2(0.f, 0.f);
    const float2 c = car(g, y, x);
    const float2 cr = hx ? car(g, y, x + 1) : z;
    const float2 cd = hy ? car(g, y + 1, x) : z;
    const float Sv = p.S[o], Sr = hx ? p.S[o + 1] : 0.f, Sd = hy ? p.S[o + g.pitch] : 0.f;
    const float2 l0 = cmulf(p.lam[o], p.inv_sigma);
    const float2 lr = hx ? cmulf(p.lam[o + 1], p.inv_sigma) : z;
    const float2 ld = hy ? cmulf(p.lam[o + g.pitch], p.inv_sigma) : z;
    const float r0 = re_mul(l0, c), rr = re_mul(lr, cr), rd = re_mul(ld, cd);
    const float dxr = hx ? rr - r0 : 0.f, dyr = hy ? rd - r0 : 0.f;
    const float2 a0 = p.chi1[o], ar = hx ? p.chi1[o + 1] : z, ad = hy ? p.chi1[o + g.pitch] : z;
    const float dxy1 = hx ? (Sr - re_mul(ar, cr)) - (Sv - re_mul(a0, c)) : 0.f;
    const float dyy1 = hy ? (Sd - re_mul(ad, cd)) - (Sv - re_mul(a0, c)) : 0.f;
    const float2 b0 = p.chi0[o], br = hx ? p.chi0[o + 1] : z, bd = hy ? p.chi0[o + g.pitch] : z;
    const float gx = hx ? (Sr - re_mul(br, cr)) - (Sv - re_mul(b0, c)) : 0.f;
    const float gy = hy ? (Sd - re_mul(bd, cd)) - (Sv - re_mul(b0, c)) : 0.f;
    const float2 dxl = hx ? csub(lr, l0) : z, dyl = hy ? csub(ld, l0) : z;
    const float2 dxc1 = hx ? csub(ar, a0) : z, dyc1 = hy ? csub(ad, a0) : z;
    const float2 dxc0 = hx ? csub(br, b0) : z, dyc0 = hy ? csub(bd, b0) : z;
    const float4 W = p.W[o];
    const float tx = dxl.x * dxc1.x + dxl.y * dxc1.y;
    const float ty = dyl.x * dyc1.x + dyl.y * dyc1.y;
    p.P[o] = make_float2(W.x * dxr, W.y * dyr);
    const float wbx = 2.f * dxy1 * dxr, wby = 2.f * dyy1 * dyr;
    const float wbcx = -2.f * sc.mu_h * tx, wbcy = -2.f * sc.mu_v * ty;
    const float e2 = sc.eps * sc.eps, ec2 = sc.eps_c * sc.eps_c;
    const float ex = gx * gx + e2, ey = gy * gy + e2;
    const float rx = cnorm(dxc0) + sc.k * gx * gx + ec2;
    const float ry = cnorm(dyc0) + sc.k * gy * gy + ec2;
    const float gbx = wbx * (-W.x * gx / ex) + wbcx * (-W.z * sc.k * gx / rx);
    const float gby = wby * (-W.y * gy / ey) + wbcy * (-W.w * sc.k * gy / ry);
    const float mbx = wbcx * (-0.5f * W.z / rx), mby = wbcy * (-0.5f * W.w / ry);
    p.GB[o] = make_float2(gbx, gby);
    p.A1[o] = cmulf(dxc0, 2.f * mbx);
    p.A2[o] = cmulf(dyc0, 2.f * mby);
    part[0] = -2.0 * (double)W.z * tx * sc.aniso - 2.0 * (double)W.w * ty;
    part[1] = (double)wbx * W.x * gx * gx / ((double)sc.eps * ex) +
              (double)wby * W.y * gy * gy / ((double)sc.eps * ey);
    part[2] = (double)wbcx * W.z * (rx - ec2) / ((double)sc.eps_c * rx) +
              (double)wbcy * W.w * (ry - ec2) / ((double)sc.eps_c * ry);
    part[3] = (double)wbcx * (-0.5 * W.z * gx * gx / rx) + (double)wbcy * (-0.5 * W.w * gy * gy / ry);
  }
  block_sum<4>(part, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double* dst = p.partials + 4 * (int64_t)(blockIdx.y * gridDim.x + blockIdx.x);
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[i] = part[i];
  }
}

// acc[i] += sum_b part[4 b + i], b in order (one CTA)
__global__ void k_adj_reduce(const double* __restrict__ part, int nb, int stride,
                             double* __restrict__ acc) {
  __shared__ double sh[4 * 256 / 32];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] += part[(int64_t)stride * b + i];
  block_sum<4>(v, sh);
  if (threadIdx.x == 0)
    for (int i = 0; i < 4 && i < stride; ++i) acc[i] += v[i];
}

__global__ void k_adj_pass_b(AdjGeom g, AdjOuter p, float* __restrict__ sbar,
                             float2* __restrict__ chib) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  const int64_t o = (int64_t)y * g.pitch + x;
  const float2 z = make_float2(0.f, 0.f);
  // DxT / DyT of the interleaved planes, component by component
  const float2 pl = x > 0 ? p.P[o - 1] : z, pc = x < g.w - 1 ? p.P[o] : z;
  const float2 pu = y > 0 ? p.P[o - g.pitch] : z, pd = y < g.h - 1 ? p.P[o] : z;
  const float2 gl = x > 0 ? p.GB[o - 1] : z, gc = x < g.w - 1 ? p.GB[o] : z;
  const float2 gu = y > 0 ? p.GB[o - g.pitch] : z, gd = y < g.h - 1 ? p.GB[o] : z;
  const float data = 2.f * ((pl.x - pc.x) + (pu.y - pd.y));
  const float ycb = (gl.x - gc.x) + (gu.y - gd.y);
  sbar[o] += data + ycb;
  const float2 c = car(g, y, x);
  const float2 t1 = dxt_c(p.A1, o, x, g.w);
  const float2 t2 = dyt_c(p.A2, o, y, g.h, g.pitch);
  // -ycb conj(c) + DxT(A1) + DyT(A2)
  chib[o] = make_float2(-ycb * c.x + t1.x + t2.x, ycb * c.y + t1.y + t2.y);
}

// ---- HolographicInit adjoint ------------------------------------------------
__global__ void k_ai_edges(AdjGeom g, AdjInit a) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  const int64_t o = (int64_t)y * g.pitch + x;
  const bool hx = x + 1 < g.w, hy = y + 1 < g.h;
  const float2 c = car(g, y, x);
  const float S0 = a.S[o];
  float e[2];
  for (int v = 0; v < 2; ++v) {
    const float2* chi = v == 0 ? a.chi1 : a.chi2;
    const float y0 = S0 - re_mul(chi[o], c);
    const float dx = hx ? (a.S[o + 1] - re_mul(chi[o + 1], car(g, y, x + 1))) - y0 : 0.f;
    const float dy = hy ? (a.S[o + g.pitch] - re_mul(chi[o + g.pitch], car(g, y + 1, x))) - y0 : 0.f;
    e[v] = fabsf(dx) + fabsf(dy);
  }
  a.a[o] = make_float2(e[0], e[1]);
}

// zero-padded 7-tap box (constant 1/7) along y, then x (BoxBlur r = 3,
// holographic_init.cpp:61-113)
__global__ void k_ai_box_v(AdjGeom g, const float2* __restrict__ in, float2* __restrict__ out) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  float2 s = make_float2(0.f, 0.f);
  for (int k = -3; k <= 3; ++k) {
    const int yy = y + k;
    if (yy >= 0 && yy < g.h) s = cadd(s, in[(int64_t)yy * g.pitch + x]);
  }
  out[(int64_t)y * g.pitch + x] = cmulf(s, 1.f / 7.f);
}
__global__ void k_ai_box_h(AdjGeom g, const float2* __restrict__ in, float2* __restrict__ out) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  float2 s = make_float2(0.f, 0.f);
  for (int k = -3; k <= 3; ++k) {
    const int xx = x + k;
    if (xx >= 0 && xx < g.w) s = cadd(s, in[(int64_t)y * g.pitch + xx]);
  }
  out[(int64_t)y * g.pitch + x] = cmulf(s, 1.f / 7.f);
}

// blend adjoint: chi0 = (chi1 w1 + chi2 w2) / (w1 + w2), w = 1 / (E + 0.5)
__global__ void k_ai_blend(AdjGeom g, AdjInit a) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  const int64_t o = (int64_t)y * g.pitch + x;
  const float2 E = a.a[o];
  const float w1 = 1.f / (E.x + 0.5f), w2 = 1.f / (E.y + 0.5f);
  const float ws = w1 + w2;
  const float2 c1 = a.chi1[o], c2 = a.chi2[o];
  const float2 c0 = make_float2((c1.x * w1 + c2.x * w2) / ws, (c1.y * w1 + c2.y * w2) / ws);
  const float2 cb = a.chi0bar[o];
  a.cb1[o] = cmulf(cb, w1 / ws);
  a.cb2[o] = cmulf(cb, w2 / ws);
  const float wb1 = (cb.x * (c1.x - c0.x) + cb.y * (c1.y - c0.y)) / ws;
  const float wb2 = (cb.x * (c2.x - c0.x) + cb.y * (c2.y - c0.y)) / ws;
  a.ebar[o] = make_float2(-wb1 * w1 * w1, -wb2 * w2 * w2);
}

__device__ __forceinline__ float sgnf(float d) { return (float)((d > 0.f) - (d < 0.f)); }

// ybar_v = DxT(sign(Dx y_v) abar_v) + DyT(sign(Dy y_v) abar_v); Sbar += ybar_v;
// the filter inputs cb_v - ybar_v conj(c) into the padded rows
__global__ void k_ai_edges_adjoint(AdjGeom g, AdjInit a, const float2* __restrict__ abar,
                                   float* __restrict__ sbar) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= g.w || y >= g.h) return;
  const int64_t o = (int64_t)y * g.pitch + x;
  const float2 c = car(g, y, x);
  float ys[2];
  for (int v = 0; v < 2; ++v) {
    const float2* chi = v == 0 ? a.chi1 : a.chi2;
    auto yv = [&](int yy, int xx) {
      const int64_t oo = (int64_t)yy * g.pitch + xx;
      return a.S[oo] - re_mul(chi[oo], car(g, yy, xx));
    };
    auto ab = [&](int64_t oo) { const float2 t = abar[oo]; return v == 0 ? t.x : t.y; };
    const float yc = yv(y, x);
    float s = 0.f;
    if (x > 0) s += sgnf(yc - yv(y, x - 1)) * ab(o - 1);
    if (x < g.w - 1) s -= sgnf(yv(y, x + 1) - yc) * ab(o);
    if (y > 0) s += sgnf(yc - yv(y - 1, x)) * ab(o - g.pitch);
    if (y < g.h - 1) s -= sgnf(yv(y + 1, x) - yc) * ab(o);
    ys[v] = s;
  }
  sbar[o] += ys[0] + ys[1];
  const int64_t plane = (int64_t)g.hp * g.pitch;
  const int64_t oi = (int64_t)(y + g.pad) * g.pitch + x;
  const float2 b1 = a.cb1[o], b2 = a.cb2[o];
  a.adj_in[oi] = make_float2(b1.x - ys[0] * c.x, b1.y + ys[0] * c.y);
  a.adj_in[plane + oi] = make_float2(b2.x - ys[1] * c.x, b2.y + ys[1] * c.y);
}

__device__ __forceinline__ int mirror101(int y, int h) {
  if (h <= 1) return 0;
  const int period = 2 * h - 2;
  y = ((y % period) + period) % period;
  return y < h ? y : period - y;
}

// one thread per column: sum the padded rows onto their mirror sources
__global__ void k_ai_fold(AdjGeom g, const float2* __restrict__ u, float* __restrict__ sbar) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= g.w) return;
  const int64_t plane = (int64_t)g.hp * g.pitch;
  for (int r = 0; r < g.hp; ++r) {
    const int sy = mirror101(r - g.pad, g.h);
    const int64_t oi = (int64_t)r * g.pitch + x;
    const float2 v = cadd(u[oi], u[plane + oi]);
    sbar[(int64_t)sy * g.pitch + x] += re_mul(v, car(g, sy, x));
  }
}

__global__ void k_adj_samples(AdjGeom g, const float* __restrict__ sbar, float inv_cpi, int fh,
                              int fw, int fal, int a0, float* __restrict__ out) {
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= fw || y >= fh) return;
  const int ay = y - fal, ax = x - a0;
  float v = 0.f;
  if (ay >= 0 && ay < g.h && ax >= 0 && ax < g.w) v = sbar[(int64_t)ay * g.pitch + ax] * inv_cpi;
  out[(int64_t)y * fw + x] = v;
}

dim3 grid_of(int w, int h) { return dim3((w + kBX - 1) / kBX, (h + kBY - 1) / kBY); }

}  // namespace

int adj_blocks(const AdjGeom& g) {
  const dim3 gr = grid_of(g.w, g.h);
  return (int)(gr.x * gr.y);
}

void launch_adj_output(const AdjGeom& g, const float* ybar, float* sbar, float2* chibar,
                       cudaStream_t st) {
  k_adj_output<<<grid_of(g.w, g.h), dim3(kBX, kBY), 0, st>>>(g, ybar, sbar, chibar);
}

void launch_adj_norm(const AdjGeom& g, const float2* chibar, double* partials, cudaStream_t st) {
  k_adj_norm<<<grid_of(g.w, g.h), dim3(kBX, kBY), 0, st>>>(g, chibar, partials);
}

void launch_adj_rhs(const AdjGeom& g, const float2* chibar, float sigma, float2* B,
                    cudaStream_t st) {
  k_adj_rhs<<<grid_of(g.w, g.h), dim3(kBX, kBY), 0, st>>>(g, chibar, sigma, B);
}

void launch_adj_outer(const AdjGeom& g, const AdjScalars& sc, const AdjOuter& o, double* acc,
                      float* sbar, float2* chibar, cudaStream_t st) {
  k_adj_pass_a<<<grid_of(g.w, g.h), dim3(kBX, kBY), 0, st>>>(g, sc, o);
  k_adj_reduce<<<1, 256, 0, st>>>(o.partials, adj_blocks(g), 4, acc);
  k_adj_pass_b<<<grid_of(g.w, g.h), dim3(kBX, kBY), 0, st>>>(g, o, sbar, chibar);
}

void launch_adj_init_pointwise(const AdjGeom& g, const AdjInit& a, float* sbar, cudaStream_t st) {
  const dim3 gr = grid_of(g.w, g.h), bl(kBX, kBY);
  k_ai_edges<<<gr, bl, 0, st>>>(g, a);
  k_ai_box_v<<<gr, bl, 0, st>>>(g, a.a, a.tmp);
  k_ai_box_h<<<gr, bl, 0, st>>>(g, a.tmp, a.a);          // a -> E
  k_ai_blend<<<gr, bl, 0, st>>>(g, a);
  k_ai_box_v<<<gr, bl, 0, st>>>(g, a.ebar, a.tmp);
  k_ai_box_h<<<gr, bl, 0, st>>>(g, a.tmp, a.ebar);       // ebar -> abar
  k_ai_edges_adjoint<<<gr, bl, 0, st>>>(g, a, a.ebar, sbar);
}

void launch_adj_fold(const AdjGeom& g, const float2* adj_out, float* sbar, cudaStream_t st) {
  k_ai_fold<<<(g.w + 127) / 128, 128, 0, st>>>(g, adj_out, sbar);
}

void launch_adj_samples(const AdjGeom& g, const float* sbar, float inv_cpi, int fh, int fw,
                        int fal, int a0, float* samples_bar, cudaStream_t st) {
  k_adj_samples<<<grid_of(fw, fh), dim3(kBX, kBY), 0, st>>>(g, sbar, inv_cpi, fh, fw, fal, a0,
                                                           samples_bar);
}

}  // namespace hvdg
