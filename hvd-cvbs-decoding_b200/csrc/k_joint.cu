// k_joint.cu -- the anchored pass of the 3-D window.
//
// SynthReference (hvd-core/src/engine/sequence.cpp:52-150): the decoded
// neighbours within nr_radius, bilinearly warped by their per-pixel motion
// with the half-line parity row offset, are blended with Geman-McClure
// weights conf eps_b^2 / (d^2 + eps_b^2); the anchor weight is
// eps_b^2 / (r^2 + eps_b^2), r the 3x3 box of |S - (Ya + Re[Ca c])|.
//
// VariationalRefineJoint (variational.cpp:558-891): Y is a free unknown
// next to chi. Per pixel the data terms (base, neighbours, anchor) form one
// 3x3 quadratic in x = (Y, Re chi, Im chi):
//   sum_t w_t (s_t - u_t . x)^2 + nu_a w_a |x - x_a|^2,   u = (1, Re c, -Im c),
// written as x^T M x - 2 b . x; the spatial Charbonnier priors act on Y and
// chi with the lagged weights (prior-renormalised by 1 + nu sum wt). The
// gradient is g = 2 (M x - b) + 2 L x and the CG runs the same single-
// reduction recurrence as the 2-D solver (g_k = g + a q, q = A d, one
// reduction point per iteration), one sweep launch plus one per-field scalar
// step per iteration, partial sums per block reduced in a fixed order.
#include <cuda_runtime.h>

#include "hvdg_common.cuh"
#include "k_joint.h"

namespace hvdg {

namespace {

constexpr int kBX = 32, kBY = 8;
constexpr int kNP = 5;  // curvature, <g,d>, <g,q>, <q,q>, <g,g>

__device__ __forceinline__ float2 car_at(const float4* lp, const float2* cp, const FieldDesc& f,
                                         int y, int x) {
  const float4 L = __ldg(lp + f.line_off + y);
  return carrier(make_float2(L.x, L.y), __ldg(cp + f.col_off + x), L.z);
}

__device__ __forceinline__ float4 f4(float a, float b, float c) { return make_float4(a, b, c, 0.f); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, 0.f);
}
__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, 0.f);
}
__device__ __forceinline__ float4 sc4(float4 a, float s) {
  return make_float4(a.x * s, a.y * s, a.z * s, 0.f);
}
__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// M v for the packed symmetric matrix
__device__ __forceinline__ float4 mv(float4 m0, float4 m1, float4 v) {
  return f4(m0.x * v.x + m0.y * v.y + m0.z * v.z, m0.y * v.x + m0.w * v.y + m1.x * v.z,
            m0.z * v.x + m1.x * v.y + m1.y * v.z);
}

// L v at one pixel: [DxT(wx Dx vY) + DyT(wy Dy vY), DxT(Wz Dx vC) + DyT(Ww Dy vC)]
// from the centre, its four neighbours and the weights at the centre, left
// and upper pixels (gradients.h:25-101 boundary rules); also the pixel's
// forward-difference energy for the curvature.
struct LapOut {
  float4 lv;
  float energy;
};
__device__ __forceinline__ LapOut lap(float4 c, float4 l, float4 r, float4 u, float4 d, float4 wc,
                                      float4 wl, float4 wu, bool hl, bool hr, bool hu, bool hd) {
  const float4 dxc = hr ? sub4(r, c) : f4(0.f, 0.f, 0.f);
  const float4 dyc = hd ? sub4(d, c) : f4(0.f, 0.f, 0.f);
  const float4 dxl = hl ? sub4(c, l) : f4(0.f, 0.f, 0.f);
  const float4 dyu = hu ? sub4(c, u) : f4(0.f, 0.f, 0.f);
  // DxT(a)(x) = a(x - 1) - a(x); a = weight * forward difference
  LapOut o;
  o.lv.x = (wl.x * dxl.x - wc.x * dxc.x) + (wu.y * dyu.x - wc.y * dyc.x);
  o.lv.y = (wl.z * dxl.y - wc.z * dxc.y) + (wu.w * dyu.y - wc.w * dyc.y);
  o.lv.z = (wl.z * dxl.z - wc.z * dxc.z) + (wu.w * dyu.z - wc.w * dyc.z);
  o.lv.w = 0.f;
  o.energy = wc.x * dxc.x * dxc.x + wc.y * dyc.x * dyc.x +
             wc.z * (dxc.y * dxc.y + dxc.z * dxc.z) + wc.w * (dyc.y * dyc.y + dyc.z * dyc.z);
  return o;
}

// The oriented chroma prior's part of L v at one pixel (gradients.h:195-279):
// D1T(w1 D1 v) + D2T(w2 D2 v) on the chroma components, with
// D1 v(y, x) = v(y+1, x+1) - v(y, x), D2 v(y, x) = v(y+1, x-1) - v(y, x)
// (zero on the last row, last / first column), the adjoints gathered as
// D1T p (y, x) = -p(y, x) + p(y-1, x-1), D2T p (y, x) = -p(y, x) + p(y-1, x+1);
// w = (mu_d wd1, mu_d wd2) at the pixel (wc), its upper-left (wul) and
// upper-right (wur) neighbours; adds the pixel's forward energy too.
struct DiagNb {
  float4 dr, dl, ul, ur;   // v at (y+1, x+1), (y+1, x-1), (y-1, x-1), (y-1, x+1)
  float4 wc, wul, wur;
  bool e1, e2, e1u, e2u;   // D1 / D2 exist at the pixel, at (y-1, x-1) / (y-1, x+1)
};
__device__ __forceinline__ void diag_lap(const DiagNb& n, float4 c, LapOut& o) {
  const float z = 0.f;
  const float p1y = n.e1 ? n.wc.x * (n.dr.y - c.y) : z, p1z = n.e1 ? n.wc.x * (n.dr.z - c.z) : z;
  const float p2y = n.e2 ? n.wc.y * (n.dl.y - c.y) : z, p2z = n.e2 ? n.wc.y * (n.dl.z - c.z) : z;
  const float q1y = n.e1u ? n.wul.x * (c.y - n.ul.y) : z, q1z = n.e1u ? n.wul.x * (c.z - n.ul.z) : z;
  const float q2y = n.e2u ? n.wur.y * (c.y - n.ur.y) : z, q2z = n.e2u ? n.wur.y * (c.z - n.ur.z) : z;
  o.lv.y += (q1y - p1y) + (q2y - p2y);
  o.lv.z += (q1z - p1z) + (q2z - p2z);
  const float d1y = n.e1 ? n.dr.y - c.y : z, d1z = n.e1 ? n.dr.z - c.z : z;
  const float d2y = n.e2 ? n.dl.y - c.y : z, d2z = n.e2 ? n.dl.z - c.z : z;
  o.energy += (n.e1 ? n.wc.x : z) * (d1y * d1y + d1z * d1z) +
              (n.e2 ? n.wc.y : z) * (d2y * d2y + d2z * d2z);
}

template <int N>
__device__ void block_sum(double (&v)[N], double* sh) {
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = t & 31, warp = t >> 5, nw = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < N; ++i) sh[warp * N + i] = v[i];
  __syncthreads();
  if (t == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double s = 0.0;
      for (int j = 0; j < nw; ++j) s += sh[j * N + i];
      v[i] = s;
    }
  }
}

__device__ __forceinline__ int64_t part_index(const JointArgs& a, int fi) {
  return ((int64_t)fi * a.by * a.bx + (int64_t)blockIdx.y * a.bx + blockIdx.x) * kNP;
}

__global__ void k_joint_load(JointArgs a, const float* __restrict__ Y,
                             const float2* __restrict__ chi) {
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x == 0 && y == 0) {
    JointCtl& c = a.ctl[a.flist[fi]];
    c.gg = c.gg0 = 0.0;
    c.alpha = c.beta = 0.f;
    c.pending = c.sel = c.done = c.iters = 0;
  }
  if (x >= f.w || y >= f.h) return;
  const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
  const float2 cv = chi[o];
  a.X[o] = f4(Y[o], cv.x, cv.y);
}

// weights (lagged), neighbour robust weights, prior scale, data matrix
__global__ void k_joint_setup(JointArgs a) {
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int64_t lo = (int64_t)y * f.pitch + x;
  const int64_t o = f.px_off + lo;
  const bool hx = x + 1 < f.w, hy = y + 1 < f.h;
  const float4 c0 = a.X[o];
  const float4 cr = hx ? a.X[o + 1] : c0, cd = hy ? a.X[o + f.pitch] : c0;
  const float gx = hx ? cr.x - c0.x : 0.f, gy = hy ? cd.x - c0.x : 0.f;
  const float dcxr = hx ? cr.y - c0.y : 0.f, dcxi = hx ? cr.z - c0.z : 0.f;
  const float dcyr = hy ? cd.y - c0.y : 0.f, dcyi = hy ? cd.z - c0.z : 0.f;
  const float e2 = a.eps * a.eps, ec2 = a.eps_c * a.eps_c;
  const float wx = a.eps / sqrtf(gx * gx + e2);
  const float wy = a.eps / sqrtf(gy * gy + e2);
  const float magx = sqrtf(dcxr * dcxr + dcxi * dcxi), magy = sqrtf(dcyr * dcyr + dcyi * dcyi);
  const float wcx = a.eps_c / sqrtf(magx * magx + a.k * gx * gx + ec2);
  const float wcy = a.eps_c / sqrtf(magy * magy + a.k * gy * gy + ec2);
  const float2 c = car_at(a.line_phasor, a.col_phasor, f, y, x);
  const float Sv = a.S[o];
  // base data term, weight 1: u = (1, Re c, -Im c)
  float m00 = 1.f, m01 = c.x, m02 = -c.y, m11 = c.x * c.x, m12 = -c.x * c.y, m22 = c.y * c.y;
  float b0 = Sv, b1 = Sv * c.x, b2 = -Sv * c.y;
  float ps = 1.f;
  const float nu = f.n_nbr > 0 ? a.nu : 0.f;
  const float et2 = a.eps_t * a.eps_t;
  for (int j = 0; j < f.n_nbr; ++j) {
    const float4 nb = a.nbr[f.nbr_off + (int64_t)j * f.plane_px + lo];
    const float cwx = c.x - nb.y, cwy = c.y - nb.z;   // c_w = c - dc
    const float Sw = Sv + nb.x;
    const float rk = Sw - c0.x - (c0.y * cwx - c0.z * cwy);
    const float wt = nb.w * et2 / (rk * rk + et2);
    const float sw = nu * wt;
    const float u1 = cwx, u2 = -cwy;
    m00 += sw;
    m01 += sw * u1;
    m02 += sw * u2;
    m11 += sw * u1 * u1;
    m12 += sw * u1 * u2;
    m22 += sw * u2 * u2;
    b0 += sw * Sw;
    b1 += sw * Sw * u1;
    b2 += sw * Sw * u2;
    ps += sw;
  }
  if (a.nu_a > 0.f) {
    const float wa = a.nu_a * a.Wa[o];
    const float2 ca = a.Ca[o];
    m00 += wa;
    m11 += wa;
    m22 += wa;
    b0 += wa * a.Ya[o];
    b1 += wa * ca.x;
    b2 += wa * ca.y;
  }
  a.W[o] = make_float4(wx * ps, wy * ps, f.mu_h * (wcx * ps), f.mu_v * (wcy * ps));
  if (a.diag) {
    // oriented diffusivities of chi (variational.cpp:787-797, prior-scaled :838-841)
    const bool e1 = hy && hx, e2 = hy && x >= 1;
    const float4 c11 = e1 ? a.X[o + f.pitch + 1] : c0, c1m = e2 ? a.X[o + f.pitch - 1] : c0;
    const float d1r = c11.y - c0.y, d1i = c11.z - c0.z, d2r = c1m.y - c0.y, d2i = c1m.z - c0.z;
    const float c1 = sqrtf(d1r * d1r + d1i * d1i) / a.eps_c;
    const float c2 = sqrtf(d2r * d2r + d2i * d2i) / a.eps_c;
    const float wd1 = 1.0f / sqrtf(1.0f + c1 * c1), wd2 = 1.0f / sqrtf(1.0f + c2 * c2);
    a.W2[o] = make_float4(f.mu_d * (wd1 * ps), f.mu_d * (wd2 * ps), 0.f, 0.f);
  }
  a.M0[o] = make_float4(m00, m01, m02, m11);
  a.M1[o] = make_float4(m12, m22, b0, b1);
  a.M2[o] = b2;
}

// g(x) = 2 (M x - b) + 2 L x -> G[0], partial ||g||^2
__global__ void k_joint_grad(JointArgs a) {
  __shared__ double sh[kNP * kBX * kBY / 32];
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  double v[kNP] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (x < f.w && y < f.h) {
    const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
    const bool hl = x > 0, hr = x + 1 < f.w, hu = y > 0, hd = y + 1 < f.h;
    const float4 c = a.X[o];
    const float4 l = hl ? a.X[o - 1] : c, r = hr ? a.X[o + 1] : c;
    const float4 u = hu ? a.X[o - f.pitch] : c, d = hd ? a.X[o + f.pitch] : c;
    const float4 wc = a.W[o];
    const float4 wl = hl ? a.W[o - 1] : wc, wu = hu ? a.W[o - f.pitch] : wc;
    LapOut L = lap(c, l, r, u, d, wc, wl, wu, hl, hr, hu, hd);
    if (a.diag) {
      DiagNb n;
      n.e1 = hd && hr;
      n.e2 = hd && hl;
      n.e1u = hu && hl;
      n.e2u = hu && hr;
      n.dr = n.e1 ? a.X[o + f.pitch + 1] : c;
      n.dl = n.e2 ? a.X[o + f.pitch - 1] : c;
      n.ul = n.e1u ? a.X[o - f.pitch - 1] : c;
      n.ur = n.e2u ? a.X[o - f.pitch + 1] : c;
      n.wc = a.W2[o];
      n.wul = n.e1u ? a.W2[o - f.pitch - 1] : n.wc;
      n.wur = n.e2u ? a.W2[o - f.pitch + 1] : n.wc;
      diag_lap(n, c, L);
    }
    const float4 m0 = a.M0[o], m1 = a.M1[o];
    const float4 b = f4(m1.z, m1.w, a.M2[o]);
    const float4 g = sc4(add4(sub4(mv(m0, m1, c), b), L.lv), 2.f);
    a.G[0][o] = g;
    v[4] = (double)dot4(g, g);
  }
  block_sum<kNP>(v, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double* dst = a.partials + part_index(a, fi);
    for (int i = 0; i < kNP; ++i) dst[i] = v[i];
  }
}

// gg0 = gg = ||g||^2, control reset for the outer
__global__ void k_joint_ctl_start(JointArgs a) {
  __shared__ double sh[kNP * 256 / 32];
  const int fi = blockIdx.x;
  const int nb = a.bx * a.by;
  double v[kNP] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    v[4] += a.partials[((int64_t)fi * nb + b) * kNP + 4];
  block_sum<kNP>(v, sh);
  if (threadIdx.x == 0) {
    JointCtl& c = a.ctl[a.flist[fi]];
    c.gg = c.gg0 = v[4];
    c.pending = 0;
    c.sel = 0;
    c.done = 0;
    c.alpha = c.beta = 0.f;
  }
}

// one fused CG sweep: pending step, g_k, d_k, q_k = A d_k and the partials
__global__ void k_joint_sweep(JointArgs a, int first) {
  __shared__ double sh[kNP * kBX * kBY / 32];
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const JointCtl c = a.ctl[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  double v[kNP] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (!c.done && x < f.w && y < f.h) {
    const int s = c.sel;
    const float al = c.alpha, be = c.beta;
    const float4* G = a.G[s];
    const float4* Q = a.Q[s];
    const float4* D = a.D[s];
    auto dk = [&](int64_t oo) {
      const float4 g = G[oo];
      if (first) return sc4(g, -1.f);
      const float4 gk = add4(g, sc4(Q[oo], al));
      return add4(sc4(gk, -1.f), sc4(D[oo], be));
    };
    const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
    const bool hl = x > 0, hr = x + 1 < f.w, hu = y > 0, hd = y + 1 < f.h;
    const float4 g0 = G[o];
    const float4 gk = first ? g0 : add4(g0, sc4(Q[o], al));
    const float4 dc = dk(o);
    const float4 dl = hl ? dk(o - 1) : dc, dr = hr ? dk(o + 1) : dc;
    const float4 du = hu ? dk(o - f.pitch) : dc, dd = hd ? dk(o + f.pitch) : dc;
    const float4 wc = a.W[o];
    const float4 wl = hl ? a.W[o - 1] : wc, wu = hu ? a.W[o - f.pitch] : wc;
    LapOut L = lap(dc, dl, dr, du, dd, wc, wl, wu, hl, hr, hu, hd);
    if (a.diag) {
      DiagNb n;
      n.e1 = hd && hr;
      n.e2 = hd && hl;
      n.e1u = hu && hl;
      n.e2u = hu && hr;
      n.dr = n.e1 ? dk(o + f.pitch + 1) : dc;
      n.dl = n.e2 ? dk(o + f.pitch - 1) : dc;
      n.ul = n.e1u ? dk(o - f.pitch - 1) : dc;
      n.ur = n.e2u ? dk(o - f.pitch + 1) : dc;
      n.wc = a.W2[o];
      n.wul = n.e1u ? a.W2[o - f.pitch - 1] : n.wc;
      n.wur = n.e2u ? a.W2[o - f.pitch + 1] : n.wc;
      diag_lap(n, dc, L);
    }
    const float4 m0 = a.M0[o], m1 = a.M1[o];
    const float4 md = mv(m0, m1, dc);
    const float4 qk = sc4(add4(md, L.lv), 2.f);
    v[0] = (double)(dot4(dc, md) + L.energy);
    v[1] = (double)dot4(gk, dc);
    v[2] = (double)dot4(gk, qk);
    v[3] = (double)dot4(qk, qk);
    v[4] = (double)dot4(gk, gk);
    a.G[s ^ 1][o] = gk;
    a.D[s ^ 1][o] = dc;
    a.Q[s ^ 1][o] = qk;
    if (!first) a.X[o] = add4(a.X[o], sc4(D[o], al));
  }
  block_sum<kNP>(v, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double* dst = a.partials + part_index(a, fi);
    for (int i = 0; i < kNP; ++i) dst[i] = v[i];
  }
}

// the scalar step of the recurrence (variational.cpp:519-549 with the
// single-reduction rewrite), per field
__global__ void k_joint_step(JointArgs a) {
  __shared__ double sh[kNP * 256 / 32];
  const int fi = blockIdx.x;
  const int fidx = a.flist[fi];
  const int nb = a.bx * a.by;
  double v[kNP] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
    for (int i = 0; i < kNP; ++i) v[i] += a.partials[((int64_t)fi * nb + b) * kNP + i];
  block_sum<kNP>(v, sh);
  if (threadIdx.x != 0) return;
  JointCtl& c = a.ctl[fidx];
  if (c.done) return;
  const FieldDesc f = a.fields[fidx];
  const double H = v[0], gd = v[1], gq = v[2], qq = v[3], ggk = v[4];
  c.sel ^= 1;
  c.gg = ggk;
  if (H <= 1e-12) {
    c.pending = 0;
    c.done = 1;
    return;
  }
  const float al = (float)(-0.5 * gd / H);
  const double gn = ggk + 2.0 * (double)al * gq + (double)al * (double)al * qq;
  c.alpha = al;
  c.beta = (float)(gn / fmax(ggk, 1e-30));
  c.pending = 1;
  c.iters += 1;
  const double tol = (double)f.cg_tol;
  if (gn < tol * tol * c.gg0 || gn < 1e-10 * (double)f.h * (double)f.w) c.done = 1;
}

// apply the pending step (end of an outer)
__global__ void k_joint_apply(JointArgs a) {
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const JointCtl c = a.ctl[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (!c.pending || x >= f.w || y >= f.h) return;
  const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
  a.X[o] = add4(a.X[o], sc4(a.D[c.sel][o], c.alpha));
}

__global__ void k_joint_clear_pending(JointArgs a) {
  const int fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi < a.nfl) a.ctl[a.flist[fi]].pending = 0;
}

__global__ void k_joint_store(JointArgs a, float* __restrict__ Y, float2* __restrict__ chi,
                              int fidelity) {
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
  const float4 v = a.X[o];
  chi[o] = make_float2(v.y, v.z);
  if (fidelity) {
    const float2 c = car_at(a.line_phasor, a.col_phasor, f, y, x);
    Y[o] = a.S[o] - (v.y * c.x - v.z * c.y);
  } else {
    Y[o] = v.x;
  }
}

__global__ void k_output_fidelity(JointArgs a, float* __restrict__ Y,
                                  const float2* __restrict__ chi) {
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int64_t o = f.px_off + (int64_t)y * f.pitch + x;
  const float2 c = car_at(a.line_phasor, a.col_phasor, f, y, x);
  const float2 v = chi[o];
  Y[o] = a.S[o] - (v.x * c.x - v.y * c.y);
}

// ---- SynthReference --------------------------------------------------------
__device__ __forceinline__ int clampi_j(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// VectorsPerPixel's bilinear interpolation between tile centres
// (temporal.cpp:45-112); the same formulas as the neighbour warps.
__device__ __forceinline__ void bracket_j(int coord, int n_tiles, int tile, int* lo, float* frac) {
  if (n_tiles > 1) {
    const float rel = (float)coord / (float)tile - 0.5f;
    *lo = clampi_j((int)floorf(rel), 0, n_tiles - 2);
    const float centre_lo = ((float)*lo + 0.5f) * (float)tile;
    *frac = fminf(fmaxf(((float)coord - centre_lo) / (float)tile, 0.0f), 1.0f);
  } else {
    *lo = 0;
    *frac = 0.0f;
  }
}

__device__ __forceinline__ float interp_j(const float* v, int tw, int iy, int iy1, int ix, int ix1,
                                          float fy, float fx) {
  const float v00 = v[iy * tw + ix], v10 = v[iy1 * tw + ix];
  const float v01 = v[iy * tw + ix1], v11 = v[iy1 * tw + ix1];
  return v00 * (1 - fy) * (1 - fx) + v10 * fy * (1 - fx) + v01 * (1 - fy) * fx + v11 * fy * fx;
}

__global__ void k_anchor_blend(AnchorArgs a) {
  const int gi = blockIdx.z;
  if (gi >= a.ngroups) return;
  const AnchorGroup G = a.groups[gi];
  const FieldDesc f = a.fields[G.field];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int64_t lo = (int64_t)y * f.pitch + x;
  const int64_t o = f.px_off + lo;
  const float Yj = a.Y[o];
  const float2 Cj = a.chi[o];
  float accY = Yj, accW = 1.0f;
  float2 accC = Cj;
  const int th = (f.h + a.tile - 1) / a.tile, tw = (f.w + a.tile - 1) / a.tile;
  int iy, ix;
  float fyb, fxb;
  bracket_j(y, th, a.tile, &iy, &fyb);
  bracket_j(x, tw, a.tile, &ix, &fxb);
  const int iy1 = min(iy + 1, th - 1), ix1 = min(ix + 1, tw - 1);
  const float eb2 = a.eps_b * a.eps_b;
  for (int q = 0; q < G.count; ++q) {
    const AnchorPair P = G.p[q];
    const FieldDesc fk = a.fields[P.k];
    const int to = a.tiles_off * P.pair;
    const float vy = interp_j(a.snap_dy + to, tw, iy, iy1, ix, ix1, fyb, fxb);
    const float vx = interp_j(a.snap_dx + to, tw, iy, iy1, ix, ix1, fyb, fxb);
    // WarpBilinearTiles (temporal.cpp:140-168)
    float sy = (float)y - vy + P.row_off;
    float sx = (float)x - vx;
    sy = fminf(fmaxf(sy, 0.0f), (float)fk.h - 1.001f);
    sx = fminf(fmaxf(sx, 0.0f), (float)fk.w - 1.001f);
    const int y0 = (int)sy, x0 = (int)sx;
    const float fy = sy - (float)y0, fx = sx - (float)x0;
    const int y1 = min(y0 + 1, fk.h - 1), x1 = min(x0 + 1, fk.w - 1);
    const int64_t b00 = fk.px_off + (int64_t)y0 * fk.pitch + x0;
    const int64_t b10 = fk.px_off + (int64_t)y1 * fk.pitch + x0;
    const int64_t b01 = fk.px_off + (int64_t)y0 * fk.pitch + x1;
    const int64_t b11 = fk.px_off + (int64_t)y1 * fk.pitch + x1;
    const float w00 = (1 - fy) * (1 - fx), w10 = fy * (1 - fx), w01 = (1 - fy) * fx, w11 = fy * fx;
    const float Yw = a.Y[b00] * w00 + a.Y[b10] * w10 + a.Y[b01] * w01 + a.Y[b11] * w11;
    const float2 k00 = a.chi[b00], k10 = a.chi[b10], k01 = a.chi[b01], k11 = a.chi[b11];
    const float cwr = k00.x * w00 + k10.x * w10 + k01.x * w01 + k11.x * w11;
    const float cwi = k00.y * w00 + k10.y * w10 + k01.y * w01 + k11.y * w11;
    const float conf = a.conf_px[a.pix_off[P.pair] + lo];
    const float dy = Yw - Yj;
    const float er = cwr - Cj.x, ei = cwi - Cj.y;
    const float d2 = dy * dy + (er * er + ei * ei);
    const float w = conf * eb2 / (d2 + eb2);
    accY += w * Yw;
    accC.x += w * cwr;
    accC.y += w * cwi;
    accW += w;
  }
  const float ya = accY / accW;
  const float2 ca = make_float2(accC.x / accW, accC.y / accW);
  a.Ya[o] = ya;
  a.Ca[o] = ca;
  const float2 c = car_at(a.line_phasor, a.col_phasor, f, y, x);
  const float s_hat = ya + (ca.x * c.x - ca.y * c.y);
  a.resid[o] = fabsf(a.S[o] - s_hat);
}

// anchor weight from the 3x3 box (zero padded, 1/3 per axis) of the residual
__global__ void k_anchor_weight(AnchorArgs a) {
  const int gi = blockIdx.z;
  if (gi >= a.ngroups) return;
  const FieldDesc f = a.fields[a.groups[gi].field];
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= f.w || y >= f.h) return;
  float s = 0.f;
  for (int yy = y - 1; yy <= y + 1; ++yy) {
    if (yy < 0 || yy >= f.h) continue;
    float rs = 0.f;
    for (int xx = x - 1; xx <= x + 1; ++xx)
      if (xx >= 0 && xx < f.w) rs += a.resid[f.px_off + (int64_t)yy * f.pitch + xx];
    s += rs * (1.0f / 3.0f);
  }
  const float r = s * (1.0f / 3.0f);
  const float eb2 = a.eps_b * a.eps_b;
  a.Wa[f.px_off + (int64_t)y * f.pitch + x] = eb2 / (r * r + eb2);
}

__global__ void k_psi_init(JointArgs a, float2* __restrict__ chi) {
  const int fi = blockIdx.z;
  const FieldDesc f = a.fields[a.flist[fi]];
  if (f.n_nbr <= 0) return;
  const int x = blockIdx.x * kBX + threadIdx.x, y = blockIdx.y * kBY + threadIdx.y;
  if (x >= f.w || y >= f.h) return;
  const int64_t lo = (int64_t)y * f.pitch + x;
  const int64_t o = f.px_off + lo;
  const float kEpsT = 6.0f;  // the refine's robust gate at the init point
  double a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0;
  double b1 = 0, b2 = 0, b3 = 0;
  double wsum = 0.0;
  auto add = [&](float Sk, float2 ck, float wk) {
    const double rc = ck.x, ic = -ck.y;
    a11 += wk;
    a12 += wk * rc;
    a13 += wk * ic;
    a22 += wk * rc * rc;
    a23 += wk * rc * ic;
    a33 += wk * ic * ic;
    b1 += wk * Sk;
    b2 += wk * Sk * rc;
    b3 += wk * Sk * ic;
  };
  const float2 c = car_at(a.line_phasor, a.col_phasor, f, y, x);
  const float Sv = a.S[o];
  const float2 cf = chi[o];
  add(Sv, c, 1.0f);
  for (int j = 0; j < f.n_nbr; ++j) {
    const float4 nb = a.nbr[f.nbr_off + (int64_t)j * f.plane_px + lo];
    // neighbour composite S + (S_w - S), carrier c - dc
    const float2 cw = make_float2(c.x - nb.y, c.y - nb.z);
    const float rt = nb.x + (cf.x * nb.y - cf.y * nb.z);
    const float wk = nb.w * kEpsT * kEpsT / (rt * rt + kEpsT * kEpsT);
    add(Sv + nb.x, cw, wk);
    wsum += wk;
  }
  const double det = a11 * (a22 * a33 - a23 * a23) - a12 * (a12 * a33 - a23 * a13) +
                     a13 * (a12 * a23 - a22 * a13);
  const double a11c = fmax(a11, 1e-9);
  const bool ok = det > 1e-3 * a11c * a11c * a11c * 0.01;
  const double d = ok ? det : 1.0;
  const double q1 = (a11 * (b2 * a33 - b3 * a23) - b1 * (a12 * a33 - a23 * a13) +
                     a13 * (a12 * b3 - b2 * a13)) / d;
  const double q2 = (a11 * (a22 * b3 - a23 * b2) - a12 * (a12 * b3 - b2 * a13) +
                     b1 * (a12 * a23 - a22 * a13)) / d;
  const float t = ok ? fminf(fmaxf((float)(wsum / 2.0), 0.0f), 1.0f) : 0.0f;
  chi[o] = make_float2(t * (float)q1 + (1.0f - t) * cf.x, t * (float)q2 + (1.0f - t) * cf.y);
}

dim3 jgrid(int max_w, int max_h, int n) {
  return dim3((max_w + kBX - 1) / kBX, (max_h + kBY - 1) / kBY, n);
}

}  // namespace

void launch_joint_load(const JointArgs& a, const float* Y, const float2* chi, int max_h, int max_w,
                       cudaStream_t st) {
  if (a.nfl <= 0) return;
  k_joint_load<<<jgrid(max_w, max_h, a.nfl), dim3(kBX, kBY), 0, st>>>(a, Y, chi);
}

void launch_joint_outer(const JointArgs& a, int n_inner, int max_h, int max_w, cudaStream_t st) {
  if (a.nfl <= 0) return;
  const dim3 gr = jgrid(max_w, max_h, a.nfl), bl(kBX, kBY);
  k_joint_setup<<<gr, bl, 0, st>>>(a);
  k_joint_grad<<<gr, bl, 0, st>>>(a);
  k_joint_ctl_start<<<a.nfl, 256, 0, st>>>(a);
  for (int it = 0; it < n_inner; ++it) {
    k_joint_sweep<<<gr, bl, 0, st>>>(a, it == 0 ? 1 : 0);
    k_joint_step<<<a.nfl, 256, 0, st>>>(a);
  }
  k_joint_apply<<<gr, bl, 0, st>>>(a);
  k_joint_clear_pending<<<(a.nfl + 63) / 64, 64, 0, st>>>(a);
}

void launch_joint_store(const JointArgs& a, float* Y, float2* chi, bool output_fidelity,
                        int max_h, int max_w, cudaStream_t st) {
  if (a.nfl <= 0) return;
  k_joint_store<<<jgrid(max_w, max_h, a.nfl), dim3(kBX, kBY), 0, st>>>(a, Y, chi,
                                                                       output_fidelity ? 1 : 0);
}

void launch_output_fidelity(const JointArgs& a, float* Y, const float2* chi, int max_h, int max_w,
                            cudaStream_t st) {
  if (a.nfl <= 0) return;
  k_output_fidelity<<<jgrid(max_w, max_h, a.nfl), dim3(kBX, kBY), 0, st>>>(a, Y, chi);
}

void launch_anchor(const AnchorArgs& a, int max_h, int max_w, cudaStream_t st) {
  if (a.ngroups <= 0) return;
  const dim3 gr = jgrid(max_w, max_h, a.ngroups), bl(kBX, kBY);
  k_anchor_blend<<<gr, bl, 0, st>>>(a);
  k_anchor_weight<<<gr, bl, 0, st>>>(a);
}

void launch_psi_init(const JointArgs& a, float2* chi, int max_h, int max_w, cudaStream_t st) {
  if (a.nfl <= 0) return;
  k_psi_init<<<jgrid(max_w, max_h, a.nfl), dim3(kBX, kBY), 0, st>>>(a, chi);
}

}  // namespace hvdg
