// k_solver.cu -- persistent IRLS + conjugate-gradient Y/C arbitration
// (kernel c) over a batch of fields of any geometry.
//
// Reference: VariationalRefine (hvd-core/src/engine/variational.cpp:198-556):
// per IRLS outer pass, Charbonnier / coupled diffusivities at the current
// chi (:406-433), then CG on the fixed-weight quadratic with
//   alpha = -0.5 <g,d> / curv(d),  beta = ||g'||^2 / ||g||^2  (:519-549),
// the gradient g(chi) = -2[DxT(wx Dx Yc) + DyT(wy Dy Yc)] conj(c)
//                       + 2[mu_h DxT(wcx Dx chi) + mu_v DyT(wcy Dy chi)]
// (:286-347), FP64 inner products (:72-95), early exits (:530, :547-548).
//
// B200 formulation (same iterates in exact arithmetic):
//  * The gradient is affine in chi, so g(chi + a d) = g(chi) + a q with
//    q = g(d) - g(0) (the stencil applied to d with S = 0), and
//    curv(d) = sum wx (Dx dY)^2 + ... is computed from the same differences.
//    One CG iteration is ONE fused sweep: apply the pending step
//    (chi += a d, g += a q), form d = -g + b d, compute q = A d, and
//    accumulate <curv>, <g,d>, <g,q>, <q,q>, <g,g> in FP64. The next ||g||^2
//    follows from ||g + a q||^2 = gg + 2a gq + a^2 qq, so each iteration
//    needs one reduction point instead of two; gg itself is re-measured
//    exactly every sweep.
//  * Work is split into units (64-column strip x band of rows, one warp).
//    Units of all fields and all phases form one ordered queue; a warp takes
//    the next item, waits (bounded) until its field completed the previous
//    phase. Units arrive in groups of 32 consecutive units: the last unit
//    of a group sums the group's partials, and the last group of the field
//    sums the group sums and publishes the field's scalars, both in a fixed
//    order. Fields therefore progress independently with no grid-wide
//    barrier, the reduction is deterministic, and the end of a phase waits
//    on two short reductions instead of one over every unit.
//  * Planes read with a halo are double-buffered (chi, g, d, q) so a unit
//    never reads a neighbour's freshly written rows.
//  * Each lane owns two adjacent pixels (128-bit loads of complex pairs);
//    horizontal neighbours come from warp shuffles, vertical neighbours from
//    a rolling window of rows kept in registers.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "hvdg_common.cuh"
#include "k_solver.h"
#include "per_device.h"

namespace hvdg {

constexpr int kNPart = 5;
constexpr int kNS = 4;  // ring slots per warp (I phase)

__device__ __forceinline__ void ld_pair(const float2* p, float2& a, float2& b) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
  a = make_float2(v.x, v.y);
  b = make_float2(v.z, v.w);
}
__device__ __forceinline__ void st_pair(float2* p, float2 a, float2 b, bool va, bool vb) {
  if (va && vb) {
    __stcg(reinterpret_cast<float4*>(p), make_float4(a.x, a.y, b.x, b.y));
  } else {
    if (va) __stcg(p, a);
    if (vb) __stcg(p + 1, b);
  }
}
__device__ __forceinline__ void ld_pairf(const float* p, float& a, float& b) {
  const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
  a = v.x;
  b = v.y;
}

struct Lanes {
  int xa, xb, hx;
  bool va, vb, hv;
  float2 Pa, Pb, Ph;
};

__device__ __forceinline__ Lanes make_lanes(const SolverArgs& A, const FieldDesc& f, int x0,
                                            int lane) {
  Lanes l;
  l.xa = x0 + 2 * lane;
  l.xb = l.xa + 1;
  l.va = l.xa < f.w;
  l.vb = l.xb < f.w;
  l.hx = lane == 0 ? x0 - 1 : x0 + kStrip;
  l.hv = (lane == 0 && x0 > 0) || (lane == 31 && x0 + kStrip < f.w);
  const float2* P = A.col_phasor + f.col_off;
  l.Pa = l.va ? __ldg(P + l.xa) : make_float2(0.f, 0.f);
  l.Pb = l.vb ? __ldg(P + l.xb) : make_float2(0.f, 0.f);
  l.Ph = l.hv ? __ldg(P + l.hx) : make_float2(0.f, 0.f);
  return l;
}

// ---------------------------------------------------------------------------
// Oriented (+-45 deg) chroma prior, diag_prior > 0 (variational.cpp:316-328,
// 371-383; gradients.h:195-279): the fluxes p1 = wd1 D1 u and p2 = wd2 D2 u
// of one row y (u = chi in the gradient, u = d in the CG sweep), with
//   D1 u(y, x) = u(y+1, x+1) - u(y, x)   (0 on the last row / column),
//   D2 u(y, x) = u(y+1, x-1) - u(y, x)   (0 on the last row / first column);
// the adjoints gather D1T p1 (y, x) = -p1(y, x) + p1(y-1, x-1) and
// D2T p2 (y, x) = -p2(y, x) + p2(y-1, x+1), so each row's fluxes are kept
// for the next row, plus one halo flux per strip edge: lane 0 carries
// p1(y, x0-1), lane 31 p2(y, x0+64). `hd` is the row's weighted energy
// wd1 |D1 u|^2 + wd2 |D2 u|^2 over this lane's pixels (the curvature term).
// ---------------------------------------------------------------------------
struct DiagFlux {
  float2 p1a, p1b, p2a, p2b, ph;
};

__device__ __forceinline__ void diag_flux(const Lanes& l, const FieldDesc& f, int lane, bool hn,
                                          float2 ua, float2 ub, float2 uh, float2 na, float2 nb,
                                          float2 nh, float2 wda, float2 wdb, float2 wdh,
                                          DiagFlux& o, float& hd) {
  // row y+1 at x+1 for pixel b and at x-1 for pixel a (neighbour lanes, or
  // the row's halo at the strip edges: lane 31 holds x0+64, lane 0 x0-1)
  float2 n_r = make_float2(__shfl_down_sync(0xffffffffu, na.x, 1),
                           __shfl_down_sync(0xffffffffu, na.y, 1));
  float2 n_l = make_float2(__shfl_up_sync(0xffffffffu, nb.x, 1),
                           __shfl_up_sync(0xffffffffu, nb.y, 1));
  if (lane == 31) n_r = nh;
  if (lane == 0) n_l = nh;
  const float2 z = make_float2(0.f, 0.f);
  // weights are read only where the difference exists (the planes' padding
  // columns hold no weights)
  const bool e1a = hn && l.xa < f.w - 1, e1b = hn && l.xb < f.w - 1;
  const bool e2a = hn && l.va && l.xa >= 1, e2b = hn && l.vb;
  const float2 d1a = e1a ? csub(nb, ua) : z;
  const float2 d1b = e1b ? csub(n_r, ub) : z;
  const float2 d2a = e2a ? csub(n_l, ua) : z;
  const float2 d2b = e2b ? csub(na, ub) : z;
  const float w1a = e1a ? wda.x : 0.f, w1b = e1b ? wdb.x : 0.f;
  const float w2a = e2a ? wda.y : 0.f, w2b = e2b ? wdb.y : 0.f;
  o.p1a = cscale(d1a, w1a);
  o.p1b = cscale(d1b, w1b);
  o.p2a = cscale(d2a, w2a);
  o.p2b = cscale(d2b, w2b);
  hd = (w1a * cnorm(d1a) + w2a * cnorm(d2a)) + (w1b * cnorm(d1b) + w2b * cnorm(d2b));
  o.ph = z;
  if (hn && l.hv) {
    if (lane == 0)
      o.ph = cscale(csub(na, uh), wdh.x);  // p1(y, x0-1): u(y+1, x0) - u(y, x0-1)
    else
      o.ph = cscale(csub(nb, uh), wdh.y);  // p2(y, x0+64): u(y+1, x0+63) - u(y, x0+64)
  }
}

// D1T p1 + D2T p2 at this lane's two pixels of row y, from the row's fluxes
// `c` and the previous row's `p` (zero above the first row).
__device__ __forceinline__ void diag_adjoint(int lane, const DiagFlux& c, const DiagFlux& p,
                                             float2& ta, float2& tb) {
  float2 q1l = make_float2(__shfl_up_sync(0xffffffffu, p.p1b.x, 1),
                           __shfl_up_sync(0xffffffffu, p.p1b.y, 1));
  float2 q2r = make_float2(__shfl_down_sync(0xffffffffu, p.p2a.x, 1),
                           __shfl_down_sync(0xffffffffu, p.p2a.y, 1));
  if (lane == 0) q1l = p.ph;   // p1(y-1, x0-1)
  if (lane == 31) q2r = p.ph;  // p2(y-1, x0+64)
  ta = cadd(csub(q1l, c.p1a), csub(p.p2b, c.p2a));
  tb = cadd(csub(p.p1a, c.p1b), csub(q2r, c.p2b));
}

// ---------------------------------------------------------------------------
// R phase: apply the pending step, recompute the IRLS weights (lagged
// diffusivity, variational.cpp:406-433) and, with neighbours, their robust
// weights, prior renormalisation and the pointwise 2x2 data term.
// ---------------------------------------------------------------------------
struct RRow {
  float2 ca, cb, xa_, xb_, xh;
  float ya, yb, yh;
  float Sa, Sb;
};

__device__ __forceinline__ void r_form(const SolverArgs& A, const FieldDesc& f, const Lanes& l,
                                       const float2* X, const float2* D, const float* S,
                                       bool pend, float alpha, int y, RRow& r) {
  const int64_t o = (int64_t)y * f.pitch + l.xa;
  const float4 L = __ldg(A.line_phasor + f.line_off + y);
  const float2 Lc = make_float2(L.x, L.y);
  r.ca = carrier(Lc, l.Pa, L.z);
  r.cb = carrier(Lc, l.Pb, L.z);
  ld_pair(X + o, r.xa_, r.xb_);
  if (pend) {
    float2 da, db;
    ld_pair(D + o, da, db);
    r.xa_ = cadd(r.xa_, cscale(da, alpha));
    r.xb_ = cadd(r.xb_, cscale(db, alpha));
  }
  ld_pairf(S + o, r.Sa, r.Sb);
  r.ya = l.va ? r.Sa - re_mul(r.xa_, r.ca) : 0.f;
  r.yb = l.vb ? r.Sb - re_mul(r.xb_, r.cb) : 0.f;
  if (!l.va) r.xa_ = make_float2(0.f, 0.f);
  if (!l.vb) r.xb_ = make_float2(0.f, 0.f);
  r.xh = make_float2(0.f, 0.f);
  r.yh = 0.f;
  if (l.hv) {  // right halo (lane 31) -- lane 0's left halo is loaded but unused
    const int64_t oh = (int64_t)y * f.pitch + l.hx;
    float2 xv = __ldcg(X + oh);
    if (pend) xv = cadd(xv, cscale(__ldcg(D + oh), alpha));
    r.xh = xv;
    r.yh = __ldcg(S + oh) - re_mul(xv, carrier(Lc, l.Ph, L.z));
  }
}

__device__ __noinline__ void phase_reweight(const SolverArgs& A, const FieldDesc& f, Unit u,
                                            int lane, FieldCtl c) {
  const Lanes l = make_lanes(A, f, u.x0, lane);
  const int64_t base = f.px_off;
  const float2* X = A.X[c.xsel] + base;
  float2* Xo = A.X[c.xsel ^ 1] + base;
  const float2* D = A.D[c.sel] + base;
  const float* S = A.S + base;
  float4* W = A.W + base;
  const bool pend = c.pending != 0;
  const float alpha = c.alpha;
  if (f.adj_flags & kAdjFixedW) {
    // weights given: only apply the pending step into the other chi buffer
    for (int y = u.y0; y < u.y1; ++y) {
      const int64_t o = (int64_t)y * f.pitch + l.xa;
      float2 xa, xb;
      ld_pair(X + o, xa, xb);
      if (pend) {
        float2 da, db;
        ld_pair(D + o, da, db);
        xa = cadd(xa, cscale(da, alpha));
        xb = cadd(xb, cscale(db, alpha));
      }
      st_pair(Xo + o, xa, xb, l.va, l.vb);
    }
    return;
  }
  const float eps = f.eps, epsc = f.eps_c, k = f.k_coupling;
  const float e2 = eps * eps, ec2 = epsc * epsc;
  RRow cur, nxt;
  r_form(A, f, l, X, D, S, pend, alpha, u.y0, cur);
  for (int y = u.y0; y < u.y1; ++y) {
    const bool hn = y + 1 < f.h;
    if (hn) r_form(A, f, l, X, D, S, pend, alpha, y + 1, nxt);
    float y_r = __shfl_down_sync(0xffffffffu, cur.ya, 1);
    float2 x_r = make_float2(__shfl_down_sync(0xffffffffu, cur.xa_.x, 1),
                             __shfl_down_sync(0xffffffffu, cur.xa_.y, 1));
    if (lane == 31) {
      y_r = cur.yh;
      x_r = cur.xh;
    }
    const float gxa = (l.xa < f.w - 1) ? cur.yb - cur.ya : 0.f;
    const float gxb = (l.xb < f.w - 1) ? y_r - cur.yb : 0.f;
    const float gya = hn ? nxt.ya - cur.ya : 0.f;
    const float gyb = hn ? nxt.yb - cur.yb : 0.f;
    const float2 dxa = (l.xa < f.w - 1) ? csub(cur.xb_, cur.xa_) : make_float2(0.f, 0.f);
    const float2 dxb = (l.xb < f.w - 1) ? csub(x_r, cur.xb_) : make_float2(0.f, 0.f);
    const float2 dya = hn ? csub(nxt.xa_, cur.xa_) : make_float2(0.f, 0.f);
    const float2 dyb = hn ? csub(nxt.xb_, cur.xb_) : make_float2(0.f, 0.f);
    const float mxa = sqrtf(cnorm(dxa)), mxb = sqrtf(cnorm(dxb));
    const float mya = sqrtf(cnorm(dya)), myb = sqrtf(cnorm(dyb));
    float4 wa, wb;
    wa.x = eps / sqrtf(gxa * gxa + e2);
    wa.y = eps / sqrtf(gya * gya + e2);
    wa.z = epsc / sqrtf(mxa * mxa + k * gxa * gxa + ec2);
    wa.w = epsc / sqrtf(mya * mya + k * gya * gya + ec2);
    wb.x = eps / sqrtf(gxb * gxb + e2);
    wb.y = eps / sqrtf(gyb * gyb + e2);
    wb.z = epsc / sqrtf(mxb * mxb + k * gxb * gxb + ec2);
    wb.w = epsc / sqrtf(myb * myb + k * gyb * gyb + ec2);
    const int64_t o = (int64_t)y * f.pitch + l.xa;
    // oriented diffusivities 1 / sqrt(1 + (|D chi| / eps_c)^2) of the +45 deg
    // difference D1 chi(y, x) = chi(y+1, x+1) - chi(y, x) and the -45 deg
    // one D2 chi(y, x) = chi(y+1, x-1) - chi(y, x), zero on the last row and
    // on the last / first column (variational.cpp:434-451, gradients.h:195-254)
    float2 wda = make_float2(0.f, 0.f), wdb = wda;
    const bool diag = f.mu_d > 0.f;
    if (diag) {
      float2 n_r = make_float2(__shfl_down_sync(0xffffffffu, nxt.xa_.x, 1),
                               __shfl_down_sync(0xffffffffu, nxt.xa_.y, 1));
      float2 n_l = make_float2(__shfl_up_sync(0xffffffffu, nxt.xb_.x, 1),
                               __shfl_up_sync(0xffffffffu, nxt.xb_.y, 1));
      if (lane == 31) n_r = nxt.xh;  // chi(y+1, x0+64)
      if (lane == 0) n_l = nxt.xh;   // chi(y+1, x0-1)
      const float2 z = make_float2(0.f, 0.f);
      const float2 d1a = (hn && l.xa < f.w - 1) ? csub(nxt.xb_, cur.xa_) : z;
      const float2 d1b = (hn && l.xb < f.w - 1) ? csub(n_r, cur.xb_) : z;
      const float2 d2a = (hn && l.va && l.xa >= 1) ? csub(n_l, cur.xa_) : z;
      const float2 d2b = (hn && l.vb) ? csub(nxt.xa_, cur.xb_) : z;
      const float c1a = sqrtf(cnorm(d1a)) / epsc, c1b = sqrtf(cnorm(d1b)) / epsc;
      const float c2a = sqrtf(cnorm(d2a)) / epsc, c2b = sqrtf(cnorm(d2b)) / epsc;
      wda = make_float2(1.0f / sqrtf(1.0f + c1a * c1a), 1.0f / sqrtf(1.0f + c2a * c2a));
      wdb = make_float2(1.0f / sqrtf(1.0f + c1b * c1b), 1.0f / sqrtf(1.0f + c2b * c2b));
    }
    if (f.has_nbr) {
      // neighbour robust weights (variational.cpp:452-462), prior
      // renormalisation (:493-516) and the pointwise data term written as
      // M = 2 nu sum wt u u^T, b = 2 nu sum wt (S_w - S) u, u = (Re dc, -Im dc).
      const float nu = f.nu, et2 = f.eps_t * f.eps_t;
      float psa = 1.f, psb = 1.f;
      float4 Ma = make_float4(0.f, 0.f, 0.f, 0.f), Mb = Ma;
      float2 ba = make_float2(0.f, 0.f), bb = ba;
      for (int j = 0; j < f.n_nbr; ++j) {
        const float4* NB = A.nbr + f.nbr_off + (int64_t)j * f.plane_px;
        const float4 na = __ldcg(NB + o);
        const float4 nbv = __ldcg(NB + o + 1);
        // na = (S_w - S, dc.x, dc.y, conf)
        const float rta = na.x + (cur.xa_.x * na.y - cur.xa_.y * na.z);
        const float rtb = nbv.x + (cur.xb_.x * nbv.y - cur.xb_.y * nbv.z);
        const float wta = na.w * et2 / (rta * rta + et2);
        const float wtb = nbv.w * et2 / (rtb * rtb + et2);
        psa += nu * wta * (na.y * na.y + na.z * na.z);
        psb += nu * wtb * (nbv.y * nbv.y + nbv.z * nbv.z);
        const float sa = 2.f * nu * wta, sb = 2.f * nu * wtb;
        Ma.x += sa * na.y * na.y;
        Ma.y -= sa * na.y * na.z;
        Ma.z += sa * na.z * na.z;
        Mb.x += sb * nbv.y * nbv.y;
        Mb.y -= sb * nbv.y * nbv.z;
        Mb.z += sb * nbv.z * nbv.z;
        ba.x += sa * na.x * na.y;
        ba.y -= sa * na.x * na.z;
        bb.x += sb * nbv.x * nbv.y;
        bb.y -= sb * nbv.x * nbv.z;
      }
      wa.x *= psa; wa.y *= psa; wa.z *= psa; wa.w *= psa;
      wb.x *= psb; wb.y *= psb; wb.z *= psb; wb.w *= psb;
      wda = cscale(wda, psa);
      wdb = cscale(wdb, psb);
      if (l.va) __stcg(A.M + base + o, Ma);
      if (l.vb) __stcg(A.M + base + o + 1, Mb);
      st_pair(A.B + base + o, ba, bb, l.va, l.vb);
    }
    if (l.va) __stcg(W + o, wa);
    if (l.vb) __stcg(W + o + 1, wb);
    if (diag) st_pair(A.W2 + base + o, wda, wdb, l.va, l.vb);
    st_pair(Xo + o, cur.xa_, cur.xb_, l.va, l.vb);
    cur = nxt;
  }
}

// ---------------------------------------------------------------------------
// G phase: the gradient at chi (with S) -> G[0], and its squared norm.
// ---------------------------------------------------------------------------
struct SRow {
  float2 ca, cb;
  float2 ua, ub, uh;   // chi, halo
  float ya, yb, yh;    // S - Re[chi c]
};

__device__ __forceinline__ void s_form(const SolverArgs& A, const FieldDesc& f, const Lanes& l,
                                       const FieldCtl& c, int y, SRow& r) {
  const int64_t base = f.px_off;
  const int64_t o = (int64_t)y * f.pitch + l.xa;
  const float4 L = __ldg(A.line_phasor + f.line_off + y);
  const float2 Lc = make_float2(L.x, L.y);
  r.ca = carrier(Lc, l.Pa, L.z);
  r.cb = carrier(Lc, l.Pb, L.z);
  const float2 z = make_float2(0.f, 0.f);
  const float2* X = A.X[c.xsel] + base;
  float Sa, Sb;
  ld_pair(X + o, r.ua, r.ub);
  ld_pairf(A.S + base + o, Sa, Sb);
  if (!l.va) r.ua = z;
  if (!l.vb) r.ub = z;
  r.ya = l.va ? Sa - re_mul(r.ua, r.ca) : 0.f;
  r.yb = l.vb ? Sb - re_mul(r.ub, r.cb) : 0.f;
  r.uh = z;
  r.yh = 0.f;
  if (l.hv) {
    const int64_t oh = (int64_t)y * f.pitch + l.hx;
    r.uh = __ldcg(X + oh);
    r.yh = __ldcg(A.S + base + oh) - re_mul(r.uh, carrier(Lc, l.Ph, L.z));
  }
}

__device__ __noinline__ double phase_gradient(const SolverArgs& A, const FieldDesc& f, Unit u,
                                              int lane, FieldCtl c) {
  const Lanes l = make_lanes(A, f, u.x0, lane);
  const int64_t base = f.px_off;
  const float4* W = A.W + base;
  const float mu_h = f.mu_h, mu_v = f.mu_v;
  const float2 z = make_float2(0.f, 0.f);
  double pgg = 0.0;
  SRow cur, nxt;
  float aypa = 0.f, aypb = 0.f;
  float2 bypa = z, bypb = z;
  const bool diag = f.mu_d > 0.f;
  const float2* W2 = A.W2 + base;
  // this lane's oriented weights at (y, own pixels) and at its halo column
  auto wd_row = [&](int y, float2& wda, float2& wdb, float2& wdh) {
    const int64_t o = (int64_t)y * f.pitch + l.xa;
    ld_pair(W2 + o, wda, wdb);
    wdh = l.hv ? __ldcg(W2 + (int64_t)y * f.pitch + l.hx) : z;
  };
  DiagFlux dprev = {z, z, z, z, z};
  float hd_unused = 0.f;
  s_form(A, f, l, c, u.y0, cur);
  if (u.y0 > 0) {
    SRow prv;
    s_form(A, f, l, c, u.y0 - 1, prv);
    const int64_t op = (int64_t)(u.y0 - 1) * f.pitch + l.xa;
    const float4 wpa = __ldcg(W + op), wpb = __ldcg(W + op + 1);
    aypa = wpa.y * (cur.ya - prv.ya);
    aypb = wpb.y * (cur.yb - prv.yb);
    bypa = cscale(csub(cur.ua, prv.ua), wpa.w);
    bypb = cscale(csub(cur.ub, prv.ub), wpb.w);
    if (diag) {
      float2 wda, wdb, wdh;
      wd_row(u.y0 - 1, wda, wdb, wdh);
      diag_flux(l, f, lane, true, prv.ua, prv.ub, prv.uh, cur.ua, cur.ub, cur.uh, wda, wdb, wdh,
                dprev, hd_unused);
    }
  }
  for (int y = u.y0; y < u.y1; ++y) {
    const bool hn = y + 1 < f.h;
    if (hn) s_form(A, f, l, c, y + 1, nxt);
    const int64_t o = (int64_t)y * f.pitch + l.xa;
    const float4 wa = __ldcg(W + o), wb = __ldcg(W + o + 1);
    float4 wh = make_float4(0.f, 0.f, 0.f, 0.f);
    if (l.hv && lane == 0) wh = __ldcg(W + (int64_t)y * f.pitch + l.hx);
    // horizontal neighbours
    float y_r = __shfl_down_sync(0xffffffffu, cur.ya, 1);
    float2 u_r = make_float2(__shfl_down_sync(0xffffffffu, cur.ua.x, 1),
                             __shfl_down_sync(0xffffffffu, cur.ua.y, 1));
    if (lane == 31) {
      y_r = cur.yh;
      u_r = cur.uh;
    }
    const bool ia = l.xa < f.w - 1, ib = l.xb < f.w - 1;
    const float dxya = ia ? cur.yb - cur.ya : 0.f;
    const float dxyb = ib ? y_r - cur.yb : 0.f;
    const float2 dxua = ia ? csub(cur.ub, cur.ua) : z;
    const float2 dxub = ib ? csub(u_r, cur.ub) : z;
    const float axa = wa.x * dxya, axb = wb.x * dxyb;
    const float2 bxa = cscale(dxua, wa.z), bxb = cscale(dxub, wb.z);
    // left neighbour of pixel a: lane - 1's pixel b, or lane 0's halo
    float axl = __shfl_up_sync(0xffffffffu, axb, 1);
    float2 bxl = make_float2(__shfl_up_sync(0xffffffffu, bxb.x, 1),
                             __shfl_up_sync(0xffffffffu, bxb.y, 1));
    if (lane == 0) {
      if (l.hv && l.hx < f.w - 1) {
        axl = wh.x * (cur.ya - cur.yh);
        bxl = cscale(csub(cur.ua, cur.uh), wh.z);
      } else {
        axl = 0.f;
        bxl = z;
      }
    }
    // vertical
    const float dyya = hn ? nxt.ya - cur.ya : 0.f;
    const float dyyb = hn ? nxt.yb - cur.yb : 0.f;
    const float2 dyua = hn ? csub(nxt.ua, cur.ua) : z;
    const float2 dyub = hn ? csub(nxt.ub, cur.ub) : z;
    const float aya = wa.y * dyya, ayb = wb.y * dyyb;
    const float2 bya = cscale(dyua, wa.w), byb = cscale(dyub, wb.w);
    // operator: -2[(ax(x-1) - ax) + (ay(y-1) - ay)] conj(c) + 2[mu_h (..) + mu_v (..)]
    const float ima = 2.f * ((axl - axa) + (aypa - aya));
    const float imb = 2.f * ((axa - axb) + (aypb - ayb));
    float2 oa = make_float2(-ima * cur.ca.x, ima * cur.ca.y);
    float2 ob = make_float2(-imb * cur.cb.x, imb * cur.cb.y);
    oa = cadd(oa, cscale(cadd(cscale(csub(bxl, bxa), mu_h), cscale(csub(bypa, bya), mu_v)), 2.f));
    ob = cadd(ob, cscale(cadd(cscale(csub(bxa, bxb), mu_h), cscale(csub(bypb, byb), mu_v)), 2.f));
    if (diag) {  // + 2 mu_d (D1T(wd1 D1 chi) + D2T(wd2 D2 chi))
      float2 wda, wdb, wdh;
      wd_row(y, wda, wdb, wdh);
      DiagFlux dcur;
      diag_flux(l, f, lane, hn, cur.ua, cur.ub, cur.uh, nxt.ua, nxt.ub, nxt.uh, wda, wdb, wdh,
                dcur, hd_unused);
      float2 ta, tb;
      diag_adjoint(lane, dcur, dprev, ta, tb);
      oa = cadd(oa, cscale(ta, 2.f * f.mu_d));
      ob = cadd(ob, cscale(tb, 2.f * f.mu_d));
      dprev = dcur;
    }
    if (f.has_nbr) {
      const float4 Ma = __ldcg(A.M + base + o), Mb = __ldcg(A.M + base + o + 1);
      // M u with u as the real 2-vector (Re, Im), plus the constant b
      oa.x += Ma.x * cur.ua.x + Ma.y * cur.ua.y;
      oa.y += Ma.y * cur.ua.x + Ma.z * cur.ua.y;
      ob.x += Mb.x * cur.ub.x + Mb.y * cur.ub.y;
      ob.y += Mb.y * cur.ub.x + Mb.z * cur.ub.y;
      float2 ba, bb;
      ld_pair(A.B + base + o, ba, bb);
      oa = cadd(oa, ba);
      ob = cadd(ob, bb);
    } else if (f.adj_flags & kAdjExtB) {
      float2 ba, bb;
      ld_pair(A.B + base + o, ba, bb);
      oa = cadd(oa, ba);
      ob = cadd(ob, bb);
    }
    if (!l.va) oa = z;
    if (!l.vb) ob = z;
    st_pair(A.G[0] + base + o, oa, ob, l.va, l.vb);
    pgg += (double)cnorm(oa) + (double)cnorm(ob);
    aypa = aya;
    aypb = ayb;
    bypa = bya;
    bypb = byb;
    cur = nxt;
  }
  return pgg;
}

// ---------------------------------------------------------------------------
// I phase with TMA-staged rows. Each warp owns a ring of kNS row slots in
// shared memory; lane 0 fills them with 1-D bulk copies (cp.async.bulk,
// mbarrier-tracked) of the g / q / d row segments (strip + 2-pixel halo
// each side), the chi row segment, the weight row segment (strip + left
// halo) and the row's line phasor, so up to kNS - 1 rows are in flight per
// warp without holding registers. Rows of one unit: [max(y0 - 1, 0),
// min(y1, h - 1)].
//
// Register economy: between rows only the operands of the vertical
// differences (d_k and its luma part -Re[d_k c]) and the vertical fluxes of
// the row above are carried; everything else of the current row (g_k,
// d_{k-1}, carriers, halo) is re-read from its slot. Each row's inner-
// product terms (at most eight per lane) are summed in FP32 and added to
// per-lane FP64 accumulators, which are reduced across the warp and the
// field in FP64 (variational.cpp:72-95 accumulates in double).
// ---------------------------------------------------------------------------
constexpr int kSlotG = (kStrip + 4) * 8;        // 544 B: columns x0-2 .. x0+65
constexpr int kSlotX = kStrip * 8;              // 512 B: columns x0 .. x0+63
constexpr int kSlotW = (kStrip + 1) * 16;       // 1040 B: columns x0-1 .. x0+63
constexpr int kOffQ = kSlotG, kOffD = 2 * kSlotG, kOffX = 3 * kSlotG, kOffW = 3 * kSlotG + kSlotX;
constexpr int kOffL = kOffW + kSlotW;           // 16 B: the row's line phasor
constexpr int kSlotBytes = kOffL + 16;          // 3200 B
// the oriented-prior variant adds the (wd1, wd2) row segment, columns
// x0-2 .. x0+65 like g (float2: 16-byte aligned at x0-2)
constexpr int kOffW2 = kSlotBytes;
template <bool kDiag>
struct RingLayout {
  static constexpr int slot = kDiag ? kSlotBytes + kSlotG : kSlotBytes;  // 3200 / 3744 B
  static constexpr int warp = kNS * slot + kNS * 8;
};
static_assert(kSlotBytes % 16 == 0 && kOffL % 16 == 0 && RingLayout<true>::slot % 16 == 0,
              "bulk copies need 16-byte slots");

struct Ring {
  char* slots;
  uint64_t* bar;
  uint32_t bits;  // per-slot phase parity
};

template <bool kDiag>
__device__ __forceinline__ void ring_issue(Ring& r, int slot, const SolverArgs& A,
                                           const FieldDesc& f, const FieldCtl& c, int x0, int y,
                                           bool first, bool need_x) {
  char* dst = r.slots + slot * RingLayout<kDiag>::slot;
  uint64_t* bar = r.bar + slot;
  const int64_t row = f.px_off + (int64_t)y * f.pitch;
  const int gs = max(x0 - 2, 0), ge = min(x0 + kStrip + 2, f.pitch);
  const uint32_t gb = (uint32_t)(ge - gs) * 8u;
  const int goff = (gs - (x0 - 2)) * 8;
  const int ws = max(x0 - 1, 0), we = min(x0 + kStrip, f.pitch);
  const uint32_t wb = (uint32_t)(we - ws) * 16u;
  const int woff = (ws - (x0 - 1)) * 16;
  const bool qd = !first;
  const bool xx = need_x && !first;
  const uint32_t total = gb + wb + 16u + (qd ? 2 * gb : 0u) + (xx ? (uint32_t)kSlotX : 0u) +
                         (kDiag ? gb : 0u);
  mbar_expect_tx(bar, total);
  if (kDiag) bulk_g2s(dst + kOffW2 + goff, A.W2 + row + gs, gb, bar);
  bulk_g2s(dst + goff, A.G[c.sel] + row + gs, gb, bar);
  if (qd) {
    bulk_g2s(dst + kOffQ + goff, A.Q[c.sel] + row + gs, gb, bar);
    bulk_g2s(dst + kOffD + goff, A.D[c.sel] + row + gs, gb, bar);
  }
  if (xx) bulk_g2s(dst + kOffX, A.X[c.xsel] + row + x0, kSlotX, bar);
  bulk_g2s(dst + kOffW + woff, A.W + row + ws, wb, bar);
  bulk_g2s(dst + kOffL, A.line_phasor + f.line_off + y, 16u, bar);
}

__device__ __forceinline__ bool ring_wait(Ring& r, int slot) {
  const bool ok = mbar_wait(r.bar + slot, (r.bits >> slot) & 1u);
  r.bits ^= 1u << slot;
  return ok;
}

// g_k = g + alpha q and d_{k-1} of this lane's two pixels, from a slot.
__device__ __forceinline__ void slot_gd(const char* slot, const FieldCtl& c, bool first, int lane,
                                        float2& gka, float2& gkb, float2& doa, float2& dob) {
  const float4 g4 = *reinterpret_cast<const float4*>(slot + 16 + 16 * lane);
  gka = make_float2(g4.x, g4.y);
  gkb = make_float2(g4.z, g4.w);
  if (first) {
    doa = make_float2(0.f, 0.f);
    dob = doa;
  } else {
    const float4 q4 = *reinterpret_cast<const float4*>(slot + kOffQ + 16 + 16 * lane);
    const float4 d4 = *reinterpret_cast<const float4*>(slot + kOffD + 16 + 16 * lane);
    gka = cadd(gka, cscale(make_float2(q4.x, q4.y), c.alpha));
    gkb = cadd(gkb, cscale(make_float2(q4.z, q4.w), c.alpha));
    doa = make_float2(d4.x, d4.y);
    dob = make_float2(d4.z, d4.w);
  }
}

// d_k = -g_k + beta d_{k-1} (zero outside the field) and its luma part.
struct DRow {
  float2 ua, ub;
  float ya, yb;
};

__device__ __forceinline__ void slot_d(const char* slot, const Lanes& l, const FieldCtl& c,
                                       bool first, int lane, DRow& r) {
  float2 gka, gkb, doa, dob;
  slot_gd(slot, c, first, lane, gka, gkb, doa, dob);
  const float4 L = *reinterpret_cast<const float4*>(slot + kOffL);
  const float2 Lc = make_float2(L.x, L.y);
  r.ua = cadd(make_float2(-gka.x, -gka.y), cscale(doa, c.beta));
  r.ub = cadd(make_float2(-gkb.x, -gkb.y), cscale(dob, c.beta));
  if (!l.va) r.ua = make_float2(0.f, 0.f);
  if (!l.vb) r.ub = make_float2(0.f, 0.f);
  r.ya = -re_mul(r.ua, carrier(Lc, l.Pa, L.z));
  r.yb = -re_mul(r.ub, carrier(Lc, l.Pb, L.z));
}

// d_k at this lane's halo column (lane 0: x0-1, lane 31: x0+64; zero for the
// other lanes and outside the field), from a slot.
__device__ __forceinline__ float2 slot_halo(const char* sl, const Lanes& l, const FieldCtl& c,
                                            bool first, int lane) {
  float2 uh = make_float2(0.f, 0.f);
  if (l.hv) {
    const int hl = lane == 0 ? 1 : kStrip + 2;  // local column of x0-1 / x0+64
    const float2 gh = *reinterpret_cast<const float2*>(sl + 8 * hl);
    if (first) {
      uh = make_float2(-gh.x, -gh.y);
    } else {
      const float2 qh = *reinterpret_cast<const float2*>(sl + kOffQ + 8 * hl);
      const float2 dd = *reinterpret_cast<const float2*>(sl + kOffD + 8 * hl);
      const float2 gkh = cadd(gh, cscale(qh, c.alpha));
      uh = cadd(make_float2(-gkh.x, -gkh.y), cscale(dd, c.beta));
    }
  }
  return uh;
}

// this lane's (wd1, wd2) at its two pixels and at its halo column, from a slot
__device__ __forceinline__ void slot_wd(const char* sl, int lane, float2& wda, float2& wdb,
                                        float2& wdh) {
  const float4 w = *reinterpret_cast<const float4*>(sl + kOffW2 + 16 + 16 * lane);
  wda = make_float2(w.x, w.y);
  wdb = make_float2(w.z, w.w);
  wdh = *reinterpret_cast<const float2*>(sl + kOffW2 + 8 * (lane == 0 ? 1 : kStrip + 2));
}

template <bool kDiag>
__device__ bool phase_iter(const SolverArgs& A, const FieldDesc& f, const Unit& u, int lane,
                           const FieldCtl& c, bool first, Ring& ring, double* part) {
  const Lanes l = make_lanes(A, f, u.x0, lane);
  const int64_t base = f.px_off;
  const float mu_h = f.mu_h, mu_v = f.mu_v;
  const float2 z = make_float2(0.f, 0.f);
  const int ybeg = max(u.y0 - 1, 0), yend = min(u.y1, f.h - 1);
  const int nrows = yend - ybeg + 1;
  double pH = 0.0, pgd = 0.0, pgq = 0.0, pqq = 0.0, pgg = 0.0;
  bool ok = true;
  // the first min(kNS, nrows) rows' copies were issued by the caller
  __syncwarp();
  auto slot_ptr = [&](int i) { return ring.slots + (i % kNS) * RingLayout<kDiag>::slot; };
  auto issue_after = [&](int i_free) {
    __syncwarp();
    const int inext = i_free + kNS;
    if (lane == 0 && inext < nrows) {
      fence_proxy_async_smem();
      const int y = ybeg + inext;
      ring_issue<kDiag>(ring, inext % kNS, A, f, c, u.x0, y, first, y >= u.y0 && y < u.y1);
    }
  };
  DRow cur, nxt;
  float aypa = 0.f, aypb = 0.f;
  float2 bypa = z, bypb = z;
  int icur = 0;
  // oriented prior: the previous row's fluxes and the next row's halo d
  DiagFlux dprev = {z, z, z, z, z};
  float2 nuh = z;
  if (u.y0 > 0) {
    DRow prv;
    ok &= ring_wait(ring, 0);
    slot_d(slot_ptr(0), l, c, first, lane, prv);
    ok &= ring_wait(ring, 1 % kNS);
    slot_d(slot_ptr(1), l, c, first, lane, cur);
    const char* w0 = slot_ptr(0) + kOffW;
    const float4 wpa = *reinterpret_cast<const float4*>(w0 + 16 * (1 + 2 * lane));
    const float4 wpb = *reinterpret_cast<const float4*>(w0 + 16 * (2 + 2 * lane));
    aypa = wpa.y * (cur.ya - prv.ya);
    aypb = wpb.y * (cur.yb - prv.yb);
    bypa = cscale(csub(cur.ua, prv.ua), wpa.w);
    bypb = cscale(csub(cur.ub, prv.ub), wpb.w);
    if (kDiag && f.mu_d > 0.f) {
      float2 wda, wdb, wdh;
      slot_wd(slot_ptr(0), lane, wda, wdb, wdh);
      float hd_unused;
      diag_flux(l, f, lane, true, prv.ua, prv.ub, slot_halo(slot_ptr(0), l, c, first, lane),
                cur.ua, cur.ub, slot_halo(slot_ptr(1), l, c, first, lane), wda, wdb, wdh, dprev,
                hd_unused);
    }
    issue_after(0);
    icur = 1;
  } else {
    ok &= ring_wait(ring, 0);
    slot_d(slot_ptr(0), l, c, first, lane, cur);
  }
  const int s2 = c.sel ^ 1;
  float2* Gw = A.G[s2] + base;
  float2* Dw = A.D[s2] + base;
  float2* Qw = A.Q[s2] + base;
  float2* Xw = A.X[c.xsel] + base;
  for (int y = u.y0; y < u.y1; ++y) {
    const bool hn = y + 1 < f.h;
    if (hn) {
      ok &= ring_wait(ring, (icur + 1) % kNS);
      slot_d(slot_ptr(icur + 1), l, c, first, lane, nxt);
      if constexpr (kDiag) nuh = slot_halo(slot_ptr(icur + 1), l, c, first, lane);
    }
    const char* sl = slot_ptr(icur);
    // the current row's g_k, d_{k-1}, carriers and halo, re-read from its slot
    float2 gka, gkb, doa, dob;
    slot_gd(sl, c, first, lane, gka, gkb, doa, dob);
    if (!l.va) gka = z;
    if (!l.vb) gkb = z;
    const float4 L = *reinterpret_cast<const float4*>(sl + kOffL);
    const float2 Lc = make_float2(L.x, L.y);
    const float2 ca = carrier(Lc, l.Pa, L.z), cb = carrier(Lc, l.Pb, L.z);
    float2 uh = z;
    float yh = 0.f;
    if (l.hv) {
      const int hl = lane == 0 ? 1 : kStrip + 2;  // local column of x0-1 / x0+64
      const float2 gh = *reinterpret_cast<const float2*>(sl + 8 * hl);
      if (first) {
        uh = make_float2(-gh.x, -gh.y);
      } else {
        const float2 qh = *reinterpret_cast<const float2*>(sl + kOffQ + 8 * hl);
        const float2 dd = *reinterpret_cast<const float2*>(sl + kOffD + 8 * hl);
        const float2 gkh = cadd(gh, cscale(qh, c.alpha));
        uh = cadd(make_float2(-gkh.x, -gkh.y), cscale(dd, c.beta));
      }
      yh = -re_mul(uh, carrier(Lc, l.Ph, L.z));
    }
    const float4 wa = *reinterpret_cast<const float4*>(sl + kOffW + 16 * (1 + 2 * lane));
    const float4 wb = *reinterpret_cast<const float4*>(sl + kOffW + 16 * (2 + 2 * lane));
    float4 wh = make_float4(0.f, 0.f, 0.f, 0.f);
    if (l.hv && lane == 0) wh = *reinterpret_cast<const float4*>(sl + kOffW);
    float y_r = __shfl_down_sync(0xffffffffu, cur.ya, 1);
    float2 u_r = make_float2(__shfl_down_sync(0xffffffffu, cur.ua.x, 1),
                             __shfl_down_sync(0xffffffffu, cur.ua.y, 1));
    if (lane == 31) {
      y_r = yh;
      u_r = uh;
    }
    const bool ia = l.xa < f.w - 1, ib = l.xb < f.w - 1;
    const float dxya = ia ? cur.yb - cur.ya : 0.f;
    const float dxyb = ib ? y_r - cur.yb : 0.f;
    const float2 dxua = ia ? csub(cur.ub, cur.ua) : z;
    const float2 dxub = ib ? csub(u_r, cur.ub) : z;
    const float axa = wa.x * dxya, axb = wb.x * dxyb;
    const float2 bxa = cscale(dxua, wa.z), bxb = cscale(dxub, wb.z);
    float axl = __shfl_up_sync(0xffffffffu, axb, 1);
    float2 bxl = make_float2(__shfl_up_sync(0xffffffffu, bxb.x, 1),
                             __shfl_up_sync(0xffffffffu, bxb.y, 1));
    if (lane == 0) {
      if (l.hv && l.hx < f.w - 1) {
        axl = wh.x * (cur.ya - yh);
        bxl = cscale(csub(cur.ua, uh), wh.z);
      } else {
        axl = 0.f;
        bxl = z;
      }
    }
    const float dyya = hn ? nxt.ya - cur.ya : 0.f;
    const float dyyb = hn ? nxt.yb - cur.yb : 0.f;
    const float2 dyua = hn ? csub(nxt.ua, cur.ua) : z;
    const float2 dyub = hn ? csub(nxt.ub, cur.ub) : z;
    const float aya = wa.y * dyya, ayb = wb.y * dyyb;
    const float2 bya = cscale(dyua, wa.w), byb = cscale(dyub, wb.w);
    const float ima = 2.f * ((axl - axa) + (aypa - aya));
    const float imb = 2.f * ((axa - axb) + (aypb - ayb));
    float2 oa = make_float2(-ima * ca.x, ima * ca.y);
    float2 ob = make_float2(-imb * cb.x, imb * cb.y);
    oa = cadd(oa, cscale(cadd(cscale(csub(bxl, bxa), mu_h), cscale(csub(bypa, bya), mu_v)), 2.f));
    ob = cadd(ob, cscale(cadd(cscale(csub(bxa, bxb), mu_h), cscale(csub(bypb, byb), mu_v)), 2.f));
    const int64_t o = (int64_t)y * f.pitch + l.xa;
    float rH = 0.f;
    if (kDiag && f.mu_d > 0.f) {  // + 2 mu_d (D1T(wd1 D1 d) + D2T(wd2 D2 d)), mu_d sum wd |D d|^2
      float2 wda, wdb, wdh;
      slot_wd(sl, lane, wda, wdb, wdh);
      DiagFlux dcur;
      float hd;
      diag_flux(l, f, lane, hn, cur.ua, cur.ub, uh, nxt.ua, nxt.ub, nuh, wda, wdb, wdh, dcur, hd);
      float2 ta, tb;
      diag_adjoint(lane, dcur, dprev, ta, tb);
      oa = cadd(oa, cscale(ta, 2.f * f.mu_d));
      ob = cadd(ob, cscale(tb, 2.f * f.mu_d));
      rH += f.mu_d * hd;
      dprev = dcur;
    }
    if (f.has_nbr) {
      const float4 Ma = __ldcg(A.M + base + o), Mb = __ldcg(A.M + base + o + 1);
      oa.x += Ma.x * cur.ua.x + Ma.y * cur.ua.y;
      oa.y += Ma.y * cur.ua.x + Ma.z * cur.ua.y;
      ob.x += Mb.x * cur.ub.x + Mb.y * cur.ub.y;
      ob.y += Mb.y * cur.ub.x + Mb.z * cur.ub.y;
      if (l.va)
        rH += 0.5f * (Ma.x * cur.ua.x * cur.ua.x + 2.f * Ma.y * cur.ua.x * cur.ua.y +
                      Ma.z * cur.ua.y * cur.ua.y);
      if (l.vb)
        rH += 0.5f * (Mb.x * cur.ub.x * cur.ub.x + 2.f * Mb.y * cur.ub.x * cur.ub.y +
                      Mb.z * cur.ub.y * cur.ub.y);
    }
    if (!l.va) oa = z;
    if (!l.vb) ob = z;
    if (l.va)
      rH += wa.x * dxya * dxya + wa.y * dyya * dyya + mu_h * wa.z * cnorm(dxua) +
            mu_v * wa.w * cnorm(dyua);
    if (l.vb)
      rH += wb.x * dxyb * dxyb + wb.y * dyyb * dyyb + mu_h * wb.z * cnorm(dxub) +
            mu_v * wb.w * cnorm(dyub);
    pH += (double)rH;
    pgd += (double)((gka.x * cur.ua.x + gka.y * cur.ua.y) + (gkb.x * cur.ub.x + gkb.y * cur.ub.y));
    pgq += (double)((gka.x * oa.x + gka.y * oa.y) + (gkb.x * ob.x + gkb.y * ob.y));
    pqq += (double)(cnorm(oa) + cnorm(ob));
    pgg += (double)(cnorm(gka) + cnorm(gkb));
    st_pair(Gw + o, gka, gkb, l.va, l.vb);
    st_pair(Dw + o, cur.ua, cur.ub, l.va, l.vb);
    st_pair(Qw + o, oa, ob, l.va, l.vb);
    if (!first) {
      const float4 x4 = *reinterpret_cast<const float4*>(sl + kOffX + 16 * lane);
      const float2 xa = cadd(make_float2(x4.x, x4.y), cscale(doa, c.alpha));
      const float2 xb = cadd(make_float2(x4.z, x4.w), cscale(dob, c.alpha));
      st_pair(Xw + o, xa, xb, l.va, l.vb);
    }
    issue_after(icur);
    aypa = aya;
    aypb = ayb;
    bypa = bya;
    bypb = byb;
    cur = nxt;
    icur += 1;
  }
  part[0] = pH;
  part[1] = pgd;
  part[2] = pgq;
  part[3] = pqq;
  part[4] = pgg;
  return ok;
}

// F phase: apply the pending step, output-fidelity luma Y = S - Re[chi c]
// (variational.cpp:552-555, sequence.cpp:1102-1114); final chi -> X[0].
__device__ __noinline__ void phase_final(const SolverArgs& A, const FieldDesc& f, Unit u, int lane,
                                         FieldCtl c) {
  const Lanes l = make_lanes(A, f, u.x0, lane);
  const int64_t base = f.px_off;
  const float2* X = A.X[c.xsel] + base;
  const float2* D = A.D[c.sel] + base;
  float2* Xo = A.X[0] + base;
  for (int y = u.y0; y < u.y1; ++y) {
    const int64_t o = (int64_t)y * f.pitch + l.xa;
    const float4 L = __ldg(A.line_phasor + f.line_off + y);
    const float2 Lc = make_float2(L.x, L.y);
    float2 xa, xb;
    ld_pair(X + o, xa, xb);
    if (c.pending) {
      float2 da, db;
      ld_pair(D + o, da, db);
      xa = cadd(xa, cscale(da, c.alpha));
      xb = cadd(xb, cscale(db, c.alpha));
    }
    float Sa, Sb;
    ld_pairf(A.S + base + o, Sa, Sb);
    const float ya = Sa - re_mul(xa, carrier(Lc, l.Pa, L.z));
    const float yb = Sb - re_mul(xb, carrier(Lc, l.Pb, L.z));
    st_pair(Xo + o, xa, xb, l.va, l.vb);
    if (l.va && l.vb) {
      __stcg(reinterpret_cast<float2*>(A.Y + base + o), make_float2(ya, yb));
    } else if (l.va) {
      __stcg(A.Y + base + o, ya);
    }
    // dense destination index; the caller's buffers carry no alignment
    // promise beyond a float's, so the wide stores are taken only where the
    // address allows them
    const int64_t od = (int64_t)y * f.w + l.xa;
    if (f.out_c) {
      float* oc = reinterpret_cast<float*>(f.out_c) + 2 * od;
      const uintptr_t ac = reinterpret_cast<uintptr_t>(oc);
      if (l.va && l.vb && (ac & 15) == 0) {
        __stcs(reinterpret_cast<float4*>(oc), make_float4(xa.x, xa.y, xb.x, xb.y));
      } else if ((ac & 7) == 0) {
        if (l.va) __stcs(reinterpret_cast<float2*>(oc), xa);
        if (l.vb) __stcs(reinterpret_cast<float2*>(oc) + 1, xb);
      } else {
        if (l.va) {
          __stcs(oc, xa.x);
          __stcs(oc + 1, xa.y);
        }
        if (l.vb) {
          __stcs(oc + 2, xb.x);
          __stcs(oc + 3, xb.y);
        }
      }
    }
    if (f.out_y) {
      if (l.va && l.vb && ((reinterpret_cast<uintptr_t>(f.out_y + od) & 7) == 0)) {
        __stcs(reinterpret_cast<float2*>(f.out_y + od), make_float2(ya, yb));
      } else {
        if (l.va) __stcs(f.out_y + od, ya);
        if (l.vb) __stcs(f.out_y + od + 1, yb);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Field-level completion: fixed-order reduction of the unit partials and the
// CG scalar logic (variational.cpp:519-549).
// ---------------------------------------------------------------------------
__device__ __noinline__ void complete_phase(const SolverArgs& A, const FieldDesc& f, int fi,
                                            int kind, int k, int p, int lane) {
  FieldCtl* c = A.ctl + fi;
  double s[kNPart];
#pragma unroll
  for (int i = 0; i < kNPart; ++i) s[i] = 0.0;
  if (kind == kPhaseG || kind == kPhaseI) {
    // the field's group sums: lane l adds groups l, l + 32, ... in that
    // order (a field has at most a few dozen groups: all loads of a lane
    // are in flight together), then a fixed butterfly across the lanes
    const int ng = (f.unit_count + kGroupUnits - 1) >> kGroupShift;
    double v[4][kNPart];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int i = 0; i < kNPart; ++i)
        v[j][i] = lane + 32 * j < ng
                      ? __ldcg(A.gpartials + (int64_t)(f.unit_begin + lane + 32 * j) * kNPart + i)
                      : 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int i = 0; i < kNPart; ++i) s[i] += v[j][i];
    for (int gg = lane + 128; gg < ng; gg += 32) {
#pragma unroll
      for (int i = 0; i < kNPart; ++i)
        s[i] += __ldcg(A.gpartials + (int64_t)(f.unit_begin + gg) * kNPart + i);
    }
#pragma unroll
    for (int i = 0; i < kNPart; ++i) s[i] = warp_allsum(s[i]);
  }
  int publish = p;
  if (lane == 0) {
    const int B = 2 + f.n_inner;
    if (kind == kPhaseR) {
      c->pending = 0;
      c->xsel ^= 1;
    } else if (kind == kPhaseG) {
      c->gg0 = s[0];
      c->gg = s[0];
      c->pending = 0;
      c->sel = 0;
    } else if (kind == kPhaseI) {
      const double H = s[0], gd = s[1], gq = s[2], qq = s[3], ggk = s[4];
      c->sel ^= 1;
      c->gg = ggk;
      const int o = p / B;
      const int last_i = o * B + 1 + f.n_inner;
      const double tol = (double)f.cg_tol;
      const double thr_rel = tol * tol * c->gg0, thr_abs = 1e-10 * (double)f.h * (double)f.w;
      if (k >= 1 && (ggk < thr_rel || ggk < thr_abs)) {
        // this sweep formed g_k = g_{k-1} + alpha q_{k-1} and applied
        // chi_k = chi_{k-1} + alpha d_{k-1} in place; ||g_k||^2, measured
        // here, is what the reference tests after its iteration k - 1
        // (variational.cpp:547-548): exit with chi_k final
        c->pending = 0;
        publish = last_i;
      } else if (H <= 1e-12) {
        c->pending = 0;
        publish = last_i;
      } else {
        const float alpha = (float)(-0.5 * gd / H);
        const double a = (double)alpha;
        const double gn = ggk + 2.0 * a * gq + a * a * qq;
        c->alpha = alpha;
        c->beta = (float)(gn / fmax(ggk, 1e-30));
        c->gg_next = gn;
        c->pending = 1;
        c->cg_iters += 1;
        // ||g_{k+1}||^2 predicted by the recurrence: the exit is taken now
        // only where the prediction lies below a threshold by more than its
        // rounding bound (FP32 terms, FP64 sums); nearer the threshold the
        // next sweep measures ||g_{k+1}||^2 and decides on that
        const double bound = 1e-5 * (ggk + 2.0 * fabs(a * gq) + a * a * qq);
        if (gn + bound < thr_rel || gn + bound < thr_abs) publish = last_i;
      }
    } else {
      c->pending = 0;
    }
    (void)k;
    // the release store orders this lane's control writes before the flag;
    // the other units' plane writes are already ordered before it by their
    // fence + arrival and this warp's fence after the last arrival
    st_release(A.done_phase + fi, publish);
  }
  __syncwarp();
}

// kDiag: the instantiation for launches with the oriented chroma prior (a
// larger ring slot and more carried state: one CTA per SM); the plain one
// keeps two.
template <bool kDiag>
__global__ void __launch_bounds__(kSolverThreads, kDiag ? 1 : 2)
    k_solver(const __grid_constant__ SolverArgs A) {
  const int lane = threadIdx.x & 31;
  extern __shared__ __align__(16) char solver_smem[];
  Ring ring;
  {
    char* wbase = solver_smem + (threadIdx.x >> 5) * RingLayout<kDiag>::warp;
    ring.slots = wbase;
    ring.bar = reinterpret_cast<uint64_t*>(wbase + kNS * RingLayout<kDiag>::slot);
    ring.bits = 0;
    if (lane == 0) {
      for (int i = 0; i < kNS; ++i) mbar_init(ring.bar + i, 1);
      fence_mbar_init();
      fence_proxy_async_smem();
    }
    __syncwarp();
  }
  const long long total = (long long)A.n_units * A.n_phases;
  for (;;) {
    long long item = 0;
    if (lane == 0) item = (long long)atomicAdd(A.queue, 1ULL);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total) break;
    const int p = (int)(item / A.n_units);
    const int ui = A.unit_base + (int)(item % A.n_units);
    const Unit u = A.units[ui];
    const FieldDesc f = A.fields[u.field];
    if (p >= f.n_phases) continue;
    int ok = 1, dp = 0;
    if (lane == 0) {
      ok = wait_at_least(A.done_phase + u.field, p - 1, A.phase_wait_limit);
      dp = ld_acquire(A.done_phase + u.field);
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    dp = __shfl_sync(0xffffffffu, dp, 0);
    if (!ok) {
      if (lane == 0) atomicOr(A.err, 1);
      break;
    }
    if (dp >= p) continue;  // phase skipped by an early CG exit
    __syncwarp();
    const int B = 2 + f.n_inner;
    int kind, k = 0;
    if (p == f.n_outer * B) {
      kind = kPhaseF;
    } else {
      const int r = p % B;
      kind = r == 0 ? kPhaseR : (r == 1 ? kPhaseG : kPhaseI);
      k = r - 2;
    }
    // A CG sweep's plane buffers follow from its position alone: the G phase
    // sets sel = 0 and every CG completion flips it (an early exit skips the
    // rest of the outer), every R completion flips xsel. So its first rows'
    // bulk copies go out before the control block's loads return, and the
    // block only supplies alpha and beta.
    FieldCtl ci;
    if (kind == kPhaseI) {
      ci.sel = k & 1;
      ci.xsel = (p / B + 1) & 1;
      if (lane == 0) {
        const int ybeg = max(u.y0 - 1, 0), yend = min(u.y1, f.h - 1);
        fence_proxy_async_global();
        fence_proxy_async_smem();
        for (int i = 0; i < min(kNS, yend - ybeg + 1); ++i) {
          const int y = ybeg + i;
          ring_issue<kDiag>(ring, i % kNS, A, f, ci, u.x0, y, k == 0, y >= u.y0 && y < u.y1);
        }
      }
    }
    FieldCtl c;
    {
      const FieldCtl* vc = A.ctl + u.field;
      c.alpha = __ldcg(&vc->alpha);
      c.beta = __ldcg(&vc->beta);
      c.pending = __ldcg(&vc->pending);
      c.sel = kind == kPhaseI ? ci.sel : __ldcg(&vc->sel);
      c.xsel = kind == kPhaseI ? ci.xsel : __ldcg(&vc->xsel);
    }
    double part[kNPart] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // the rarely taken phases are out of line (their registers do not
    // constrain the CG sweep); they read the field from its global copy
    const FieldDesc& fg = A.fields[u.field];
    if (kind == kPhaseR) {
      phase_reweight(A, fg, u, lane, c);
    } else if (kind == kPhaseG) {
      part[0] = part[4] = phase_gradient(A, fg, u, lane, c);
    } else if (kind == kPhaseI) {
      if (!phase_iter<kDiag>(A, f, u, lane, c, k == 0, ring, part)) {
        if (lane == 0) atomicOr(A.err, 2);
        break;
      }
    } else {
      phase_final(A, fg, u, lane, c);
    }
    if (kind == kPhaseG || kind == kPhaseI) {
#pragma unroll
      for (int i = 0; i < kNPart; ++i) {
        const double v = warp_sum(part[i]);
        if (lane == 0) __stcg(A.partials + (int64_t)ui * kNPart + i, v);
      }
    }
    // two-level arrival: the last unit of a group of kGroupUnits consecutive
    // units sums the group's partials (one load per lane, a fixed butterfly)
    // into the group's slot and arrives at the field; the field's last group
    // completes the phase. The end-of-phase reduction then reads a few dozen
    // group sums instead of every unit's partials.
    __threadfence();
    const int gj = (ui - f.unit_begin) >> kGroupShift;
    const int gslot = f.unit_begin + gj;
    const int gfirst = f.unit_begin + (gj << kGroupShift);
    const int gsize = min(kGroupUnits, f.unit_count - (gj << kGroupShift));
    // the counters only grow (zeroed before the launch): every unit of a
    // field arrives in a phase or none does (a phase skipped by an early
    // exit is skipped by all), so the group's last arrival of a phase is the
    // one that makes its count a multiple of the group size -- no reset
    // store for the fence below to wait on
    int last = 0;
    if (lane == 0) last = (atomicAdd(A.garrive + gslot, 1) + 1) % gsize == 0;
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) continue;
    __threadfence();
    if (kind == kPhaseG || kind == kPhaseI) {
      double gv[kNPart];
#pragma unroll
      for (int i = 0; i < kNPart; ++i)
        gv[i] = lane < gsize ? __ldcg(A.partials + (int64_t)(gfirst + lane) * kNPart + i) : 0.0;
#pragma unroll
      for (int i = 0; i < kNPart; ++i) {
        const double v = warp_sum(gv[i]);
        if (lane == 0) __stcg(A.gpartials + (int64_t)gslot * kNPart + i, v);
      }
      __threadfence();
    }
    const int ng = (f.unit_count + kGroupUnits - 1) >> kGroupShift;
    if (lane == 0) last = (atomicAdd(A.arrive + u.field, 1) + 1) % ng == 0;
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
      __threadfence();
      complete_phase(A, fg, u.field, kind, k, p, lane);
    }
  }
}

template <bool kDiag>
constexpr int solver_smem() {
  return (kSolverThreads / 32) * RingLayout<kDiag>::warp;
}

static PerDeviceOnce solver_once;

static void configure_solver() {
  solver_once([] {
    cudaFuncSetAttribute(k_solver<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         solver_smem<false>());
    cudaFuncSetAttribute(k_solver<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         solver_smem<true>());
  });
}

int solver_max_blocks_per_sm(bool diag) {
  configure_solver();
  int n = 0;
  if (diag)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solver<true>, kSolverThreads,
                                                  solver_smem<true>());
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_solver<false>, kSolverThreads,
                                                  solver_smem<false>());
  return n;
}

cudaError_t launch_solver(const SolverArgs& args, int grid, cudaStream_t st) {
  configure_solver();
  SolverArgs a = args;
  void* params[] = {&a};
  if (a.W2) {
    // the oriented-prior instantiation holds fewer CTAs per SM; the
    // persistent grid never exceeds what is co-resident
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    grid = std::max(1, std::min(grid, sms * std::max(1, solver_max_blocks_per_sm(true))));
    return cudaLaunchCooperativeKernel((const void*)k_solver<true>, dim3(grid),
                                       dim3(kSolverThreads), params, solver_smem<true>(), st);
  }
  return cudaLaunchCooperativeKernel((const void*)k_solver<false>, dim3(grid),
                                     dim3(kSolverThreads), params, solver_smem<false>(), st);
}

}  // namespace hvdg
