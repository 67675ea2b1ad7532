"""TEST INFRASTRUCTURE -- FP64 oracle of the decode adjoint.

The reference has no adjoint; this module differentiates the forward path as
restated in oracle/hvd_oracle.py: HolographicInit (hvd-core/src/engine/
holographic_init.cpp:200-317) followed by the IRLS + CG VariationalRefine
(variational.cpp:198-556; lagged-diffusivity weights :406-433, gradient
:286-347, curvature :352-399), and the output luma Y = S - Re[chi c]
(sequence.cpp:1102-1114). Only tests/ import it, as the checker of the
device adjoint.

Formulation (implicit function, per IRLS outer o): chi_{o+1} minimises the
quadratic E_o(chi; W_o, S, mu) whose weights W_o = W(chi_o) are frozen at
the start of the outer, so g_o(chi_{o+1}) = 0 and, with H_o the (real,
symmetric) Hessian applied by the CG operator q = g(d) - g(0),
    lambda_o = H_o^-1 chibar_{o+1},   dL/dp = -<lambda_o, dg_o/dp>,
where <a, b> = Re sum conj(a) b. The chain to chi_o runs only through the
lagged weights W(chi_o). This is exact for converged inner solves; with a
truncated CG budget it is the gradient of the converged IRLS map.

Held at their forward values (no gradient through them): the lock-in
carrier phase and the chroma-anisotropy split (an order statistic).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import hvd_oracle as O


def rdot(a, b) -> float:
    """Real inner product of complex (or real) planes."""
    return float(np.sum(np.real(np.conj(a) * b)))


@dataclass
class Weights:
    wx: np.ndarray
    wy: np.ndarray
    wcx: np.ndarray
    wcy: np.ndarray
    gx: np.ndarray
    gy: np.ndarray
    rx: np.ndarray      # mx^2 + k gx^2 + eps_c^2
    ry: np.ndarray


def weights(s, c, chi, eps, eps_c, k) -> Weights:
    """Lagged-diffusivity weights at chi (variational.cpp:406-433)."""
    yc = s - np.real(chi * c)
    gx, gy = O.Dx(yc), O.Dy(yc)
    mx2, my2 = np.abs(O.Dx(chi)) ** 2, np.abs(O.Dy(chi)) ** 2
    rx = mx2 + k * gx * gx + eps_c * eps_c
    ry = my2 + k * gy * gy + eps_c * eps_c
    return Weights(eps / np.sqrt(gx * gx + eps * eps), eps / np.sqrt(gy * gy + eps * eps),
                   eps_c / np.sqrt(rx), eps_c / np.sqrt(ry), gx, gy, rx, ry)


def hess(c, d, W: Weights, mu_h, mu_v):
    """H d = g(d) - g(0): the CG operator (gradient of E at d with S = 0)."""
    r = np.real(d * c)
    img = 2.0 * (O.DxT(W.wx * O.Dx(r)) + O.DyT(W.wy * O.Dy(r)))
    cpr = 2.0 * (mu_h * O.DxT(W.wcx * O.Dx(d)) + mu_v * O.DyT(W.wcy * O.Dy(d)))
    return img * np.conj(c) + cpr


def grad(s, c, chi, W: Weights, mu_h, mu_v):
    """g(chi) (variational.cpp:286-347), 2-D."""
    yc = s - np.real(chi * c)
    img = 2.0 * (O.DxT(W.wx * O.Dx(yc)) + O.DyT(W.wy * O.Dy(yc)))
    cpr = 2.0 * (mu_h * O.DxT(W.wcx * O.Dx(chi)) + mu_v * O.DyT(W.wcy * O.Dy(chi)))
    return -img * np.conj(c) + cpr


def cg_solve(apply, b, tol=1e-13, maxit=20000):
    """CG for H x = b in the real inner product, from x = 0, until
    ||r|| <= tol ||b||."""
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = rdot(r, r)
    rr0 = rr
    it = 0
    while it < maxit and rr > tol * tol * rr0 and rr > 0.0:
        q = apply(p)
        a = rr / rdot(p, q)
        x = x + a * p
        r = r - a * q
        rn = rdot(r, r)
        p = r + (rn / rr) * p
        rr = rn
        it += 1
    return x, it


def refine_forward(s, c, chi0, cfg, aniso, tol=1e-13, maxit=20000):
    """IRLS outers with each quadratic solved by CG to ||g|| <= tol ||g_0||.
    Returns the iterates chi_0 .. chi_n (chi_0 = chi0)."""
    s = np.asarray(s, np.float64)
    c = np.asarray(c, np.complex128)
    eps, eps_c, k = float(cfg.charbonnier_eps), float(cfg.chroma_eps), float(cfg.structure_coupling)
    mu_h, mu_v = float(cfg.lambda_c) * aniso, float(cfg.lambda_c)
    n_outer = max(1, int(cfg.irls_outer))
    chis = [np.array(chi0, np.complex128)]
    for _ in range(n_outer):
        chi = chis[-1]
        W = weights(s, c, chi, eps, eps_c, k)
        g = grad(s, c, chi, W, mu_h, mu_v)
        delta, _ = cg_solve(lambda d: hess(c, d, W, mu_h, mu_v), -g, tol, maxit)
        chis.append(chi + delta)
    return chis


def refine_forward_budget(s, c, chi0, cfg, aniso):
    """IRLS outers with the reference's CG budget and exits
    (variational.cpp:224-230, 519-549), one VariationalRefine call per outer
    so that every iterate chi_o is kept; the anisotropy split is the one
    resolved from the init chi0."""
    irls_outer, n_inner, tol = O.solver_budget(cfg)
    c1 = _config_copy(cfg, irls_outer=1, cg_iterations=n_inner, fast=0, cg_tol=tol,
                      chroma_aniso=aniso)
    chis = [np.array(chi0, np.complex128)]
    for _ in range(irls_outer):
        _, chi = O.variational_refine(s, c, chis[-1], c1)
        chis.append(chi)
    return chis


def _config_copy(cfg, **kw):
    import copy
    c = copy.copy(cfg)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def refine_adjoint(s, c, chis, cfg, aniso, y_bar, chi_bar, tol=1e-13, maxit=20000):
    """Cotangents of (Y, chi) = refine(...) -> (S_bar, chi0_bar, scalar grads)
    for the scalars lambda_c, eps (charbonnier_eps), eps_c (chroma_eps) and
    k (structure_coupling)."""
    s = np.asarray(s, np.float64)
    c = np.asarray(c, np.complex128)
    eps, eps_c, k = float(cfg.charbonnier_eps), float(cfg.chroma_eps), float(cfg.structure_coupling)
    mu_h, mu_v = float(cfg.lambda_c) * aniso, float(cfg.lambda_c)
    y_bar = np.asarray(y_bar, np.float64)
    s_bar = y_bar.copy()
    chib = np.asarray(chi_bar, np.complex128) - y_bar * np.conj(c)
    gl = {"lambda_c": 0.0, "eps": 0.0, "eps_c": 0.0, "k": 0.0}
    for o in reversed(range(len(chis) - 1)):
        chi_o, chi1 = chis[o], chis[o + 1]
        W = weights(s, c, chi_o, eps, eps_c, k)
        lam, _ = cg_solve(lambda d: hess(c, d, W, mu_h, mu_v), chib, tol, maxit)
        r = np.real(lam * c)
        # data term: dg/dS
        s_bar += 2.0 * (O.DxT(W.wx * O.Dx(r)) + O.DyT(W.wy * O.Dy(r)))
        # chroma priors: dg/dmu
        tx = np.real(np.conj(O.Dx(lam)) * O.Dx(chi1))
        ty = np.real(np.conj(O.Dy(lam)) * O.Dy(chi1))
        gl["lambda_c"] += -2.0 * float(np.sum(W.wcx * tx)) * aniso - 2.0 * float(np.sum(W.wcy * ty))
        # dg/dW at chi_{o+1}
        yc1 = s - np.real(chi1 * c)
        wbx = 2.0 * O.Dx(yc1) * O.Dx(r)
        wby = 2.0 * O.Dy(yc1) * O.Dy(r)
        wbcx = -2.0 * mu_h * tx
        wbcy = -2.0 * mu_v * ty
        # W(chi_o; eps, eps_c, k)
        ex = W.gx * W.gx + eps * eps
        ey = W.gy * W.gy + eps * eps
        gbx = wbx * (-W.wx * W.gx / ex) + wbcx * (-W.wcx * k * W.gx / W.rx)
        gby = wby * (-W.wy * W.gy / ey) + wbcy * (-W.wcy * k * W.gy / W.ry)
        mbx = wbcx * (-0.5 * W.wcx / W.rx)
        mby = wbcy * (-0.5 * W.wcy / W.ry)
        gl["eps"] += float(np.sum(wbx * W.wx * W.gx ** 2 / (eps * ex))
                           + np.sum(wby * W.wy * W.gy ** 2 / (eps * ey)))
        gl["eps_c"] += float(np.sum(wbcx * W.wcx * (W.rx - eps_c ** 2) / (eps_c * W.rx))
                             + np.sum(wbcy * W.wcy * (W.ry - eps_c ** 2) / (eps_c * W.ry)))
        gl["k"] += float(np.sum(wbcx * (-0.5 * W.wcx * W.gx ** 2 / W.rx))
                         + np.sum(wbcy * (-0.5 * W.wcy * W.gy ** 2 / W.ry)))
        ycb = O.DxT(gbx) + O.DyT(gby)
        s_bar += ycb
        chib = (-ycb * np.conj(c) + O.DxT(2.0 * mbx * O.Dx(chi_o))
                + O.DyT(2.0 * mby * O.Dy(chi_o)))
    return s_bar, chib, gl


def _init_ops(s, g):
    h, w = s.shape
    pad = min(16, h - 1 if h > 1 else 0)
    hp = h + 2 * pad
    rows = O.mirror_row(np.arange(hp) - pad, h)
    masks = []
    for (mhz, cph) in O.INIT_VARIANTS:
        gy, gx = O.gaussian_lpf(hp, w, g, mhz, cph, h)
        masks.append(gy[:, None] * gx[None, :])
    return pad, hp, rows, masks


def init_parts(s, c, g):
    """HolographicInit (holographic_init.cpp:200-317) with its intermediates."""
    s = np.asarray(s, np.float64)
    pad, hp, rows, masks = _init_ops(s, g)
    h = s.shape[0]
    spec = np.fft.fft2((s * np.conj(c))[rows])
    chis, wts = [], []
    for m in masks:
        chi_v = np.fft.ifft2(spec * m)[pad:pad + h] * 2.0
        y_v = s - np.real(chi_v * c)
        chis.append(chi_v)
        wts.append(1.0 / (O.edge_energy(y_v) + 0.5))
    wsum = wts[0] + wts[1]
    chi0 = (chis[0] * wts[0] + chis[1] * wts[1]) / wsum
    return chis, wts, chi0


def init_adjoint(s, c, g, chi0_bar):
    """S_bar of chi0 = HolographicInit(S, c) for the cotangent chi0_bar."""
    s = np.asarray(s, np.float64)
    c = np.asarray(c, np.complex128)
    h, w = s.shape
    pad, hp, rows, masks = _init_ops(s, g)
    chis, wts, chi0 = init_parts(s, c, g)
    wsum = wts[0] + wts[1]
    s_bar = np.zeros((h, w))
    u_bar = np.zeros((hp, w), np.complex128)
    for chi_v, wt, m in zip(chis, wts, masks):
        cb = chi0_bar * (wt / wsum)
        w_bar = np.real(np.conj(chi0_bar) * (chi_v - chi0)) / wsum
        e_bar = -w_bar * wt * wt
        a_bar = O.box_blur_same(e_bar, 3)          # the zero-padded box is self-adjoint
        y_v = s - np.real(chi_v * c)
        dx, dy = O.Dx(y_v), O.Dy(y_v)
        yb = O.DxT(np.sign(dx) * a_bar) + O.DyT(np.sign(dy) * a_bar)
        s_bar += yb
        cb = cb - yb * np.conj(c)
        emb = np.zeros((hp, w), np.complex128)
        emb[pad:pad + h] = cb
        u_bar += np.fft.ifft2(np.fft.fft2(emb) * m) * 2.0   # real mask: the op is self-adjoint
    fold = np.zeros((h, w), np.complex128)
    np.add.at(fold, rows, u_bar)
    return s_bar + np.real(fold * c)


@dataclass
class DecodeGrad:
    loss: float
    samples_bar: np.ndarray   # d loss / d raw sample code, field_height x field_width
    scalars: dict             # lambda_c, eps, eps_c, k
    y: np.ndarray
    chi: np.ndarray


def decode_loss_and_grad(field_ire, g, cfg, y_true, chi_true, codes_per_ire, parity=0,
                         tol=1e-13, carrier=None, aniso=None):
    """Forward (init + converged IRLS) and the full gradient of
    L = mean((Y - Y_true)^2) + mean(|chi - chi_true|^2) with respect to the
    raw field samples (through S; the lock-in carrier held) and the four
    scalars. `carrier` / `aniso` override the forward's (FD checks pass the
    unperturbed ones)."""
    obs = O.prepare_field(field_ire, g, cfg, parity)
    c = obs.carrier if carrier is None else carrier
    s = obs.s
    _, _, chi0 = init_parts(s, c, g)
    if aniso is None:
        aniso = O.resolve_chroma_aniso(chi0, cfg, O.uses_vswitch(g))
    chis = refine_forward(s, c, chi0, cfg, aniso, tol)
    chi = chis[-1]
    y = s - np.real(chi * c)
    n = y.size
    loss = float(np.mean((y - y_true) ** 2) + np.mean(np.abs(chi - chi_true) ** 2))
    y_bar = 2.0 * (y - y_true) / n
    chi_bar = 2.0 * (chi - chi_true) / n
    s_bar, chi0_bar, gl = refine_adjoint(s, c, chis, cfg, aniso, y_bar, chi_bar, tol)
    s_bar = s_bar + init_adjoint(s, c, g, chi0_bar)
    fb = np.zeros((g.field_height, g.field_width))
    fal, lal = g.first_active_field_line, O.last_active_line(g)
    fb[fal:lal, g.active_video_start:g.active_video_end] = s_bar / codes_per_ire
    return DecodeGrad(loss, fb, gl, y, chi), c, aniso
