"""TEST INFRASTRUCTURE -- the FP64 oracle of the hvd-core hot path.

A float64 NumPy restatement of the reference engine's algorithm (hvd-core,
NOT research/hvd/decoder.py: the two differ, e.g. the C++ init's reflect-101
pad and the per-field 2-D path). Every function cites the reference
file:line it follows (paths relative to hvd-core/src/). Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg import this module,
and only as the checker.

Pinned (tests/test_oracle_pins.py) against
  * the reference's own analytic tests (lockin_test.cpp, pal_lockin_test.cpp,
    gradients_test.cpp, lossless_identity_test.cpp, motion_test.cpp), and
  * the compiled reference engine (oracle/_ref/libhvdref.so, float32) on the
    same seeded inputs, and the committed fixtures in tests/golden/.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PI = math.pi

STD_NTSC, STD_PAL, STD_PAL_M = 0, 1, 2


# --------------------------------------------------------------------------
# Geometry (engine/ntsc_geometry.h:142-267)
# --------------------------------------------------------------------------

def uses_vswitch(g) -> bool:
    return g.standard in (STD_PAL, STD_PAL_M)


def phase_per_sample(g) -> float:
    """FieldGeometry::phase_per_sample (ntsc_geometry.h:200-203)."""
    if g.subcarrier_hz <= 0.0:
        return 0.5 * PI
    return 2.0 * PI * g.subcarrier_hz / g.sample_rate


def line_advance(g) -> float:
    """FieldGeometry::line_advance (ntsc_geometry.h:216-251)."""
    if g.subcarrier_hz <= 0.0:
        if g.standard == STD_PAL:
            return 2.0 * PI * 0.7516
        if g.standard == STD_PAL_M:
            return 0.5 * PI
        return PI
    cycles = g.subcarrier_hz * g.field_width / g.sample_rate
    return 2.0 * PI * (cycles - math.floor(cycles))


def nominal_burst_ire(g) -> float:
    """ntsc_geometry.h:256-258."""
    return 21.43 if g.standard == STD_PAL else 20.0


def active_lines(g) -> int:
    lal = g.last_active_field_line if g.last_active_field_line != 0 else g.field_height
    return lal - g.first_active_field_line


def last_active_line(g) -> int:
    return g.last_active_field_line if g.last_active_field_line != 0 else g.field_height


def sample_to_ire(s, blanking, white):
    """SampleToIre (ntsc_geometry.h:301-304)."""
    return (np.asarray(s, np.float64) - blanking) / ((white - blanking) / 100.0)


def wrap_pi(a):
    """WrapPi (lockin.cpp:93-95): atan2(sin, cos), range (-pi, pi]."""
    return np.arctan2(np.sin(a), np.cos(a))


def upper_median(v) -> float:
    """MedianOf in lockin.cpp:85-90 / Median in ntsc_geometry.cpp:384-389:
    nth_element at n/2, no averaging."""
    v = np.asarray(v, np.float64)
    if v.size == 0:
        return 0.0
    k = v.size // 2
    return float(np.partition(v, k)[k])


def mean_median(v) -> float:
    """MedianOf in sequence.cpp:29-39 / Median in motion.cpp:80-91: averages
    the two middle values for even n (numpy.median)."""
    v = np.asarray(v, np.float64)
    if v.size == 0:
        return 0.0
    return float(np.median(v))


# --------------------------------------------------------------------------
# Burst lock-in (engine/lockin.cpp)
# --------------------------------------------------------------------------

def burst_lockin_z(field, g):
    """BurstLockin (lockin.cpp:103-130): z[line] = mean((seg - mean(seg)) *
    exp(-i w0 x)) over the burst window, x the absolute sample index."""
    f = np.asarray(field, np.float64)
    x0, x1 = g.colour_burst_start, g.colour_burst_end
    n = max(0, x1 - x0)
    h = f.shape[0]
    if n == 0:
        return np.zeros(h, np.complex128), np.zeros(h)
    w0 = phase_per_sample(g)
    seg = f[:, x0:x1]
    seg = seg - seg.mean(axis=1, keepdims=True)
    xs = np.arange(x0, x1)
    z = (seg * np.exp(-1j * w0 * xs)[None, :]).sum(axis=1) / n
    return z, np.abs(z)


def tridiag_smooth(d, a, lam):
    """TridiagSmooth (lockin.cpp:133-167): solve (diag(a) + lam L) x = a d,
    L the Neumann 1-D Laplacian, by the Thomas algorithm."""
    d = np.asarray(d, np.float64)
    a = np.asarray(a, np.float64)
    n = d.size
    x = np.zeros(n)
    if n == 0:
        return x
    if n == 1:
        x[0] = d[0] if a[0] > 0 else 0.0
        return x
    diag = a + 2.0 * lam
    diag[0] -= lam
    diag[-1] -= lam
    off = -lam
    rhs = a * d
    c = np.zeros(n - 1)
    dd = np.zeros(n)
    c[0] = off / diag[0]
    dd[0] = rhs[0] / diag[0]
    for i in range(1, n):
        m = diag[i] - off * c[i - 1]
        if i < n - 1:
            c[i] = off / m
        dd[i] = (rhs[i] - off * dd[i - 1]) / m
    x[n - 1] = dd[n - 1]
    for i in range(n - 2, -1, -1):
        x[i] = dd[i] - c[i] * x[i + 1]
    return x


def _robust_trajectory(d, amp, good, lam=25.0):
    """Amplitude weights + tridiag + one Huber IRLS (lockin.cpp:231-250,
    399-414)."""
    med_amp = upper_median(amp[good]) + 1e-9
    a = np.where(good, np.clip(amp / med_amp, 0.0, 2.0), 0.0)
    x = tridiag_smooth(d, a, lam)
    r = np.abs(d - x)
    a2 = a * 0.15 / np.maximum(r, 0.15)
    return tridiag_smooth(d, a2, lam)


def burst_lockin_phase(field, g):
    """BurstLockinPhase (lockin.cpp:169-254), NTSC."""
    z, amp = burst_lockin_z(field, g)
    h = z.size
    theta = np.angle(z) - 0.5 * PI
    amp_max = amp.max() if h else 0.0
    thresh = amp_max * 0.2 if amp_max > 0 else 1.0
    good = amp > thresh
    if not good.any():
        return theta
    fg = int(np.argmax(good))
    adv = line_advance(g)
    model = theta[fg] + adv * (np.arange(h) - fg)
    d = wrap_pi(theta - model)
    x = _robust_trajectory(d, amp, good)
    return model + x


def burst_lockin_phase_pal(field, g):
    """BurstLockinPhasePal (lockin.cpp:325-417): joint phase + V-switch
    parity by two-hypothesis amplitude-weighted scoring."""
    z, amp = burst_lockin_z(field, g)
    h = z.size
    adv = line_advance(g)
    q = 0.25 * PI
    amp_max = amp.max() if h else 0.0
    thresh = amp_max * 0.2 if amp_max > 0 else 1.0
    good = amp > thresh
    ys = np.arange(h)
    if not good.any():
        theta = adv * ys
        vs = np.where(ys % 2 == 0, 1, -1).astype(np.int8)
        return theta, vs
    fg = int(np.argmax(good))
    a_meas = np.angle(z)
    best_score = -1e30
    best = None
    for hyp in (0, 1):
        s_ref = 1.0 if hyp == 0 else -1.0
        theta_ref = a_meas[fg] - 0.5 * PI + s_ref * q
        m = theta_ref + adv * (ys - fg)
        same = ((ys - fg) % 2) == 0
        sy = np.where(same, s_ref, -s_ref)
        dev = wrap_pi(a_meas - (m + 0.5 * PI - sy * q))
        score = float(np.sum(np.where(good, np.cos(dev) * amp, 0.0)))
        if score > best_score:
            best_score = score
            best = (m, sy)
    model, sy = best
    vs = np.where(sy > 0, 1, -1).astype(np.int8)
    theta_meas = a_meas - 0.5 * PI + sy * q
    d = wrap_pi(theta_meas - model)
    x = _robust_trajectory(d, amp, good)
    return model + x, vs


def burst_amplitude_ire(field, g) -> float:
    """BurstAmplitudeIre (lockin.cpp:256-323): median over lines of the
    median sliding one-cycle envelope."""
    f = np.asarray(field, np.float64)
    x0, x1 = g.colour_burst_start, g.colour_burst_end
    if x1 - x0 < 4:
        return nominal_burst_ire(g)
    w0 = phase_per_sample(g)
    ph = np.exp(-1j * w0 * np.arange(x0, x1))
    prod = f[:, x0:x1] * ph[None, :]
    nseg = (x1 - x0) - 4 + 1
    acc = sum(prod[:, k:k + nseg] for k in range(4))
    env = 2.0 * np.abs(acc) * 0.25
    per_line = np.array([upper_median(env[y]) for y in range(f.shape[0])])
    if per_line.size == 0:
        return nominal_burst_ire(g)
    med_all = upper_median(per_line)
    good = per_line[per_line > 0.25 * med_all]
    return nominal_burst_ire(g) if good.size == 0 else upper_median(good)


def acc_gain(median_burst_ire, nominal):
    """AccGain (colour.cpp:24-27)."""
    return float(np.clip(nominal / max(median_burst_ire, 1.0), 0.5, 2.0))


# --------------------------------------------------------------------------
# Carrier (ntsc_geometry.h:341-352, ntsc_geometry.cpp:392-456)
# --------------------------------------------------------------------------

def apply_chroma_phase(theta, vswitch, deg, g):
    """ApplyChromaPhase (ntsc_geometry.h:341-352)."""
    theta = np.array(theta, np.float64)
    if deg == 0.0:
        return theta
    off = -deg * PI / 180.0
    signed = uses_vswitch(g) and vswitch is not None and len(vswitch) == len(theta)
    if signed:
        return theta + np.where(np.asarray(vswitch) < 0, -off, off)
    return theta + off


def make_carrier(theta_active, vswitch_active, g):
    """MakeCarrier / MakeCarrierPal: c = exp(i (theta + w0 (a0 + x))), and
    -conj(c) on V-switched lines."""
    w0 = phase_per_sample(g)
    xs = g.active_video_start + np.arange(g.active_video_end - g.active_video_start)
    c = np.exp(1j * (np.asarray(theta_active, np.float64)[:, None] + w0 * xs[None, :]))
    if uses_vswitch(g):
        sw = np.asarray(vswitch_active) < 0
        c = np.where(sw[:, None], -np.conj(c), c)
    return c


@dataclass
class FieldObs:
    s: np.ndarray          # active composite, IRE
    carrier: np.ndarray    # complex
    theta: np.ndarray      # full-field per-line phase (after trim)
    vswitch: np.ndarray    # full-field per-line V-switch
    parity: int = 0


def prepare_field(field_ire, g, cfg, parity=0) -> FieldObs:
    """PrepareFieldObs (sequence.cpp:229-268)."""
    f = np.asarray(field_ire, np.float64)
    if uses_vswitch(g):
        theta, vs = burst_lockin_phase_pal(f, g)
    else:
        theta = burst_lockin_phase(f, g)
        vs = np.ones(f.shape[0], np.int8)
    theta = apply_chroma_phase(theta, vs if uses_vswitch(g) else None, cfg.chroma_phase_deg, g)
    fal, lal = g.first_active_field_line, last_active_line(g)
    a0, a1 = g.active_video_start, g.active_video_end
    s = f[fal:lal, a0:a1].copy()
    car = make_carrier(theta[fal:lal], vs[fal:lal], g)
    return FieldObs(s, car, theta, vs, parity)


# --------------------------------------------------------------------------
# Difference operators (engine/gradients.h) -- Neumann, exact adjoints
# --------------------------------------------------------------------------

def Dx(a):
    """gradients.h:25-41."""
    d = np.zeros_like(a)
    d[:, :-1] = a[:, 1:] - a[:, :-1]
    return d


def Dy(a):
    """gradients.h:43-59."""
    d = np.zeros_like(a)
    d[:-1] = a[1:] - a[:-1]
    return d


def DxT(a):
    """gradients.h:61-82."""
    d = np.zeros_like(a)
    w = a.shape[1]
    if w < 2:
        return d
    d[:, 0] = -a[:, 0]
    d[:, 1:-1] = a[:, :-2] - a[:, 1:-1]
    d[:, -1] = a[:, -2]
    return d


def DyT(a):
    """gradients.h:84-101."""
    d = np.zeros_like(a)
    h = a.shape[0]
    if h < 2:
        return d
    d[0] = -a[0]
    d[1:-1] = a[:-2] - a[1:-1]
    d[-1] = a[-2]
    return d


def D1(a):
    """+45 deg (gradients.h:195-211): d[:-1, :-1] = a[1:, 1:] - a[:-1, :-1]."""
    d = np.zeros_like(a)
    d[:-1, :-1] = a[1:, 1:] - a[:-1, :-1]
    return d


def D1T(a):
    """Adjoint of D1 (gradients.h:213-236)."""
    d = np.zeros_like(a)
    d[:-1, :-1] -= a[:-1, :-1]
    d[1:, 1:] += a[:-1, :-1]
    return d


def D2(a):
    """-45 deg (gradients.h:238-254): d[:-1, 1:] = a[1:, :-1] - a[:-1, 1:]."""
    d = np.zeros_like(a)
    d[:-1, 1:] = a[1:, :-1] - a[:-1, 1:]
    return d


def D2T(a):
    """Adjoint of D2 (gradients.h:256-279)."""
    d = np.zeros_like(a)
    d[:-1, 1:] -= a[:-1, 1:]
    d[1:, :-1] += a[:-1, 1:]
    return d


# --------------------------------------------------------------------------
# Holographic init (engine/holographic_init.cpp)
# --------------------------------------------------------------------------

def gaussian_lpf(h, w, g, lpf_h_mhz, lpf_v_cph, h_ref):
    """GaussianLpf (holographic_init.cpp:33-56): separable Gaussian mask on
    numpy fftfreq grids; vertical cutoff against the REAL height h_ref."""
    fx = np.fft.fftfreq(w, 1.0 / g.sample_rate)
    fy = np.fft.fftfreq(h, 1.0)
    cx = lpf_h_mhz * 1.0e6
    cy = lpf_v_cph / (2.0 * h_ref)
    gx = np.exp(-0.5 * (fx / cx) ** 2)
    gy = np.exp(-0.5 * (fy / cy) ** 2)
    return gy, gx


def mirror_row(y, h):
    """MirrorRow (holographic_init.cpp:126-131): reflect-101."""
    if h <= 1:
        return np.zeros_like(y)
    period = 2 * h - 2
    y = np.mod(y, period)
    return np.where(y < h, y, period - y)


def box_blur_same(a, r):
    """BoxBlur (holographic_init.cpp:61-113): zero-padded 'same' box of
    length 2r+1 per axis, constant 1/(2r+1) normalisation. Same semantics
    as motion.cpp's BoxBlur (motion.cpp:21-55, 391-395)."""
    a = np.asarray(a, np.float64)
    h, w = a.shape
    k = 2 * r + 1
    c = np.zeros((h + 1, w))
    c[1:] = np.cumsum(a, axis=0)
    y = np.arange(h)
    y0 = np.maximum(y - r, 0)
    y1 = np.minimum(y + r + 1, h)
    b = (c[y1] - c[y0]) / k
    c2 = np.zeros((h, w + 1))
    c2[:, 1:] = np.cumsum(b, axis=1)
    x = np.arange(w)
    x0 = np.maximum(x - r, 0)
    x1 = np.minimum(x + r + 1, w)
    return (c2[:, x1] - c2[:, x0]) / k


def edge_energy(y):
    """EdgeEnergy (holographic_init.cpp:185-196)."""
    return box_blur_same(np.abs(Dx(y)) + np.abs(Dy(y)), 3)


INIT_VARIANTS = ((0.8, 120.0), (1.8, 30.0))  # holographic_init.cpp:236


def symmetry_certify(spec, gy, gx):
    """The third variant's spectrum (holographic_init.cpp:265-290): each bin
    weighted by min(|D[k]|, |D[-k]|) / (|D[k]| + 1e-6) -- bin k pairs with
    its point reflection ((hp - y) mod hp, (w - x) mod w) -- and the
    {1.3 MHz, 60 c/ph} Gaussian crop."""
    hp, w = spec.shape
    mag = np.abs(spec)
    ry = (hp - np.arange(hp)) % hp
    rx = (w - np.arange(w)) % w
    mr = mag[ry][:, rx]
    sym = np.minimum(mag, mr) / (mag + 1e-6)
    return spec * sym * gy[:, None] * gx[None, :]


def holographic_init(s, carrier, g, symmetry_variant=False):
    """HolographicInit (holographic_init.cpp:200-317), with the optional
    spectral-symmetry third variant (:265-306)."""
    s = np.asarray(s, np.float64)
    h, w = s.shape
    demod = s * np.conj(carrier)
    pad = min(16, h - 1 if h > 1 else 0)
    hp = h + 2 * pad
    rows = mirror_row(np.arange(hp) - pad, h)
    spec = np.fft.fft2(demod[rows])
    num = np.zeros((h, w), np.complex128)
    wsum = np.zeros((h, w))
    crops = []
    for (mhz, cph) in INIT_VARIANTS:
        gy, gx = gaussian_lpf(hp, w, g, mhz, cph, h)
        crops.append(spec * gy[:, None] * gx[None, :])
    if symmetry_variant:
        gy, gx = gaussian_lpf(hp, w, g, 1.3, 60.0, h)
        crops.append(symmetry_certify(spec, gy, gx))
    for crop in crops:
        chi_v = np.fft.ifft2(crop)[pad:pad + h] * 2.0
        y_v = s - np.real(chi_v * carrier)
        wt = 1.0 / (edge_energy(y_v) + 0.5)
        num += chi_v * wt
        wsum += wt
    chi0 = num / wsum
    return s - np.real(chi0 * carrier), chi0


def init_row_kernels(g, w):
    """Spatial form of the two horizontal crops: k_v = IDFT_w(gx_v), so that
    IDFT(gx_v * DFT(row)) is the circular convolution of the row with k_v."""
    out = []
    for (mhz, cph) in INIT_VARIANTS:
        gx = np.exp(-0.5 * (np.fft.fftfreq(w, 1.0 / g.sample_rate) / (mhz * 1e6)) ** 2)
        out.append(np.fft.ifft(gx))
    return out


# --------------------------------------------------------------------------
# Variational refine (engine/variational.cpp)
# --------------------------------------------------------------------------

def resolve_chroma_aniso(chi0, cfg, is_pal):
    """ResolveChromaAniso (variational.cpp:130-196)."""
    if cfg.chroma_aniso > 0.0:
        return float(cfg.chroma_aniso)
    group = 4 if is_pal else 2
    h, w = chi0.shape
    Hh = h // group
    pav = chi0[:Hh * group].reshape(Hh, group, w).mean(axis=1)
    ts = np.arange(1, Hh, 2)
    xs = np.arange(1, w, 3)
    gx = np.abs(pav[ts][:, xs] - pav[ts][:, xs - 1]).ravel()
    gy = np.abs(pav[ts][:, xs] - pav[ts - 1][:, xs]).ravel()

    def p98(v):
        if v.size == 0:
            return 0.0
        k = v.size - 1 - v.size // 50
        return float(np.partition(v, k)[k])
    px, py = p98(gx), p98(gy)
    r = py / max(px, 1e-6)
    if is_pal:
        return float(np.clip(0.7 + 0.9 * (r - 1.3), 0.55, 1.0))
    return float(np.clip(0.5 + 1.1 * (r - 1.3), 0.5, 1.0))


@dataclass
class Neighbor:
    composite: np.ndarray   # S_w
    carrier: np.ndarray     # c_w
    confidence: np.ndarray  # conf


def solver_budget(cfg):
    """variational.cpp:224-230."""
    irls_outer = max(1, int(cfg.irls_outer))
    cg_total = (cfg.cg_iterations * 2) // 3 if cfg.fast else cfg.cg_iterations
    n_inner = max(1, cg_total // irls_outer)
    tol = cfg.cg_tol if cfg.cg_tol > 0.0 else (0.10 if cfg.fast else 0.02)
    return irls_outer, n_inner, float(tol)


def variational_refine(s, carrier, chi0, cfg, is_pal=False, neighbors=(), stats=None,
                       return_weights=False):
    """VariationalRefine (variational.cpp:198-556), FP64 throughout,
    including the oriented +-45 deg chroma prior of diag_prior > 0
    (variational.cpp:207-222, 316-328, 371-383, 434-451)."""
    s = np.asarray(s, np.float64)
    c = np.asarray(carrier, np.complex128)
    eps, eps_c = float(cfg.charbonnier_eps), float(cfg.chroma_eps)
    aniso = resolve_chroma_aniso(np.asarray(chi0, np.complex128), cfg, is_pal)
    mu_h = cfg.lambda_c * aniso
    mu_v = float(cfg.lambda_c)
    # oriented prior weight, distance-normalised by 1/2, and the total prior
    # mass kept: mu_h, mu_v, mu_d scaled by tot0 / (tot0 + 2 mu_d)
    mu_d = float(cfg.lambda_c) * float(cfg.diag_prior) * 0.5
    if mu_d > 0.0:
        tot0 = float(cfg.lambda_c) * (1.0 + aniso)
        scale = tot0 / (tot0 + 2.0 * mu_d)
        mu_h, mu_v, mu_d = mu_h * scale, mu_v * scale, mu_d * scale
    k = float(cfg.structure_coupling)
    nbrs = list(neighbors)
    nu = float(cfg.temporal_strength) if nbrs else 0.0
    eps_t = float(cfg.temporal_eps)
    irls_outer, n_inner, tol = solver_budget(cfg)
    N = s.size
    chi = np.array(chi0, np.complex128)
    dcs = [c - np.asarray(nb.carrier, np.complex128) for nb in nbrs]
    wts = [None] * len(nbrs)
    e2, ec2, et2 = eps * eps, eps_c * eps_c, eps_t * eps_t

    def trm(ch, j):
        return (np.asarray(nbrs[j].composite, np.float64) - s) + np.real(ch * dcs[j])

    W = {}

    def grad(ch):
        yc = s - np.real(ch * c)
        img = 2.0 * (DxT(W["wx"] * Dx(yc)) + DyT(W["wy"] * Dy(yc)))
        cpr = 2.0 * (mu_h * DxT(W["wcx"] * Dx(ch)) + mu_v * DyT(W["wcy"] * Dy(ch)))
        if mu_d > 0.0:
            cpr = cpr + 2.0 * mu_d * (D1T(W["wd1"] * D1(ch)) + D2T(W["wd2"] * D2(ch)))
        out = -img * np.conj(c) + cpr
        for j in range(len(nbrs)):
            out = out + 2.0 * nu * wts[j] * trm(ch, j) * np.conj(dcs[j])
        return out

    def curv(dd):
        dy = -np.real(dd * c)
        hh = (np.sum(W["wx"] * Dx(dy) ** 2) + np.sum(W["wy"] * Dy(dy) ** 2)
              + mu_h * np.sum(W["wcx"] * np.abs(Dx(dd)) ** 2)
              + mu_v * np.sum(W["wcy"] * np.abs(Dy(dd)) ** 2))
        if mu_d > 0.0:
            hh += mu_d * (np.sum(W["wd1"] * np.abs(D1(dd)) ** 2)
                          + np.sum(W["wd2"] * np.abs(D2(dd)) ** 2))
        for j in range(len(nbrs)):
            re = np.real(dd * dcs[j])
            hh += nu * np.sum(wts[j] * re * re)
        return float(hh)

    iters = 0
    outer_log = []     # per outer: (CG iterations, nearest |gg - threshold| / threshold)
    for _outer in range(irls_outer):
        yc = s - np.real(chi * c)
        gxY, gyY = Dx(yc), Dy(yc)
        mx, my = np.abs(Dx(chi)), np.abs(Dy(chi))
        W["wx"] = eps / np.sqrt(gxY ** 2 + e2)
        W["wy"] = eps / np.sqrt(gyY ** 2 + e2)
        W["wcx"] = eps_c / np.sqrt(mx ** 2 + k * gxY ** 2 + ec2)
        W["wcy"] = eps_c / np.sqrt(my ** 2 + k * gyY ** 2 + ec2)
        if mu_d > 0.0:
            W["wd1"] = 1.0 / np.sqrt(1.0 + (np.abs(D1(chi)) / eps_c) ** 2)
            W["wd2"] = 1.0 / np.sqrt(1.0 + (np.abs(D2(chi)) / eps_c) ** 2)
        if nu > 0.0:
            for j in range(len(nbrs)):
                rt = trm(chi, j)
                wts[j] = np.asarray(nbrs[j].confidence, np.float64) * et2 / (rt * rt + et2)
            ps = np.ones_like(s)
            for j in range(len(nbrs)):
                ps += nu * wts[j] * np.abs(dcs[j]) ** 2
            for key in ("wx", "wy", "wcx", "wcy") + (("wd1", "wd2") if mu_d > 0.0 else ()):
                W[key] = W[key] * ps
        g = grad(chi)
        d = -g
        gg = float(np.sum(np.abs(g) ** 2))
        gg0 = gg
        thr = max(tol * tol * gg0, 1e-10 * N)
        near, n_it = np.inf, 0
        for _it in range(n_inner):
            hh = curv(d)
            if hh <= 1e-12:
                break
            gd = float(np.sum(np.real(np.conj(g) * d)))
            alpha = -0.5 * gd / hh
            chi = chi + alpha * d
            gn = grad(chi)
            ggn = float(np.sum(np.abs(gn) ** 2))
            beta = ggn / max(gg, 1e-30)
            d = -gn + beta * d
            g, gg = gn, ggn
            iters += 1
            n_it += 1
            if n_it < n_inner:
                near = min(near, abs(gg - thr) / thr)
            if gg < tol * tol * gg0:
                break
            if gg < 1e-10 * N:
                break
        outer_log.append((n_it, near))
    if stats is not None:
        stats["cg_iterations"] = iters
        stats["outer_log"] = outer_log
        stats["aniso"] = aniso
    luma = s - np.real(chi * c)
    if return_weights:
        return luma, chi, W
    return luma, chi


def estimate_noise_ire(s) -> float:
    """EstimateNoiseIre (ntsc_geometry.cpp:49-71)."""
    s = np.asarray(s, np.float64)
    h, w = s.shape
    if w <= 8 or h <= 0:
        return 0.0
    d = (s[:, :w - 8] - 2.0 * s[:, 4:w - 4] + s[:, 8:]).ravel()
    med = upper_median(d)
    a = np.abs(d - med)
    k = a.size // 4
    q = float(np.partition(a, k)[k])
    return q / 0.3186 / math.sqrt(6.0)


def decode_fields_2d(fields_ire, parities, g, cfg, stats=None):
    """PrepareFieldObs + DecodeFieldWindow with temporal terms off
    (sequence.cpp:229-281, 423-449, 660-669, 1076-1114): per field
    HolographicInit + VariationalRefine, output-fidelity luma. `stats`, if
    a list, receives each field's solver statistics (variational_refine)."""
    out = []
    for f, p in zip(fields_ire, parities):
        obs = prepare_field(f, g, cfg, p)
        _, chi0 = holographic_init(obs.s, obs.carrier, g,
                                   bool(getattr(cfg, "symmetry_variant", 0)))
        st = {} if stats is not None else None
        y, chi = variational_refine(obs.s, obs.carrier, chi0, cfg, is_pal=uses_vswitch(g),
                                    stats=st)
        if stats is not None:
            stats.append(st)
        if cfg.output_fidelity:
            y = obs.s - np.real(chi * obs.carrier)
        out.append((y, chi, obs))
    return out


# --------------------------------------------------------------------------
# Motion estimation (engine/motion.cpp) and warps (engine/temporal.cpp)
# --------------------------------------------------------------------------

def decimate(a, f):
    """Decimate (motion.cpp:59-78): f x f block mean, remainder cropped."""
    h, w = a.shape
    hh, ww = h // f, w // f
    return a[:hh * f, :ww * f].reshape(hh, f, ww, f).mean(axis=(1, 3))


def range_from_centre(lo, hi):
    """RangeFromCentre (motion.cpp:286-298)."""
    v = []
    if lo > hi:
        return v
    if lo <= 0 <= hi:
        v.append(0)
    for d in range(1, max(-lo, hi) + 1):
        if lo <= -d <= hi:
            v.append(-d)
        if lo <= d <= hi:
            v.append(d)
    return v if v else list(range(lo, hi + 1))


def _lround(x):
    return np.where(x >= 0, np.floor(x + 0.5), -np.floor(-x + 0.5))


def bm_pass(A, B, tile, dys, dxs, base_dy=None, base_dx=None):
    """BmPass (motion.cpp:105-260) without the partial-distortion bail-out
    (which cannot change the winner): biased SSD, visit order, strict-less
    update. Returns (mdy, mdx, best, cost0)."""
    A = np.asarray(A, np.float64)
    B = np.asarray(B, np.float64)
    h, w = A.shape
    th, tw = -(-h // tile), -(-w // tile)
    max_s = max([abs(d) for d in dys] + [abs(d) for d in dxs])
    if base_dy is not None:
        max_s += int(max(np.abs(base_dy).max(), np.abs(base_dx).max()))
    pad = max_s + 1
    Bp = np.pad(B, pad, mode="edge")
    mdy = np.zeros((th, tw))
    mdx = np.zeros((th, tw))
    best = np.full((th, tw), np.inf)
    cost0 = np.zeros((th, tw)) if base_dy is None else None
    ty_of = np.minimum(np.arange(h) // tile, th - 1)
    tx_of = np.minimum(np.arange(w) // tile, tw - 1)
    if base_dy is not None:
        rby = _lround(np.asarray(base_dy)).astype(int)
        rbx = _lround(np.asarray(base_dx)).astype(int)
    yy, xx = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    for dy in dys:
        for dx in dxs:
            bias = 1.0 + 0.02 * (abs(dy) + abs(dx))
            if base_dy is None:
                src = Bp[pad - dy:pad - dy + h, pad - dx:pad - dx + w]
            else:
                sy = rby[ty_of][:, tx_of] + dy
                sx = rbx[ty_of][:, tx_of] + dx
                src = Bp[yy + pad - sy, xx + pad - sx]
            e = (A - src) ** 2
            se = np.zeros((th, tw))
            np.add.at(se, (ty_of[:, None].repeat(w, 1), tx_of[None, :].repeat(h, 0)), e)
            if base_dy is None and dy == 0 and dx == 0:
                cost0 = se.copy()
            cost = se * bias
            upd = cost < best
            best = np.where(upd, cost, best)
            if base_dy is None:
                mdy = np.where(upd, float(dy), mdy)
                mdx = np.where(upd, float(dx), mdx)
            else:
                mdy = np.where(upd, np.asarray(base_dy) + dy, mdy)
                mdx = np.where(upd, np.asarray(base_dx) + dx, mdx)
    return mdy, mdx, best, cost0


def motion_confidence(A, best, tile):
    """MotionConfidence (motion.cpp:321-387), edge tiles normalised by their
    real pixel count."""
    A = np.asarray(A, np.float64)
    h, w = A.shape
    th, tw = best.shape
    ty = np.minimum(np.arange(h) // tile, th - 1)
    tx = np.minimum(np.arange(w) // tile, tw - 1)
    idx = (ty[:, None] * tw + tx[None, :]).ravel()
    n = np.bincount(idx, minlength=th * tw).reshape(th, tw).astype(np.float64)
    s1 = np.bincount(idx, A.ravel(), minlength=th * tw).reshape(th, tw)
    s2 = np.bincount(idx, (A * A).ravel(), minlength=th * tw).reshape(th, tw)
    norm = 1.0 / np.maximum(1.0, n)
    tmean = s1 * norm
    tvar = s2 * norm - tmean * tmean
    energy = (tvar + 1.0) * np.maximum(1.0, n)
    conf = np.clip(1.0 - best / energy, 0.0, 1.0)
    ratios = best / np.maximum(1.0, n)
    med = mean_median(ratios.ravel())
    excess = np.maximum(0.0, ratios - med)
    conf = conf * (med + 1.0) / (med + 1.0 + excess)
    conf = conf * 6.0 / (6.0 + med)
    return conf


def estimate_motion(y_ref, y_cur, tile=32, search=8):
    """EstimateMotion (motion.cpp:397-488)."""
    A = box_blur_same(y_cur, 2)
    B = box_blur_same(y_ref, 2)
    h, w = A.shape
    th, tw = -(-h // tile), -(-w // tile)
    cs = max(1, (search + 3) // 4)
    Ad, Bd = decimate(A, 4), decimate(B, 4)
    ct = max(4, tile // 4)
    rc = range_from_centre(-cs, cs)
    cdy, cdx, _, _ = bm_pass(Ad, Bd, ct, rc, rc)
    hh, ww = cdy.shape
    gy = np.minimum((np.arange(th) * hh) // th, hh - 1)
    gx = np.minimum((np.arange(tw) * ww) // tw, ww - 1)
    base_dy = cdy[gy][:, gx] * 4.0
    base_dx = cdx[gy][:, gx] * 4.0
    r3 = range_from_centre(-3, 3)
    mdy, mdx, bestr, _ = bm_pass(A, B, tile, r3, r3, base_dy, base_dx)
    costs = {}
    for (oy, ox) in ((-1, 0), (1, 0), (0, -1), (0, 1)):
        costs[(oy, ox)] = bm_pass(A, B, tile, [0], [0], mdy + oy, mdx + ox)[2]

    def parabolic(cm, c0, cp):
        den = cm - 2.0 * c0 + cp
        sub = np.where(den > 1e-9, 0.5 * (cm - cp) / np.maximum(den, 1e-9), 0.0)
        return np.clip(sub, -0.5, 0.5)
    sdy = parabolic(costs[(-1, 0)], bestr, costs[(1, 0)])
    sdx = parabolic(costs[(0, -1)], bestr, costs[(0, 1)])
    _, _, best0, cost0 = bm_pass(A, B, tile, [0], [0])
    best = bestr.copy()
    z = best0 < best
    mdy = np.where(z, 0.0, mdy)
    mdx = np.where(z, 0.0, mdx)
    best = np.where(z, best0, best)
    m = best > 0.85 * cost0
    mdy = np.where(m, 0.0, mdy)
    mdx = np.where(m, 0.0, mdx)
    best = np.where(m, cost0, best)
    sdy = np.where(m, 0.0, sdy)
    sdx = np.where(m, 0.0, sdx)
    conf = motion_confidence(A, best, tile)
    return mdy + sdy, mdx + sdx, conf


# --------------------------------------------------------------------------
# Integer-SAD motion mode (me_mode 1). No reference counterpart for the cost:
# the reference's EstimateMotion uses float SSD. This mode keeps its control
# structure (motion.cpp:397-488: centre-out visit order RangeFromCentre
# :286-298, strict-less update :244, bias 1 + 0.02 (|dy| + |dx|), zero-motion
# margin 0.85 :455-473, parabolic sub-pel :437-452, MotionConfidence
# :321-387) with every decision exact in integers.
# --------------------------------------------------------------------------
QUANT_ZERO = np.float32(16384.0)    # 0 IRE
QUANT_SCALE = np.float32(348.16)    # codes per IRE (100 IRE = 51200)


def quantise_luma(y):
    """uint16 codes of float32 IRE luma: rint(16384 + 348.16 y) in float32
    (multiply, then add), clamped to [0, 65535]."""
    t = QUANT_ZERO + QUANT_SCALE * np.asarray(y, np.float32)
    return np.clip(np.rint(t), 0, 65535).astype(np.int64)


def box_blur_int(q, r=2):
    """Integer BoxBlur: zero-padded (2r+1)^2 window sum, rounded division by
    (2r+1)^2 ((sum + k2 // 2) // k2)."""
    q = np.asarray(q, np.int64)
    h, w = q.shape
    k = 2 * r + 1
    p = np.pad(q, r)
    v = np.zeros((h, w + 2 * r), np.int64)
    for d in range(k):
        v += p[d:d + h, :]
    o = np.zeros((h, w), np.int64)
    for d in range(k):
        o += v[:, d:d + w]
    k2 = k * k
    return (o + k2 // 2) // k2


def _centre_out_index(d):
    return 0 if d == 0 else (2 * d if d > 0 else -2 * d - 1)


def _tile_sums(e, tile, th, tw):
    """Per-tile sums; the last tile row / column holds the remainder
    (th = ceil(h / tile)), so zero padding to th x tw whole tiles is exact."""
    h, w = e.shape
    p = np.zeros((th * tile, tw * tile), e.dtype)
    p[:h, :w] = e
    return p.reshape(th, tile, tw, tile).sum(axis=(1, 3))


def _shifted(B, dy, dx):
    """B(clamp(y - dy), clamp(x - dx)) over the whole plane."""
    h, w = B.shape
    sy = np.clip(np.arange(h) - dy, 0, h - 1)
    sx = np.clip(np.arange(w) - dx, 0, w - 1)
    return B[sy][:, sx]


def _shifted_tiles(B, dyt, dxt, tile):
    """Per-pixel source with a per-tile integer vector."""
    h, w = B.shape
    th, tw = dyt.shape
    ty = np.minimum(np.arange(h) // tile, th - 1)
    tx = np.minimum(np.arange(w) // tile, tw - 1)
    vy = dyt[ty][:, tx]
    vx = dxt[ty][:, tx]
    yy, xx = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    return B[np.clip(yy - vy, 0, h - 1), np.clip(xx - vx, 0, w - 1)]


def estimate_motion_sad(y_ref, y_cur, block=16, search=16):
    """Exhaustive +-search integer-SAD block matching of block x block tiles
    on quantised, integer-blurred luma (me_mode 1). Returns per-tile
    (dy, dx, confidence) as float32, like estimate_motion."""
    A = box_blur_int(quantise_luma(y_cur))
    B = box_blur_int(quantise_luma(y_ref))
    h, w = A.shape
    th, tw = -(-h // block), -(-w // block)
    rc = range_from_centre(-search, search)
    n = len(rc)
    best = np.full((th, tw), np.iinfo(np.int64).max, np.int64)
    bci = np.zeros((th, tw), np.int64)
    sad0 = None
    for i, dy in enumerate(rc):
        for j, dx in enumerate(rc):
            sad = _tile_sums(np.abs(A - _shifted(B, dy, dx)), block, th, tw)
            if dy == 0 and dx == 0:
                sad0 = sad.copy()
            cost = sad * (50 + abs(dy) + abs(dx))
            upd = cost < best                      # strict-less in visit order
            best = np.where(upd, cost, best)
            bci = np.where(upd, i * n + j, bci)
    mdy = np.array([[rc[c // n] for c in row] for row in bci], np.int64)
    mdx = np.array([[rc[c % n] for c in row] for row in bci], np.int64)
    # parabolic sub-pel from the unbiased SADs either side (x50 scale, exact)
    def sad_at(vy, vx):
        return _tile_sums(np.abs(A - _shifted_tiles(B, vy, vx, block)), block, th, tw)

    def parabolic(sm, sp):
        num = 50 * sm - 50 * sp
        den = 50 * sm - 2 * best + 50 * sp
        sub = np.where(den > 0, 0.5 * num.astype(np.float64) / np.maximum(den, 1), 0.0)
        return np.clip(sub, -0.5, 0.5)
    sdy = parabolic(sad_at(mdy - 1, mdx), sad_at(mdy + 1, mdx))
    sdx = parabolic(sad_at(mdy, mdx - 1), sad_at(mdy, mdx + 1))
    cost0 = 50 * sad0
    m = 20 * best > 17 * cost0                     # best > 0.85 cost0
    mdy = np.where(m, 0, mdy)
    mdx = np.where(m, 0, mdx)
    sdy = np.where(m, 0.0, sdy)
    sdx = np.where(m, 0.0, sdx)
    # MotionConfidence on the IRE scale from exact integer sums: the biased
    # SSD at the chosen vector and the tile statistics of A
    ssd = _tile_sums((A - _shifted_tiles(B, mdy, mdx, block)) ** 2, block, th, tw)
    l1 = np.abs(mdy) + np.abs(mdx)
    npx = _tile_sums(np.ones_like(A), block, th, tw).astype(np.float64)
    s1 = _tile_sums(A, block, th, tw).astype(np.float64)
    s2 = _tile_sums(A * A, block, th, tw).astype(np.float64)
    sc2 = float(QUANT_SCALE) * float(QUANT_SCALE)
    bestv = (ssd * (50 + l1)).astype(np.float64) / (50.0 * sc2)
    norm = 1.0 / np.maximum(1.0, npx)
    tmean = s1 * norm
    tvar = (s2 * norm - tmean * tmean) / sc2
    energy = (tvar + 1.0) * np.maximum(1.0, npx)
    conf = np.clip(1.0 - bestv / energy, 0.0, 1.0)
    ratios = bestv / np.maximum(1.0, npx)
    v = np.sort(ratios.ravel())
    k = v.size // 2
    med = v[k] if v.size % 2 else 0.5 * (v[k] + v[k - 1])
    excess = np.maximum(0.0, ratios - med)
    conf = conf * ((med + 1.0) / (med + 1.0 + excess))
    conf = conf * (6.0 / (6.0 + med))
    dy = (mdy.astype(np.float64) + sdy).astype(np.float32)
    dx = (mdx.astype(np.float64) + sdx).astype(np.float32)
    return dy, dx, conf.astype(np.float32)


def _median3(v):
    """Median3 (temporal.cpp:20-41): 3x3 edge-padded median; < 3 tiles: copy."""
    th, tw = v.shape
    if th < 3 or tw < 3:
        return v.copy()
    p = np.pad(v, 1, mode="edge")
    stack = np.stack([p[dy:dy + th, dx:dx + tw] for dy in range(3) for dx in range(3)])
    return np.partition(stack, 4, axis=0)[4]


def vectors_per_pixel(mdy, mdx, tile, out_h, out_w):
    """VectorsPerPixel (temporal.cpp:45-112)."""
    mdy = np.asarray(mdy, np.float64)
    mdx = np.asarray(mdx, np.float64)
    th, tw = mdy.shape
    my, mx = _median3(mdy), _median3(mdx)
    dis = np.abs(mdy - my) + np.abs(mdx - mx)
    mdy = np.where(dis > 3.0, my, mdy)
    mdx = np.where(dis > 3.0, mx, mdx)

    def bracket(n_px, n_t):
        c = np.arange(n_px, dtype=np.float64)
        if n_t > 1:
            lo = np.clip(np.floor(c / tile - 0.5).astype(int), 0, n_t - 2)
            frac = np.clip((c - (lo + 0.5) * tile) / tile, 0.0, 1.0)
        else:
            lo = np.zeros(n_px, int)
            frac = np.zeros(n_px)
        return lo, frac
    iy, fy = bracket(out_h, th)
    ix, fx = bracket(out_w, tw)
    iy1 = np.minimum(iy + 1, th - 1)
    ix1 = np.minimum(ix + 1, tw - 1)
    fy, fx = fy[:, None], fx[None, :]

    def interp(v):
        return (v[iy][:, ix] * (1 - fy) * (1 - fx) + v[iy1][:, ix] * fy * (1 - fx)
                + v[iy][:, ix1] * (1 - fy) * fx + v[iy1][:, ix1] * fy * fx)
    return interp(mdy), interp(mdx)


def warp_by_tiles(a, vdy, vdx):
    """WarpByTiles / WarpByTilesComplex (temporal.cpp:118-133, 210-225)."""
    h, w = a.shape
    yy, xx = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    sy = np.clip(yy - _lround(vdy).astype(int), 0, h - 1)
    sx = np.clip(xx - _lround(vdx).astype(int), 0, w - 1)
    return a[sy, sx]


def upsample_confidence(conf, tile, out_h, out_w, fast=False):
    """UpsampleConfidence (temporal.cpp:227-243) / UpsampleConfidenceFast
    (temporal.cpp:245-254)."""
    conf = np.asarray(conf, np.float64)
    if fast:
        c2 = conf * conf
        return vectors_per_pixel(c2, c2, tile, out_h, out_w)[0]
    th, tw = conf.shape
    ty = np.minimum(np.arange(out_h) // tile, th - 1)
    tx = np.minimum(np.arange(out_w) // tile, tw - 1)
    px = conf[ty][:, tx] ** 2
    return box_blur_same(px, 8)


# --------------------------------------------------------------------------
# Frame bridge (hvd-core/src/frame_bridge.cpp)
# --------------------------------------------------------------------------

def frame_line_offset(fp, line):
    """FrameLineOffset (frame_bridge.h:106-112)."""
    off = line * fp.frame_width
    for i in range(fp.extra_sample_line_count):
        if fp.extra_sample_lines[i] < line:
            off += 1
    return off


def split_frame_fields(frame, fp):
    """SplitFrameFields (frame_bridge.cpp:61-99): block 1 / block 2 in IRE."""
    fw, fh, f1 = fp.frame_width, fp.frame_height, fp.field1_lines
    f2 = fh - f1
    top = np.full((f1, fw), float(fp.blanking_level))
    bot = np.full((f1, fw), float(fp.blanking_level))
    fr = np.asarray(frame).ravel()
    for y in range(f1):
        if y < f1:
            o = frame_line_offset(fp, y)
            top[y] = fr[o:o + fw]
        if y < f2:
            o = frame_line_offset(fp, f1 + y)
            bot[y] = fr[o:o + fw]
    return (sample_to_ire(top, fp.blanking_level, fp.white_level),
            sample_to_ire(bot, fp.blanking_level, fp.white_level))


def geometry_from_params(fp, Geometry):
    """FieldGeometryFromParams (frame_bridge.cpp:43-59)."""
    g = Geometry()
    g.field_width = fp.frame_width
    g.field_height = fp.field1_lines
    g.active_video_start = fp.active_video_start
    g.active_video_end = fp.active_video_end
    g.colour_burst_start = fp.colour_burst_start
    g.colour_burst_end = fp.colour_burst_end
    g.first_active_field_line = fp.first_active_frame_line // 2
    g.last_active_field_line = fp.last_active_frame_line // 2 if fp.last_active_frame_line else 0
    g.sample_rate = fp.sample_rate
    g.subcarrier_hz = fp.subcarrier_hz
    g.standard = fp.standard
    return g


def detect_field_parity(b1, b2, fp, g) -> int:
    """DetectFieldParity (frame_bridge.cpp:102-149)."""
    fal, lal = g.first_active_field_line, last_active_line(g)
    a0, a1 = fp.active_video_start, fp.active_video_end
    lines, width = lal - fal, a1 - a0
    if lines < 8 or width < 32:
        return 0
    ystep = max(1, lines // 120)
    ep = em = 0.0
    n = 0
    for r in range(fal + 1, lal - 1, ystep):
        for x in range(a0, a1 - 3, 16):
            lp = lambda p, row: 0.25 * (p[row, x] + p[row, x + 1] + p[row, x + 2] + p[row, x + 3])
            b = lp(b2, r)
            ac, au, ad = lp(b1, r), lp(b1, r - 1), lp(b1, r + 1)
            ep += abs(b - 0.5 * (ac + ad))
            em += abs(b - 0.5 * (ac + au))
            n += 1
    if n == 0:
        return 0
    ep /= n
    em /= n
    lo, hi = min(ep, em), max(ep, em)
    if hi <= 1e-9 or (hi - lo) / hi < 0.02:
        return 0
    return 1 if ep < em else -1


def drizzle_frame(j0, Ys, chis, parities, cfg, scale=2):
    """DrizzleFrame (sequence.cpp:283-421) in FP64: each target field of the
    frame (j0, j0 + 1) collects the motion-compensated samples of the fields
    within 2 nr_radius (itself with zero motion and confidence 1), weighted
    by confidence x eps_b^2 / (d^2 + eps_b^2) against its own decode at the
    rounded warp and split linearly between the two fine rows around
    (2 (y + vy) + p_k) scale; coverage-blended with the interpolated weave."""
    L, W = np.asarray(Ys[j0]).shape
    HF = 2 * L * scale
    n = len(Ys)
    tile, search, r = cfg.mc_tile, cfg.mc_search, cfg.nr_radius
    eps_b = cfg.nr_eps if cfg.nr_eps > 0 else 3.0
    acc = np.zeros((4, HF, W))
    yy, xx = np.mgrid[0:L, 0:W].astype(np.float64)
    Ys = [np.asarray(y, np.float64) for y in Ys]
    chis = [np.asarray(c, np.complex128) for c in chis]
    for jt in (j0, j0 + 1):
        for k in range(max(0, j0 - 2 * r), min(n, j0 + 2 + 2 * r)):
            if k in (j0, j0 + 1) and k != jt:
                continue
            if k == jt:
                vy = np.zeros((L, W))
                vx = np.zeros((L, W))
                cpx = np.ones((L, W))
            else:
                mdy, mdx, conf = estimate_motion(Ys[k], Ys[jt], tile, search)
                vy, vx = vectors_per_pixel(mdy, mdx, tile, L, W)
                th, tw = conf.shape
                cpx = conf[np.minimum(yy.astype(int) // tile, th - 1),
                           np.minimum(xx.astype(int) // tile, tw - 1)]
            syi = np.clip(_lround(yy - vy), 0, L - 1).astype(int)
            sxi = np.clip(_lround(xx - vx), 0, W - 1).astype(int)
            dY = Ys[k] - Ys[jt][syi, sxi]
            d2 = dY * dY + np.abs(chis[k] - chis[jt][syi, sxi]) ** 2
            wgt = cpx * eps_b * eps_b / (d2 + eps_b * eps_b)
            yf = (2.0 * (yy + vy) + parities[k]) * scale
            xs = np.clip(_lround(xx + vx), 0, W - 1).astype(int)
            y0 = np.floor(yf).astype(int)
            fy = yf - y0
            for off in (0, 1):
                yt = np.clip(y0 + off, 0, HF - 1)
                ww = wgt * ((1.0 - fy) if off == 0 else fy)
                for i, v in enumerate((ww * Ys[k], ww * chis[k].real, ww * chis[k].imag, ww)):
                    np.add.at(acc[i], (yt.ravel(), xs.ravel()), v.ravel())
    p0, p1 = parities[j0], parities[j0 + 1]
    wy = np.zeros((2 * L, W))
    wc = np.zeros((2 * L, W), np.complex128)
    wy[p0::2], wc[p0::2] = Ys[j0], chis[j0]
    wy[p1::2], wc[p1::2] = Ys[j0 + 1], chis[j0 + 1]
    fine = np.arange(HF) / scale
    f0 = np.clip(np.floor(fine).astype(int), 0, 2 * L - 2)
    ff = (fine - f0)[:, None]
    base_y = wy[f0] * (1 - ff) + wy[f0 + 1] * ff
    base_c = wc[f0] * (1 - ff) + wc[f0 + 1] * ff
    aw = acc[3]
    mix = aw / (aw + 0.35)
    den = np.maximum(aw, 1e-9)
    dz_y = np.where(aw > 0, acc[0] / den, 0.0)
    dz_c = np.where(aw > 0, (acc[1] + 1j * acc[2]) / den, 0.0)
    return mix * dz_y + (1 - mix) * base_y, mix * dz_c + (1 - mix) * base_c


def ambiguous_boxes(Y, chi, max_area=0.45):
    """AmbiguousBoxes (frame_bridge.cpp:402-580) in float32 / float64 as the
    reference: [] = stay 2-D, None = full 3-D, else [(fy0, fy1, x0, x1)]."""
    T, HX, HY, K = 16, 48, 16, 8
    ya = np.asarray(Y, np.float32)
    ca = np.abs(np.asarray(chi, np.complex64)).astype(np.float32)
    h, w = ya.shape
    th, tw = (h + T - 1) // T, (w + T - 1) // T

    def box_mean(a):
        def along(a, axis):
            n = a.shape[axis]
            acc = np.zeros_like(a)
            cnt = np.zeros(n, np.int64)
            for d in range(-K // 2, K - K // 2):
                lo, hi = max(0, -d), min(n, n - d)
                if hi <= lo:
                    continue
                if axis == 0:
                    acc[lo:hi] = acc[lo:hi] + a[lo + d:hi + d]
                else:
                    acc[:, lo:hi] = acc[:, lo:hi] + a[:, lo + d:hi + d]
                cnt[lo:hi] += 1
            c = np.maximum(cnt, 1).astype(np.float32)
            return acc / (c[:, None] if axis == 0 else c[None, :])
        return along(along(a, 0), 1)

    dy = (ya - box_mean(ya)).astype(np.float64)
    dc = (ca - box_mean(ca)).astype(np.float64)
    score = np.zeros((th, tw), np.float32)
    for ty in range(th):
        for tx in range(tw):
            sl = (slice(ty * T, min(h, ty * T + T)), slice(tx * T, min(w, tx * T + T)))
            n = dy[sl].size
            ey = np.cumsum((dy[sl] * dy[sl]).ravel())[-1]   # sequential, raster order
            ec = np.cumsum((dc[sl] * dc[sl]).ravel())[-1]
            score[ty, tx] = np.float32(math.sqrt((ey / n) * (ec / n)))
    flat = score.ravel().copy()
    k = flat.size // 2
    med = np.float32(np.partition(flat, k)[k])
    flagged = score >= np.float32(4.0) * med
    dense = np.zeros((th, tw), bool)
    for ty in range(1, th - 1):
        for tx in range(1, tw - 1):
            if flagged[ty, tx]:
                nb = int(flagged[ty - 1:ty + 2, tx - 1:tx + 2].sum()) - 1
                dense[ty, tx] = nb >= 2
    bands = []
    for ty in range(th):
        if dense[ty].sum() < 2:
            continue
        if bands and ty - bands[-1][1] <= 1:
            bands[-1][1] = ty
        else:
            bands.append([ty, ty])
    if not bands:
        return None if med > np.float32(3.0) else []
    while len(bands) > 4:
        gaps = [bands[i + 1][0] - bands[i][1] for i in range(len(bands) - 1)]
        bi = int(np.argmin(gaps))           # first of the smallest gaps
        bands[bi][1] = bands[bi + 1][1]
        del bands[bi + 1]
    boxes = []
    for tr0, tr1 in bands:
        col = dense[tr0:tr1 + 1].any(axis=0)
        y0 = max(0, tr0 * T - HY)
        y0 -= y0 % 2
        y1 = min(h, (tr1 + 1) * T + HY)
        runs = []
        for tx in range(tw):
            if not col[tx]:
                continue
            if runs and tx - runs[-1][1] <= 2:
                runs[-1][1] = tx
            else:
                runs.append([tx, tx])
        first = len(boxes)
        for c0, c1 in runs:
            if c1 - c0 < 1:
                continue
            x0, x1 = max(0, c0 * T - HX), min(w, (c1 + 1) * T + HX)
            if len(boxes) > first and x0 <= boxes[-1][3]:
                boxes[-1][3] = x1
            else:
                boxes.append([y0, y1, x0, x1])
    area = sum(float(b[1] - b[0]) * (b[3] - b[2]) for b in boxes)
    if area > float(np.float32(max_area)) * h * w:
        return None
    return [tuple(b) for b in boxes]


# --------------------------------------------------------------------------
# Temporal (3-D) field window (engine/sequence.cpp:423-1116), the subset with
# no anchor pass, no coherence gate, no trajectory fit, no PSI init.
# --------------------------------------------------------------------------

def _smooth_rows(src):
    """smooth_rows (sequence.cpp:860-889): sqrt of the mean over [x-2, x+2]
    clipped to the row."""
    h, w = src.shape
    c = np.zeros((h, w + 1))
    c[:, 1:] = np.cumsum(src, axis=1)
    x = np.arange(w)
    lo = np.maximum(x - 2, 0)
    hi = np.minimum(x + 2, w - 1)
    n = hi - lo + 1
    return np.sqrt((c[:, hi + 1] - c[:, lo]) / n)


def envelope_gate(Y, chi, eps_t, odd_gate_floor):
    """Odd-offset half-line envelope gate (sequence.cpp:797-932, 1000-1026):
    returns max(floor_i, e2 / (e2 + b^2)) per pixel."""
    h, w = Y.shape
    ym = np.maximum(np.arange(h) - 1, 0)
    yp = np.minimum(np.arange(h) + 1, h - 1)
    dyu = Y - Y[ym]
    dyd = Y[yp] - Y
    dcu = np.abs(chi - chi[ym])
    dcd = np.abs(chi[yp] - chi)
    gmag = np.maximum(dyu ** 2 + dcu ** 2, dyd ** 2 + dcd ** 2)
    ly = Y - 0.5 * (Y[ym] + Y[yp])
    lc = np.abs(chi - 0.5 * (chi[ym] + chi[yp]))
    lapmag = ly ** 2 + lc ** 2
    vgrad = _smooth_rows(gmag)
    med = mean_median(vgrad.ravel()[::7])
    vgrad = np.sqrt(np.maximum(0.0, vgrad ** 2 - 2.25 * med * med))
    traw = _smooth_rows(lapmag)
    t = np.where(vgrad > 1e-6, np.clip(traw / np.where(vgrad > 1e-6, vgrad, 1.0), 0.0, 1.0), 0.0)
    lapsm = 1.0 - t * t
    e2 = eps_t * eps_t
    floor_i = float(np.clip(odd_gate_floor, 0.0, 1.0)) * lapsm
    return np.maximum(floor_i, e2 / (e2 + vgrad ** 2))


def temporal_offsets(cfg, pal):
    """sequence.cpp:451-468."""
    if cfg.extended_temporal:
        if pal:
            return [-4, -3, -2, -1, 1, 2, 3, 4] if cfg.bidirectional else [-4, -3, -2, -1]
        return [-3, -2, -1, 1, 2, 3] if cfg.bidirectional else [-3, -2, -1]
    return [-2, -1, 1, 2] if cfg.bidirectional else [-2, -1]


def adaptive_strength(S_list, carriers, stride, nr_eps):
    """The adaptive temporal strength (sequence.cpp:526-646) in the
    reference's float32 operations and order: per same-parity pair (j,
    j + stride), at rows 2, 5, ... < h - 2 and columns 4, 8, ... (x + 7 < w)
    where the two fields' 4-sample means agree within nr_eps, the triangle-7
    demodulations d = sum_k w_k S conj(c) / 16 and e = |d_j - d_k|^2 / 4
    summed in double per band of 8 rows in row order; the pair's ambiguity
    is the sqrt of the p95 band mean (bands with >= 8 terms; else of the
    mean of all terms); the median over pairs, the noise floor 0.29 nr_eps/3
    removed. Returns (strength, ambiguity)."""
    f32 = np.float32
    kW = np.array([1, 2, 3, 4, 3, 2, 1], f32)
    eps = f32(nr_eps)
    ambs = []
    for j in range(len(S_list) - stride):
        Sj = np.asarray(S_list[j], f32)
        Sk = np.asarray(S_list[j + stride], f32)
        cj = np.asarray(carriers[j], np.complex64)
        ck = np.asarray(carriers[j + stride], np.complex64)
        h, w = Sj.shape
        xs = np.arange(4, w - 7, 4)
        bands = []
        for yi, y in enumerate(range(2, h - 2, 3)):
            if yi // 8 >= len(bands):
                bands.append([])
            mj = np.zeros(len(xs), f32)
            mk = np.zeros(len(xs), f32)
            for q in range(4):
                mj = mj + Sj[y, xs + q]
                mk = mk + Sk[y, xs + q]
            keep = ~(np.abs(mj - mk) * f32(0.25) > eps)

            def demod(S, c):
                dr = np.zeros(len(xs), f32)
                di = np.zeros(len(xs), f32)
                for q in range(7):
                    sv = kW[q] * S[y, xs + q]
                    cc = c[y, xs + q]
                    dr = dr + sv * cc.real.astype(f32)
                    di = di + sv * (-cc.imag.astype(f32))
                return dr * f32(1.0 / 16.0), di * f32(1.0 / 16.0)

            djr, dji = demod(Sj, cj)
            dkr, dki = demod(Sk, ck)
            er, ei = djr - dkr, dji - dki
            e = 0.25 * (er * er + ei * ei).astype(np.float64)
            bands[yi // 8].append(e[keep])
        band_e = [np.concatenate(b) if b else np.zeros(0) for b in bands]
        n = sum(len(b) for b in band_e)
        if n == 0:
            continue
        # sequential double sums (np.cumsum adds in order)
        brms = [f32(np.cumsum(b)[-1] / len(b)) for b in band_e if len(b) >= 8]
        if brms:
            k95 = min(len(brms) - 1, int(0.95 * len(brms)))
            ambs.append(np.sqrt(np.sort(np.array(brms, f32))[k95]))
        else:
            acc = np.cumsum(np.concatenate(band_e))[-1]
            ambs.append(np.sqrt(f32(acc / n)))
    amb = f32(0.0)
    if ambs:
        v = np.sort(np.array(ambs, f32))
        k = len(v) // 2
        amb = v[k] if len(v) % 2 else f32(f32(0.5) * (v[k] + v[k - 1]))
    sigma_d = f32(eps / f32(3.0)) if eps > 0 else f32(1.0)
    floor = sigma_d * f32(0.29)
    amb = np.sqrt(max(f32(0.0), f32(amb * amb - floor * floor)))
    strength = min(max(f32(f32(0.5) * amb - f32(0.05)), f32(0.0)), f32(1.5))
    return float(strength), float(amb)


def decode_window_temporal(fields_ire, parities, g, cfg, strength):
    """DecodeFieldWindowWithInits with a fixed temporal strength > 0, one
    pass: per field (in the reference's sweep order) EstimateMotion on the
    current luma state, integer warps of the neighbours' composite and
    carrier, confidence upsample, odd-offset envelope gate, VariationalRefine
    with neighbour terms; output-fidelity luma."""
    import copy
    pal = uses_vswitch(g)
    obs = [prepare_field(f, g, cfg, p) for f, p in zip(fields_ire, parities)]
    nf = len(obs)
    sig = [estimate_noise_ire(o.s) for o in obs]
    sigma = mean_median(sig)
    eps_t = cfg.temporal_eps if cfg.temporal_eps > 0 else float(np.clip(7 * sigma, 4, 20))
    c2 = copy.copy(cfg)
    c2.temporal_strength = strength
    c2.temporal_eps = eps_t
    Ys, chis = [], []
    for o in obs:
        y0, chi0 = holographic_init(o.s, o.carrier, g, bool(getattr(cfg, "symmetry_variant", 0)))
        Ys.append(y0)
        chis.append(chi0)
    offs = temporal_offsets(cfg, pal)
    max_off = max(abs(o) for o in offs)
    reach = max(max_off, cfg.nr_radius if cfg.nr_anchor > 0 else 0)
    if cfg.fast and cfg.parallel_across_fields:
        order = [list(range(c, nf, reach + 1)) for c in range(reach + 1)]
    else:
        order = [[j] for j in range(nf)]
    h, w = obs[0].s.shape
    for colour in order:
        state = [(Y.copy(), c.copy()) for Y, c in zip(Ys, chis)]
        for j in colour:
            Yj, chij = state[j]
            nbrs = []
            gate = None
            for o in offs:
                k = j + o
                if k < 0 or k >= nf:
                    continue
                if getattr(cfg, "me_mode", 0) == 1:
                    tile = cfg.me_block
                    dy, dx, conf = estimate_motion_sad(state[k][0], Yj, cfg.me_block, cfg.me_range)
                else:
                    tile = cfg.mc_tile
                    dy, dx, conf = estimate_motion(state[k][0], Yj, cfg.mc_tile, cfg.mc_search)
                vdy, vdx = vectors_per_pixel(dy, dx, tile, h, w)
                comp = warp_by_tiles(obs[k].s, vdy, vdx)
                car = warp_by_tiles(obs[k].carrier, vdy, vdx)
                cf = upsample_confidence(conf, tile, h, w, fast=bool(cfg.fast))
                if o & 1:
                    if gate is None:
                        gate = envelope_gate(Yj, chij, eps_t, cfg.odd_gate_floor)
                    cf = cf * gate
                nbrs.append(Neighbor(comp, car, cf))
            y, chi = variational_refine(obs[j].s, obs[j].carrier, chij, c2, is_pal=pal,
                                        neighbors=nbrs)
            Ys[j], chis[j] = y, chi
    out = []
    for j in range(nf):
        out.append((obs[j].s - np.real(chis[j] * obs[j].carrier), chis[j]))
    return out
