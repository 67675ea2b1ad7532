"""Pins of the FP64 oracle (oracle/hvd_oracle.py), CPU only:

1. the reference's own analytic tests, restated (file:line of each);
2. the golden fixtures in tests/golden/ -- outputs of the reference engine
   itself, compiled from its own sources and run on seeded inputs
   (tests/golden/make_golden.py);
3. the algebra the device kernels rely on (cyclic-convolution form of the
   FFT crop, the single-reduction CG recurrence), checked in FP64.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from hvdg import _cabi
from oracle import hvd_oracle as O

GOLD = Path(__file__).resolve().parent / "golden"


def wrap(a):
    return np.arctan2(np.sin(a), np.cos(a))


def geom_from(arr, sr):
    g = _cabi.Geometry()
    (g.field_width, g.field_height, g.active_video_start, g.active_video_end,
     g.colour_burst_start, g.colour_burst_end, g.first_active_field_line,
     g.last_active_field_line, g.standard) = [int(v) for v in arr]
    g.sample_rate = float(sr)
    return g


def cfg_from(arr):
    c = _cabi.default_config()
    c.irls_outer, c.cg_iterations, c.fast = int(arr[0]), int(arr[1]), int(arr[2])
    c.cg_tol, c.temporal_strength, c.chroma_aniso, c.lambda_c = map(float, arr[3:7])
    return c


# ---------------------------------------------------------------------------
# 1. restated reference tests
# ---------------------------------------------------------------------------

def test_lockin_ntsc_recovers_phase_and_amplitude():
    """lockin_test.cpp:28-67: a -A sin(phi) burst on 30 lines of 200 samples,
    theta recovered to 0.05 rad, amplitude 20 +/- 1, TridiagSmooth's low-lambda
    limit returns the data."""
    g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_NTSC), field_width=200,
                            colour_burst_start=20, colour_burst_end=60)
    h = 30
    field = np.zeros((h, 200))
    ys = np.arange(h)
    tt = 0.3 + math.pi * ys + 0.05 * np.sin(0.2 * ys)
    x = np.arange(20, 60)
    field[:, 20:60] = -20.0 * np.sin(tt[:, None] + 0.5 * math.pi * x[None, :])
    th = O.burst_lockin_phase(field, g)
    assert np.abs(wrap(th[2:h - 2] - tt[2:h - 2])).max() < 0.05
    assert abs(O.burst_amplitude_ire(field, g) - 20.0) < 1.0
    xs = O.tridiag_smooth([1, 2, 3, 4], [1, 1, 1, 1], 1e-6)
    assert np.allclose(xs, [1, 2, 3, 4], atol=1e-3)


def _pal_field(g, theta, sw, Y, U, V, burst):
    """pal_lockin_test.cpp:44-62."""
    h = len(theta)
    x = np.arange(g.field_width)
    phi = theta[:, None] + 0.5 * math.pi * x[None, :]
    s = np.where(np.asarray(sw) > 0, 1.0, -1.0)[:, None]
    bs = burst / math.sqrt(2.0)
    f = np.zeros((h, g.field_width))
    bm = (x >= g.colour_burst_start) & (x < g.colour_burst_end)
    am = (x >= g.active_video_start) & (x < g.active_video_end)
    f[:, bm] = (-bs * np.sin(phi) + s * bs * np.cos(phi))[:, bm]
    f[:, am] = (Y + U * np.sin(phi) + s * V * np.cos(phi))[:, am]
    return f


def test_lockin_pal_joint_phase_and_parity():
    """pal_lockin_test.cpp:75-155: exact parity, 0.03 rad clean, 0.08 rad with
    8 bursts destroyed; effective-carrier identity < 1e-3; line advance
    2 pi * 0.7516."""
    g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_PAL), field_width=300,
                            colour_burst_start=20, colour_burst_end=60, active_video_start=80,
                            active_video_end=280, first_active_field_line=0,
                            last_active_field_line=0, field_height=40)
    h = 40
    ys = np.arange(h)
    adv = 2 * math.pi * 0.7516
    tt = 0.4 + adv * ys + 0.05 * np.sin(0.15 * ys)
    sw = np.where(ys % 2 == 0, 1, -1)
    field = _pal_field(g, tt, sw, 50.0, -12.0, 20.0, 21.43)
    th, vs = O.burst_lockin_phase_pal(field, g)
    assert (vs == sw).all()
    assert np.abs(wrap(th - tt)).max() < 0.03
    dmg = field.copy()
    dmg[12:20, 20:60] = 0.0
    th2, vs2 = O.burst_lockin_phase_pal(dmg, g)
    assert (vs2 == sw).all()
    assert np.abs(wrap(th2 - tt)).max() < 0.08
    c = O.make_carrier(tt, sw, g)
    chi = 20.0 - 1j * (-12.0)
    recon = 50.0 + np.real(chi * c)
    assert np.abs(recon - field[:, 80:280]).max() < 1e-3
    cyc = 4433618.75 / 15625.0
    assert abs(O.line_advance(g) - 2 * math.pi * (cyc - math.floor(cyc))) < 1e-5


@pytest.mark.parametrize("shape", [(1, 1), (1, 8), (8, 1), (17, 23), (64, 48)])
def test_gradient_adjoints(shape):
    """gradients_test.cpp:40-67: <Da, b> == <a, D^T b> for Dx, Dy (real and
    complex planes)."""
    rng = np.random.default_rng(3)
    a = rng.uniform(-1, 1, shape)
    b = rng.uniform(-1, 1, shape)
    assert abs(np.sum(O.Dx(a) * b) - np.sum(a * O.DxT(b))) < 1e-12
    assert abs(np.sum(O.Dy(a) * b) - np.sum(a * O.DyT(b))) < 1e-12
    ac = a + 1j * rng.uniform(-1, 1, shape)
    bc = b + 1j * rng.uniform(-1, 1, shape)
    assert abs(np.vdot(O.Dx(ac), bc) - np.vdot(ac, O.DxT(bc))) < 1e-12
    # the oriented +-45 deg differences (gradients.h:195-279)
    assert abs(np.sum(O.D1(a) * b) - np.sum(a * O.D1T(b))) < 1e-12
    assert abs(np.sum(O.D2(a) * b) - np.sum(a * O.D2T(b))) < 1e-12
    assert abs(np.vdot(O.D1(ac), bc) - np.vdot(ac, O.D1T(bc))) < 1e-12
    assert abs(np.vdot(O.D2(ac), bc) - np.vdot(ac, O.D2T(bc))) < 1e-12


def test_box_blur_equals_naive_convolution():
    """motion_v2_test.cpp: BoxBlur == zero-padded 'same' convolution with a
    constant 1/(2r+1) kernel per axis."""
    rng = np.random.default_rng(5)
    a = rng.normal(size=(23, 31))
    for r in (1, 2, 3, 8):
        k = np.ones(2 * r + 1) / (2 * r + 1)
        rows = np.array([np.convolve(a[:, x], k, mode="same") for x in range(a.shape[1])]).T
        naive = np.array([np.convolve(rows[y], k, mode="same") for y in range(a.shape[0])])
        assert np.abs(O.box_blur_same(a, r) - naive).max() < 1e-12


def test_motion_recovers_shift():
    """motion_test.cpp:78-127 (own texture): a (3, -2) shift of a textured
    128 x 128 plane is recovered within 0.6 px on confident interior tiles,
    and unconfident tiles are flagged."""
    rng = np.random.default_rng(11)
    h = w = 128
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    blocks = rng.uniform(-15, 15, size=(h // 4, w // 4))
    tex = (40 * np.sin(yy * 0.31) * np.cos(xx * 0.27) + 15 * np.sin(xx * 0.23 + yy * 0.17)
           + blocks[(yy // 4).astype(int), (xx // 4).astype(int)])
    cur = tex[np.clip(np.arange(h) - 3, 0, h - 1)][:, np.clip(np.arange(w) + 2, 0, w - 1)]
    dy, dx, cf = O.estimate_motion(tex, cur, 32, 8)
    inner = (slice(1, -1), slice(1, -1))
    conf = cf[inner] > 0.15
    assert conf.sum() >= 1
    assert np.abs(dy[inner][conf] - 3).max() <= 0.6
    assert np.abs(dx[inner][conf] + 2).max() <= 0.6


def test_sad_motion_recovers_integer_shift():
    """Integer-SAD mode (me_mode 1): an integer (3, -5) shift of a textured
    plane is found exactly on interior blocks, with |sub-pel| <= 0.5."""
    rng = np.random.default_rng(12)
    h, w = 96, 128
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    tex = (40 * np.sin(yy * 0.31) * np.cos(xx * 0.27) + 15 * np.sin(xx * 0.23 + yy * 0.17)
           + rng.uniform(-10, 10, size=(h, w)) + 50).astype(np.float32)
    cur = tex[np.clip(np.arange(h) - 3, 0, h - 1)][:, np.clip(np.arange(w) + 5, 0, w - 1)]
    dy, dx, cf = O.estimate_motion_sad(tex, cur, 16, 8)
    inner = (slice(1, -1), slice(1, -1))
    assert np.array_equal(np.round(dy[inner]), np.full_like(dy[inner], 3))
    assert np.array_equal(np.round(dx[inner]), np.full_like(dx[inner], -5))
    assert np.abs(dy - np.round(dy)).max() <= 0.5 and np.abs(dx - np.round(dx)).max() <= 0.5
    assert cf[inner].min() > 0.0


def test_sad_motion_ties_pick_zero_first():
    """Strict-less update in centre-out order: on a flat plane every
    candidate ties and the zero vector (visited first) is kept."""
    a = np.full((40, 56), 37.25, np.float32)
    dy, dx, _ = O.estimate_motion_sad(a, a, 16, 6)
    assert not dy.any() and not dx.any()


def test_sad_quantise_and_integer_blur():
    """0 IRE -> 16384, 100 IRE -> 51200, clamped to uint16; the integer
    blur is the zero-padded 5 x 5 box sum with rounded division."""
    q = O.quantise_luma(np.array([[0.0, 100.0, -100.0, 200.0]], np.float32))
    assert q.tolist() == [[16384, 51200, 0, 65535]]
    rng = np.random.default_rng(3)
    a = rng.integers(0, 65536, size=(19, 23))
    b = O.box_blur_int(a, 2)
    p = np.pad(a, 2)
    naive = np.array([[p[y:y + 5, x:x + 5].sum() for x in range(23)] for y in range(19)])
    assert np.array_equal(b, (naive + 12) // 25)


def test_lossless_identity():
    """lossless_identity_test.cpp:40-101: init and refine keep
    |S - Y - Re[chi c]| < 1e-3."""
    d = np.load(GOLD / "field_ntsc_small.npz")
    g = geom_from(d["geometry"], d["sample_rate"])
    cfg = cfg_from(d["cfg"])
    s, c = d["s"].astype(np.float64), d["carrier"].astype(np.complex128)
    y0, chi0 = O.holographic_init(s, c, g)
    assert np.abs(s - y0 - np.real(chi0 * c)).max() < 1e-3
    y, chi = O.variational_refine(s, c, chi0, cfg)
    assert np.abs(s - y - np.real(chi * c)).max() < 1e-3


# ---------------------------------------------------------------------------
# 2. golden fixtures (the reference engine's own outputs)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("tag", ["ntsc", "pal"])
def test_oracle_matches_reference_golden(tag):
    d = np.load(GOLD / f"field_{tag}_small.npz")
    g = geom_from(d["geometry"], d["sample_rate"])
    cfg = cfg_from(d["cfg"])
    ire = ((d["samples"].astype(np.float32) - np.float32(16384.0)) /
           np.float32((51200.0 - 16384.0) / 100.0)).astype(np.float64)
    if O.uses_vswitch(g):
        th, vs = O.burst_lockin_phase_pal(ire, g)
        assert (vs == d["vswitch"]).all()
    else:
        th = O.burst_lockin_phase(ire, g)
    assert np.abs(wrap(th - d["theta"])).max() < 2e-3
    assert abs(O.burst_amplitude_ire(ire, g) - float(d["amplitude"])) < 1e-3
    # init / refine from the reference's own prepared field
    s, c = d["s"].astype(np.float64), d["carrier"].astype(np.complex128)
    y0, chi0 = O.holographic_init(s, c, g)
    assert np.abs(chi0 - d["chi0"]).max() < 5e-3
    assert np.abs(y0 - d["y0"]).max() < 5e-3
    y, chi = O.variational_refine(s, c, d["chi0"].astype(np.complex128), cfg,
                                  is_pal=O.uses_vswitch(g))
    assert np.abs(chi - d["chi_refine"]).max() < 5e-3
    assert np.abs(y - d["y_refine"]).max() < 5e-3
    # whole 2-D field decode from the raw samples
    (yd, chid, _), = O.decode_fields_2d([ire], [0], g, cfg)
    assert np.abs(yd - d["y_decode"]).max() < 2e-2
    assert np.abs(chid - d["chi_decode"]).max() < 2e-2


def test_oracle_motion_matches_reference_golden():
    d = np.load(GOLD / "motion_small.npz")
    dy, dx, cf = O.estimate_motion(d["y_ref"], d["y_cur"], int(d["tile"]), int(d["search"]))
    # same integer vectors and sub-pel fits (FP64 vs the reference's FP32)
    assert np.abs(dy - d["dy"]).max() < 1e-4 and np.abs(dx - d["dx"]).max() < 1e-4
    assert np.abs(cf - d["conf"]).max() < 1e-4


# ---------------------------------------------------------------------------
# 3. algebra behind the device kernels
# ---------------------------------------------------------------------------

def _khat(k, n, M, scale=1.0):
    kt = np.zeros(M, np.complex128)
    for j in range(-(n - 1), n):
        kt[j % M] = k[j % n]
    return np.fft.fft(kt) * scale / M


def test_init_cyclic_convolution_equals_fft_crop():
    """k_init_rows / k_init_cols: IDFT(gy gx DFT(x)) on the padded field equals
    a row cyclic convolution (length 2048) followed by a column one (length
    1024) with the kernels' spectra."""
    d = np.load(GOLD / "field_pal_small.npz")
    g = geom_from(d["geometry"], d["sample_rate"])
    s, c = d["s"].astype(np.float64), d["carrier"].astype(np.complex128)
    h, w = s.shape
    pad = min(16, h - 1)
    hp = h + 2 * pad
    X = (s * np.conj(c))[O.mirror_row(np.arange(hp) - pad, h)]
    for (mhz, cph) in O.INIT_VARIANTS:
        gy, gx = O.gaussian_lpf(hp, w, g, mhz, cph, h)
        want = np.fft.ifft2(np.fft.fft2(X) * gy[:, None] * gx[None, :])
        xp = np.zeros((hp, 2048), complex)
        xp[:, :w] = X
        R = np.fft.ifft(np.fft.fft(xp, axis=1) * _khat(np.fft.ifft(gx), w, 2048)[None, :],
                        axis=1)[:, :w] * 2048
        cp = np.zeros((1024, w), complex)
        cp[:hp] = R
        got = np.fft.ifft(np.fft.fft(cp, axis=0) * _khat(np.fft.ifft(gy), hp, 1024)[:, None],
                          axis=0)[:hp] * 1024
        assert np.abs(got - want).max() < 1e-10


@pytest.mark.parametrize("h,w,row_m,col_m", [(96, 1135, 4096, 1024), (600, 96, 2048, 2048),
                                             (1000, 96, 2048, 4096), (40, 2048, 4096, 1024)])
def test_init_cyclic_convolution_long_lengths(h, w, row_m, col_m):
    """The same identity at the lengths of the planes past the register
    transforms: rows of more than 1024 samples at 4096 (k_init_rows_long),
    field columns of 513-1024 padded lines at 2048, columns of more than 1024
    padded lines at 4096 (k_init_cols_long); the widest plane (2048 samples:
    row convolution 4095 <= 4096)."""
    rng = np.random.default_rng(h * 7 + w)
    g = _cabi.default_geometry(_cabi.STD_PAL)
    pad = min(16, h - 1)
    hp = h + 2 * pad
    assert 2 * w - 1 <= row_m and 2 * hp - 1 <= col_m
    X = rng.normal(size=(hp, w)) + 1j * rng.normal(size=(hp, w))
    for (mhz, cph) in O.INIT_VARIANTS:
        gy, gx = O.gaussian_lpf(hp, w, g, mhz, cph, h)
        want = np.fft.ifft2(np.fft.fft2(X) * gy[:, None] * gx[None, :])
        xp = np.zeros((hp, row_m), complex)
        xp[:, :w] = X
        R = np.fft.ifft(np.fft.fft(xp, axis=1) * _khat(np.fft.ifft(gx), w, row_m)[None, :],
                        axis=1)[:, :w] * row_m
        cp = np.zeros((col_m, w), complex)
        cp[:hp] = R
        got = np.fft.ifft(np.fft.fft(cp, axis=0) * _khat(np.fft.ifft(gy), hp, col_m)[:, None],
                          axis=0)[:hp] * col_m
        assert np.abs(got - want).max() < 1e-10 * max(1.0, np.abs(want).max())


def test_single_reduction_cg_recurrence():
    """k_solver: with q = g(d) - g(0), g(chi + a d) = g(chi) + a q and
    curv(d) = <d, q> / 2, so ||g + a q||^2 = gg + 2 a <g,q> + a^2 <q,q>
    reproduces the reference's recomputed residual norm."""
    d = np.load(GOLD / "field_ntsc_small.npz")
    cfg = cfg_from(d["cfg"])
    s, c = d["s"].astype(np.float64), d["carrier"].astype(np.complex128)
    chi = d["chi0"].astype(np.complex128)
    _, _, W = O.variational_refine(s, c, chi, _cabi.config_copy(cfg, irls_outer=1, cg_iterations=1),
                                   return_weights=True)
    mu_h = cfg.lambda_c * O.resolve_chroma_aniso(chi, cfg, False)
    mu_v = cfg.lambda_c

    def grad(ch, ss):
        yc = ss - np.real(ch * c)
        img = 2 * (O.DxT(W["wx"] * O.Dx(yc)) + O.DyT(W["wy"] * O.Dy(yc)))
        return -img * np.conj(c) + 2 * (mu_h * O.DxT(W["wcx"] * O.Dx(ch)) +
                                        mu_v * O.DyT(W["wcy"] * O.Dy(ch)))
    rng = np.random.default_rng(1)
    dd = rng.normal(size=s.shape) + 1j * rng.normal(size=s.shape)
    g0 = grad(chi, s)
    q = grad(dd, np.zeros_like(s))
    a = 0.37
    g1 = grad(chi + a * dd, s)
    assert np.abs(g1 - (g0 + a * q)).max() < 1e-9
    dy = -np.real(dd * c)
    curv = (np.sum(W["wx"] * O.Dx(dy) ** 2) + np.sum(W["wy"] * O.Dy(dy) ** 2) +
            mu_h * np.sum(W["wcx"] * np.abs(O.Dx(dd)) ** 2) +
            mu_v * np.sum(W["wcy"] * np.abs(O.Dy(dd)) ** 2))
    assert abs(curv - 0.5 * np.real(np.vdot(dd, q))) < 1e-8 * abs(curv)
    gg = np.vdot(g0, g0).real
    pred = gg + 2 * a * np.real(np.vdot(g0, q)) + a * a * np.vdot(q, q).real
    assert abs(pred - np.vdot(g1, g1).real) < 1e-9 * gg


@pytest.mark.parametrize("tag", ["ntsc", "pal"])
def test_oracle_symmetry_variant_matches_reference(tag):
    """HolographicInit's optional spectral-symmetry third variant
    (holographic_init.cpp:265-306): the oracle's restatement against the
    compiled reference on the golden field's prepared S and carrier."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    from hvdg import api
    d = np.load(GOLD / f"field_{tag}_small.npz")
    g = geom_from(d["geometry"], d["sample_rate"])
    s, c = d["s"].astype(np.float64), d["carrier"].astype(np.complex128)
    y0, chi0 = O.holographic_init(s, c, g, symmetry_variant=True)
    _, chi_plain = O.holographic_init(s, c, g)
    assert np.abs(chi0 - chi_plain).max() > 0.5     # the variant changes the init
    ry0, rchi0 = ref.holographic_init(d["s"], d["carrier"], g,
                                      api.default_config(symmetry_variant=1))
    assert np.abs(chi0 - rchi0).max() < 1e-4
    assert np.abs(y0 - ry0).max() < 1e-4


@pytest.mark.parametrize("tag", ["ntsc", "pal"])
def test_oracle_diag_prior_matches_reference(tag):
    """The oriented chroma prior (diag_prior > 0: D1 / D2 diffusivities,
    gradient and curvature terms and the prior-mass renormalisation,
    variational.cpp:207-222, 316-328, 371-383, 434-451): the oracle's 2-D
    decode against the compiled reference, at 0.5 -- the two agree as
    closely as without the oriented terms, and the terms move the decode."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    from hvdg import api, synth
    std = _cabi.STD_NTSC if tag == "ntsc" else _cabi.STD_PAL
    g = _cabi.default_geometry(std)
    f = synth.make_field(41 + std, std, noise_sigma=0.5)
    ire = synth.to_ire(f.samples)
    got = {}
    for dp in (0.0, 0.5):
        cfg = api.default_config(irls_outer=2, cg_iterations=30, fast=0, cg_tol=1e-6,
                                 temporal_strength=-1.0, diag_prior=dp)
        (yo, co, _), = O.decode_fields_2d([ire], [0], g, cfg)
        (yr,), (cr,) = ref.decode_fields([ire], [0], [g], [cfg], across_fields=False)
        assert np.abs(yo - yr).max() < 0.02 and np.abs(co - cr).max() < 0.02, dp
        got[dp] = yo
    assert np.abs(got[0.5] - got[0.0]).max() > 0.1


def test_oracle_drizzle_matches_reference():
    """DrizzleFrame (sequence.cpp:283-421): the FP64 restatement against the
    compiled reference on the reference's own 2-D decodes of a moving NTSC
    window. Deposit positions are rounding decisions on motion vectors that
    agree to ~1e-4 px, so a few samples land one row / column apart; the
    rest agrees to float rounding."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    from hvdg import api, synth
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    fs = synth.make_sequence(5, _cabi.STD_NTSC, 8, noise_sigma=0.5, moving=True)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6,
                             temporal_strength=-1.0)
    par = [f.parity for f in fs]
    ys, cs, _ = ref.decode_field_window([synth.to_ire(f.samples) for f in fs], par, g, cfg)
    ry, rc = ref.drizzle_frame(4, ys, cs, par, cfg, 2)
    oy, oc = O.drizzle_frame(4, ys, cs, par, cfg, 2)
    assert ry.shape == (2 * 2 * g.active_lines, g.active_width)
    d, dc = np.abs(oy - ry), np.abs(oc - rc)
    assert d.mean() < 1e-4 and dc.mean() < 1e-4
    assert (d > 1e-3).mean() < 1e-3 and (dc > 1e-3).mean() < 1e-3


@pytest.mark.parametrize("case", ["pal_m", "custom_fsc"])
def test_oracle_other_standards_match_reference(case):
    """PAL-M (90 deg / line, V-switch) and a declared subcarrier frequency
    (exact column phasors, fractional line advance): the oracle's 2-D decode
    against the compiled reference on the same field."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    from hvdg import api, synth
    if case == "pal_m":
        g, std = _cabi.default_geometry(_cabi.STD_PAL_M), _cabi.STD_PAL_M
    else:
        g, std = _cabi.default_geometry(_cabi.STD_NTSC), _cabi.STD_NTSC
        g.subcarrier_hz = _cabi.FSC_NTSC * (1.0 + 3e-4)
    f = synth.make_field(31, std, noise_sigma=0.5, geometry=g)
    cfg = api.default_config(irls_outer=3, cg_iterations=60, fast=0, cg_tol=1e-6,
                             temporal_strength=-1.0)
    ire = synth.to_ire(f.samples)
    (yo, co, _), = O.decode_fields_2d([ire], [0], g, cfg)
    (yr,), (cr,) = ref.decode_fields([ire], [0], [g], [cfg], across_fields=False)
    assert np.abs(yo - yr).max() < 2e-2 and np.abs(co - cr).max() < 2e-2


@pytest.mark.parametrize("std,seed", [(0, 61), (1, 62)])
def test_oracle_adaptive_strength_matches_reference(std, seed):
    """The adaptive temporal strength (sequence.cpp:526-646): the oracle's
    float32 restatement, fed the compiled reference's own prepared S and
    carrier planes and its calibrated nr_eps, gives the reference's
    ambiguity and resolved strength exactly."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    from hvdg import api, synth
    g = _cabi.default_geometry(std)
    nf = 6 if std == _cabi.STD_NTSC else 10
    fs = synth.make_sequence(seed, std, nf, noise_sigma=0.8, moving=True)
    ires = [synth.to_ire(f.samples) for f in fs]
    par = [f.parity for f in fs]
    cfg = api.default_config(irls_outer=1, cg_iterations=2, fast=1, temporal_strength=0.0,
                             passes=1)
    _, _, diag = ref.decode_field_window(ires, par, g, cfg)
    sc = [ref.prepare_field(i, g, cfg, p) for i, p in zip(ires, par)]
    stride = 4 if O.uses_vswitch(g) else 2
    strength, amb = O.adaptive_strength([s for s, _ in sc], [c for _, c in sc], stride,
                                        float(diag[4]))
    print(f"std={std}: reference amb {diag[1]!r} strength {diag[0]!r}; oracle {amb!r} {strength!r}")
    assert amb > 0.0
    assert np.float32(amb) == diag[1]
    assert np.float32(strength) == diag[0]


@pytest.mark.parametrize("case", ["pal_full_line", "tall1000"])
def test_oracle_long_planes_match_reference(case):
    """Planes past the device init's register transforms (a whole 1135-sample
    PAL line; 1000 lines, padded 1032): the oracle's init (plain and
    symmetry variant) and 2-D decode against the compiled reference, whose
    FFTs run at the plane's own size (holographic_init.cpp:214-222)."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    from hvdg import api, synth
    if case == "pal_full_line":
        g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_PAL), active_video_start=0,
                                active_video_end=1135, first_active_field_line=22,
                                last_active_field_line=118)
    else:
        g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_NTSC), field_height=1020,
                                first_active_field_line=10, last_active_field_line=1010,
                                active_video_start=134, active_video_end=230)
    f = synth.make_field(251, g.standard, noise_sigma=0.5, geometry=g)
    cfg = api.default_config(irls_outer=3, cg_iterations=60, fast=0, cg_tol=1e-6,
                             temporal_strength=-1.0)
    ire = synth.to_ire(f.samples)
    rs, rc = ref.prepare_field(ire, g, cfg, 0)
    for sym in (0, 1):
        y0, chi0 = O.holographic_init(rs.astype(np.float64), rc.astype(np.complex128), g,
                                      symmetry_variant=bool(sym))
        ry0, rchi0 = ref.holographic_init(rs, rc, g, api.default_config(symmetry_variant=sym))
        assert np.abs(chi0 - rchi0).max() < 1e-4 and np.abs(y0 - ry0).max() < 1e-4
    (yo, co, _), = O.decode_fields_2d([ire], [0], g, cfg)
    (yr,), (cr,) = ref.decode_fields([ire], [0], [g], [cfg], across_fields=False)
    assert np.abs(yo - yr).max() < 2e-2 and np.abs(co - cr).max() < 2e-2
