"""CPU pins for the woven-frame path (no GPU): the reference's own
sensitivity to the carrier phase precision on a woven PAL frame, which sets
the PAL u / v tolerance of tests/test_gpu_frame_buffer.py.

WeaveAndBuildCarrier (engine.cpp:53-126) weaves the two fields' active
pictures and per-line phases; MakeCarrierPal (ntsc_geometry.cpp:438-456)
evaluates theta[y] + w0 x in float. On PAL theta reaches ~1500 rad, so the
float phase carries ~1e-4 rad of rounding. Re-running the reference's
HolographicInit + VariationalRefine with the same phases evaluated in double
moves its u / v by ~0.1 codes (5.6 codes / IRE)."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth


def _woven(ref, std, frame, field1_bottom=False):
    fp = api.frame_params(std)
    g = _cabi.default_geometry(std)
    top, bot = ref.split_frame_fields(frame, fp)
    if field1_bottom:
        top, bot = bot, top     # the field on the even woven rows first
    fal, lal = g.first_active_field_line, g.last_active_line
    a0, a1 = g.active_video_start, g.active_video_end
    th_t, vs_t = ref.burst_lockin(top, g)
    th_b, vs_b = ref.burst_lockin(bot, g)
    n = lal - fal
    s = np.zeros((2 * n, a1 - a0), np.float32)
    th = np.zeros(2 * n, np.float32)
    vs = np.zeros(2 * n, np.int8)
    s[0::2], s[1::2] = top[fal:lal, a0:a1], bot[fal:lal, a0:a1]
    th[0::2], th[1::2] = th_t[fal:lal], th_b[fal:lal]
    vs[0::2], vs[1::2] = vs_t[fal:lal], vs_b[fal:lal]
    return g, s, th, vs


def _carrier(th, vs, a0, a1, double):
    x = np.arange(a0, a1)
    if double:
        c = np.exp(1j * (th.astype(np.float64)[:, None] + 0.5 * np.pi * x[None, :]))
    else:
        ph = th[:, None] + np.float32(0.5 * np.pi) * x[None, :].astype(np.float32)
        c = np.cos(ph) + 1j * np.sin(ph)
    c = np.where(vs[:, None] < 0, -np.conj(c), c)
    return c.astype(np.complex64)


def pal_carrier_sensitivity(ref, frame, cfg, field1_bottom=False):
    """Max |u / v| (codes) the reference's woven-frame init + solve moves by
    when the carrier phase of one PAL frame is evaluated in double instead
    of float."""
    g, s, th, vs = _woven(ref, _cabi.STD_PAL, frame, field1_bottom)
    assert th.max() > 1000.0  # the phases the float carrier rounds
    chis = []
    for double in (False, True):
        c = _carrier(th, vs, g.active_video_start, g.active_video_end, double)
        _, chi0 = ref.holographic_init(s, c, g, cfg)
        _, chi = ref.variational_refine(s, c, chi0, cfg, is_pal=True)
        chis.append(chi)
    return np.abs(chis[0] - chis[1]).max() * 5.6


def test_reference_pal_weave_carrier_sensitivity():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    frames, _ = synth.make_frames(62, _cabi.STD_PAL, 1, noise_sigma=1.0)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6)
    codes = pal_carrier_sensitivity(ref, frames[0], cfg)
    print(f"reference u/v move under a double carrier phase: {codes:.3f} codes")
    assert 0.03 < codes < 0.15
