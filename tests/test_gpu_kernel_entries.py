"""The exported kernel-level entries on their own: hvdg_burst_amplitude
(BurstAmplitudeIre, lockin.cpp:256-323) against the FP64 oracle and the
compiled reference, and hvdg_variational_refine (VariationalRefine,
variational.cpp:198-556) started from the oracle's init against the FP64
oracle's refine, on NTSC and PAL, with and without the oriented chroma
prior. Tolerances: amplitude within 1e-3 IRE; refine max |dY|, |dC| below
0.05 IRE and PSNR against ground truth within 0.05 dB of the oracle's."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


def psnr(a, b, peak=100.0):
    d = np.asarray(a) - np.asarray(b)
    return 10 * np.log10(peak ** 2 / np.mean(np.abs(d.astype(np.complex128)) ** 2))


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
@pytest.mark.parametrize("burst_gain", [1.0, 0.6])
def test_burst_amplitude_entry(ctx, std, burst_gain):
    """The chroma part (active chroma and burst) scaled by `burst_gain`, as a
    tape with a weak burst gives the ACC stage."""
    g = _cabi.default_geometry(std)
    _, y_part, c_part, noise = synth.make_field(70 + std, std, noise_sigma=0.8, return_parts=True)
    ire = (y_part + burst_gain * c_part + noise).astype(np.float32)
    got = ctx.burst_amplitude(ire, g)
    want = O.burst_amplitude_ire(ire, g)
    print(f"std={std} gain={burst_gain}: device {got:.6f} oracle {want:.6f}")
    assert abs(got - want) < 1e-3
    from oracle import ref
    if ref.available():
        r = ref.burst_amplitude(ire, g)
        print(f"  reference {r:.6f}")
        assert abs(got - r) < 1e-3


def test_burst_amplitude_entry_short_burst_window(ctx):
    """A burst window under 4 samples returns the standard's nominal burst
    amplitude (lockin.cpp:262-264), as the oracle does."""
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    f = synth.make_field(75, _cabi.STD_NTSC, noise_sigma=0.5)
    g.colour_burst_end = g.colour_burst_start + 3
    ire = synth.to_ire(f.samples)
    assert abs(ctx.burst_amplitude(ire, g) - O.burst_amplitude_ire(ire, g)) < 1e-6


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
@pytest.mark.parametrize("diag_prior", [0.0, 0.5])
def test_variational_refine_entry(ctx, std, diag_prior):
    g = _cabi.default_geometry(std)
    f = synth.make_field(80 + std, std, noise_sigma=0.5)
    cfg = api.default_config(irls_outer=4, cg_iterations=120, fast=0, cg_tol=1e-6,
                             temporal_strength=-1.0, diag_prior=diag_prior)
    obs = O.prepare_field(synth.to_ire(f.samples), g, cfg, 0)
    fal, lal = g.first_active_field_line, g.last_active_line
    th = obs.theta[fal:lal].astype(np.float32)
    sw = obs.vswitch[fal:lal].astype(np.int8)
    carrier = O.make_carrier(th, sw, g)
    _, chi0 = O.holographic_init(obs.s, carrier, g)
    y, chi = ctx.variational_refine(obs.s.astype(np.float32), th, sw, chi0.astype(np.complex64),
                                    g, cfg)
    yo, co = O.variational_refine(obs.s, carrier, chi0, cfg, is_pal=O.uses_vswitch(g))
    dy, dc = np.abs(y - yo).max(), np.abs(chi - co).max()
    yt, ct = f.y_true, f.chi_true
    print(f"std={std} diag={diag_prior}: max dY {dy:.3g} max dC {dc:.3g}")
    assert dy < 0.05 and dc < 0.05
    assert abs(psnr(y, yt) - psnr(yo, yt)) < 0.05
    assert abs(psnr(chi, ct) - psnr(co, ct)) < 0.05


def test_variational_refine_entry_refuses_bad_geometry(ctx):
    """A chi0 plane whose geometry the refine cannot take is refused with a
    status before any plane is read: the active width above the
    2048-sample limit (arrays sized to the refused geometry)."""
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    g.field_width = g.active_video_start + 2049 + 8
    g.active_video_end = g.active_video_start + 2049
    h = g.last_active_line - g.first_active_field_line
    s = np.zeros((h, 2049), np.float32)
    th = np.zeros(h, np.float32)
    sw = np.zeros(h, np.int8)
    with pytest.raises(RuntimeError, match="hvdg_variational_refine"):
        ctx.variational_refine(s, th, sw, np.zeros((h, 2049), np.complex64), g,
                               api.default_config(temporal_strength=-1.0))
