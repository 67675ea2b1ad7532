"""GPU parity of the 2-D field decode (lock-in -> init -> IRLS + CG) against
the FP64 oracle (oracle/hvd_oracle.py) and, where built, the compiled
reference engine. Tolerances: PSNR against ground truth within 0.05 dB of
the oracle's; max |dY|, |dC| small in IRE."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


def psnr(a, b, peak=100.0):
    d = np.asarray(a) - np.asarray(b)
    return 10 * np.log10(peak ** 2 / np.mean(np.abs(d.astype(np.complex128)) ** 2))


def _cfg(**kw):
    base = dict(irls_outer=5, cg_iterations=150, fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    base.update(kw)
    return api.default_config(**base)


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
def test_decode_field_matches_oracle(ctx, std):
    g = _cabi.default_geometry(std)
    f = synth.make_field(11 + std, std, noise_sigma=0.5)
    cfg = _cfg()
    out = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg, want_theta=True)[0]
    ire = synth.to_ire(f.samples)
    (yo, chio, obs), = O.decode_fields_2d([ire], [0], g, cfg)
    # lock-in phases (FP64 on both sides)
    dth = np.abs(np.angle(np.exp(1j * (out.theta.astype(np.float64) - obs.theta))))
    assert dth.max() < 1e-4
    if std == _cabi.STD_PAL:
        assert (out.vswitch == obs.vswitch).all()
    dY = np.abs(out.luma - yo).max()
    dC = np.abs(out.chroma - chio).max()
    p_gpu = psnr(out.luma, f.y_true)
    p_orc = psnr(yo, f.y_true)
    pc_gpu = psnr(out.chroma, f.chi_true)
    pc_orc = psnr(chio, f.chi_true)
    print(f"std={std} maxdY={dY:.4g} maxdC={dC:.4g} PSNR Y gpu={p_gpu:.3f} oracle={p_orc:.3f} "
          f"C gpu={pc_gpu:.3f} oracle={pc_orc:.3f} vs-oracle={psnr(out.luma, yo):.1f} dB")
    assert abs(p_gpu - p_orc) < 0.05
    assert abs(pc_gpu - pc_orc) < 0.05
    assert dY < 0.05 and dC < 0.05
    # lossless split: Y + Re[chi c] == S
    s = obs.s
    assert np.abs(out.luma + np.real(out.chroma * obs.carrier) - s).max() < 2e-3


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
def test_symmetry_variant_vs_oracle(ctx, std):
    """HolographicInit's spectral-symmetry third variant
    (holographic_init.cpp:265-306: exact hp x w 2-D DFT by Bluestein rows /
    columns on the device, certified spectrum, inverse, blended third) --
    the init alone and the whole 2-D decode against the FP64 oracle."""
    g = _cabi.default_geometry(std)
    f = synth.make_field(21 + std, std, noise_sigma=0.5)
    cfg = _cfg(symmetry_variant=1)
    ire = synth.to_ire(f.samples)
    obs = O.prepare_field(ire, g, cfg, 0)
    fal, lal = g.first_active_field_line, g.last_active_line
    th = obs.theta[fal:lal].astype(np.float32)
    sw = obs.vswitch[fal:lal].astype(np.int8)
    y0, chi0 = ctx.holographic_init(obs.s.astype(np.float32), th, sw, g, cfg)
    yo, co = O.holographic_init(obs.s, O.make_carrier(th, sw, g), g, symmetry_variant=True)
    _, cplain = O.holographic_init(obs.s, O.make_carrier(th, sw, g), g)
    dc, dy = np.abs(chi0 - co).max(), np.abs(y0 - yo).max()
    print(f"std={std} init: max dchi {dc:.3g} max dY {dy:.3g} "
          f"(variant moves chi by {np.abs(co - cplain).max():.3g})")
    assert np.abs(co - cplain).max() > 0.5
    assert dc < 5e-3 and dy < 5e-3
    out = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg)[0]
    (yd, cd, _), = O.decode_fields_2d([ire], [0], g, cfg)
    print(f"std={std} decode: max dY {np.abs(out.luma - yd).max():.3g} "
          f"max dC {np.abs(out.chroma - cd).max():.3g}")
    assert abs(psnr(out.luma, f.y_true) - psnr(yd, f.y_true)) < 0.05
    assert abs(psnr(out.chroma, f.chi_true) - psnr(cd, f.chi_true)) < 0.05
    assert np.abs(out.luma - yd).max() < 0.05 and np.abs(out.chroma - cd).max() < 0.05


def _geometry_case(case):
    if case == "pal_m":
        # PAL-M: 525-line raster, PAL V-switch, 90 deg per line (ntsc_geometry.h:40-47, 165-166)
        return _cabi.default_geometry(_cabi.STD_PAL_M), _cabi.STD_PAL_M
    # a declared, non-standard subcarrier: w0 = 2 pi fsc / fs != pi / 2 and
    # the per-line advance from the fractional cycles per line
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    g.subcarrier_hz = _cabi.FSC_NTSC * (1.0 + 3e-4)
    return g, _cabi.STD_NTSC


@pytest.mark.parametrize("case", ["pal_m", "custom_fsc"])
def test_other_standards_vs_oracle_and_reference(ctx, case):
    """PAL-M and a declared subcarrier frequency (the lock-in's PAL-family
    parity search at 90 deg / line; exact column phasors exp(i w0 x) instead
    of the 4fsc quadrants) against the FP64 oracle and the compiled
    reference."""
    g, std = _geometry_case(case)
    f = synth.make_field(31, std, noise_sigma=0.5, geometry=g)
    cfg = _cfg()
    out = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg, want_theta=True)[0]
    ire = synth.to_ire(f.samples)
    (yo, chio, obs), = O.decode_fields_2d([ire], [0], g, cfg)
    dth = np.abs(np.angle(np.exp(1j * (out.theta.astype(np.float64) - obs.theta))))
    assert dth.max() < 1e-4
    if std == _cabi.STD_PAL_M:
        assert (out.vswitch == obs.vswitch).all()
    dY, dC = np.abs(out.luma - yo).max(), np.abs(out.chroma - chio).max()
    print(f"{case}: maxdY={dY:.3g} maxdC={dC:.3g} PSNR Y gpu={psnr(out.luma, f.y_true):.2f} "
          f"oracle={psnr(yo, f.y_true):.2f}")
    assert abs(psnr(out.luma, f.y_true) - psnr(yo, f.y_true)) < 0.05
    assert abs(psnr(out.chroma, f.chi_true) - psnr(chio, f.chi_true)) < 0.05
    assert dY < 0.05 and dC < 0.05
    assert psnr(out.luma, f.y_true) > 35.0     # the decode actually separates
    from oracle import ref
    if ref.available():
        (yr,), (cr,) = ref.decode_fields([ire], [0], [g], [cfg], across_fields=False)
        assert np.abs(out.luma - yr).max() < 0.05 and np.abs(out.chroma - cr).max() < 0.05


def test_pinned_outputs_written_by_the_solver(ctx):
    """Page-locked output buffers are written by the solver's final phase
    itself (mapped host memory), overlapping the other fields' solves; the
    results equal those copied into pageable buffers, bit for bit, for a
    mixed NTSC / PAL batch with an odd-width geometry (unaligned dense rows)."""
    torch = pytest.importorskip("torch")
    fs = synth.mixed_batch(5, 3, 2, outer_range=(2, 3), cg_per_outer=10)
    geoms = [_cabi.default_geometry(f.standard) for f in fs]
    g_odd = _cabi.geometry_copy(geoms[0], active_video_end=geoms[0].active_video_end - 1)
    geoms[0] = g_odd
    cfg = _cfg()
    fields = [api.Field(f.samples, g, parity=f.parity, irls_outer=f.irls_outer,
                        cg_iterations=f.cg_iterations) for f, g in zip(fs, geoms)]
    ref_out = ctx.decode_fields(fields, cfg)
    pinned, keep = [], []
    for g in geoms:
        ty = torch.zeros((g.active_lines, g.active_width), dtype=torch.float32, pin_memory=True)
        tc = torch.zeros((g.active_lines, g.active_width, 2), dtype=torch.float32,
                         pin_memory=True)
        keep += [ty, tc]
        pinned.append(api.Decoded(ty.numpy(), tc.numpy().view(np.complex64)[..., 0]))
    got = ctx.decode_fields(fields, cfg, out=pinned)
    for a, b in zip(got, ref_out):
        assert np.array_equal(a.luma, b.luma)
        assert np.array_equal(a.chroma, b.chroma)
