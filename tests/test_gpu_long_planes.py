"""Planes past the register transforms of the holographic init, against the
FP64 oracle. Rows longer than 1024 active samples and padded columns longer
than 1024 lines run their cyclic convolutions at length 4096 through the
shared-memory FFT (k_init_rows_long, k_init_cols_long, k_sym_cols_long,
k_sym_rows<4096>); field planes of 481-992 lines take the 2048-point column
pass of woven frames. The reference has no such lengths: FFTW runs at the
plane's own size (holographic_init.cpp:214-222), which the oracle restates.

Cases: a full PAL line (1135 samples), the widest plane (2048 samples), a
600-line and a 1000-line field, the init alone (and its symmetry variant)
on long rows and long columns, one batch mixing long and standard
geometries, the decode adjoint on a long-row field, the 3-D field window on
long rows against the compiled reference, and one past each limit
(HVDG_ERR_UNSUPPORTED)."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_adjoint as A
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu

CPI = (51200.0 - 16384.0) / 100.0


def _cfg(**kw):
    base = dict(irls_outer=3, cg_iterations=60, fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    base.update(kw)
    return api.default_config(**base)


def _full_pal_line():
    # the whole 4fsc PAL line as the active window: 1135 samples
    g = _cabi.default_geometry(_cabi.STD_PAL)
    return _cabi.geometry_copy(g, active_video_start=0, active_video_end=1135,
                               first_active_field_line=22, last_active_field_line=118)


def _widest():
    # 2048 active samples (row convolution 4095 <= 4096), 40 lines
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    return _cabi.geometry_copy(g, field_width=2140, active_video_start=60,
                               active_video_end=2108, first_active_field_line=20,
                               last_active_field_line=60)


def _tall(lines):
    # NTSC columns, `lines` active lines, 96 samples wide
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    return _cabi.geometry_copy(g, field_height=lines + 20, first_active_field_line=10,
                               last_active_field_line=lines + 10, active_video_start=134,
                               active_video_end=230)


def _vs_oracle(ctx, g, seed, tol=0.05):
    f = synth.make_field(seed, g.standard, noise_sigma=0.5, geometry=g)
    cfg = _cfg()
    out = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg)[0]
    (yo, co, _), = O.decode_fields_2d([synth.to_ire(f.samples)], [0], g, cfg)
    dy, dc = np.abs(out.luma - yo).max(), np.abs(out.chroma - co).max()
    print(f"h={g.active_lines} w={g.active_width}: max dY {dy:.3g} max dC {dc:.3g}")
    assert out.luma.shape == (g.active_lines, g.active_width)
    assert dy < tol and dc < tol


@pytest.mark.parametrize("case", ["pal_full_line", "widest", "tall600", "tall1000"])
def test_long_plane_decode_vs_oracle(ctx, case):
    g = {"pal_full_line": _full_pal_line, "widest": _widest,
         "tall600": lambda: _tall(600), "tall1000": lambda: _tall(1000)}[case]()
    _vs_oracle(ctx, g, 201 + len(case))


@pytest.mark.parametrize("case", ["pal_full_line", "tall1000"])
@pytest.mark.parametrize("sym", [0, 1])
def test_long_plane_init_vs_oracle(ctx, case, sym):
    """The init alone on long rows (PAL full line) and long columns (1000
    lines, padded 1032), plain and with the symmetry variant (Bluestein at
    length 4096 for the exact-length DFTs)."""
    g = _full_pal_line() if case == "pal_full_line" else _tall(1000)
    f = synth.make_field(211 + sym, g.standard, noise_sigma=0.5, geometry=g)
    cfg = _cfg(symmetry_variant=sym)
    obs = O.prepare_field(synth.to_ire(f.samples), g, cfg, 0)
    fal, lal = g.first_active_field_line, g.last_active_line
    th = obs.theta[fal:lal].astype(np.float32)
    sw = obs.vswitch[fal:lal].astype(np.int8)
    y0, chi0 = ctx.holographic_init(obs.s.astype(np.float32), th, sw, g, cfg)
    yo, co = O.holographic_init(obs.s, O.make_carrier(th, sw, g), g, symmetry_variant=bool(sym))
    dc, dy = np.abs(chi0 - co).max(), np.abs(y0 - yo).max()
    print(f"{case} sym={sym}: max dchi {dc:.3g} max dY {dy:.3g}")
    tol = 5e-3 if sym else 1e-3
    assert dc < tol and dy < tol


def test_mixed_long_and_standard_batch(ctx):
    """One batched call over a standard NTSC field, a full PAL line and a
    1000-line field: the register and shared-memory kernels share the init
    grids, each taking its own geometries' rows and columns."""
    gs = [_cabi.default_geometry(_cabi.STD_NTSC), _full_pal_line(), _tall(1000)]
    fs = [synth.make_field(221 + i, g.standard, noise_sigma=0.5, geometry=g)
          for i, g in enumerate(gs)]
    cfg = _cfg()
    outs = ctx.decode_fields([api.Field(f.samples, g, parity=0) for f, g in zip(fs, gs)], cfg)
    for f, g, out in zip(fs, gs, outs):
        (yo, co, _), = O.decode_fields_2d([synth.to_ire(f.samples)], [0], g, cfg)
        dy, dc = np.abs(out.luma - yo).max(), np.abs(out.chroma - co).max()
        print(f"h={g.active_lines} w={g.active_width}: max dY {dy:.3g} max dC {dc:.3g}")
        assert dy < 0.05 and dc < 0.05


def test_long_row_adjoint_vs_fp64_oracle(ctx):
    """The decode adjoint on a field 1160 samples wide: the adjoint of the
    init's filter passes runs through the long-row kernel (adjoint mode)."""
    g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_NTSC), field_width=1300,
                            active_video_start=100, active_video_end=1260,
                            first_active_field_line=20, last_active_field_line=84)
    f = synth.make_field(231, _cabi.STD_NTSC, 0.5, geometry=g)
    cfg = api.default_config(irls_outer=3, cg_iterations=80, fast=0, cg_tol=1e-6,
                             temporal_strength=-1.0)
    fld = api.Field(f.samples, g, parity=0)
    dec = ctx.decode_fields([fld], cfg)[0]
    n = dec.luma.size
    yb = (2 * (dec.luma.astype(np.float64) - f.y_true) / n).astype(np.float32)
    cb = (2 * (dec.chroma.astype(np.complex128) - f.chi_true) / n).astype(np.complex64)
    sbar, sc, _ = ctx.decode_fields_adjoint([fld], cfg, [yb], [cb], 300)
    obs = O.prepare_field(synth.to_ire(f.samples), g, cfg)
    _, _, chi0 = A.init_parts(obs.s, obs.carrier, g)
    aniso = O.resolve_chroma_aniso(chi0, cfg, False)
    chis = A.refine_forward_budget(obs.s, obs.carrier, chi0, cfg, aniso)
    s_bar, chi0_bar, gl = A.refine_adjoint(obs.s, obs.carrier, chis, cfg, aniso, yb, cb, 1e-8, 3000)
    s_bar = s_bar + A.init_adjoint(obs.s, obs.carrier, g, chi0_bar)
    for k_gpu, k_orc in (("lambda_c", "lambda_c"), ("charbonnier_eps", "eps")):
        print(k_gpu, sc[k_gpu], gl[k_orc])
        assert abs(sc[k_gpu] - gl[k_orc]) <= 1e-3 * abs(gl[k_orc]) + 1e-9
    fal, lal = g.first_active_field_line, g.last_active_line
    a0, a1 = g.active_video_start, g.active_video_end
    got = sbar[0][fal:lal, a0:a1].astype(np.float64)
    want = s_bar / CPI
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    print("sample gradient rel L2", rel)
    assert rel < 1e-3


def test_long_row_window_vs_reference(ctx):
    """The temporal (3-D) field window -- motion search, neighbour terms,
    envelope gate -- on PAL fields 1140 samples wide (long-row init) against
    the compiled reference on the same fields: PSNR against ground truth
    within 0.05 dB of the reference's, field by field."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_PAL), field_width=1300,
                            active_video_start=150, active_video_end=1290)
    nf = 6
    sc = synth.make_scene(261, _cabi.STD_PAL, n_rects=4, geometry=g)
    seq = [synth.make_field(261, _cabi.STD_PAL, 1.0, field_index=j, parity=j % 2, scene=sc,
                            theta_base=0.3, geometry=g) for j in range(nf)]
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6,
                             temporal_strength=0.5, passes=1, nr_anchor=0.0, coherence_gate=0.0,
                             trajectory_fit=0)
    outs = ctx.decode_field_window([api.Field(f.samples, g, parity=f.parity) for f in seq], cfg)
    ys, cs, _ = ref.decode_field_window([synth.to_ire(f.samples) for f in seq],
                                        [f.parity for f in seq], g, cfg)

    def psnr(a, b):
        d = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
        return 10 * np.log10(100.0 ** 2 / np.mean(np.abs(d) ** 2))

    for j in range(nf):
        pg, pr = psnr(outs[j].luma, seq[j].y_true), psnr(ys[j], seq[j].y_true)
        cg, cr = psnr(outs[j].chroma, seq[j].chi_true), psnr(cs[j], seq[j].chi_true)
        print(f"wide window field {j}: Y gpu {pg:.3f} ref {pr:.3f}  C gpu {cg:.3f} ref {cr:.3f}")
        assert abs(pg - pr) < 0.05 and abs(cg - cr) < 0.05


def test_one_past_each_limit(ctx):
    """2049 active samples (row convolution 4097 > 4096) and 1025 lines per
    field (the lock-in's line table) are refused; the context stays usable."""
    wide = _widest()
    tall = _tall(1000)
    for g, edit in ((wide, dict(active_video_end=wide.active_video_end + 1)),
                    (tall, dict(field_height=1025, last_active_field_line=1015))):
        bad = _cabi.geometry_copy(g, **edit)
        f = synth.make_field(241, g.standard, 0.5, geometry=bad)
        with pytest.raises(api.HvdgError) as e:
            ctx.decode_fields([api.Field(f.samples, bad, parity=0)], _cfg())
        assert e.value.status == _cabi.ERR_UNSUPPORTED
    _vs_oracle(ctx, _cabi.default_geometry(_cabi.STD_NTSC), 242)
