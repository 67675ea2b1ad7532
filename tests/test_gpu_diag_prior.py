"""The oriented (+-45 deg) chroma prior, diag_prior > 0 (variational.cpp:
207-222 weights and renormalisation, 316-328 gradient, 371-383 curvature,
434-451 diffusivities; the anchored pass's copy at 572-578, 682-697,
745-757, 787-797, 838-841): the 2-D decode against the FP64 oracle and the
compiled reference, the frame-buffer decode and the default two-pass 3-D
window (the anchored joint solve included) against the compiled reference.
The decoder stage exposes this knob (hvd_chroma_decoder_stage.cpp:1670).

Tolerances: as the decode tests without the prior -- max |dY|, |dC| <
0.05 IRE and PSNR within 0.05 dB of the oracle; the window within 0.05 dB
window-mean / 0.15 dB per field of the reference (near-tie motion flips in
the anchored pass's re-estimated motion, test_gpu_window3d.py)."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


def psnr(a, b, peak=100.0):
    d = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
    return 10 * np.log10(peak ** 2 / np.mean(np.abs(d) ** 2))


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
def test_decode_diag_prior_vs_oracle_and_reference(ctx, std):
    g = _cabi.default_geometry(std)
    f = synth.make_field(41 + std, std, noise_sigma=0.5)
    ire = synth.to_ire(f.samples)
    cfg = api.default_config(irls_outer=3, cg_iterations=60, fast=0, cg_tol=1e-6,
                             temporal_strength=-1.0, diag_prior=0.5)
    out = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg)[0]
    (yo, co, _), = O.decode_fields_2d([ire], [0], g, cfg)
    cfg0 = api.default_config(irls_outer=3, cg_iterations=60, fast=0, cg_tol=1e-6,
                              temporal_strength=-1.0)
    plain = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg0)[0]
    dY, dC = np.abs(out.luma - yo).max(), np.abs(out.chroma - co).max()
    print(f"std={std} diag 0.5: max dY {dY:.3g} dC {dC:.3g} IRE; PSNR Y gpu "
          f"{psnr(out.luma, f.y_true):.3f} oracle {psnr(yo, f.y_true):.3f}; the prior moves "
          f"Y by {np.abs(out.luma - plain.luma).max():.3g} IRE")
    assert np.abs(out.luma - plain.luma).max() > 0.1     # the oriented terms are applied
    assert dY < 0.05 and dC < 0.05
    assert abs(psnr(out.luma, f.y_true) - psnr(yo, f.y_true)) < 0.05
    assert abs(psnr(out.chroma, f.chi_true) - psnr(co, f.chi_true)) < 0.05
    from oracle import ref
    if ref.available():
        (yr,), (cr,) = ref.decode_fields([ire], [0], [g], [cfg], across_fields=False)
        assert np.abs(out.luma - yr).max() < 0.05 and np.abs(out.chroma - cr).max() < 0.05


def test_batched_diag_prior_equals_single_field_decodes(ctx):
    """A mixed NTSC / PAL batch with the prior: each field as decoded alone."""
    fs = synth.mixed_batch(88, 2, 2, outer_range=(2, 3), cg_per_outer=20)
    cfg = api.default_config(fast=0, cg_tol=1e-6, temporal_strength=-1.0, diag_prior=0.8)
    hf = [api.Field(f.samples, _cabi.default_geometry(f.standard), parity=f.parity,
                    irls_outer=f.irls_outer, cg_iterations=f.cg_iterations) for f in fs]
    batch = ctx.decode_fields(hf, cfg)
    for i, h in enumerate(hf):
        one = ctx.decode_fields([h], cfg)[0]
        assert np.abs(one.luma - batch[i].luma).max() <= 1e-5, i
        assert np.abs(one.chroma - batch[i].chroma).max() <= 1e-5, i


def test_frame_buffer_diag_prior_vs_reference(ctx):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    frames, _ = synth.make_frames(58, _cabi.STD_NTSC, 1, noise_sigma=0.5)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6, diag_prior=0.5)
    got = ctx.decode_frame_buffer(frames[0], fp, cfg)
    want = ref.decode_frame_buffer(frames[0], fp, cfg)
    for key in ("luma", "chroma"):
        d = np.abs(got[key].astype(np.int32) - want[key].astype(np.int32))
        print(f"frame {key}: max {d.max()} frac>0 {(d > 0).mean():.2e}")
        assert d.max() <= 1 and (d > 0).mean() < 2e-3
    for key in ("u", "v"):
        assert np.abs(got[key] - want[key]).max() < 0.05


@pytest.mark.parametrize("fast", [0, 1])
def test_window_anchored_diag_prior_vs_reference(ctx, fast):
    """The default two-pass 3-D window (pass 0 with neighbour terms, pass 1
    anchored: the joint Y / chi solve) with the oriented prior."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    std, nf = _cabi.STD_NTSC, 8
    seq = synth.make_sequence(73, std, nf, noise_sigma=1.0, moving=True)
    g = _cabi.default_geometry(std)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=fast, cg_tol=1e-6,
                             temporal_strength=0.5, diag_prior=0.5)
    assert cfg.passes == 2 and cfg.nr_anchor > 0
    outs = ctx.decode_field_window([api.Field(f.samples, g, parity=f.parity) for f in seq], cfg)
    ires = [synth.to_ire(f.samples) for f in seq]
    ys, cs, _ = ref.decode_field_window(ires, [f.parity for f in seq], g, cfg)
    dys, dcs = [], []
    for j in range(nf):
        dys.append(psnr(outs[j].luma, seq[j].y_true) - psnr(ys[j], seq[j].y_true))
        dcs.append(psnr(outs[j].chroma, seq[j].chi_true) - psnr(cs[j], seq[j].chi_true))
        print(f"diag window fast={fast} field {j}: dPSNR Y {dys[-1]:.4f} C {dcs[-1]:.4f}")
    assert abs(np.mean(dys)) < 0.05 and abs(np.mean(dcs)) < 0.05
    assert np.max(np.abs(dys)) < 0.15 and np.max(np.abs(dcs)) < 0.15
