"""The decode adjoint on the GPU (hvdg_decode_fields_adjoint and the
torch.autograd binding) on full NTSC fields with the gradient configuration
(10 IRLS x 50 CG): against the FP64 adjoint oracle run on the same
cotangents (scalars and the sample gradient within 1e-3 relative), against
central differences of the device forward for lambda_c and charbonnier_eps
(1e-3 relative), and the recomputed checkpointed forward against the
one-launch decode."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_adjoint as A
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu

CPI = (51200.0 - 16384.0) / 100.0


def _cfg(**kw):
    base = dict(irls_outer=10, cg_iterations=500, fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    base.update(kw)
    return api.default_config(**base)


def _loss_and_cot(dec, f):
    y, chi = dec.luma.astype(np.float64), dec.chroma.astype(np.complex128)
    n = y.size
    loss = float(np.mean((y - f.y_true) ** 2) + np.mean(np.abs(chi - f.chi_true) ** 2))
    return loss, (2 * (y - f.y_true) / n).astype(np.float32), (2 * (chi - f.chi_true) / n).astype(np.complex64)


def test_adjoint_vs_fp64_oracle(ctx):
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    f = synth.make_field(41, _cabi.STD_NTSC, 0.5)
    cfg = _cfg()
    fld = api.Field(f.samples, g, parity=0)
    dec = ctx.decode_fields([fld], cfg)[0]
    _, yb, cb = _loss_and_cot(dec, f)
    sbar, sc, fwd = ctx.decode_fields_adjoint([fld], cfg, [yb], [cb], 300, want_forward=True)
    # the checkpointed forward (one launch per outer) is the decode
    assert np.abs(fwd[0].luma - dec.luma).max() <= 1e-4
    assert np.abs(fwd[0].chroma - dec.chroma).max() <= 1e-4
    obs = O.prepare_field(synth.to_ire(f.samples), g, cfg)
    _, _, chi0 = A.init_parts(obs.s, obs.carrier, g)
    aniso = O.resolve_chroma_aniso(chi0, cfg, False)
    chis = A.refine_forward_budget(obs.s, obs.carrier, chi0, cfg, aniso)
    s_bar, chi0_bar, gl = A.refine_adjoint(obs.s, obs.carrier, chis, cfg, aniso, yb, cb, 1e-8, 3000)
    s_bar = s_bar + A.init_adjoint(obs.s, obs.carrier, g, chi0_bar)
    for k_gpu, k_orc in (("lambda_c", "lambda_c"), ("charbonnier_eps", "eps"),
                         ("chroma_eps", "eps_c"), ("structure_coupling", "k")):
        print(k_gpu, sc[k_gpu], gl[k_orc])
        assert abs(sc[k_gpu] - gl[k_orc]) <= 1e-3 * abs(gl[k_orc]) + 1e-9
    fal, lal = g.first_active_field_line, g.last_active_line
    a0, a1 = g.active_video_start, g.active_video_end
    got = sbar[0][fal:lal, a0:a1].astype(np.float64)
    want = s_bar / CPI
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    print("sample gradient rel L2", rel)
    assert rel < 1e-3
    outside = sbar[0].copy()
    outside[fal:lal, a0:a1] = 0.0
    assert not outside.any()


def test_adjoint_vs_device_central_differences(ctx):
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    f = synth.make_field(43, _cabi.STD_NTSC, 0.8)
    cfg = _cfg()
    fld = api.Field(f.samples, g, parity=1)
    _, yb, cb = _loss_and_cot(ctx.decode_fields([fld], cfg)[0], f)
    _, sc, _ = ctx.decode_fields_adjoint([fld], cfg, [yb], [cb], 300)
    for name in ("lambda_c", "charbonnier_eps"):
        v = getattr(cfg, name)
        h = 1e-2 * abs(v)
        lp = _loss_and_cot(ctx.decode_fields([fld], _cabi.config_copy(cfg, **{name: v + h}))[0], f)[0]
        lm = _loss_and_cot(ctx.decode_fields([fld], _cabi.config_copy(cfg, **{name: v - h}))[0], f)[0]
        fd = (lp - lm) / (2 * h)
        print(name, sc[name], fd)
        assert abs(sc[name] - fd) <= 1e-3 * abs(fd)


def test_torch_autograd_binding(ctx):
    torch = pytest.importorskip("torch")
    from hvdg import autograd as AG
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    fs = [synth.make_field(50 + i, _cabi.STD_NTSC, 0.5) for i in range(2)]
    cfg = _cfg(irls_outer=2, cg_iterations=60)
    samples = torch.tensor(np.stack([f.samples.astype(np.float32) for f in fs]), requires_grad=True)
    lc = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    eps = torch.tensor(float(cfg.charbonnier_eps), dtype=torch.float64, requires_grad=True)
    epc = torch.tensor(float(cfg.chroma_eps), dtype=torch.float64, requires_grad=True)
    k = torch.tensor(float(cfg.structure_coupling), dtype=torch.float64, requires_grad=True)
    y, chi = AG.decode(ctx, samples, g, lc, eps, epc, k, cfg=cfg, parity=[0, 1],
                       sample_type=_cabi.SAMPLES_U16)
    yt = torch.tensor(np.stack([f.y_true for f in fs]), dtype=torch.float32)
    ct = torch.tensor(np.stack([np.stack([f.chi_true.real, f.chi_true.imag], -1) for f in fs]),
                      dtype=torch.float32)
    loss = ((y - yt) ** 2).mean() + 2.0 * ((chi - ct) ** 2).mean()
    loss.backward()
    # the same gradient through the C ABI directly
    flds = [api.Field(f.samples, g, parity=i) for i, f in enumerate(fs)]
    n = yt[0].numel()
    yb = [(2 * (y[i] - yt[i]) / (2 * n)).detach().numpy() for i in range(2)]
    cb = [(2 * (chi[i] - ct[i]) / (2 * n)).detach().numpy().view(np.complex64)[..., 0] for i in range(2)]
    sbar, sc, _ = ctx.decode_fields_adjoint(flds, cfg, yb, cb)
    assert np.allclose(samples.grad.numpy(), np.stack(sbar), rtol=1e-5, atol=1e-12)
    assert abs(lc.grad.item() - sc["lambda_c"]) <= 1e-6 * abs(sc["lambda_c"]) + 1e-12
    assert abs(k.grad.item() - sc["structure_coupling"]) <= 1e-6 * abs(sc["structure_coupling"]) + 1e-12


def test_adjoint_config4_batch_vs_fp64_oracle(ctx):
    """Config 4 as configured: 8 NTSC fields in one batched adjoint call at
    10 IRLS x 50 CG. Each field's sample gradient against the FP64 adjoint
    oracle (1e-3 relative), and the batch's scalar gradients against the sum
    of the oracle's per-field ones (1e-3 relative). The oracle runs field-
    parallel in a spawn pool."""
    from oracle import jobs
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    fs = [synth.make_field(200 + i, _cabi.STD_NTSC, 0.5) for i in range(8)]
    cfg = _cfg()
    flds = [api.Field(f.samples, g, parity=i % 2) for i, f in enumerate(fs)]
    decs = ctx.decode_fields(flds, cfg)
    cots = [_loss_and_cot(d, f)[1:] for d, f in zip(decs, fs)]
    sbar, sc, _ = ctx.decode_fields_adjoint(flds, cfg, [c[0] for c in cots], [c[1] for c in cots],
                                            300)
    kw = dict(irls_outer=10, cg_iterations=500, fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    orc = jobs.adjoint_fields_parallel([(f.samples, _cabi.STD_NTSC, i % 2, kw, c[0], c[1])
                                        for i, (f, c) in enumerate(zip(fs, cots))])
    fal, lal = g.first_active_field_line, g.last_active_line
    a0, a1 = g.active_video_start, g.active_video_end
    for i, (s_bar, _) in enumerate(orc):
        got = sbar[i][fal:lal, a0:a1].astype(np.float64)
        rel = np.linalg.norm(got - s_bar / CPI) / np.linalg.norm(s_bar / CPI)
        print(f"field {i}: sample gradient rel L2 {rel:.2e}")
        assert rel < 1e-3
    for k_gpu, k_orc in (("lambda_c", "lambda_c"), ("charbonnier_eps", "eps"),
                         ("chroma_eps", "eps_c"), ("structure_coupling", "k")):
        want = sum(gl[k_orc] for _, gl in orc)
        print(k_gpu, sc[k_gpu], want)
        assert abs(sc[k_gpu] - want) <= 1e-3 * abs(want) + 1e-9
