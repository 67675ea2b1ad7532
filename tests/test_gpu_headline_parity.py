"""Parity at the benchmark's own settings: the batched mixed NTSC / PAL
decode (hvdg_decode_fields over fields of both geometries in one call, the
per-field work queue, per-field completion flags and uneven IRLS budgets of
4-12 outers x 50 CG, sigma 0.2-2 IRE) against the FP64 oracle field by
field; the plain one-field-per-launch path against the batched one; the CG
tolerance exits (variational.cpp:530, 547-548) against the oracle's; and
the 3-D window at config 1's solver budget (10 IRLS x 500 CG, slow sweep)
against the compiled reference.

Tolerances: PSNR against ground truth within 0.05 dB of the oracle's,
max |dY|, |dC| < 0.05 IRE; plain = batched to 1e-5 IRE."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import jobs

pytestmark = pytest.mark.gpu


def psnr(a, b, peak=100.0):
    d = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
    return 10 * np.log10(peak ** 2 / np.mean(np.abs(d) ** 2))


FIXED = dict(fast=0, cg_tol=1e-6, temporal_strength=-1.0)


def _mixed_fields(seed=2024, n_ntsc=5, n_pal=3):
    fs = synth.mixed_batch(seed, n_ntsc, n_pal, outer_range=(4, 12), cg_per_outer=50)
    geoms = [_cabi.default_geometry(f.standard) for f in fs]
    hf = [api.Field(f.samples, g, parity=f.parity, irls_outer=f.irls_outer,
                    cg_iterations=f.cg_iterations) for f, g in zip(fs, geoms)]
    return fs, hf


@pytest.fixture(scope="module")
def mixed():
    """Oracle decodes of the mixed batch, computed once in a spawn pool."""
    fs, hf = _mixed_fields()
    job_list = [(f.samples, f.standard, f.parity,
                 dict(FIXED, irls_outer=f.irls_outer, cg_iterations=f.cg_iterations))
                for f in fs]
    return fs, hf, jobs.decode_fields_2d_parallel(job_list)


def test_mixed_batch_matches_oracle(ctx, mixed):
    fs, hf, orc = mixed
    assert len({f.standard for f in fs}) == 2
    assert len({f.irls_outer for f in fs}) > 2
    cfg = api.default_config(**FIXED)
    ctx.set_batching(True)
    out = ctx.decode_fields(hf, cfg)
    worst = dict(dY=0.0, dC=0.0, dpY=0.0, dpC=0.0)
    for i, (f, d, (yo, co, st)) in enumerate(zip(fs, out, orc)):
        dY = float(np.abs(d.luma - yo).max())
        dC = float(np.abs(d.chroma - co).max())
        dpY = abs(psnr(d.luma, f.y_true) - psnr(yo, f.y_true))
        dpC = abs(psnr(d.chroma, f.chi_true) - psnr(co, f.chi_true))
        print(f"field {i} std={f.standard} sigma={f.noise_sigma:.2f} outer={f.irls_outer}: "
              f"max dY {dY:.3g} max dC {dC:.3g} IRE, dPSNR Y {dpY:.4f} C {dpC:.4f} dB, "
              f"oracle iters {st['cg_iterations']}")
        for k, v in (("dY", dY), ("dC", dC), ("dpY", dpY), ("dpC", dpC)):
            worst[k] = max(worst[k], v)
    print("worst:", worst)
    assert worst["dY"] < 0.05 and worst["dC"] < 0.05
    assert worst["dpY"] < 0.05 and worst["dpC"] < 0.05
    # cg_tol 1e-6 leaves the absolute floor ||g||^2 < 1e-10 N (variational.cpp:548)
    # to end the later outers early, in the oracle as on the device: the
    # batch ran the oracle's iterations, field for field summed
    orc_iters = sum(st["cg_iterations"] for _, _, st in orc)
    near = sum(1 for _, _, st in orc for _, m in st["outer_log"] if m < 1e-3)
    print(f"CG iterations: device {ctx.last_diag.cg_iterations_run} oracle {orc_iters} "
          f"(budgets {sum(f.cg_iterations for f in fs)})")
    assert abs(ctx.last_diag.cg_iterations_run - orc_iters) <= near


def test_plain_path_equals_batched(ctx, mixed):
    """The metric's denominator, hvdg_set_batching(ctx, 0): one field per
    launch sequence. Same kernels with a per-field tiling, so the results
    equal the batched decode up to the reduction order of the partials."""
    fs, hf, orc = mixed
    cfg = api.default_config(**FIXED)
    ctx.set_batching(True)
    batched = ctx.decode_fields(hf, cfg)
    runs_batched = ctx.last_diag.cg_iterations_run
    ctx.set_batching(False)
    try:
        plain = ctx.decode_fields(hf, cfg)
        runs = ctx.last_diag.cg_iterations_run
    finally:
        ctx.set_batching(True)
    assert runs == runs_batched
    for i, (a, b, (yo, co, _)) in enumerate(zip(plain, batched, orc)):
        dy = float(np.abs(a.luma - b.luma).max())
        dc = float(np.abs(a.chroma - b.chroma).max())
        print(f"field {i}: plain vs batched max dY {dy:.3g} dC {dc:.3g}")
        assert dy <= 1e-5 and dc <= 1e-5, (i, dy, dc)
        assert np.abs(a.luma - yo).max() < 0.05 and np.abs(a.chroma - co).max() < 0.05


@pytest.mark.parametrize("fast", [1, 0])
def test_cg_tolerance_exits_match_oracle(ctx, fast):
    """Early CG exits at the reference's automatic tolerance (cg_tol 0 ->
    0.10 fast / 0.02 slow, variational.cpp:224-230) and its absolute floor
    (1e-10 N): every field's executed CG iteration count equals the FP64
    oracle's, except that an outer whose tested ||g||^2 came within 1e-3
    (relative) of its threshold may end one iteration either side."""
    fs = synth.mixed_batch(515 + fast, 3, 2, outer_range=(3, 6), cg_per_outer=40)
    job_list = [(f.samples, f.standard, f.parity,
                 dict(fast=fast, cg_tol=0.0, temporal_strength=-1.0, irls_outer=f.irls_outer,
                      cg_iterations=f.cg_iterations)) for f in fs]
    orc = jobs.decode_fields_2d_parallel(job_list)
    cfg = api.default_config(fast=fast, cg_tol=0.0, temporal_strength=-1.0)
    n_exact = 0
    for i, (f, (yo, co, st)) in enumerate(zip(fs, orc)):
        g = _cabi.default_geometry(f.standard)
        d = ctx.decode_fields([api.Field(f.samples, g, parity=f.parity, irls_outer=f.irls_outer,
                                         cg_iterations=f.cg_iterations)], cfg)[0]
        dev_iters = ctx.last_diag.cg_iterations_run
        near = sum(1 for _, m in st["outer_log"] if m < 1e-3)
        budget = f.cg_iterations * 2 // 3 if fast else f.cg_iterations
        print(f"field {i} std={f.standard} fast={fast}: device {dev_iters} oracle "
              f"{st['cg_iterations']} of {budget} (per outer {[n for n, _ in st['outer_log']]}, "
              f"near-threshold outers {near})")
        assert st["cg_iterations"] < budget        # the tolerance exits were taken
        assert abs(dev_iters - st["cg_iterations"]) <= near
        n_exact += dev_iters == st["cg_iterations"]
        assert np.abs(d.luma - yo).max() < 0.05 and np.abs(d.chroma - co).max() < 0.05
        assert abs(psnr(d.luma, f.y_true) - psnr(yo, f.y_true)) < 0.05
    assert n_exact >= len(fs) - 1


def test_window_config1_budget_vs_reference(ctx):
    """Config 1's solver settings on a 6-field NTSC window of moving
    content: temporal strength 0.5, one pass, no anchor / coherence gate /
    trajectory fit, 10 IRLS x 500 CG (n_inner 50), slow (sequential) sweep,
    the reference's float-SSD motion search; per-field PSNR against ground
    truth within 0.05 dB of the compiled reference's."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    std, nf = _cabi.STD_NTSC, 6
    seq = synth.make_sequence(101, std, nf, noise_sigma=0.5, moving=True)
    g = _cabi.default_geometry(std)
    cfg = api.default_config(irls_outer=10, cg_iterations=500, fast=0, cg_tol=1e-6,
                             temporal_strength=0.5, passes=1, nr_anchor=0.0, coherence_gate=0.0,
                             trajectory_fit=0)
    outs = ctx.decode_field_window([api.Field(f.samples, g, parity=f.parity) for f in seq], cfg)
    assert ctx.last_diag.cg_iterations_run > 0
    ys, cs, _ = ref.decode_field_window([synth.to_ire(f.samples) for f in seq],
                                        [f.parity for f in seq], g, cfg)
    for j in range(nf):
        pg, pr = psnr(outs[j].luma, seq[j].y_true), psnr(ys[j], seq[j].y_true)
        cg, cr = psnr(outs[j].chroma, seq[j].chi_true), psnr(cs[j], seq[j].chi_true)
        print(f"cfg1 field {j}: Y gpu {pg:.3f} ref {pr:.3f}  C gpu {cg:.3f} ref {cr:.3f}  "
              f"max dY {np.abs(outs[j].luma - ys[j]).max():.3g}")
        assert abs(pg - pr) < 0.05
        assert abs(cg - cr) < 0.05
