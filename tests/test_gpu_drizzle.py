"""DrizzleFrame (sequence.cpp:283-421) on the device (hvdg_drizzle_frame):
float motion estimation bit-exact with the reference's, per-pixel vectors,
robust-weighted deposits onto the fine grid (float atomics) and the coverage
blend, against the compiled reference and the FP64 oracle on the
reference's own 2-D decodes of moving windows. The deposit positions follow
the reference's float arithmetic exactly, so only the accumulation order
differs: sums agree to rounding."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("std,scale", [(_cabi.STD_NTSC, 2), (_cabi.STD_PAL, 3)])
def test_drizzle_vs_reference(ctx, std, scale):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    g = _cabi.default_geometry(std)
    fs = synth.make_sequence(5 + std, std, 8, noise_sigma=0.5, moving=True)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6,
                             temporal_strength=-1.0)
    par = [f.parity for f in fs]
    ys, cs, _ = ref.decode_field_window([synth.to_ire(f.samples) for f in fs], par, g, cfg)
    for j0 in (0, 4):
        gy, gc = ctx.drizzle_frame(j0, ys, cs, par, cfg, scale)
        ry, rc = ref.drizzle_frame(j0, ys, cs, par, cfg, scale)
        d, dc = np.abs(gy - ry), np.abs(gc - rc)
        print(f"std={std} j0={j0} scale={scale}: max dY {d.max():.3g} mean {d.mean():.3g} "
              f"max dC {dc.max():.3g}")
        assert d.max() < 1e-3 and dc.max() < 1e-3
    oy, oc = O.drizzle_frame(4, ys, cs, par, cfg, scale)
    d = np.abs(gy - oy)
    assert d.mean() < 1e-4 and (d > 1e-3).mean() < 1e-3


def test_drizzle_rejects_bad_arguments(ctx):
    ys = [np.zeros((10, 12), np.float32)] * 2
    cs = [np.zeros((10, 12), np.complex64)] * 2
    with pytest.raises(api.HvdgError) as e:
        ctx.drizzle_frame(1, ys, cs, [0, 1], api.default_config(), 2)   # j0 + 1 out of range
    assert e.value.status == _cabi.ERR_BAD_ARGUMENT
