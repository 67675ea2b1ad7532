"""Edge cases of the 2-D decode at the boundary, against the FP64 oracle:
ragged geometries (odd active width and start, a line count that no solver
band divides), a tiny plane (8 x 16), the largest planes the device path
takes (active width 1024: row convolution 2047 <= 2048; 480 active lines:
padded 512, column convolution 1023 <= 1024) and one past each limit
(HVDG_ERR_UNSUPPORTED), non-finite samples (HVDG_ERR_NONFINITE_INPUT, the
context stays usable) and the empty batch."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


def _cfg():
    return api.default_config(irls_outer=3, cg_iterations=60, fast=0, cg_tol=1e-6,
                              temporal_strength=-1.0)


def _vs_oracle(ctx, g, std, seed, tol=0.05):
    f = synth.make_field(seed, std, noise_sigma=0.5, geometry=g)
    cfg = _cfg()
    out = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg)[0]
    (yo, co, _), = O.decode_fields_2d([synth.to_ire(f.samples)], [0], g, cfg)
    dy, dc = np.abs(out.luma - yo).max(), np.abs(out.chroma - co).max()
    print(f"h={g.active_lines} w={g.active_width}: max dY {dy:.3g} max dC {dc:.3g}")
    assert out.luma.shape == (g.active_lines, g.active_width)
    assert dy < tol and dc < tol
    return out


def test_ragged_geometry(ctx):
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    g.active_video_start, g.active_video_end = 135, 894      # odd start, width 759
    g.first_active_field_line, g.last_active_field_line = 23, 202   # 179 lines
    _vs_oracle(ctx, g, _cabi.STD_NTSC, 71)


def test_tiny_plane(ctx):
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    g.field_height = 40
    g.active_video_start, g.active_video_end = 134, 150      # 16 samples
    g.first_active_field_line, g.last_active_field_line = 20, 28    # 8 lines
    _vs_oracle(ctx, g, _cabi.STD_NTSC, 72)


def test_largest_planes_and_one_past(ctx):
    wide = _cabi.default_geometry(_cabi.STD_PAL)
    wide.active_video_start, wide.active_video_end = 100, 1124      # width 1024
    _vs_oracle(ctx, wide, _cabi.STD_PAL, 73)
    tall = _cabi.default_geometry(_cabi.STD_NTSC)
    tall.field_height = 500
    tall.first_active_field_line, tall.last_active_field_line = 10, 490   # 480 lines
    tall.active_video_start, tall.active_video_end = 134, 390
    _vs_oracle(ctx, tall, _cabi.STD_NTSC, 74)
    for g, edit in ((wide, dict(active_video_end=1125)), (tall, dict(last_active_field_line=491))):
        bad = _cabi.geometry_copy(g, **edit)
        f = synth.make_field(75, g.standard, 0.5, geometry=g)
        with pytest.raises(api.HvdgError) as e:
            ctx.decode_fields([api.Field(f.samples, bad, parity=0)], _cfg())
        assert e.value.status == _cabi.ERR_UNSUPPORTED


def test_nonfinite_input_and_empty_batch(ctx):
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    f = synth.make_field(76, _cabi.STD_NTSC, 0.5)
    ire = synth.to_ire(f.samples).astype(np.float32)
    ire[100, 400] = np.nan
    with pytest.raises(api.HvdgError) as e:
        ctx.decode_fields([api.Field(ire, g, parity=0)], _cfg())
    assert e.value.status == _cabi.ERR_NONFINITE_INPUT
    assert ctx.decode_fields([], _cfg()) == []
    _vs_oracle(ctx, g, _cabi.STD_NTSC, 76)     # the context still decodes
