"""Edge cases of the 2-D decode at the boundary, against the FP64 oracle:
ragged geometries (odd active width and start, a line count that no solver
band divides), a tiny plane (8 x 16), the largest planes of the init's
register transforms (active width 1024: row convolution 2047 <= 2048; 480
active lines: padded 512, column convolution 1023 <= 1024) and one past
each, which the shared-memory transforms take (test_gpu_long_planes.py
covers those and the refusals past them), non-finite samples
(HVDG_ERR_NONFINITE_INPUT, the
context stays usable), the empty batch, and caller output planes that
start off any vector boundary."""
import ctypes as C

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


def test_largest_register_planes_and_one_past(ctx):
    wide = _cabi.default_geometry(_cabi.STD_PAL)
    wide.active_video_start, wide.active_video_end = 100, 1124      # width 1024
    _vs_oracle(ctx, wide, _cabi.STD_PAL, 73)
    tall = _cabi.default_geometry(_cabi.STD_NTSC)
    tall.field_height = 500
    tall.first_active_field_line, tall.last_active_field_line = 10, 490   # 480 lines
    tall.active_video_start, tall.active_video_end = 134, 390
    _vs_oracle(ctx, tall, _cabi.STD_NTSC, 74)
    # one past each: row length 4096, column length 2048
    _vs_oracle(ctx, _cabi.geometry_copy(wide, active_video_end=1125), _cabi.STD_PAL, 75)
    _vs_oracle(ctx, _cabi.geometry_copy(tall, last_active_field_line=491), _cabi.STD_NTSC, 75)


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


def test_unaligned_caller_output_buffers(ctx):
    """Output planes at any float offset: page-locked host planes (written by
    the solver through their mapped addresses) and device planes, starting
    4 bytes past a 16-byte boundary, decode exactly like aligned ones."""
    import torch
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    f = synth.make_field(77, _cabi.STD_NTSC, 0.5)
    cfg = _cfg()
    want = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg)[0]
    h, w = g.active_lines, g.active_width
    ybuf = torch.zeros(h * w + 4, dtype=torch.float32, pin_memory=True)
    cbuf = torch.zeros(2 * h * w + 4, dtype=torch.float32, pin_memory=True)
    y = ybuf.numpy()[1:1 + h * w].reshape(h, w)
    c = cbuf.numpy()[1:1 + 2 * h * w].view(np.complex64).reshape(h, w)
    assert y.ctypes.data % 16 == 4 and c.ctypes.data % 16 == 4
    got = ctx.decode_fields([api.Field(f.samples, g, parity=0)], cfg, out=[api.Decoded(y, c)])[0]
    assert np.array_equal(got.luma, want.luma) and np.array_equal(got.chroma, want.chroma)
    # device-resident buffers at the same offsets
    d_in = torch.from_numpy(f.samples.view(np.int16)).cuda()
    d_y = torch.zeros(h * w + 4, dtype=torch.float32, device="cuda")
    d_c = torch.zeros(2 * h * w + 4, dtype=torch.float32, device="cuda")
    fin = (_cabi.FieldIn * 1)()
    fout = (_cabi.FieldOut * 1)()
    fin[0].samples = d_in.data_ptr()
    fin[0].sample_type = _cabi.SAMPLES_U16
    fin[0].parity = 0
    fin[0].blanking_level = 16384.0
    fin[0].white_level = 51200.0
    fin[0].geometry = C.pointer(g)
    fin[0].irls_outer = 0
    fin[0].cg_iterations = -1
    fout[0].luma = d_y.data_ptr() + 4
    fout[0].chroma = d_c.data_ptr() + 4
    ctx.decode_fields_device(fin, fout, 1, cfg)
    torch.cuda.synchronize()
    gy = d_y.cpu().numpy()[1:1 + h * w].reshape(h, w)
    gc = d_c.cpu().numpy()[1:1 + 2 * h * w].view(np.complex64).reshape(h, w)
    assert np.array_equal(gy, want.luma) and np.array_equal(gc, want.chroma)
