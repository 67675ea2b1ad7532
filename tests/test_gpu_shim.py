"""The drop-in shim (hvd-cvbs-decoding_b200/shim/frame_bridge_b200.cpp):
hvd::DecodeFrameSequenceWindow, DecodeFrameBuffer and DecodeYcFrameBuffer
with the reference's own C++ signatures and types (built against the
reference's headers, oracle/Makefile), served by the B200 library. Through
the shim the results equal the library's direct C ABI bit for bit, and the
reference's within the frame-bridge tolerances; invalid windows come back
empty, as the reference returns them."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth

pytestmark = pytest.mark.gpu


def _shim():
    from oracle import shim
    if not shim.available():
        pytest.skip("shim not built (needs the reference's headers)")
    return shim


def _same(a, b, tag):
    for key in ("luma", "chroma", "u", "v"):
        assert np.array_equal(a[key], b[key]), (tag, key)


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
def test_shim_sequence_window_equals_library(ctx, std):
    shim = _shim()
    frames, _ = synth.make_frames(51 + std, std, 3, noise_sigma=1.0)
    fp = api.frame_params(std)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6,
                             temporal_strength=-1.0)
    direct = ctx.decode_frame_sequence_window(frames, 1, 3, fp, cfg)
    via = shim.decode_frame_sequence_window(frames, 1, 3, fp, cfg)
    assert len(via) == len(direct) == 2
    from oracle import ref
    if ref.available():
        want = ref.decode_frame_sequence_window(frames, 1, 3, fp, cfg)
        for g, r in zip(via, want):
            d = np.abs(g["luma"].astype(np.int32) - r["luma"].astype(np.int32))
            assert d.max() <= 1 and (d > 0).mean() < 5e-3
    # same library, same configuration, same (automatic) solver tiling
    for t, (g, r) in enumerate(zip(via, direct)):
        _same(g, r, t)


def test_shim_frame_buffers_equal_library(ctx):
    shim = _shim()
    frames, _ = synth.make_frames(53, _cabi.STD_NTSC, 1, noise_sigma=1.0)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6)
    via = shim.decode_frame_buffer(frames[0], fp, cfg)
    direct = ctx.decode_frame_buffer(frames[0], fp, cfg)
    assert via is not None
    _same(via, direct, "composite")
    ys, cs, _ = synth.make_yc_frames(54, _cabi.STD_PAL, 1, noise_sigma=0.7)
    fpp = api.frame_params(_cabi.STD_PAL)
    fpp.chroma_dc = 512.0
    via = shim.decode_yc_frame_buffer(ys[0], cs[0], fpp, cfg)
    direct = ctx.decode_yc_frame_buffer(ys[0], cs[0], fpp, cfg)
    _same(via, direct, "yc")      # init only: no solver tiling involved


def test_shim_empty_window(ctx):
    shim = _shim()
    frames, _ = synth.make_frames(3, _cabi.STD_NTSC, 1)
    fp = api.frame_params(_cabi.STD_NTSC)
    assert shim.decode_frame_sequence_window(frames, 1, 1, fp, api.default_config()) == []


def test_shim_worker_threads_leave_no_device_memory(ctx):
    """Each export worker of the stage builds its own HvdEngine on its own
    thread (hvd_chroma_decoder_stage.cpp:991, 1115, 1166). The shim keeps
    one library context per thread and destroys it when the thread exits,
    so a stream of short-lived workers leaves the device's free memory where
    it was (before: one context with its arena per engine, never freed)."""
    torch = pytest.importorskip("torch")
    shim = _shim()
    frames, _ = synth.make_frames(57, _cabi.STD_NTSC, 1, noise_sigma=1.0)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = api.default_config(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6)
    assert shim.decode_frame_buffer_workers(frames[0], fp, cfg, 2) == 2   # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert shim.decode_frame_buffer_workers(frames[0], fp, cfg, 24) == 24
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    print(f"device free memory: {free0 / 2**20:.0f} MiB before, {free1 / 2**20:.0f} MiB after "
          f"24 worker threads")
    assert free1 >= free0 - (64 << 20)
