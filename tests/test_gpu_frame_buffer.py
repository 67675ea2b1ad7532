"""Woven-frame entry points against the reference on the same int16 frames:

- hvdg_decode_frame_buffer ~ hvd::DecodeFrameBuffer (frame_bridge.cpp:161-255,
  engine DecodeFrame engine.cpp:141-195): split, field-order vote, per-field
  lock-in, weave, holographic init (column length 2048: woven NTSC pads to
  516 rows, PAL to 614) + IRLS / CG on the woven frame, lossless chroma
  S - Y, ACC, re-weave, 10-bit requantisation;
- hvdg_decode_yc_frame_buffer ~ hvd::DecodeYcFrameBuffer
  (frame_bridge.cpp:263-377, engine DecodeChromaOnly engine.cpp:197-237):
  C channel de-woven around chroma_dc, init only, chroma = Re[chi c], luma
  passed through.

Codes are compared exactly up to rare +-1 rounding flips (the float chi of
the two implementations differs in its last bits: FFT-convolution init,
reduction order of the FP32 solver, FP64 carrier phases here), u / v within
0.05 codes on NTSC. PAL's per-line phases grow to ~1500 rad, where the
reference's float carrier phase (MakeCarrierPal, ntsc_geometry.cpp:438-456)
carries ~1e-4 rad of rounding: ~0.02 codes of chroma per sample. The
reference itself moves by 0.10 codes of u / v on the PAL frame of
test_frame_buffer_vs_reference when only its carrier phase is evaluated in
double instead of float, so PAL is held to 0.15 codes of u / v and 0.5 % of
+-1 code flips.
Pass-through luma and everything outside the active picture must be
identical."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    return ref


def _compare(got, want, tag, pal=False, uv_tol=None):
    flip_frac, uv_default = (5e-3, 0.15) if pal else (2e-3, 0.05)
    uv_tol = uv_default if uv_tol is None else uv_tol
    for key in ("luma", "chroma"):
        d = np.abs(got[key].astype(np.int32) - want[key].astype(np.int32))
        print(f"{tag} {key}: max {d.max()} frac>0 {(d > 0).mean():.2e}")
        assert d.max() <= 1, (tag, key)
        assert (d > 0).mean() < flip_frac, (tag, key)
    for key in ("u", "v"):
        du = np.abs(got[key] - want[key])
        print(f"{tag} {key}: max {du.max():.3e}")
        assert du.max() < uv_tol, (tag, key)
        # zero exactly where the reference is zero (outside the active picture)
        assert np.all(got[key][want[key] == 0.0] == 0.0), (tag, key)


def _cfg(**kw):
    base = dict(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6)
    base.update(kw)
    return api.default_config(**base)


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
@pytest.mark.parametrize("field_order", [0, 2])
def test_frame_buffer_vs_reference(ctx, std, field_order):
    ref = _ref()
    frames, _ = synth.make_frames(61 + std, std, 1, noise_sigma=1.0)
    fp = api.frame_params(std)
    cfg = _cfg(field_order=field_order)
    got = ctx.decode_frame_buffer(frames[0], fp, cfg)
    want = ref.decode_frame_buffer(frames[0], fp, cfg)
    _compare(got, want, f"composite std={std} order={field_order}", pal=std == _cabi.STD_PAL)


@pytest.mark.parametrize("opts", [dict(monochrome=1), dict(acc=0, chroma_gain=1.3),
                                  dict(cg_iterations=0), dict(chroma_phase_deg=20.0),
                                  dict(field_order=1, chroma_aniso=0.7),
                                  dict(symmetry_variant=1)])
def test_frame_buffer_options_vs_reference(ctx, opts):
    ref = _ref()
    std = _cabi.STD_PAL if "chroma_phase_deg" in opts else _cabi.STD_NTSC
    frames, _ = synth.make_frames(71, std, 1, noise_sigma=1.0)
    fp = api.frame_params(std)
    cfg = _cfg(**opts)
    got = ctx.decode_frame_buffer(frames[0], fp, cfg)
    want = ref.decode_frame_buffer(frames[0], fp, cfg)
    _compare(got, want, f"composite {opts}", pal=std == _cabi.STD_PAL)


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
@pytest.mark.parametrize("field_order", [0, 2])
def test_yc_frame_buffer_vs_reference(ctx, std, field_order):
    ref = _ref()
    ys, cs, _ = synth.make_yc_frames(81 + std, std, 1, noise_sigma=0.7)
    fp = api.frame_params(std)
    fp.chroma_dc = 512.0
    cfg = _cfg(field_order=field_order)
    got = ctx.decode_yc_frame_buffer(ys[0], cs[0], fp, cfg)
    want = ref.decode_yc_frame_buffer(ys[0], cs[0], fp, cfg)
    _compare(got, want, f"yc std={std} order={field_order}", pal=std == _cabi.STD_PAL)
    # luma passes straight through, line by line through FrameLineOffset
    assert np.array_equal(got["luma"], want["luma"])


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
def test_field1_bottom_vote_vs_reference(ctx, std):
    """Frames whose field 1 is the bottom field: the automatic order (the
    device vote) must weave them as the reference's DetectFieldParity does.
    The reference's auto decode equals its forced-bottom decode (its vote
    said bottom), the device's auto decode equals the device's forced-bottom
    decode bit for bit, and the two implementations agree as usual -- on PAL
    u / v within twice the reference's own movement on this frame when its
    carrier phase is evaluated in double (0.09 codes here)."""
    ref = _ref()
    frames, _ = synth.make_frames(63 + std, std, 1, noise_sigma=1.0, field1_bottom=True)
    fp = api.frame_params(std)
    uv_tol = None
    if std == _cabi.STD_PAL:
        from test_frame_buffer_pins import pal_carrier_sensitivity
        uv_tol = 2.0 * pal_carrier_sensitivity(ref, frames[0], _cfg(), field1_bottom=True)
    want = ref.decode_frame_buffer(frames[0], fp, _cfg(field_order=0))
    want_b = ref.decode_frame_buffer(frames[0], fp, _cfg(field_order=2))
    for key in ("luma", "chroma", "u", "v"):
        assert np.array_equal(want[key], want_b[key]), key
    got = ctx.decode_frame_buffer(frames[0], fp, _cfg(field_order=0))
    got_b = ctx.decode_frame_buffer(frames[0], fp, _cfg(field_order=2))
    for key in ("luma", "chroma", "u", "v"):
        assert np.array_equal(got[key], got_b[key]), key
    _compare(got, want, f"bottom-first std={std}", pal=std == _cabi.STD_PAL, uv_tol=uv_tol)


def _ramp_frame(fp, slope, offset):
    """Block 1 lines at 100 + slope y codes (levels 100 / 900: 8 codes per
    IRE, so every term of the vote is exact), block 2 at the same ramp plus
    `offset` codes. Offsets 99 put the vote's two means exactly 2 % apart
    (the threshold: decided), 101 just inside it (undecided)."""
    f1, fh, fw = fp.field1_lines, fp.frame_height, fp.frame_width
    y = np.concatenate([np.arange(f1), np.arange(fh - f1)])
    base = (100 + (slope * y if slope > 0 else 800 + slope * y)).astype(np.int32)
    base[f1:] += offset
    return np.repeat(base[:, None], fw, axis=1).astype(np.int16).ravel()


def test_detect_field_parity_vs_reference(ctx):
    """The device vote equals the reference's DetectFieldParity on every
    frame: synthetic top- and bottom-first frames, a flat frame (0), and
    ramps whose means sit exactly on the 2 % threshold (the case the
    parallel sum hands to the in-order FP64 re-sum) or just inside it."""
    ref = _ref()
    for std in (_cabi.STD_NTSC, _cabi.STD_PAL):
        fp = api.frame_params(std)
        frames = []
        for fb in (False, True):
            fr, _ = synth.make_frames(81 + std, std, 2, noise_sigma=1.0, moving=True,
                                      field1_bottom=fb)
            frames += fr
        size = api.frame_buffer_size(fp)
        frames.append(np.full(size, int(fp.blanking_level), np.int16))
        votes = ctx.detect_field_parity(frames, fp)
        want = [ref.detect_field_parity(*ref.split_frame_fields(f, fp), fp) for f in frames]
        assert list(votes) == want, (std, list(votes), want)
        assert want[:4] == [1, 1, -1, -1] and want[4] == 0
    fp = api.frame_params(_cabi.STD_NTSC)
    fp.blanking_level, fp.white_level = 100.0, 900.0
    ramps = [_ramp_frame(fp, 2, 99), _ramp_frame(fp, -2, 99), _ramp_frame(fp, 2, 101)]
    votes = ctx.detect_field_parity(ramps, fp)
    want = [ref.detect_field_parity(*ref.split_frame_fields(f, fp), fp) for f in ramps]
    assert list(votes) == want == [1, -1, 0]


def test_mixed_field_orders_in_one_batch(ctx):
    """A batch whose frames vote differently: each frame is woven by its own
    vote, bit for bit as its single-frame call (band height pinned)."""
    order = [False, True, True, False]
    frames, _ = synth.make_frames(93, _cabi.STD_NTSC, 4, noise_sigma=1.0, moving=True,
                                  field1_bottom=order)
    fp = api.frame_params(_cabi.STD_NTSC)
    ctx.set_tuning(16, 0)
    try:
        batch = ctx.decode_frame_buffers(frames, fp, _cfg(field_order=0))
        for t, f in enumerate(frames):
            forced = ctx.decode_frame_buffer(f, fp, _cfg(field_order=2 if order[t] else 1))
            for key in ("luma", "chroma", "u", "v"):
                assert np.array_equal(batch[t][key], forced[key]), (t, key)
    finally:
        ctx.set_tuning(0, 0)


def test_batched_frames_equal_single_calls(ctx):
    """With the solver band height pinned (the automatic one depends on the
    batch size), a batch of frames decodes bit-for-bit like one-frame calls:
    every reduction is per unit in a fixed order."""
    frames, _ = synth.make_frames(91, _cabi.STD_NTSC, 3, noise_sigma=1.0, moving=True)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = _cfg()
    ctx.set_tuning(16, 0)
    try:
        _batched_vs_single(ctx, frames, fp, cfg)
    finally:
        ctx.set_tuning(0, 0)


def _batched_vs_single(ctx, frames, fp, cfg):
    batch = ctx.decode_frame_buffers(frames, fp, cfg)
    assert ctx.last_diag.kernel_launches > 0
    for t, f in enumerate(frames):
        one = ctx.decode_frame_buffer(f, fp, cfg)
        for key in ("luma", "chroma", "u", "v"):
            assert np.array_equal(batch[t][key], one[key]), (t, key)
    ys, cs, _ = synth.make_yc_frames(92, _cabi.STD_PAL, 2, noise_sigma=0.7)
    fpp = api.frame_params(_cabi.STD_PAL)
    fpp.chroma_dc = 512.0
    yb = ctx.decode_yc_frame_buffers(ys, cs, fpp, cfg)
    for t in range(2):
        one = ctx.decode_yc_frame_buffer(ys[t], cs[t], fpp, cfg)
        for key in ("luma", "chroma", "u", "v"):
            assert np.array_equal(yb[t][key], one[key]), (t, key)


def test_frame_buffer_lossless_split(ctx):
    """luma + chroma reconstructs the composite to one code inside the
    active picture (the YcFrameS16 contract, frame_bridge.h:114-122)."""
    frames, _ = synth.make_frames(95, _cabi.STD_NTSC, 1, noise_sigma=0.5)
    fp = api.frame_params(_cabi.STD_NTSC)
    got = ctx.decode_frame_buffer(frames[0], fp, _cfg())
    src = frames[0].astype(np.int32)
    rec = got["luma"].astype(np.int32) + got["chroma"].astype(np.int32)
    active = got["u"] != 0.0
    assert np.abs(rec - src)[active].max() <= 1
    assert np.array_equal(got["luma"][~active], frames[0][~active])


def test_frame_buffer_error_statuses(ctx):
    """Statuses at the boundary, as the reference's empty-result convention
    maps onto them: bad frame parameters -> BAD_GEOMETRY, a woven plane
    beyond the device-path limits -> UNSUPPORTED (a PAL frame 1100 samples
    wide is within them, on the long-row transforms, and matches the
    reference), n = 0 -> OK, nothing decoded; the context stays usable."""
    frames, _ = synth.make_frames(97, _cabi.STD_NTSC, 1, noise_sigma=0.5)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = _cfg()
    bad = api.frame_params(_cabi.STD_NTSC)
    bad.white_level = bad.blanking_level          # zero codes per IRE
    with pytest.raises(api.HvdgError) as e:
        ctx.decode_frame_buffer(frames[0], bad, cfg)
    assert e.value.status == _cabi.ERR_BAD_GEOMETRY
    tall = api.frame_params(_cabi.STD_NTSC)
    tall.active_video_start, tall.active_video_end = 0, 910   # 2 w - 1 > 2048 is fine; w = 910
    tall.first_active_frame_line = 0                           # 263 lines -> 526-row woven plane
    out = ctx.decode_frame_buffer(frames[0], tall, cfg)        # still within the limits
    assert out["luma"].shape == frames[0].shape
    pal_frames, _ = synth.make_frames(98, _cabi.STD_PAL, 1, noise_sigma=0.5)
    wide = api.frame_params(_cabi.STD_PAL)
    wide.active_video_start, wide.active_video_end = 10, 1110  # 2 w - 1 > 2048: rows of 4096
    out = ctx.decode_frame_buffer(pal_frames[0], wide, cfg)
    ref = _ref()
    _compare(out, ref.decode_frame_buffer(pal_frames[0], wide, cfg), "wide PAL frame", pal=True)
    past = api.frame_params(_cabi.STD_NTSC)
    past.frame_width = 2100
    past.active_video_start, past.active_video_end = 20, 2069  # 2049 samples: 2 w - 1 > 4096
    blank = np.full((past.frame_height, past.frame_width), 16384, np.uint16)
    with pytest.raises(api.HvdgError) as e:
        ctx.decode_frame_buffer(blank, past, cfg)
    assert e.value.status == _cabi.ERR_UNSUPPORTED
    assert ctx.decode_frame_buffers([], fp, cfg) == []
    ok = ctx.decode_frame_buffer(frames[0], fp, cfg)
    assert np.abs(ok["u"]).max() > 0
