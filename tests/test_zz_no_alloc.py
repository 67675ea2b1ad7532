"""The allocation-free holographic init (hvdg_holographic_init_noalloc).

It exists for callers that cannot call cudaMalloc (a plugin inside a host
that owns the CUDA allocator, a real-time path that must not stall on an
allocation): its scratch is a fixed file-scope device array. This test calls
it through the C ABI twice in a row -- an NTSC field, then a PAL field, which
reuses the same scratch with a different layout -- and checks each result
against the context-based hvdg_holographic_init on the same inputs. It sits
in its own file named to be collected last; it passes alone in a fresh
process and after the other tests. Its no-alloc calls come before it opens
any context, so run alone it also covers the cold path: the first call in a
process does the per-device set-up (the array's address, the init kernels'
attributes and twiddle constants) itself."""
import ctypes as C

import numpy as np
import pytest

from hvdg import _cabi, api, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


def _prepared(std, seed):
    g = _cabi.default_geometry(std)
    f = synth.make_field(seed, std, noise_sigma=0.5)
    cfg = api.default_config()
    obs = O.prepare_field(synth.to_ire(f.samples), g, cfg)
    fal, lal = g.first_active_field_line, g.last_active_line
    th = obs.theta[fal:lal].astype(np.float32)
    sw = obs.vswitch[fal:lal].astype(np.int8)
    return g, cfg, np.ascontiguousarray(obs.s, np.float32), th, sw


def test_noalloc_init_matches_context_init_twice():
    lib = _cabi.load_library()
    cases = [(_cabi.STD_NTSC, 31), (_cabi.STD_PAL, 32)]
    got = []
    for std, seed in cases:     # no context exists yet in this test
        g, cfg, s, th, sw = _prepared(std, seed)
        y = np.zeros_like(s)
        c = np.zeros(s.shape, np.complex64)
        st = lib.hvdg_holographic_init_noalloc(s.ctypes.data, th.ctypes.data, sw.ctypes.data,
                                               C.byref(g), y.ctypes.data, c.ctypes.data)
        assert st == _cabi.OK, _cabi.STATUS_NAMES.get(st, st)
        got.append((g, cfg, s, th, sw, y, c))
    with api.Context(0) as ctx:
        for g, cfg, s, th, sw, y, c in got:
            y_ref, c_ref = ctx.holographic_init(s, th, sw, g, cfg)
            assert np.abs(y - y_ref).max() <= 1e-5
            assert np.abs(c - c_ref).max() <= 1e-5


def test_noalloc_rejects_oversized_geometry():
    lib = _cabi.load_library()
    g = _cabi.geometry_copy(_cabi.default_geometry(_cabi.STD_NTSC), field_width=2000,
                            active_video_end=1900)
    s = np.zeros((g.active_lines, g.active_width), np.float32)
    th = np.zeros(g.active_lines, np.float32)
    y = np.zeros_like(s)
    c = np.zeros(s.shape, np.complex64)
    st = lib.hvdg_holographic_init_noalloc(s.ctypes.data, th.ctypes.data, None, C.byref(g),
                                           y.ctypes.data, c.ctypes.data)
    assert st == _cabi.ERR_UNSUPPORTED
