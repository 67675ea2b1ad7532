"""TEST INFRASTRUCTURE -- ctypes view of oracle/_ref/libhvdshim.so: the
reference's own C++ frame-bridge signatures (hvd::DecodeFrameSequenceWindow,
DecodeFrameBuffer, DecodeYcFrameBuffer) served by the B200 shim
(hvd-cvbs-decoding_b200/shim/frame_bridge_b200.cpp) on the product library,
built against the reference's headers by oracle/Makefile. Lets the tests
drive the drop-in exactly as the decode-orc plugin would."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from hvdg import _cabi

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libhvdshim.so"
_LIB = None


def available() -> bool:
    return LIB_PATH.exists()


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        L = C.CDLL(str(LIB_PATH))
        vp, P = C.c_void_p, C.POINTER
        L.hvdshim_decode_frame_sequence_window.argtypes = [
            P(vp), C.c_int, C.c_int, C.c_int, P(_cabi.FrameParams), P(_cabi.Config),
            P(vp), P(vp), P(vp), P(vp)]
        L.hvdshim_decode_frame_sequence_window.restype = C.c_int
        L.hvdshim_decode_frame_buffer.argtypes = [vp, P(_cabi.FrameParams), P(_cabi.Config),
                                                  vp, vp, vp, vp]
        L.hvdshim_decode_frame_buffer.restype = C.c_int
        L.hvdshim_decode_yc_frame_buffer.argtypes = [vp, vp, P(_cabi.FrameParams),
                                                     P(_cabi.Config), vp, vp, vp, vp]
        L.hvdshim_decode_yc_frame_buffer.restype = C.c_int
        L.hvdshim_decode_frame_buffer_workers.argtypes = [vp, P(_cabi.FrameParams),
                                                          P(_cabi.Config), C.c_int]
        L.hvdshim_decode_frame_buffer_workers.restype = C.c_int
        _LIB = L
    return _LIB


def _out(fp):
    sz = fp.frame_width * fp.frame_height
    return dict(luma=np.zeros(sz, np.int16), chroma=np.zeros(sz, np.int16),
                u=np.zeros(sz, np.float64), v=np.zeros(sz, np.float64))


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def decode_frame_sequence_window(frames, core_begin, core_end, fp, cfg):
    fr = [np.ascontiguousarray(f, dtype=np.int16) for f in frames]
    outs = [_out(fp) for _ in range(max(core_end - core_begin, 0))]
    V = C.c_void_p
    arr = lambda lst: (V * max(len(lst), 1))(*[a.ctypes.data for a in lst])
    got = lib().hvdshim_decode_frame_sequence_window(
        arr(fr), len(fr), core_begin, core_end, C.byref(fp), C.byref(cfg),
        arr([o["luma"] for o in outs]), arr([o["chroma"] for o in outs]),
        arr([o["u"] for o in outs]), arr([o["v"] for o in outs]))
    return outs[:got]


def decode_frame_buffer(frame, fp, cfg):
    fr = np.ascontiguousarray(frame, dtype=np.int16)
    o = _out(fp)
    ok = lib().hvdshim_decode_frame_buffer(_ptr(fr), C.byref(fp), C.byref(cfg), _ptr(o["luma"]),
                                           _ptr(o["chroma"]), _ptr(o["u"]), _ptr(o["v"]))
    return o if ok else None


def decode_yc_frame_buffer(luma, chroma, fp, cfg):
    y = np.ascontiguousarray(luma, dtype=np.int16)
    c = np.ascontiguousarray(chroma, dtype=np.int16)
    o = _out(fp)
    ok = lib().hvdshim_decode_yc_frame_buffer(_ptr(y), _ptr(c), C.byref(fp), C.byref(cfg),
                                              _ptr(o["luma"]), _ptr(o["chroma"]), _ptr(o["u"]),
                                              _ptr(o["v"]))
    return o if ok else None


def decode_frame_buffer_workers(frame, fp, cfg, n_threads):
    """hvd::DecodeFrameBuffer on `n_threads` short-lived worker threads, one
    fresh HvdEngine each (the stage's export pattern); returns the number of
    non-empty results."""
    fr = np.ascontiguousarray(frame, dtype=np.int16)
    return lib().hvdshim_decode_frame_buffer_workers(_ptr(fr), C.byref(fp), C.byref(cfg),
                                                     int(n_threads))
