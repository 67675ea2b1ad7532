"""TEST INFRASTRUCTURE (oracle): ctypes access to the UNMODIFIED reference
engine compiled from its own sources (oracle/_ref/libhvdref.so, built by
oracle/Makefile). Used only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs, as the checker -- never by the product.

Each wrapper names the reference function it reaches (through
oracle/ref_capi.cpp)."""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
from hvdg import _cabi  # noqa: E402  (ABI struct layouts shared with the C header)

LIB_PATH = HERE / "_ref" / "libhvdref.so"
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"reference engine not built: {LIB_PATH} (run make -C oracle)")
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L):
    P, vp = C.POINTER, C.c_void_p
    L.hvdref_set_threads.argtypes = [C.c_int]
    L.hvdref_set_threads.restype = C.c_int
    L.hvdref_burst_lockin.argtypes = [vp, P(_cabi.Geometry), vp, vp]
    L.hvdref_burst_amplitude.argtypes = [vp, P(_cabi.Geometry)]
    L.hvdref_burst_amplitude.restype = C.c_float
    L.hvdref_tridiag_smooth.argtypes = [vp, vp, C.c_int, C.c_float, vp]
    L.hvdref_make_carrier.argtypes = [vp, vp, C.c_int, P(_cabi.Geometry), vp]
    L.hvdref_prepare_field.argtypes = [vp, P(_cabi.Geometry), P(_cabi.Config), C.c_int, vp, vp]
    L.hvdref_holographic_init.argtypes = [vp, vp, C.c_int, C.c_int, P(_cabi.Geometry),
                                          P(_cabi.Config), vp, vp]
    L.hvdref_variational_refine.argtypes = [vp, vp, vp, C.c_int, C.c_int, P(_cabi.Config),
                                            C.c_int, C.c_int, P(vp), P(vp), P(vp), vp, vp]
    L.hvdref_estimate_motion.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]
    L.hvdref_verify_motion.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp]
    L.hvdref_box_blur.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.hvdref_vectors_per_pixel.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           vp, vp]
    L.hvdref_upsample_confidence.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, vp]
    L.hvdref_estimate_noise.argtypes = [vp, C.c_int, C.c_int]
    L.hvdref_estimate_noise.restype = C.c_float
    L.hvdref_decode_field_window.argtypes = [P(vp), vp, C.c_int, P(_cabi.Geometry),
                                             P(_cabi.Config), P(vp), P(vp), vp]
    L.hvdref_decode_fields.argtypes = [P(vp), vp, C.c_int, P(vp), P(vp), P(vp), P(vp), C.c_int]
    L.hvdref_decode_frame_sequence_window.argtypes = [P(vp), C.c_int, C.c_int, C.c_int,
                                                      P(_cabi.FrameParams), P(_cabi.Config),
                                                      P(vp), P(vp), P(vp), P(vp)]
    L.hvdref_split_frame_fields.argtypes = [vp, P(_cabi.FrameParams), vp, vp]
    L.hvdref_decode_frame_sequence_window_debug.argtypes = [
        P(vp), C.c_int, C.c_int, C.c_int, P(_cabi.FrameParams), P(_cabi.Config), C.c_char_p,
        C.c_int64, P(vp), P(vp), P(vp), P(vp)]
    L.hvdref_drizzle_frame.argtypes = [P(vp), P(vp), vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                       P(_cabi.Config), C.c_int, vp, vp]
    L.hvdref_decode_frame_buffer.argtypes = [vp, P(_cabi.FrameParams), P(_cabi.Config), vp, vp,
                                             vp, vp]
    L.hvdref_decode_yc_frame_buffer.argtypes = [vp, vp, P(_cabi.FrameParams), P(_cabi.Config),
                                                vp, vp, vp, vp]
    L.hvdref_detect_field_parity.argtypes = [vp, vp, P(_cabi.FrameParams)]
    L.hvdref_fft2d.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp]


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex64)


def set_threads(n: int) -> int:
    return lib().hvdref_set_threads(int(n))


def burst_lockin(field_ire: np.ndarray, g: _cabi.Geometry):
    f = _f32(field_ire)
    th = np.zeros(g.field_height, np.float32)
    sw = np.zeros(g.field_height, np.int8)
    lib().hvdref_burst_lockin(_p(f), C.byref(g), _p(th), _p(sw))
    return th, sw


def burst_amplitude(field_ire, g) -> float:
    f = _f32(field_ire)
    return float(lib().hvdref_burst_amplitude(_p(f), C.byref(g)))


def tridiag_smooth(d, a, lam):
    d, a = _f32(d), _f32(a)
    x = np.zeros_like(d)
    lib().hvdref_tridiag_smooth(_p(d), _p(a), len(d), C.c_float(lam), _p(x))
    return x


def make_carrier(theta_active, vswitch_active, g):
    th = _f32(theta_active)
    sw = np.ascontiguousarray(vswitch_active, dtype=np.int8)
    out = np.zeros((len(th), g.active_width), np.complex64)
    lib().hvdref_make_carrier(_p(th), _p(sw), len(th), C.byref(g), _p(out))
    return out


def prepare_field(field_ire, g, cfg, parity=0):
    f = _f32(field_ire)
    s = np.zeros((g.active_lines, g.active_width), np.float32)
    c = np.zeros((g.active_lines, g.active_width), np.complex64)
    lib().hvdref_prepare_field(_p(f), C.byref(g), C.byref(cfg), int(parity), _p(s), _p(c))
    return s, c


def holographic_init(s, carrier, g, cfg):
    s, c = _f32(s), _c64(carrier)
    h, w = s.shape
    y0 = np.zeros_like(s)
    chi0 = np.zeros((h, w), np.complex64)
    lib().hvdref_holographic_init(_p(s), _p(c), h, w, C.byref(g), C.byref(cfg), _p(y0), _p(chi0))
    return y0, chi0


def variational_refine(s, carrier, chi0, cfg, is_pal=False, neighbors=()):
    s, c, x0 = _f32(s), _c64(carrier), _c64(chi0)
    h, w = s.shape
    nb = [(_f32(a), _c64(b), _f32(cf)) for (a, b, cf) in neighbors]
    n = len(nb)
    arr = lambda k: (C.c_void_p * max(n, 1))(*[_p(t[k]).value for t in nb])
    y = np.zeros_like(s)
    chi = np.zeros((h, w), np.complex64)
    lib().hvdref_variational_refine(_p(s), _p(c), _p(x0), h, w, C.byref(cfg), int(is_pal), n,
                                    arr(0), arr(1), arr(2), _p(y), _p(chi))
    return y, chi


def estimate_motion(y_ref, y_cur, tile=32, search=16):
    a, b = _f32(y_ref), _f32(y_cur)
    h, w = a.shape
    th, tw = -(-h // tile), -(-w // tile)
    dy = np.zeros((th, tw), np.float32)
    dx = np.zeros_like(dy)
    cf = np.zeros_like(dy)
    lib().hvdref_estimate_motion(_p(a), _p(b), h, w, tile, search, _p(dy), _p(dx), _p(cf))
    return dy, dx, cf


def verify_motion(y_ref, y_cur, pdy, pdx, tile=32):
    """VerifyMotion (motion.cpp:490-530) of the compiled reference."""
    a, b = _f32(y_ref), _f32(y_cur)
    h, w = a.shape
    pdy, pdx = _f32(pdy), _f32(pdx)
    dy, dx, cf = (np.zeros(pdy.shape, np.float32) for _ in range(3))
    lib().hvdref_verify_motion(_p(a), _p(b), h, w, int(tile), _p(pdy), _p(pdx), _p(dy), _p(dx),
                               _p(cf))
    return dy, dx, cf


def box_blur(a, r):
    a = _f32(a).copy()
    lib().hvdref_box_blur(_p(a), a.shape[0], a.shape[1], int(r))
    return a


def vectors_per_pixel(mdy, mdx, tile, out_h, out_w):
    mdy, mdx = _f32(mdy), _f32(mdx)
    dy = np.zeros((out_h, out_w), np.float32)
    dx = np.zeros_like(dy)
    lib().hvdref_vectors_per_pixel(_p(mdy), _p(mdx), mdy.shape[0], mdy.shape[1], tile,
                                   out_h, out_w, _p(dy), _p(dx))
    return dy, dx


def upsample_confidence(conf, tile, out_h, out_w, fast=False):
    cf = _f32(conf)
    out = np.zeros((out_h, out_w), np.float32)
    lib().hvdref_upsample_confidence(_p(cf), cf.shape[0], cf.shape[1], tile, out_h, out_w,
                                     int(bool(fast)), _p(out))
    return out


def estimate_noise(s) -> float:
    s = _f32(s)
    return float(lib().hvdref_estimate_noise(_p(s), s.shape[0], s.shape[1]))


def decode_field_window(fields_ire, parities, g, cfg):
    """PrepareFieldObs x n + DecodeFieldWindow. Returns ([Y], [chi], diag5)."""
    fs = [_f32(f) for f in fields_ire]
    n = len(fs)
    par = np.ascontiguousarray(parities, dtype=np.int32)
    ys = [np.zeros((g.active_lines, g.active_width), np.float32) for _ in range(n)]
    cs = [np.zeros((g.active_lines, g.active_width), np.complex64) for _ in range(n)]
    V = C.c_void_p * n
    diag = np.zeros(5, np.float32)
    lib().hvdref_decode_field_window(V(*[_p(f).value for f in fs]), _p(par), n, C.byref(g),
                                     C.byref(cfg), V(*[_p(y).value for y in ys]),
                                     V(*[_p(c).value for c in cs]), _p(diag))
    return ys, cs, diag


def decode_fields(fields_ire, parities, geoms, cfgs, across_fields=True):
    """Independent 2-D fields, each with its own geometry / config."""
    fs = [_f32(f) for f in fields_ire]
    n = len(fs)
    par = np.ascontiguousarray(parities, dtype=np.int32)
    ys = [np.zeros((g.active_lines, g.active_width), np.float32) for g in geoms]
    cs = [np.zeros((g.active_lines, g.active_width), np.complex64) for g in geoms]
    V = C.c_void_p * n
    gp = V(*[C.cast(C.pointer(g), C.c_void_p).value for g in geoms])
    cp = V(*[C.cast(C.pointer(c), C.c_void_p).value for c in cfgs])
    lib().hvdref_decode_fields(V(*[_p(f).value for f in fs]), _p(par), n, gp, cp,
                               V(*[_p(y).value for y in ys]), V(*[_p(c).value for c in cs]),
                               int(bool(across_fields)))
    return ys, cs


def decode_frame_sequence_window(frames, core_begin, core_end, fp, cfg):
    fr = [np.ascontiguousarray(f, dtype=np.int16) for f in frames]
    n = len(fr)
    m = max(core_end - core_begin, 0)
    sz = fp.frame_width * fp.frame_height
    L = [np.zeros(sz, np.int16) for _ in range(m)]
    Cc = [np.zeros(sz, np.int16) for _ in range(m)]
    U = [np.zeros(sz, np.float64) for _ in range(m)]
    Vv = [np.zeros(sz, np.float64) for _ in range(m)]
    Vp = C.c_void_p
    arr = lambda lst: (Vp * max(len(lst), 1))(*[_p(a).value for a in lst])
    got = lib().hvdref_decode_frame_sequence_window(arr(fr), n, core_begin, core_end,
                                                    C.byref(fp), C.byref(cfg),
                                                    arr(L), arr(Cc), arr(U), arr(Vv))
    return [dict(luma=L[t], chroma=Cc[t], u=U[t], v=Vv[t]) for t in range(got)]


def drizzle_frame(j0, Ys, chis, parities, cfg, scale=2):
    """hvd::DrizzleFrame: (luma, chroma) of (2 h scale) x w."""
    ys = [_f32(y) for y in Ys]
    cs = [_c64(c) for c in chis]
    n = len(ys)
    h, w = ys[0].shape
    par = np.ascontiguousarray(parities, dtype=np.int32)
    oy = np.zeros((2 * h * scale, w), np.float32)
    oc = np.zeros((2 * h * scale, w), np.complex64)
    V = C.c_void_p * n
    lib().hvdref_drizzle_frame(V(*[_p(y).value for y in ys]), V(*[_p(c).value for c in cs]),
                               _p(par), n, j0, h, w, C.byref(cfg), scale, _p(oy), _p(oc))
    return oy, oc


def _yc_out(fp):
    sz = fp.frame_width * fp.frame_height
    return (np.zeros(sz, np.int16), np.zeros(sz, np.int16), np.zeros(sz, np.float64),
            np.zeros(sz, np.float64))


def decode_frame_buffer(frame, fp, cfg):
    """hvd::DecodeFrameBuffer on one int16 frame: dict(luma, chroma, u, v)."""
    fr = np.ascontiguousarray(frame, dtype=np.int16)
    L, Cc, U, Vv = _yc_out(fp)
    lib().hvdref_decode_frame_buffer(_p(fr), C.byref(fp), C.byref(cfg), _p(L), _p(Cc), _p(U),
                                     _p(Vv))
    return dict(luma=L, chroma=Cc, u=U, v=Vv)


def decode_yc_frame_buffer(luma, chroma, fp, cfg):
    """hvd::DecodeYcFrameBuffer on one Y/C int16 frame pair."""
    y = np.ascontiguousarray(luma, dtype=np.int16)
    c = np.ascontiguousarray(chroma, dtype=np.int16)
    L, Cc, U, Vv = _yc_out(fp)
    lib().hvdref_decode_yc_frame_buffer(_p(y), _p(c), C.byref(fp), C.byref(cfg), _p(L), _p(Cc),
                                        _p(U), _p(Vv))
    return dict(luma=L, chroma=Cc, u=U, v=Vv)


def decode_frame_sequence_window_debug(frames, core_begin, core_end, fp, cfg, debug_dir,
                                       base_frame_id=0):
    """DecodeFrameSequenceWindow with HvdConfig::debug_dir set: the
    diagnostic maps land in debug_dir."""
    fr = [np.ascontiguousarray(f, dtype=np.int16) for f in frames]
    m = max(core_end - core_begin, 0)
    outs = [_yc_out(fp) for _ in range(m)]
    Vp = C.c_void_p
    arr = lambda lst: (Vp * max(len(lst), 1))(*[_p(a).value for a in lst])
    got = lib().hvdref_decode_frame_sequence_window_debug(
        arr(fr), len(fr), core_begin, core_end, C.byref(fp), C.byref(cfg),
        str(debug_dir).encode(), int(base_frame_id), arr([o[0] for o in outs]),
        arr([o[1] for o in outs]), arr([o[2] for o in outs]), arr([o[3] for o in outs]))
    return [dict(luma=o[0], chroma=o[1], u=o[2], v=o[3]) for o in outs[:got]]


def split_frame_fields(frame, fp):
    fr = np.ascontiguousarray(frame, dtype=np.int16)
    top = np.zeros((fp.field1_lines, fp.frame_width), np.float32)
    bot = np.zeros_like(top)
    lib().hvdref_split_frame_fields(_p(fr), C.byref(fp), _p(top), _p(bot))
    return top, bot


def detect_field_parity(b1, b2, fp) -> int:
    a, b = _f32(b1), _f32(b2)
    return int(lib().hvdref_detect_field_parity(_p(a), _p(b), C.byref(fp)))


def fft2d(a, inverse=False):
    a = _c64(a)
    out = np.zeros_like(a)
    lib().hvdref_fft2d(_p(a), a.shape[0], a.shape[1], int(bool(inverse)), _p(out))
    return out
