"""Python mirror of the engine interface, over the C ABI (include/hvdg.h).

Names and argument meanings follow hvd-core: decode_field_window ~
PrepareFieldObs + DecodeFieldWindow (sequence.h:60-101), burst_lockin ~
BurstLockinPhase[Pal] (lockin.h:31-59), holographic_init ~ HolographicInit,
variational_refine ~ VariationalRefine, estimate_motion ~ EstimateMotion,
decode_frame_sequence_window ~ hvd::DecodeFrameSequenceWindow. Errors are
raised as HvdgError carrying the C status.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _cabi
from ._cabi import Config, Diag, FieldIn, FieldOut, Geometry


class HvdgError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{_cabi.STATUS_NAMES.get(status, status)}: {msg}")


@dataclass
class Field:
    """One composite field in (FieldInput + parity + per-field budget)."""
    samples: np.ndarray             # (field_height, field_width) uint16 / int16 / float32 IRE
    geometry: Geometry
    parity: int = 0
    blanking_level: float = 16384.0
    white_level: float = 51200.0
    irls_outer: int = 0             # <= 0: config value
    cg_iterations: int = -1         # < 0: config value


@dataclass
class Decoded:
    luma: np.ndarray                # (active_lines, active_width) float32
    chroma: np.ndarray              # (active_lines, active_width) complex64, chi = V - iU
    theta: np.ndarray | None = None
    vswitch: np.ndarray | None = None


def _ptr(a) -> int:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a)


_SAMPLE_TYPES = {np.dtype(np.uint16): _cabi.SAMPLES_U16, np.dtype(np.int16): _cabi.SAMPLES_S16,
                 np.dtype(np.float32): _cabi.SAMPLES_F32_IRE}


class Context:
    """hvdg_ctx: one per thread (same contract as one HvdEngine per thread)."""

    def __init__(self, device: int = 0, lib_path=None):
        self.lib = _cabi.load_library(lib_path)
        h = C.c_void_p()
        st = self.lib.hvdg_create(int(device), C.byref(h))
        if st != _cabi.OK:
            raise HvdgError(st, "hvdg_create")
        self._h = h
        self.last_diag = Diag()

    def close(self):
        if getattr(self, "_h", None):
            self.lib.hvdg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int, what: str):
        if st != _cabi.OK:
            err = self.lib.hvdg_last_error(self._h)
            raise HvdgError(st, f"{what}: {err.decode() if err else ''}")

    def set_batching(self, batched: bool):
        self._check(self.lib.hvdg_set_batching(self._h, int(bool(batched))), "set_batching")

    def set_tuning(self, band_rows: int = 0, ctas_per_sm: int = 0):
        self._check(self.lib.hvdg_set_tuning(self._h, int(band_rows), int(ctas_per_sm)), "set_tuning")

    def set_device_wait_limit(self, polls: int = 0):
        """Polls of a field's phase flag before the solver gives up with
        HVDG_ERR_DEVICE_TIMEOUT (<= 0: the default, ~2 s)."""
        self._check(self.lib.hvdg_set_device_wait_limit(self._h, int(polls)),
                    "set_device_wait_limit")

    # ---- engine level ----------------------------------------------------
    def _build_fields(self, fields):
        n = len(fields)
        arr = (FieldIn * max(n, 1))()
        keep = []
        for i, f in enumerate(fields):
            s = np.ascontiguousarray(f.samples)
            st = _SAMPLE_TYPES.get(s.dtype)
            if st is None:
                s = np.ascontiguousarray(s, dtype=np.float32)
                st = _cabi.SAMPLES_F32_IRE
            g = f.geometry
            if s.shape != (g.field_height, g.field_width):
                raise ValueError(f"field {i}: samples {s.shape} != geometry "
                                 f"({g.field_height}, {g.field_width})")
            keep.append(s)
            arr[i].samples = s.ctypes.data
            arr[i].sample_type = st
            arr[i].parity = int(f.parity)
            arr[i].blanking_level = float(f.blanking_level)
            arr[i].white_level = float(f.white_level)
            arr[i].geometry = C.pointer(g)
            arr[i].irls_outer = int(f.irls_outer)
            arr[i].cg_iterations = int(f.cg_iterations)
            keep.append(arr[i].geometry)
        return arr, keep

    def _alloc_out(self, fields, want_theta: bool, out=None):
        outs, res = (FieldOut * max(len(fields), 1))(), []
        if out is not None and len(out) != len(fields):
            raise ValueError(f"out: {len(out)} buffers for {len(fields)} fields")
        for i, f in enumerate(fields):
            g = f.geometry
            shape = (g.active_lines, g.active_width)
            if out is not None:
                d = out[i]
                if (d.luma.shape != shape or d.luma.dtype != np.float32
                        or not d.luma.flags.c_contiguous or d.chroma.shape != shape
                        or d.chroma.dtype != np.complex64 or not d.chroma.flags.c_contiguous):
                    raise ValueError(f"out[{i}]: need C-contiguous float32 luma and complex64 "
                                     f"chroma of shape {shape}")
            else:
                d = Decoded(np.zeros(shape, np.float32), np.zeros(shape, np.complex64))
            outs[i].luma = d.luma.ctypes.data
            outs[i].chroma = d.chroma.ctypes.data
            if want_theta and (d.theta is None or d.vswitch is None):
                d.theta = np.zeros(g.field_height, np.float32)
                d.vswitch = np.zeros(g.field_height, np.int8)
                outs[i].theta = d.theta.ctypes.data
                outs[i].vswitch = d.vswitch.ctypes.data
            res.append(d)
        return outs, res

    def decode_fields(self, fields, cfg: Config, want_theta: bool = False,
                      out: list[Decoded] | None = None) -> list[Decoded]:
        """Independent 2-D fields (mixed geometry / budget) in one batch.
        `out` optionally supplies the output buffers (one Decoded per field,
        e.g. views of page-locked memory, which the device writes at full
        copy bandwidth); they are filled in place and returned."""
        arr, keep = self._build_fields(fields)
        outs, res = self._alloc_out(fields, want_theta, out)
        self.last_diag = Diag()
        st = self.lib.hvdg_decode_fields(self._h, arr, len(fields), C.byref(cfg), outs,
                                         C.byref(self.last_diag))
        self._check(st, "hvdg_decode_fields")
        del keep
        return res

    def decode_field_window(self, fields, cfg: Config, want_theta: bool = False) -> list[Decoded]:
        """PrepareFieldObs x n + DecodeFieldWindow (one geometry per window)."""
        arr, keep = self._build_fields(fields)
        outs, res = self._alloc_out(fields, want_theta)
        self.last_diag = Diag()
        st = self.lib.hvdg_decode_field_window(self._h, arr, len(fields), C.byref(cfg), outs,
                                               C.byref(self.last_diag))
        self._check(st, "hvdg_decode_field_window")
        del keep
        return res

    def decode_fields_device(self, fields_in, outs, n, cfg: Config) -> Diag:
        """Device-resident variant: `fields_in` / `outs` are prepared FieldIn /
        FieldOut arrays holding DEVICE pointers (e.g. torch tensor data_ptr)."""
        d = Diag()
        st = self.lib.hvdg_decode_fields_device(self._h, fields_in, int(n), C.byref(cfg), outs,
                                                C.byref(d))
        self._check(st, "hvdg_decode_fields_device")
        return d

    def decode_fields_device_async(self, fields_in, outs, n, cfg: Config, stream: int = 0):
        """Asynchronous device-resident decode ordered against `stream` (a raw
        cudaStream_t, e.g. torch.cuda.Stream().cuda_stream); complete it with
        wait()."""
        st = self.lib.hvdg_decode_fields_device_async(self._h, fields_in, int(n), C.byref(cfg),
                                                      outs, C.c_void_p(stream or None))
        self._check(st, "hvdg_decode_fields_device_async")

    def wait(self) -> Diag:
        d = Diag()
        self._check(self.lib.hvdg_wait(self._h, C.byref(d)), "hvdg_wait")
        return d

    def decode_fields_adjoint(self, fields, cfg: Config, y_bar, chi_bar,
                              adjoint_cg_iterations: int = 0, want_forward: bool = False):
        """Gradients of a scalar loss through the 2-D decode of `fields`
        (hvdg_decode_fields_adjoint). y_bar[i] / chi_bar[i]: the loss
        cotangents of field i's decoded luma (float) and chroma (complex).
        Returns (samples_bar, scalars, forward): samples_bar[i] is d loss /
        d sample (field_height x field_width), scalars maps lambda_c,
        charbonnier_eps, chroma_eps, structure_coupling to their gradients,
        forward is the recomputed decode (list of Decoded) or None."""
        arr, keep = self._build_fields(fields)
        n = len(fields)
        yb = [np.ascontiguousarray(a, np.float32) for a in y_bar]
        cb = [np.ascontiguousarray(a, np.complex64) for a in chi_bar]
        sb = [np.zeros((f.geometry.field_height, f.geometry.field_width), np.float32)
              for f in fields]
        for i, f in enumerate(fields):
            shape = (f.geometry.active_lines, f.geometry.active_width)
            if yb[i].shape != shape or cb[i].shape != shape:
                raise ValueError(f"field {i}: cotangents must have shape {shape}")
        ybp = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in yb])
        cbp = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in cb])
        sbp = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in sb])
        sc = (C.c_double * 4)()
        outs, res = (self._alloc_out(fields, False) if want_forward else (None, None))
        self.last_diag = Diag()
        st = self.lib.hvdg_decode_fields_adjoint(self._h, arr, n, C.byref(cfg), ybp, cbp, sbp, sc,
                                                 int(adjoint_cg_iterations), outs,
                                                 C.byref(self.last_diag))
        self._check(st, "hvdg_decode_fields_adjoint")
        del keep
        names = ("lambda_c", "charbonnier_eps", "chroma_eps", "structure_coupling")
        return sb, dict(zip(names, list(sc))), res

    # ---- kernel level --------------------------------------------------------
    def burst_lockin(self, field_ire: np.ndarray, g: Geometry):
        f = np.ascontiguousarray(field_ire, dtype=np.float32)
        th = np.zeros(g.field_height, np.float32)
        sw = np.zeros(g.field_height, np.int8)
        self._check(self.lib.hvdg_burst_lockin(self._h, f.ctypes.data, C.byref(g), th.ctypes.data,
                                               sw.ctypes.data), "hvdg_burst_lockin")
        return th, sw

    def burst_amplitude(self, field_ire: np.ndarray, g: Geometry) -> float:
        f = np.ascontiguousarray(field_ire, dtype=np.float32)
        v = C.c_float()
        self._check(self.lib.hvdg_burst_amplitude(self._h, f.ctypes.data, C.byref(g), C.byref(v)),
                    "hvdg_burst_amplitude")
        return float(v.value)

    def holographic_init(self, s, theta_active, vswitch_active, g: Geometry, cfg: Config):
        s = np.ascontiguousarray(s, dtype=np.float32)
        th = np.ascontiguousarray(theta_active, dtype=np.float32)
        sw = np.ascontiguousarray(vswitch_active, dtype=np.int8)
        y0 = np.zeros_like(s)
        chi0 = np.zeros(s.shape, np.complex64)
        self._check(self.lib.hvdg_holographic_init(self._h, s.ctypes.data, th.ctypes.data,
                                                   sw.ctypes.data, C.byref(g), C.byref(cfg),
                                                   y0.ctypes.data, chi0.ctypes.data),
                    "hvdg_holographic_init")
        return y0, chi0

    def variational_refine(self, s, theta_active, vswitch_active, chi0, g: Geometry, cfg: Config):
        s = np.ascontiguousarray(s, dtype=np.float32)
        th = np.ascontiguousarray(theta_active, dtype=np.float32)
        sw = np.ascontiguousarray(vswitch_active, dtype=np.int8)
        x0 = np.ascontiguousarray(chi0, dtype=np.complex64)
        y = np.zeros_like(s)
        chi = np.zeros(s.shape, np.complex64)
        self._check(self.lib.hvdg_variational_refine(self._h, s.ctypes.data, th.ctypes.data,
                                                     sw.ctypes.data, x0.ctypes.data, C.byref(g),
                                                     C.byref(cfg), y.ctypes.data, chi.ctypes.data),
                    "hvdg_variational_refine")
        return y, chi

    def estimate_motion(self, y_ref, y_cur, tile: int = 32, search: int = 16, me_mode: int = 0):
        a = np.ascontiguousarray(y_ref, dtype=np.float32)
        b = np.ascontiguousarray(y_cur, dtype=np.float32)
        h, w = a.shape
        th, tw = -(-h // tile), -(-w // tile)
        dy = np.zeros((th, tw), np.float32)
        dx = np.zeros_like(dy)
        cf = np.zeros_like(dy)
        self._check(self.lib.hvdg_estimate_motion(self._h, a.ctypes.data, b.ctypes.data, h, w,
                                                  tile, search, me_mode, dy.ctypes.data,
                                                  dx.ctypes.data, cf.ctypes.data),
                    "hvdg_estimate_motion")
        return dy, dx, cf

    def verify_motion(self, y_ref, y_cur, pdy, pdx, tile: int = 32):
        """VerifyMotion (motion.cpp:490-530): per-tile predictions audited
        against zero; returns (dy, dx, confidence) per tile."""
        a = np.ascontiguousarray(y_ref, dtype=np.float32)
        b = np.ascontiguousarray(y_cur, dtype=np.float32)
        h, w = a.shape
        pdy = np.ascontiguousarray(pdy, dtype=np.float32)
        pdx = np.ascontiguousarray(pdx, dtype=np.float32)
        if pdy.shape != (-(-h // tile), -(-w // tile)) or pdx.shape != pdy.shape:
            raise ValueError("predictions must have one value per tile")
        dy, dx, cf = (np.zeros(pdy.shape, np.float32) for _ in range(3))
        self._check(self.lib.hvdg_verify_motion(self._h, a.ctypes.data, b.ctypes.data, h, w, tile,
                                                pdy.ctypes.data, pdx.ctypes.data, dy.ctypes.data,
                                                dx.ctypes.data, cf.ctypes.data),
                    "hvdg_verify_motion")
        return dy, dx, cf


def default_config(**kw) -> Config:
    return _cabi.config_copy(_cabi.default_config(), **kw)


def ambiguous_boxes(luma: np.ndarray, chroma: np.ndarray, max_area: float = 0.45):
    """AmbiguousBoxes (the selective 3-D detector) on one decoded field:
    a list of (fy0, fy1, x0, x1), [] = stay 2-D, None = full 3-D."""
    lib = _cabi.load_library()
    y = np.ascontiguousarray(luma, dtype=np.float32)
    c = np.ascontiguousarray(chroma, dtype=np.complex64)
    h, w = y.shape
    buf = np.zeros(4 * 64, np.int32)
    n = C.c_int(0)
    st = lib.hvdg_ambiguous_boxes(y.ctypes.data, c.ctypes.data, h, w, float(max_area),
                                  buf.ctypes.data, 64, C.byref(n))
    if st != 0:
        raise HvdgError(st, "hvdg_ambiguous_boxes")
    if n.value < 0:
        return None
    return [tuple(int(v) for v in buf[4 * i:4 * i + 4]) for i in range(min(n.value, 64))]


def default_geometry(standard: int) -> Geometry:
    return _cabi.default_geometry(standard)


def frame_params(standard: int, blanking=240.0, white=800.0, black=None) -> _cabi.FrameParams:
    """FrameParams (frame_bridge.h:40-101) for the 4fsc frame layouts. PAL
    frames carry 4 extra samples (709 379 per frame, EBU Tech. 3280-E): two on
    frame line 312 and two on 624; FrameLineOffset counts one sample per
    listed entry, so each of those lines is listed twice."""
    fp = _cabi.FrameParams()
    g = _cabi.default_geometry(standard)
    fp.standard = standard
    fp.frame_width = g.field_width
    if standard == _cabi.STD_PAL:
        fp.frame_height, fp.field1_lines = 625, 313
        for i, ln in enumerate((312, 312, 624, 624)):
            fp.extra_sample_lines[i] = ln
        fp.extra_sample_line_count = 4
    else:
        fp.frame_height, fp.field1_lines = 525, 263
    fp.active_video_start, fp.active_video_end = g.active_video_start, g.active_video_end
    fp.colour_burst_start, fp.colour_burst_end = g.colour_burst_start, g.colour_burst_end
    fp.first_active_frame_line = 2 * g.first_active_field_line
    fp.last_active_frame_line = 0
    fp.blanking_level = blanking
    fp.white_level = white
    fp.black_level = blanking if black is None else black
    fp.chroma_dc = 0.0
    fp.sample_rate = g.sample_rate
    fp.subcarrier_hz = 0.0
    return fp


def frame_buffer_size(fp: _cabi.FrameParams) -> int:
    return fp.frame_width * fp.frame_height + fp.extra_sample_line_count


def _decode_frames(self, frames, core_begin, core_end, fp, cfg, base_frame_id=0):
    """hvd::DecodeFrameSequenceWindow: frames are flat int16 field-sequential
    buffers; returns one dict(luma, chroma, u, v) per core frame."""
    n = len(frames)
    fr = [np.ascontiguousarray(f, dtype=np.int16) for f in frames]
    ptrs = (C.c_void_p * max(n, 1))(*[f.ctypes.data for f in fr])
    m = max(core_end - core_begin, 0)
    sz = fp.frame_width * fp.frame_height
    res = [dict(luma=np.zeros(sz, np.int16), chroma=np.zeros(sz, np.int16),
                u=np.zeros(sz, np.float64), v=np.zeros(sz, np.float64)) for _ in range(m)]
    outs = (_cabi.YcFrame * max(m, 1))()
    for t, r in enumerate(res):
        outs[t].luma = r["luma"].ctypes.data
        outs[t].chroma = r["chroma"].ctypes.data
        outs[t].u_plane = r["u"].ctypes.data
        outs[t].v_plane = r["v"].ctypes.data
    self.last_diag = Diag()
    st = self.lib.hvdg_decode_frame_sequence_window_at(self._h, ptrs, n, core_begin, core_end,
                                                       int(base_frame_id), C.byref(fp),
                                                       C.byref(cfg), outs, C.byref(self.last_diag))
    self._check(st, "hvdg_decode_frame_sequence_window")
    return res


Context.decode_frame_sequence_window = _decode_frames


def _set_debug_dir(self, path):
    """HvdConfig::debug_dir: diagnostic maps of the sequence frame bridge
    (None = off)."""
    self._check(self.lib.hvdg_set_debug_dir(self._h, None if path is None else str(path).encode()),
                "hvdg_set_debug_dir")


Context.set_debug_dir = _set_debug_dir


def _yc_frames(fp, m, out=None):
    sz = fp.frame_width * fp.frame_height
    if out is not None:
        # caller-owned (e.g. pinned) planes: dicts of contiguous arrays of sz
        # elements (luma / chroma int16, u / v float64)
        if len(out) != m:
            raise ValueError("one output dict per frame")
        for r in out:
            for key, dt in (("luma", np.int16), ("chroma", np.int16), ("u", np.float64),
                            ("v", np.float64)):
                a = r[key]
                if a.dtype != dt or a.size != sz or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"output plane {key}: {sz} contiguous {np.dtype(dt)}")
        res = out
    else:
        res = [dict(luma=np.zeros(sz, np.int16), chroma=np.zeros(sz, np.int16),
                    u=np.zeros(sz, np.float64), v=np.zeros(sz, np.float64)) for _ in range(m)]
    outs = (_cabi.YcFrame * max(m, 1))()
    for t, r in enumerate(res):
        outs[t].luma = r["luma"].ctypes.data
        outs[t].chroma = r["chroma"].ctypes.data
        outs[t].u_plane = r["u"].ctypes.data
        outs[t].v_plane = r["v"].ctypes.data
    return res, outs


def _ptrs(arrs):
    return (C.c_void_p * max(len(arrs), 1))(*[a.ctypes.data for a in arrs])


def _decode_frame_buffer(self, frame, fp, cfg):
    """hvd::DecodeFrameBuffer: one flat int16 field-sequential composite
    frame -> dict(luma, chroma, u, v) (frame_width x frame_height each)."""
    fr = np.ascontiguousarray(frame, dtype=np.int16)
    res, outs = _yc_frames(fp, 1)
    st = self.lib.hvdg_decode_frame_buffer(self._h, fr.ctypes.data, C.byref(fp), C.byref(cfg),
                                           outs)
    self._check(st, "hvdg_decode_frame_buffer")
    return res[0]


def _decode_frame_buffers(self, frames, fp, cfg, out=None):
    """n independent frames of decode_frame_buffer in one batch; `out`
    (optional) = caller-owned output dicts (see _yc_frames)."""
    fr = [np.ascontiguousarray(f, dtype=np.int16) for f in frames]
    res, outs = _yc_frames(fp, len(fr), out)
    self.last_diag = Diag()
    st = self.lib.hvdg_decode_frame_buffers(self._h, _ptrs(fr), len(fr), C.byref(fp),
                                            C.byref(cfg), outs, C.byref(self.last_diag))
    self._check(st, "hvdg_decode_frame_buffers")
    return res


def _detect_field_parity(self, frames, fp):
    """DetectFieldParity of each int16 frame (split as SplitFrameFields
    splits it): +1 field 1 on top, -1 field 1 at the bottom, 0 no vote."""
    fr = [np.ascontiguousarray(f, dtype=np.int16) for f in frames]
    votes = np.zeros(max(len(fr), 1), np.int32)
    st = self.lib.hvdg_detect_field_parity(self._h, _ptrs(fr), len(fr), C.byref(fp),
                                           votes.ctypes.data)
    self._check(st, "hvdg_detect_field_parity")
    return votes[:len(fr)]


def _decode_yc_frame_buffer(self, luma, chroma, fp, cfg):
    """hvd::DecodeYcFrameBuffer: Y and C int16 frames -> dict(luma, chroma, u, v)."""
    y = np.ascontiguousarray(luma, dtype=np.int16)
    c = np.ascontiguousarray(chroma, dtype=np.int16)
    res, outs = _yc_frames(fp, 1)
    st = self.lib.hvdg_decode_yc_frame_buffer(self._h, y.ctypes.data, c.ctypes.data, C.byref(fp),
                                              C.byref(cfg), outs)
    self._check(st, "hvdg_decode_yc_frame_buffer")
    return res[0]


def _decode_yc_frame_buffers(self, lumas, chromas, fp, cfg, out=None):
    """n independent frames of decode_yc_frame_buffer in one batch."""
    ys = [np.ascontiguousarray(a, dtype=np.int16) for a in lumas]
    cs = [np.ascontiguousarray(a, dtype=np.int16) for a in chromas]
    if len(ys) != len(cs):
        raise ValueError("one chroma frame per luma frame")
    res, outs = _yc_frames(fp, len(ys), out)
    self.last_diag = Diag()
    st = self.lib.hvdg_decode_yc_frame_buffers(self._h, _ptrs(ys), _ptrs(cs), len(ys),
                                               C.byref(fp), C.byref(cfg), outs,
                                               C.byref(self.last_diag))
    self._check(st, "hvdg_decode_yc_frame_buffers")
    return res


def _drizzle_frame(self, j0, lumas, chromas, parities, cfg, scale=2):
    """DrizzleFrame: the frame of fields j0, j0 + 1 on a (2 h scale)-row
    grid from the motion-compensated deposits of the fields around it."""
    ys = [np.ascontiguousarray(y, dtype=np.float32) for y in lumas]
    cs = [np.ascontiguousarray(c, dtype=np.complex64) for c in chromas]
    n = len(ys)
    h, w = ys[0].shape
    par = np.ascontiguousarray(parities, dtype=np.int32)
    oy = np.zeros((2 * h * scale, w), np.float32)
    oc = np.zeros((2 * h * scale, w), np.complex64)
    st = self.lib.hvdg_drizzle_frame(self._h, _ptrs(ys), _ptrs(cs), par.ctypes.data, n, j0, h, w,
                                     C.byref(cfg), scale, oy.ctypes.data, oc.ctypes.data)
    self._check(st, "hvdg_drizzle_frame")
    return oy, oc


Context.drizzle_frame = _drizzle_frame
Context.decode_frame_buffer = _decode_frame_buffer
Context.detect_field_parity = _detect_field_parity
Context.decode_frame_buffers = _decode_frame_buffers
Context.decode_yc_frame_buffer = _decode_yc_frame_buffer
Context.decode_yc_frame_buffers = _decode_yc_frame_buffers
