"""ctypes mirror of include/hvdg.h (structs, enums, library loading).

The C header is the source of truth; every struct here must match it field
for field (tests/test_cabi.py checks sizes against the compiled library).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR.parent / "lib" / "libhvdg.so"

HVDG_ABI_VERSION = 1

# hvdg_status
OK = 0
ERR_BAD_ARGUMENT = 1
ERR_BAD_GEOMETRY = 2
ERR_NONFINITE_INPUT = 3
ERR_DEVICE_TIMEOUT = 4
ERR_CUDA = 5
ERR_OUT_OF_MEMORY = 6
ERR_UNSUPPORTED = 7
ERR_NO_DEVICE = 8

STATUS_NAMES = {
    0: "HVDG_OK", 1: "HVDG_ERR_BAD_ARGUMENT", 2: "HVDG_ERR_BAD_GEOMETRY",
    3: "HVDG_ERR_NONFINITE_INPUT", 4: "HVDG_ERR_DEVICE_TIMEOUT", 5: "HVDG_ERR_CUDA",
    6: "HVDG_ERR_OUT_OF_MEMORY", 7: "HVDG_ERR_UNSUPPORTED", 8: "HVDG_ERR_NO_DEVICE",
}

# hvdg_standard
STD_NTSC = 0
STD_PAL = 1
STD_PAL_M = 2

# hvdg_sample_type
SAMPLES_F32_IRE = 0
SAMPLES_U16 = 1
SAMPLES_S16 = 2


class Geometry(C.Structure):
    _fields_ = [
        ("field_width", C.c_int32),
        ("field_height", C.c_int32),
        ("active_video_start", C.c_int32),
        ("active_video_end", C.c_int32),
        ("colour_burst_start", C.c_int32),
        ("colour_burst_end", C.c_int32),
        ("first_active_field_line", C.c_int32),
        ("last_active_field_line", C.c_int32),
        ("sample_rate", C.c_double),
        ("standard", C.c_int32),
        ("reserved0", C.c_int32),
        ("subcarrier_hz", C.c_double),
    ]

    # convenience accessors mirroring FieldGeometry (ntsc_geometry.h:260-266)
    @property
    def active_width(self) -> int:
        return self.active_video_end - self.active_video_start

    @property
    def last_active_line(self) -> int:
        return self.last_active_field_line if self.last_active_field_line != 0 else self.field_height

    @property
    def active_lines(self) -> int:
        return self.last_active_line - self.first_active_field_line

    @property
    def uses_vswitch(self) -> bool:
        return self.standard in (STD_PAL, STD_PAL_M)


class Config(C.Structure):
    _fields_ = [
        ("lambda_c", C.c_float),
        ("chroma_aniso", C.c_float),
        ("charbonnier_eps", C.c_float),
        ("chroma_eps", C.c_float),
        ("structure_coupling", C.c_float),
        ("diag_prior", C.c_float),
        ("cg_iterations", C.c_int32),
        ("irls_outer", C.c_int32),
        ("cg_tol", C.c_float),
        ("fast", C.c_int32),
        ("parallel_across_fields", C.c_int32),
        ("symmetry_variant", C.c_int32),
        ("acc", C.c_int32),
        ("chroma_gain", C.c_float),
        ("monochrome", C.c_int32),
        ("chroma_phase_deg", C.c_float),
        ("field_order", C.c_int32),
        ("temporal_strength", C.c_float),
        ("bidirectional", C.c_int32),
        ("passes", C.c_int32),
        ("temporal_eps", C.c_float),
        ("nr_anchor", C.c_float),
        ("nr_eps", C.c_float),
        ("nr_radius", C.c_int32),
        ("mc_tile", C.c_int32),
        ("mc_search", C.c_int32),
        ("trajectory_fit", C.c_int32),
        ("extended_temporal", C.c_int32),
        ("coherence_gate", C.c_float),
        ("odd_gate_floor", C.c_float),
        ("output_fidelity", C.c_int32),
        ("psi_init", C.c_int32),
        ("selective_3d", C.c_int32),
        ("selective_max_area", C.c_float),
        ("me_mode", C.c_int32),
        ("me_block", C.c_int32),
        ("me_range", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


MAX_EXTRA_SAMPLE_LINES = 8


class FrameParams(C.Structure):
    _fields_ = [
        ("standard", C.c_int32),
        ("frame_width", C.c_int32),
        ("frame_height", C.c_int32),
        ("field1_lines", C.c_int32),
        ("active_video_start", C.c_int32),
        ("active_video_end", C.c_int32),
        ("colour_burst_start", C.c_int32),
        ("colour_burst_end", C.c_int32),
        ("first_active_frame_line", C.c_int32),
        ("last_active_frame_line", C.c_int32),
        ("black_level", C.c_float),
        ("white_level", C.c_float),
        ("blanking_level", C.c_float),
        ("chroma_dc", C.c_float),
        ("sample_rate", C.c_double),
        ("subcarrier_hz", C.c_double),
        ("extra_sample_lines", C.c_int32 * MAX_EXTRA_SAMPLE_LINES),
        ("extra_sample_line_count", C.c_int32),
        ("reserved0", C.c_int32),
    ]


class FieldIn(C.Structure):
    _fields_ = [
        ("samples", C.c_void_p),
        ("sample_type", C.c_int32),
        ("parity", C.c_int32),
        ("blanking_level", C.c_float),
        ("white_level", C.c_float),
        ("geometry", C.POINTER(Geometry)),
        ("irls_outer", C.c_int32),
        ("cg_iterations", C.c_int32),
    ]


class FieldOut(C.Structure):
    _fields_ = [
        ("luma", C.c_void_p),
        ("chroma", C.c_void_p),
        ("theta", C.c_void_p),
        ("vswitch", C.c_void_p),
    ]


class YcFrame(C.Structure):
    _fields_ = [
        ("luma", C.c_void_p),
        ("chroma", C.c_void_p),
        ("u_plane", C.c_void_p),
        ("v_plane", C.c_void_p),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("resolved_strength", C.c_float),
        ("ambiguity_ire", C.c_float),
        ("sigma_ire", C.c_float),
        ("temporal_eps", C.c_float),
        ("nr_eps", C.c_float),
        ("acc_gain", C.c_float),
        ("ms_total", C.c_float),
        ("ms_solver", C.c_float),
        ("ms_init", C.c_float),
        ("ms_motion", C.c_float),
        ("cg_iterations_run", C.c_int64),
        ("solver_pixel_iters", C.c_int64),
        ("solver_pixel_outers", C.c_int64),
        ("kernel_launches", C.c_int32),
        ("reserved", C.c_int32),
    ]


# ---------------------------------------------------------------------------
# Defaults, restated from the reference so that host-only code (tests, the
# synthetic generator) does not need the shared library.
# ---------------------------------------------------------------------------

def default_config() -> Config:
    """hvd::HvdConfig defaults (hvd_config.h:21-419) + build extensions."""
    c = Config()
    c.lambda_c = 1.0
    c.chroma_aniso = 0.0
    c.charbonnier_eps = 0.5
    c.chroma_eps = 1.0
    c.structure_coupling = 0.25
    c.diag_prior = 0.0
    c.cg_iterations = 2
    c.irls_outer = 4
    c.cg_tol = 0.0
    c.fast = 1
    c.parallel_across_fields = 1
    c.symmetry_variant = 0
    c.acc = 1
    c.chroma_gain = 1.0
    c.monochrome = 0
    c.chroma_phase_deg = 0.0
    c.field_order = 0
    c.temporal_strength = 0.0
    c.bidirectional = 1
    c.passes = 2
    c.temporal_eps = 0.0
    c.nr_anchor = 1.0
    c.nr_eps = 0.0
    c.nr_radius = 2
    c.mc_tile = 32
    c.mc_search = 16
    c.trajectory_fit = 1
    c.extended_temporal = 1
    c.coherence_gate = 0.6
    c.odd_gate_floor = 0.35
    c.output_fidelity = 1
    c.psi_init = 0
    c.selective_3d = 0
    c.selective_max_area = 0.45
    c.me_mode = 0
    c.me_block = 16
    c.me_range = 16
    return c


FSC_NTSC = 315.0e6 / 88.0
FS_NTSC = 4.0 * FSC_NTSC
FSC_PAL = 4433618.75
FS_PAL = 4.0 * FSC_PAL


def default_geometry(standard: int) -> Geometry:
    """FieldGeometry defaults (ntsc_geometry.h:143-152) for NTSC; the PAL
    4fsc geometry of research/reference-pal/hvd_pal/tbc.py:34-50."""
    g = Geometry()
    if standard == STD_PAL:
        g.field_width, g.field_height = 1135, 313
        g.active_video_start, g.active_video_end = 185, 1107
        g.colour_burst_start, g.colour_burst_end = 98, 138
        g.first_active_field_line, g.last_active_field_line = 22, 0
        g.sample_rate = FS_PAL
    else:
        g.field_width, g.field_height = 910, 263
        g.active_video_start, g.active_video_end = 134, 894
        g.colour_burst_start, g.colour_burst_end = 78, 110
        g.first_active_field_line, g.last_active_field_line = 21, 0
        g.sample_rate = FS_NTSC
    g.standard = standard
    g.subcarrier_hz = 0.0
    return g


def config_copy(c: Config, **kw) -> Config:
    o = Config()
    C.memmove(C.byref(o), C.byref(c), C.sizeof(Config))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def geometry_copy(g: Geometry, **kw) -> Geometry:
    o = Geometry()
    C.memmove(C.byref(o), C.byref(g), C.sizeof(Geometry))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


_LIB = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libhvdg.so (built in-tree by __graft_entry__.build()). Raises if
    it is missing: there is no fallback implementation."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"libhvdg.so not found at {p}: build it first "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(str(p))
    _declare(lib)
    if path is None:
        _LIB = lib
    return lib


def _declare(lib: C.CDLL) -> None:
    P = C.POINTER
    vp = C.c_void_p
    lib.hvdg_abi_version.restype = C.c_int
    lib.hvdg_status_string.restype = C.c_char_p
    lib.hvdg_status_string.argtypes = [C.c_int]
    lib.hvdg_config_default.argtypes = [P(Config)]
    lib.hvdg_config_default.restype = None
    lib.hvdg_geometry_default.argtypes = [C.c_int, P(Geometry)]
    lib.hvdg_geometry_default.restype = None
    lib.hvdg_create.argtypes = [C.c_int, P(vp)]
    lib.hvdg_create.restype = C.c_int
    lib.hvdg_destroy.argtypes = [vp]
    lib.hvdg_destroy.restype = None
    lib.hvdg_last_error.argtypes = [vp]
    lib.hvdg_last_error.restype = C.c_char_p
    lib.hvdg_set_batching.argtypes = [vp, C.c_int]
    lib.hvdg_set_batching.restype = C.c_int
    lib.hvdg_set_tuning.argtypes = [vp, C.c_int, C.c_int]
    lib.hvdg_set_tuning.restype = C.c_int
    lib.hvdg_set_device_wait_limit.argtypes = [vp, C.c_int64]
    lib.hvdg_set_device_wait_limit.restype = C.c_int
    for name in ("hvdg_decode_field_window", "hvdg_decode_fields", "hvdg_decode_fields_device"):
        f = getattr(lib, name)
        f.argtypes = [vp, P(FieldIn), C.c_int, P(Config), P(FieldOut), P(Diag)]
        f.restype = C.c_int
    lib.hvdg_decode_fields_device_async.argtypes = [vp, P(FieldIn), C.c_int, P(Config),
                                                    P(FieldOut), vp]
    lib.hvdg_decode_fields_device_async.restype = C.c_int
    lib.hvdg_wait.argtypes = [vp, P(Diag)]
    lib.hvdg_wait.restype = C.c_int
    lib.hvdg_decode_frame_sequence_window.argtypes = [
        vp, P(vp), C.c_int, C.c_int, C.c_int, P(FrameParams), P(Config), P(YcFrame), P(Diag)]
    lib.hvdg_decode_frame_sequence_window.restype = C.c_int
    lib.hvdg_decode_frame_sequence_window_at.argtypes = [
        vp, P(vp), C.c_int, C.c_int, C.c_int, C.c_int64, P(FrameParams), P(Config), P(YcFrame),
        P(Diag)]
    lib.hvdg_decode_frame_sequence_window_at.restype = C.c_int
    lib.hvdg_set_debug_dir.argtypes = [vp, C.c_char_p]
    lib.hvdg_set_debug_dir.restype = C.c_int
    lib.hvdg_drizzle_frame.argtypes = [vp, P(vp), P(vp), vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                       P(Config), C.c_int, vp, vp]
    lib.hvdg_drizzle_frame.restype = C.c_int
    lib.hvdg_ambiguous_boxes.argtypes = [vp, vp, C.c_int, C.c_int, C.c_float, vp, C.c_int,
                                         P(C.c_int)]
    lib.hvdg_ambiguous_boxes.restype = C.c_int
    lib.hvdg_detect_field_parity.argtypes = [vp, P(vp), C.c_int, P(FrameParams), vp]
    lib.hvdg_detect_field_parity.restype = C.c_int
    lib.hvdg_decode_frame_buffer.argtypes = [vp, vp, P(FrameParams), P(Config), P(YcFrame)]
    lib.hvdg_decode_frame_buffer.restype = C.c_int
    lib.hvdg_decode_frame_buffers.argtypes = [vp, P(vp), C.c_int, P(FrameParams), P(Config),
                                              P(YcFrame), P(Diag)]
    lib.hvdg_decode_frame_buffers.restype = C.c_int
    lib.hvdg_decode_yc_frame_buffer.argtypes = [vp, vp, vp, P(FrameParams), P(Config), P(YcFrame)]
    lib.hvdg_decode_yc_frame_buffer.restype = C.c_int
    lib.hvdg_decode_yc_frame_buffers.argtypes = [vp, P(vp), P(vp), C.c_int, P(FrameParams),
                                                 P(Config), P(YcFrame), P(Diag)]
    lib.hvdg_decode_yc_frame_buffers.restype = C.c_int
    lib.hvdg_burst_lockin.argtypes = [vp, vp, P(Geometry), vp, vp]
    lib.hvdg_burst_lockin.restype = C.c_int
    lib.hvdg_burst_amplitude.argtypes = [vp, vp, P(Geometry), P(C.c_float)]
    lib.hvdg_burst_amplitude.restype = C.c_int
    lib.hvdg_holographic_init.argtypes = [vp, vp, vp, vp, P(Geometry), P(Config), vp, vp]
    lib.hvdg_holographic_init.restype = C.c_int
    lib.hvdg_variational_refine.argtypes = [vp, vp, vp, vp, vp, P(Geometry), P(Config), vp, vp]
    lib.hvdg_variational_refine.restype = C.c_int
    lib.hvdg_estimate_motion.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_int, vp, vp, vp]
    lib.hvdg_estimate_motion.restype = C.c_int
    lib.hvdg_verify_motion.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp]
    lib.hvdg_verify_motion.restype = C.c_int
    lib.hvdg_holographic_init_noalloc.argtypes = [vp, vp, vp, P(Geometry), vp, vp]
    lib.hvdg_holographic_init_noalloc.restype = C.c_int
    lib.hvdg_decode_fields_adjoint.argtypes = [vp, P(FieldIn), C.c_int, P(Config), P(vp), P(vp),
                                               P(vp), P(C.c_double), C.c_int, P(FieldOut), P(Diag)]
    lib.hvdg_decode_fields_adjoint.restype = C.c_int
