"""CPU checks of the C ABI boundary: the shared library loads, exports every
function include/hvdg.h declares, and the ctypes mirrors have the C layout.
No compute calls (no GPU here)."""
import ctypes as C
import re
import subprocess
import textwrap
from pathlib import Path

import pytest

from hvdg import _cabi

REPO = Path(__file__).resolve().parent.parent
HDR = REPO / "include" / "hvdg.h"


def declared_functions():
    text = HDR.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hvdg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_cabi.LIB_PATH))
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_library_binds_with_declared_signatures():
    lib = _cabi.load_library()
    assert lib.hvdg_abi_version() == _cabi.HVDG_ABI_VERSION
    assert lib.hvdg_status_string(7) == b"HVDG_ERR_UNSUPPORTED"


def test_defaults_match_header_defaults():
    lib = _cabi.load_library()
    c = _cabi.Config()
    lib.hvdg_config_default(C.byref(c))
    d = _cabi.default_config()
    for name, _ in _cabi.Config._fields_:
        if name == "reserved":
            continue
        assert getattr(c, name) == pytest.approx(getattr(d, name)), name
    for std in (0, 1):
        g = _cabi.Geometry()
        lib.hvdg_geometry_default(std, C.byref(g))
        h = _cabi.default_geometry(std)
        for name, _ in _cabi.Geometry._fields_:
            assert getattr(g, name) == getattr(h, name), (std, name)


def test_struct_layouts_match_c(tmp_path):
    names = {"hvdg_geometry": _cabi.Geometry, "hvdg_config": _cabi.Config,
             "hvdg_frame_params": _cabi.FrameParams, "hvdg_field_in": _cabi.FieldIn,
             "hvdg_field_out": _cabi.FieldOut, "hvdg_yc_frame": _cabi.YcFrame,
             "hvdg_diag": _cabi.Diag}
    src = tmp_path / "sz.c"
    body = "".join(f'  printf("{n} %zu\\n", sizeof({n}));\n' for n in names)
    src.write_text(f'#include <stdio.h>\n#include "hvdg.h"\nint main(void){{\n{body}  return 0;\n}}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    for line in out.strip().splitlines():
        n, sz = line.split()
        assert C.sizeof(names[n]) == int(sz), n


def test_no_device_is_reported_not_faulted():
    """Without a CUDA device the context refuses with HVDG_ERR_NO_DEVICE."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _cabi.load_library()
    h = C.c_void_p()
    assert lib.hvdg_create(0, C.byref(h)) == _cabi.ERR_NO_DEVICE


def test_shim_library_exports_the_reference_entry_points():
    """The drop-in shim, built against the reference's headers, exports the
    reference's C++ frame-bridge functions (mangled hvd:: names) on top of
    the product library; no GPU needed to load it."""
    import subprocess
    from oracle import shim
    if not shim.available():
        pytest.skip("shim not built (needs the reference's headers)")
    shim.lib()
    syms = subprocess.run(["nm", "-D", "--defined-only", str(shim.LIB_PATH)],
                          capture_output=True, text=True).stdout
    for name in ("DecodeFrameSequenceWindow", "DecodeFrameBuffer", "DecodeYcFrameBuffer"):
        assert f"3hvd{len(name)}{name}" in syms, name
