"""hvdg: Python binding of the B200 holographic-variational Y/C separator.

The product is the C-ABI library ``lib/libhvdg.so`` (include/hvdg.h). This
package loads it with ctypes and mirrors the reference engine's interface
for tests, benchmarks and the research adjoint.
"""
from . import _cabi  # noqa: F401
