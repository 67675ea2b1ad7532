"""Failure paths of the device-side waits, without a GPU fault.

The persistent solver's warps wait (bounded) on a field's phase flag before
taking a unit of the next phase. A wait that runs out must end the launch
with an error status the host reads (HVDG_ERR_DEVICE_TIMEOUT), and leave
the context usable. The test shortens the bound to one poll, so warps that
take a unit of the next phase while the current one is still running give
up; every other wait in the kernel keeps its bound, nothing traps, and the
next call (default bound) decodes the same fields to the same results."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth

pytestmark = pytest.mark.gpu


def _fields():
    fs = synth.mixed_batch(404, 2, 1, outer_range=(2, 3), cg_per_outer=10)
    return [api.Field(f.samples, _cabi.default_geometry(f.standard), parity=f.parity,
                      irls_outer=f.irls_outer, cg_iterations=f.cg_iterations) for f in fs]


def test_solver_wait_timeout_returns_status_and_context_recovers():
    cfg = api.default_config(fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    hf = _fields()
    with api.Context(0) as ctx:
        good = ctx.decode_fields(hf, cfg)
        ctx.set_device_wait_limit(1)
        with pytest.raises(api.HvdgError) as err:
            ctx.decode_fields(hf, cfg)
        assert err.value.status == _cabi.ERR_DEVICE_TIMEOUT, err.value
        assert "wait" in ctx.lib.hvdg_last_error(ctx._h).decode()
        ctx.set_device_wait_limit(0)       # back to the default bound
        again = ctx.decode_fields(hf, cfg)
        for a, b in zip(again, good):
            assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma)
