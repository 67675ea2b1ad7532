"""Burst lock-in (BurstLockinPhase / BurstLockinPhasePal, engine/lockin.cpp)
on fields whose bursts are missing on some lines: those lines get zero
weight in the trajectory smoother, which the device solves by parallel
cyclic reduction where the reference sweeps serially (TridiagSmooth,
lockin.cpp:65-99). Phases agree with the FP64 oracle to the float rounding
of the returned theta; the PAL V-switch sequence is identical."""
import numpy as np
import pytest

from hvdg import _cabi, synth
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu


def _wrap(a):
    return np.angle(np.exp(1j * a))


def _kill(ire, g, rows):
    out = ire.copy()
    out[rows, g.colour_burst_start:g.colour_burst_end] = 0.0
    return out


@pytest.mark.parametrize("std", [_cabi.STD_NTSC, _cabi.STD_PAL])
@pytest.mark.parametrize("pattern", ["ends_and_band", "one_good_line", "every_other"])
def test_lockin_with_missing_bursts_vs_oracle(ctx, std, pattern):
    g = _cabi.default_geometry(std)
    f = synth.make_field(41 + std, std, noise_sigma=0.5)
    ire = synth.to_ire(f.samples).astype(np.float32)
    h = g.field_height
    if pattern == "ends_and_band":
        rows = np.r_[0:5, 100:112, h - 3:h]
    elif pattern == "one_good_line":
        rows = np.r_[0:150, 151:h]
    else:
        rows = np.r_[30:h:2]
    ire = _kill(ire, g, rows)
    th, sw = ctx.burst_lockin(ire, g)
    if std == _cabi.STD_PAL:
        tho, swo = O.burst_lockin_phase_pal(ire.astype(np.float64), g)
        assert (sw == swo).all()
    else:
        tho = O.burst_lockin_phase(ire.astype(np.float64), g)
    d = np.abs(_wrap(th.astype(np.float64) - tho))
    print(f"std={std} {pattern}: max |dtheta| {d.max():.2e} rad")
    assert d.max() < 1e-4
