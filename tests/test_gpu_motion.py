"""GPU motion estimation (EstimateMotion, motion.cpp:397-488) against the
reference engine's own outputs: bit-exact vectors and confidences."""
from pathlib import Path

import numpy as np
import pytest

from hvdg import synth, _cabi
from oracle import hvd_oracle as O

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def test_motion_bit_exact_vs_reference_golden(ctx):
    d = np.load(GOLD / "motion_small.npz")
    dy, dx, cf = ctx.estimate_motion(d["y_ref"], d["y_cur"], int(d["tile"]), int(d["search"]))
    assert np.array_equal(dy, d["dy"])
    assert np.array_equal(dx, d["dx"])
    assert np.array_equal(cf, d["conf"])


@pytest.mark.parametrize("std,tile,search", [(_cabi.STD_NTSC, 32, 16), (_cabi.STD_PAL, 16, 8),
                                             (_cabi.STD_NTSC, 80, 8)])
def test_motion_full_field_vs_reference(ctx, std, tile, search):
    """Two consecutive same-parity fields' init luma, full field size. Tiles
    up to 64 rows refine with a warp per tile (the visit replayed from
    per-row sums), larger ones with a thread per tile: both bit-exact."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    seq = synth.make_sequence(5 + std, std, 3, moving=True)
    g = _cabi.default_geometry(std)
    cfg = _cabi.default_config()
    ys = []
    for f in (seq[0], seq[2]):
        s, c = ref.prepare_field(synth.to_ire(f.samples), g, cfg)
        y0, _ = ref.holographic_init(s, c, g, cfg)
        ys.append(y0)
    dy, dx, cf = ctx.estimate_motion(ys[0], ys[1], tile, search)
    rdy, rdx, rcf = ref.estimate_motion(ys[0], ys[1], tile, search)
    assert np.array_equal(dy, rdy) and np.array_equal(dx, rdx) and np.array_equal(cf, rcf)
    ody, odx, _ = O.estimate_motion(ys[0], ys[1], tile, search)
    # FP64 oracle: same vectors up to float rounding of the sub-pel fit
    agree = (np.abs(ody - dy) < 1e-3) & (np.abs(odx - dx) < 1e-3)
    assert agree.mean() > 0.95


def _sad_pair(kind):
    if kind == "ntsc" or kind == "pal":
        std = _cabi.STD_NTSC if kind == "ntsc" else _cabi.STD_PAL
        seq = synth.make_sequence(9 + std, std, 3, moving=True)
        return seq[0].y_true.astype(np.float32), seq[2].y_true.astype(np.float32)
    rng = np.random.default_rng(17)
    a = (rng.normal(50, 25, size=(37, 53))).astype(np.float32)
    b = np.roll(a, (2, -3), axis=(0, 1)) + rng.normal(0, 1, size=a.shape).astype(np.float32)
    return a, b.astype(np.float32)


@pytest.mark.parametrize("kind,block,rng_", [("ntsc", 16, 16), ("pal", 16, 16), ("odd", 16, 5),
                                             ("odd", 8, 7), ("ntsc", 32, 22)])
def test_sad_motion_bit_exact_vs_restatement(ctx, kind, block, rng_):
    """Integer-SAD mode (me_mode 1) against its CPU restatement: identical
    vectors, sub-pel offsets and confidences, including partial edge
    blocks and ties."""
    a, b = _sad_pair(kind)
    dy, dx, cf = ctx.estimate_motion(a, b, block, rng_, me_mode=1)
    ody, odx, ocf = O.estimate_motion_sad(a, b, block, rng_)
    assert np.array_equal(dy, ody)
    assert np.array_equal(dx, odx)
    assert np.array_equal(cf, ocf)


@pytest.mark.parametrize("kind,tile", [("ntsc", 32), ("pal", 32), ("odd", 16)])
def test_verify_motion_bit_exact_vs_reference(ctx, kind, tile):
    """VerifyMotion (motion.cpp:490-530) -- the fast 3-D window's audit of
    its trajectory predictions -- through hvdg_verify_motion against the
    compiled reference: identical vectors and confidences, with predictions
    that win (near the true shift), lose to zero and tie with it."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    if kind == "odd":
        a, b = _sad_pair("odd")
    else:
        std = _cabi.STD_NTSC if kind == "ntsc" else _cabi.STD_PAL
        seq = synth.make_sequence(19 + std, std, 3, moving=True)
        a, b = seq[0].y_true.astype(np.float32), seq[2].y_true.astype(np.float32)
    h, w = a.shape
    th, tw = -(-h // tile), -(-w // tile)
    rng = np.random.default_rng(tile + h)
    mdy, mdx, _ = ctx.estimate_motion(a, b, tile, 8)
    # predictions: the searched vectors, perturbed by up to +-1.5 px, some
    # exactly zero (ties with the zero candidate)
    pdy = (mdy + rng.uniform(-1.5, 1.5, (th, tw))).astype(np.float32)
    pdx = (mdx + rng.uniform(-1.5, 1.5, (th, tw))).astype(np.float32)
    pdy[rng.random((th, tw)) < 0.15] = 0.0
    pdx[rng.random((th, tw)) < 0.15] = 0.0
    dy, dx, cf = ctx.verify_motion(a, b, pdy, pdx, tile)
    rdy, rdx, rcf = ref.verify_motion(a, b, pdy, pdx, tile)
    kept = (dy == pdy) & (dx == pdx)
    print(f"{kind} tile {tile}: {kept.mean():.2f} of the predictions kept")
    assert 0.0 < kept.mean() < 1.0
    assert np.array_equal(dy, rdy) and np.array_equal(dx, rdx) and np.array_equal(cf, rcf)
