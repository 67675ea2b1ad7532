"""Generates the committed golden fixtures in this directory by running the
REFERENCE engine itself (hvd-core compiled from its own sources by
oracle/Makefile into oracle/_ref/libhvdref.so) on small seeded synthetic
inputs. Run in the build container (it needs the reference tree to build
the library):  python tests/golden/make_golden.py

Small geometries keep the fixtures to a few hundred KB; the algorithms are
geometry-generic (the reference tests use the same trick, e.g.
lockin_test.cpp's 200-sample lines)."""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
sys.path.insert(0, str(REPO))

from hvdg import _cabi, synth  # noqa: E402
from oracle import ref  # noqa: E402


def small_geometry(std):
    g = _cabi.default_geometry(std)
    if std == _cabi.STD_PAL:
        return _cabi.geometry_copy(g, field_width=288, field_height=56, colour_burst_start=16,
                                   colour_burst_end=56, active_video_start=72,
                                   active_video_end=288, first_active_field_line=8)
    return _cabi.geometry_copy(g, field_width=256, field_height=48, colour_burst_start=16,
                               colour_burst_end=48, active_video_start=64, active_video_end=256,
                               first_active_field_line=8)


def geom_array(g):
    return np.array([g.field_width, g.field_height, g.active_video_start, g.active_video_end,
                     g.colour_burst_start, g.colour_burst_end, g.first_active_field_line,
                     g.last_active_field_line, g.standard], np.int64), np.float64(g.sample_rate)


def cfg_array(c):
    return np.array([c.irls_outer, c.cg_iterations, c.fast, c.cg_tol, c.temporal_strength,
                     c.chroma_aniso, c.lambda_c], np.float64)


def main():
    ref.set_threads(1)
    for std, tag, seed in ((_cabi.STD_NTSC, "ntsc", 101), (_cabi.STD_PAL, "pal", 202)):
        g = small_geometry(std)
        f = synth.make_field(seed, std, noise_sigma=0.5, geometry=g)
        ire = synth.to_ire(f.samples)
        cfg = _cabi.config_copy(_cabi.default_config(), irls_outer=3, cg_iterations=45, fast=0,
                                cg_tol=1e-6, temporal_strength=-1.0)
        theta, vsw = ref.burst_lockin(ire, g)
        amp = ref.burst_amplitude(ire, g)
        s, car = ref.prepare_field(ire, g, cfg, 0)
        y0, chi0 = ref.holographic_init(s, car, g, cfg)
        y, chi = ref.variational_refine(s, car, chi0, cfg, is_pal=(std == _cabi.STD_PAL))
        ys, cs, _ = ref.decode_field_window([ire], [0], g, cfg)
        ga, sr = geom_array(g)
        np.savez_compressed(
            HERE / f"field_{tag}_small.npz", samples=f.samples, geometry=ga, sample_rate=sr,
            cfg=cfg_array(cfg), theta=theta, vswitch=vsw, amplitude=np.float32(amp), s=s,
            carrier=car, y0=y0, chi0=chi0, y_refine=y, chi_refine=chi, y_decode=ys[0],
            chi_decode=cs[0], y_true=f.y_true, chi_true=f.chi_true)
    # motion: textured plane and a shifted copy (motion_test.cpp's construction,
    # own texture), tile 16 / search 8
    rng = np.random.default_rng(7)
    h, w = 96, 128
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    blocks = rng.uniform(-15, 15, size=(h // 4 + 1, w // 4 + 1))
    tex = (40 * np.sin(yy * 0.31) * np.cos(xx * 0.27) + 15 * np.sin(xx * 0.23 + yy * 0.17)
           + blocks[(yy // 4).astype(int), (xx // 4).astype(int)]).astype(np.float32)
    sy, sx = 3, -2
    cur = tex[np.clip(np.arange(h) - sy, 0, h - 1)][:, np.clip(np.arange(w) - sx, 0, w - 1)]
    dy, dx, cf = ref.estimate_motion(tex, cur, 16, 8)
    np.savez_compressed(HERE / "motion_small.npz", y_ref=tex, y_cur=cur, tile=16, search=8,
                        dy=dy, dx=dx, conf=cf, shift=np.array([sy, sx]))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
