"""Selective 3-D detector (AmbiguousBoxes, frame_bridge.cpp:402-580), no GPU:

* the oracle's restatement (oracle/hvd_oracle.py: ambiguous_boxes) and the
  library's host implementation (hvdg_ambiguous_boxes) give the same boxes
  on the compiled reference's own 2-D decode of a window;
* the compiled reference's selective decode (DecodeWindowSelective,
  frame_bridge.cpp:596-718) differs from its plain 2-D decode only inside
  those boxes -- which pins the restatement to the reference's behaviour.

Scenes: flat, colourless content with a localized luma grating near the
subcarrier (hvdg.synth.grille_scene), NTSC static and PAL with moving
rectangles (two bands)."""
import numpy as np
import pytest

from hvdg import _cabi, api, synth

CFG2D = dict(irls_outer=2, cg_iterations=16, fast=1, cg_tol=1e-6)
CFG3D = dict(CFG2D, temporal_strength=0.5, passes=1, nr_anchor=0.0, coherence_gate=0.0,
             trajectory_fit=0)


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    return ref


def _window(std, n_rects):
    sc = synth.grille_scene(7, std, n_rects=n_rects)
    frames, _ = synth.make_frames(7, std, 3, noise_sigma=0.7, moving=n_rects > 0, scene=sc)
    return frames, api.frame_params(std)


@pytest.mark.parametrize("std,n_rects,n_boxes", [(_cabi.STD_NTSC, 0, 1), (_cabi.STD_PAL, 2, 2)])
def test_boxes_oracle_vs_library_vs_reference(std, n_rects, n_boxes):
    from oracle import hvd_oracle as O
    ref = _ref()
    frames, fp = _window(std, n_rects)
    g = _cabi.default_geometry(std)
    fields, par = [], []
    for f in frames:
        t, b = ref.split_frame_fields(f, fp)
        fields += [t, b]
        par += [0, 1]
    ys, cs, _ = ref.decode_field_window(fields, par, g, api.default_config(temporal_strength=-1.0,
                                                                            **CFG2D))
    boxes = O.ambiguous_boxes(ys[0], cs[0])
    assert boxes == api.ambiguous_boxes(ys[0], cs[0])
    assert boxes is not None and len(boxes) == n_boxes
    # the reference's selective window moves only the pixels inside the boxes
    sel = ref.decode_frame_sequence_window(frames, 1, 2, fp,
                                           api.default_config(selective_3d=1, **CFG3D))
    two = ref.decode_frame_sequence_window(frames, 1, 2, fp,
                                           api.default_config(temporal_strength=-1.0, **CFG2D))
    inside = np.zeros((fp.frame_height, fp.frame_width), bool)
    fal, a0, f1 = g.first_active_field_line, g.active_video_start, fp.field1_lines
    for fy0, fy1, x0, x1 in boxes:
        inside[fal + fy0:fal + fy1, a0 + x0:a0 + x1] = True
        inside[f1 + fal + fy0:f1 + fal + fy1, a0 + x0:a0 + x1] = True
    for key in ("luma", "chroma", "u", "v"):
        moved = (sel[0][key] != two[0][key]).reshape(inside.shape)
        assert moved.any(), key
        assert not (moved & ~inside).any(), key


def test_boxes_edge_cases():
    from oracle import hvd_oracle as O
    h, w = 242, 760
    rng = np.random.default_rng(3)
    # flat with a little noise: no tile reaches 4 x the median, stay 2-D
    flat_y = (50 + 0.2 * rng.standard_normal((h, w))).astype(np.float32)
    flat_c = (0.2 * (rng.standard_normal((h, w)) + 1j * rng.standard_normal((h, w)))).astype(
        np.complex64)
    assert O.ambiguous_boxes(flat_y, flat_c) == [] == api.ambiguous_boxes(flat_y, flat_c)
    # exactly flat: every score is 0 = 4 x the median, every tile counts,
    # the boxes overflow the area cap -> full 3-D (the reference's degenerate case)
    zy, zc = np.full((h, w), 50.0, np.float32), np.zeros((h, w), np.complex64)
    assert O.ambiguous_boxes(zy, zc) is None and api.ambiguous_boxes(zy, zc) is None
    # uniformly textured (median above 3 IRE^2, no localized peak): full 3-D
    y = (50 + 6 * rng.standard_normal((h, w))).astype(np.float32)
    c = (6 * (rng.standard_normal((h, w)) + 1j * rng.standard_normal((h, w)))).astype(np.complex64)
    assert O.ambiguous_boxes(y, c) is None and api.ambiguous_boxes(y, c) is None
