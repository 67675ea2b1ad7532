"""Seeded synthetic composite fields (the benchmark workloads).

The reference publishes no dataset for this path; its own quality benches
are synthetic (research/bench_*.py). These generators build the workloads
the benchmark configurations describe, from a seed:

* luma: 20 random Gaussian blobs + 5 random-orientation step edges, clipped
  to 0..100 IRE;
* chroma: I/Q (NTSC) or U/V (PAL) patches uniform in +/-40 IRE, low-passed
  horizontally (Gaussian, sigma_f = 1.3 MHz for I / U / V, 0.5 MHz for Q);
* composite S = Y + Re[chi * c], chi = V - iU, with the carrier
  c = exp(i phi) on NTSC and the PAL V-switch folded in as
  c = -exp(-i phi) on switched lines (ntsc_geometry.h:8-11, 241-253);
  phi = theta_field + adv * line + (pi/2) * sample, adv = pi (NTSC) or
  2 pi * 0.7516 (PAL), and per-field phase steps of 270 deg (NTSC) /
  135 deg (PAL) so consecutive fields keep the physical carrier relation;
* every line: a -40 IRE sync pulse, a burst at 180 deg (NTSC, +/-20 IRE,
  9 cycles) or +/-135 deg (PAL, 21.43 IRE, 10 cycles) covering the burst
  window;
* Gaussian noise, then quantisation to uint16 with 0 IRE = 16384 and
  100 IRE = 51200 (348.16 codes per IRE).

Moving sequences add four foreground rectangles translating by seeded
per-frame motions of up to +/-12 px and +/-6 lines (integer + half-pel),
rendered with exact area coverage so half-pel positions are meaningful.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _cabi

BLANK_CODE = 16384.0
WHITE_CODE = 51200.0
CODES_PER_IRE = (WHITE_CODE - BLANK_CODE) / 100.0


@dataclass
class FieldSample:
    samples: np.ndarray          # (field_height, field_width) uint16
    parity: int
    standard: int
    y_true: np.ndarray           # (active_lines, active_width) float32 IRE
    chi_true: np.ndarray         # (active_lines, active_width) complex64 IRE
    theta_true: np.ndarray       # (field_height,) float64 carrier phase at sample 0
    vswitch_true: np.ndarray     # (field_height,) int8
    noise_sigma: float = 0.0
    irls_outer: int = 0
    cg_iterations: int = -1


@dataclass
class Scene:
    """A static background plus optional moving rectangles, evaluated on the
    frame grid (frame row = 2 * field line + parity)."""
    rng_seed: int
    standard: int
    frame_rows: int
    width: int
    blobs: list = field(default_factory=list)
    edges: list = field(default_factory=list)
    patches: list = field(default_factory=list)
    rects: list = field(default_factory=list)
    grilles: list = field(default_factory=list)


def _lowpass_rows(a: np.ndarray, sigma_px: float) -> np.ndarray:
    """Gaussian low-pass along x (rows), zero-phase, reflect-padded."""
    if sigma_px <= 0:
        return a
    r = int(np.ceil(4 * sigma_px))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma_px) ** 2)
    k /= k.sum()
    ap = np.pad(a, ((0, 0), (r, r)), mode="reflect")
    out = np.zeros_like(a, dtype=np.float64)
    for i, kv in enumerate(k):
        out += kv * ap[:, i:i + a.shape[1]]
    return out


def make_scene(seed: int, standard: int, n_rects: int = 0,
               geometry: _cabi.Geometry | None = None, grille=None) -> Scene:
    """`grille` (optional): (r0, r1, c0, c1, period_px, amp_ire) with the
    box in fractions of the frame -- a localized luma grating near the
    subcarrier (a fan grille / blinds), the Y/C-ambiguous content selective
    3-D targets."""
    g = geometry or _cabi.default_geometry(standard)
    rng = np.random.default_rng(seed)
    rows = 2 * g.active_lines
    w = g.active_width
    sc = Scene(seed, standard, rows, w)
    for _ in range(20):
        sc.blobs.append((rng.uniform(0, rows), rng.uniform(0, w),
                         rng.uniform(6, 60), rng.uniform(8, 120),
                         rng.uniform(-45, 45)))
    for _ in range(5):
        ang = rng.uniform(0, np.pi)
        sc.edges.append((np.cos(ang), np.sin(ang), rng.uniform(-0.4, 0.4),
                         rng.uniform(-30, 30)))
    for _ in range(14):
        r0 = rng.uniform(-0.1, 0.9) * rows
        c0 = rng.uniform(-0.1, 0.9) * w
        sc.patches.append((r0, r0 + rng.uniform(0.15, 0.6) * rows,
                           c0, c0 + rng.uniform(0.1, 0.5) * w,
                           rng.uniform(-40, 40), rng.uniform(-40, 40)))
    for _ in range(n_rects):
        hh = rng.uniform(0.12, 0.3) * rows
        ww = rng.uniform(0.08, 0.22) * w
        sc.rects.append(dict(
            r0=rng.uniform(0.1, 0.9) * rows - hh / 2, c0=rng.uniform(0.1, 0.9) * w - ww / 2,
            h=hh, w=ww,
            # per-frame motion: integer or half-pel, +/-12 px, +/-6 frame lines
            vx=rng.integers(-24, 25) / 2.0, vy=rng.integers(-12, 13) / 2.0,
            y=rng.uniform(10, 90), a=rng.uniform(-40, 40), b=rng.uniform(-40, 40)))
    if grille is not None:
        r0, r1, c0, c1, period, amp = grille
        sc.grilles.append((r0 * rows, r1 * rows, c0 * w, c1 * w, period, amp))
    return sc


def _coverage_1d(lo: float, hi: float, n: int) -> np.ndarray:
    """Fraction of each unit cell [i, i+1) covered by [lo, hi)."""
    i = np.arange(n, dtype=np.float64)
    return np.clip(np.minimum(i + 1, hi) - np.maximum(i, lo), 0.0, 1.0)


def render(sc: Scene, frame_rows: np.ndarray, t_frames: float):
    """Luma (IRE), chroma components (a, b) at the given frame rows (float
    array, one per output line), all columns. a/b are I/Q on NTSC, U/V on
    PAL, before horizontal band limiting."""
    w = sc.width
    x = np.arange(w, dtype=np.float64)[None, :]
    y = frame_rows.astype(np.float64)[:, None]
    luma = np.full((len(frame_rows), w), 50.0)
    for (cy, cx, sy, sx, amp) in sc.blobs:
        luma += amp * np.exp(-0.5 * (((y - cy) / sy) ** 2 + ((x - cx) / sx) ** 2))
    for (nx, ny, off, step) in sc.edges:
        d = nx * (x / w - 0.5) + ny * (y / sc.frame_rows - 0.5) - off
        luma += step * (d > 0)
    ca = np.zeros_like(luma)
    cb = np.zeros_like(luma)
    for (r0, r1, c0, c1, va, vb) in sc.patches:
        m = (y >= r0) & (y < r1) & (x >= c0) & (x < c1)
        ca = np.where(m, va, ca)
        cb = np.where(m, vb, cb)
    for (r0, r1, c0, c1, period, amp) in sc.grilles:
        m = (y >= r0) & (y < r1) & (x >= c0) & (x < c1)
        luma = luma + np.where(m, amp * np.cos(2 * np.pi * x / period), 0.0)
    for r in sc.rects:
        rr0 = r["r0"] + r["vy"] * t_frames
        cc0 = r["c0"] + r["vx"] * t_frames
        cov_x = _coverage_1d(cc0, cc0 + r["w"], w)[None, :]
        # rows are sampled at frame_rows (points); coverage of a 1-line cell
        cov_y = np.clip(np.minimum(y + 1.0, rr0 + r["h"]) - np.maximum(y, rr0), 0, 1)
        cov = cov_y * cov_x
        luma = luma * (1 - cov) + r["y"] * cov
        ca = ca * (1 - cov) + r["a"] * cov
        cb = cb * (1 - cov) + r["b"] * cov
    return np.clip(luma, 0.0, 100.0), ca, cb


def _field_phase(standard: int, field_index: int, base: float) -> float:
    # carrier phase steps per field: NTSC 0.75 cycle (270 deg), PAL 0.375 (135 deg)
    step = 1.5 * np.pi if standard == _cabi.STD_NTSC else 0.75 * np.pi
    return base + step * field_index


def make_field(seed: int, standard: int = _cabi.STD_NTSC, noise_sigma: float = 0.5,
               field_index: int = 0, parity: int | None = None, scene: Scene | None = None,
               theta_base: float | None = None,
               geometry: _cabi.Geometry | None = None, return_parts: bool = False):
    """One composite field as uint16 codes, plus its ground truth. With
    return_parts: (field, luma part, chroma part, noise) in IRE, the parts
    being the noiseless luma (+ sync) and chroma (+ burst) of the field."""
    g = geometry or _cabi.default_geometry(standard)
    rng = np.random.default_rng(np.uint64(seed) * np.uint64(7919) + np.uint64(field_index))
    sc = scene or make_scene(seed, standard, geometry=g)
    if parity is None:
        parity = field_index % 2
    fh, fw = g.field_height, g.field_width
    fal, lal = g.first_active_field_line, g.last_active_line
    a0, a1 = g.active_video_start, g.active_video_end
    lines = lal - fal
    if theta_base is None:
        theta_base = float(np.random.default_rng(seed + 17).uniform(-np.pi, np.pi))
    th0 = _field_phase(standard, field_index, theta_base)
    pal = standard in (_cabi.STD_PAL, _cabi.STD_PAL_M)
    adv = 2 * np.pi * 0.7516 if standard == _cabi.STD_PAL else (
        0.5 * np.pi if standard == _cabi.STD_PAL_M else np.pi)
    line_idx = np.arange(fh)
    theta = th0 + adv * line_idx
    # V-switch alternates per line; its phase per field alternates too
    vsw = np.where(((line_idx + field_index) % 2) == 0, 1, -1).astype(np.int8) if pal \
        else np.ones(fh, np.int8)

    # scene in the active window
    frame_rows = 2.0 * np.arange(lines) + parity
    t = field_index / 2.0
    luma, ca, cb = render(sc, frame_rows, t)
    fs = g.sample_rate
    sig_a = fs / (2 * np.pi * 1.3e6)
    sig_b = fs / (2 * np.pi * (1.3e6 if pal else 0.5e6))
    ca = _lowpass_rows(ca, sig_a)
    cb = _lowpass_rows(cb, sig_b)
    if pal:
        u, v = ca, cb
    else:
        # I/Q -> U/V (33 deg rotation)
        s33, c33 = np.sin(np.deg2rad(33.0)), np.cos(np.deg2rad(33.0))
        u = -ca * s33 + cb * c33
        v = ca * c33 + cb * s33
    chi = v - 1j * u

    xs = np.arange(fw)
    w0 = 0.5 * np.pi
    if g.subcarrier_hz > 0.0:
        # a declared subcarrier: w0 = 2 pi fsc / fs, per-line advance from the
        # fractional cycles per line (FieldGeometry::phase_per_sample /
        # line_advance, ntsc_geometry.h:124-177)
        w0 = 2.0 * np.pi * g.subcarrier_hz / g.sample_rate
        cyc = g.subcarrier_hz * fw / g.sample_rate
        theta = th0 + 2.0 * np.pi * (cyc - np.floor(cyc)) * line_idx
    phi = theta[:, None] + w0 * xs[None, :]
    car = np.exp(1j * phi)
    if pal:
        car = np.where(vsw[:, None] < 0, -np.conj(car), car)

    # luma part (active luma + sync) and chroma part (active chroma + burst)
    y_part = np.zeros((fh, fw))
    c_part = np.zeros((fh, fw))
    y_part[fal:lal, a0:a1] = luma
    c_part[fal:lal, a0:a1] = np.real(chi * car[fal:lal, a0:a1])
    # sync pulse (4.7 us)
    sync_len = min(int(round(4.7e-6 * fs)), max(0, g.colour_burst_start - 8))
    y_part[:, :sync_len] = -40.0
    # burst: 9 (NTSC) / 10 (PAL) cycles centred on the burst window
    b0, b1 = g.colour_burst_start, g.colour_burst_end
    ncyc = 10 if pal else 9
    blen = 4 * ncyc
    bs = (b0 + b1) // 2 - blen // 2
    amp = 21.43 if standard == _cabi.STD_PAL else 20.0
    if pal:
        chi_b = amp * (np.sin(np.pi / 4) + 1j * np.cos(np.pi / 4))
    else:
        chi_b = 1j * amp
    c_part[:, bs:bs + blen] = np.real(chi_b * car[:, bs:bs + blen])
    ire = y_part + c_part
    noise = rng.normal(0.0, noise_sigma, size=ire.shape)
    ire += noise
    codes = np.clip(np.rint(BLANK_CODE + ire * CODES_PER_IRE), 0, 65535).astype(np.uint16)
    fsmp = FieldSample(codes, parity, standard, luma.astype(np.float32),
                       chi.astype(np.complex64), theta, vsw, noise_sigma)
    if return_parts:
        return fsmp, y_part, c_part, noise
    return fsmp


def make_sequence(seed: int, standard: int, n_fields: int, noise_sigma: float = 0.5,
                  moving: bool = True, grille=None, scene: Scene | None = None
                  ) -> list[FieldSample]:
    """Consecutive fields (two per frame, parity alternating) of one scene
    (`scene` overrides the seeded one)."""
    sc = scene or make_scene(seed, standard, n_rects=4 if moving else 0, grille=grille)
    base = float(np.random.default_rng(seed + 17).uniform(-np.pi, np.pi))
    return [make_field(seed, standard, noise_sigma, field_index=j, parity=j % 2,
                       scene=sc, theta_base=base) for j in range(n_fields)]


def to_ire(codes: np.ndarray) -> np.ndarray:
    """SampleToIre (ntsc_geometry.h:225-228) with the synthetic levels."""
    return ((codes.astype(np.float32) - np.float32(BLANK_CODE)) /
            np.float32((WHITE_CODE - BLANK_CODE) / 100.0)).astype(np.float32)


def mixed_batch(seed: int, n_ntsc: int = 40, n_pal: int = 24,
                outer_range=(4, 12), cg_per_outer: int = 50) -> list[FieldSample]:
    """The batched mixed workload: NTSC and PAL fields in seeded random
    order, per-field noise sigma ~ U[0.2, 2] IRE and per-field IRLS count
    ~ U{outer_range}, cg_per_outer CG iterations per outer."""
    rng = np.random.default_rng(seed)
    stds = [_cabi.STD_NTSC] * n_ntsc + [_cabi.STD_PAL] * n_pal
    rng.shuffle(stds)
    out = []
    for i, s in enumerate(stds):
        sigma = float(rng.uniform(0.2, 2.0))
        outer = int(rng.integers(outer_range[0], outer_range[1] + 1))
        f = make_field(seed * 1000 + i, s, sigma, field_index=i % 4, parity=i % 2)
        f.irls_outer = outer
        f.cg_iterations = outer * cg_per_outer
        out.append(f)
    return out


def make_frames(seed: int, standard: int, n_frames: int, noise_sigma: float = 0.5,
                moving: bool = False, blanking: float = 240.0, white: float = 800.0,
                grille=None, scene: Scene | None = None, field1_bottom=False):
    """Field-sequential 10-bit int16 frame buffers (the plugin's CVBS frame
    layout, frame_bridge.h:12-23): field 1 lines, then field 2 lines, with the
    PAL extra samples on frame lines 312 and 624. field1_bottom (a bool, or
    one per frame): field 1 is the bottom (odd-parity) field of the pair.
    Returns (frames, fields)."""
    fields = make_sequence(seed, standard, 2 * n_frames, noise_sigma, moving, grille=grille,
                           scene=scene)
    g = _cabi.default_geometry(standard)
    fw = g.field_width
    if standard == _cabi.STD_PAL:
        fh, f1, extra = 625, 313, (312, 624)
    else:
        fh, f1, extra = 525, 263, ()
    f2 = fh - f1
    cpi = (white - blanking) / 100.0
    frames = []
    for t in range(n_frames):
        top = to_ire(fields[2 * t].samples)
        bot = to_ire(fields[2 * t + 1].samples)
        fb = field1_bottom[t] if isinstance(field1_bottom, (list, tuple)) else field1_bottom
        if fb:
            top, bot = bot, top
        lines = [top[y] for y in range(f1)] + [bot[y] for y in range(f2)]
        buf = []
        for i, ln in enumerate(lines):
            codes = np.clip(np.rint(blanking + ln * cpi), -32768, 32767).astype(np.int16)
            buf.append(codes)
            if i in extra:
                buf.append(codes[-2:])  # the two extra samples of this line
        frames.append(np.concatenate(buf))
    return frames, fields


def make_yc_frames(seed: int, standard: int, n_frames: int, noise_sigma: float = 0.5,
                   moving: bool = False, blanking: float = 240.0, white: float = 800.0,
                   chroma_dc: float = 512.0):
    """Y/C-native frame pairs in the same field-sequential int16 layout as
    make_frames: the Y channel (luma + sync, levels as make_frames) and the C
    channel (chroma + burst, centred on chroma_dc), each with its own noise.
    Returns (luma_frames, chroma_frames, fields)."""
    sc = make_scene(seed, standard, n_rects=4 if moving else 0)
    base = float(np.random.default_rng(seed + 17).uniform(-np.pi, np.pi))
    g = _cabi.default_geometry(standard)
    if standard == _cabi.STD_PAL:
        fh, f1, extra = 625, 313, (312, 624)
    else:
        fh, f1, extra = 525, 263, ()
    f2 = fh - f1
    cpi = (white - blanking) / 100.0
    rng = np.random.default_rng(seed + 101)
    ys, cs, fields = [], [], []
    for t in range(n_frames):
        parts = [make_field(seed, standard, noise_sigma, field_index=2 * t + k, parity=k,
                            scene=sc, theta_base=base, return_parts=True) for k in range(2)]
        fields += [p[0] for p in parts]
        yl = [parts[0][1][y] for y in range(f1)] + [parts[1][1][y] for y in range(f2)]
        cl = [parts[0][2][y] for y in range(f1)] + [parts[1][2][y] for y in range(f2)]
        ybuf, cbuf = [], []
        for i, (ly, lc) in enumerate(zip(yl, cl)):
            yc_ = np.rint(blanking + (ly + rng.normal(0, noise_sigma, ly.shape)) * cpi)
            cc_ = np.rint(chroma_dc + (lc + rng.normal(0, noise_sigma, lc.shape)) * cpi)
            yc_ = np.clip(yc_, -32768, 32767).astype(np.int16)
            cc_ = np.clip(cc_, -32768, 32767).astype(np.int16)
            ybuf.append(yc_)
            cbuf.append(cc_)
            if i in extra:
                ybuf.append(yc_[-2:])
                cbuf.append(cc_[-2:])
        ys.append(np.concatenate(ybuf))
        cs.append(np.concatenate(cbuf))
    return ys, cs, fields


def grille_scene(seed: int, standard: int, grille=(0.35, 0.6, 0.3, 0.55, 4.6, 18.0),
                 n_rects: int = 0) -> Scene:
    """A flat, colourless scene (one broad luma blob) with one localized luma
    grating near the subcarrier: the case selective 3-D is for -- the
    ambiguity detector should find the grating's box and nothing else."""
    g = _cabi.default_geometry(standard)
    rows, w = 2 * g.active_lines, g.active_width
    sc = Scene(seed, standard, rows, w)
    sc.blobs.append((rows / 2, w / 2, 0.6 * rows, 0.6 * w, 20.0))
    r0, r1, c0, c1, period, amp = grille
    sc.grilles.append((r0 * rows, r1 * rows, c0 * w, c1 * w, period, amp))
    rng = np.random.default_rng(seed)
    for _ in range(n_rects):
        hh, ww = rng.uniform(0.12, 0.2) * rows, rng.uniform(0.06, 0.12) * w
        sc.rects.append(dict(r0=rng.uniform(0.1, 0.9) * rows - hh / 2,
                             c0=rng.uniform(0.1, 0.9) * w - ww / 2, h=hh, w=ww,
                             vx=rng.integers(-8, 9) / 2.0, vy=rng.integers(-4, 5) / 2.0,
                             y=rng.uniform(30, 70), a=0.0, b=0.0))
    return sc
