"""Benchmark: batched 2-D field decode on B200 (fields/s).

Workload (one step): 64 composite fields in one batch -- 40 NTSC 910x263
and 24 PAL 1135x313 uint16 fields in seeded random order, per-field noise
sigma ~ U[0.2, 2] IRE, per-field IRLS outer count ~ U{4..12} with 50 CG
iterations per outer, fixed iteration counts (cg_tol 1e-6, fast off),
temporal terms off. Synthetic data (hvdg.synth), seeded per rank.

  value     : fields/s with the inputs already resident in HBM
              (hvdg_decode_fields_device), device time from CUDA events on
              the library's stream, L2 flushed between steps.
  e2e       : the same through the host-buffer C ABI (hvdg_decode_fields),
              pinned uint16 inputs in, float Y/chi out, copies included,
              wall clock of the synchronous call.
  plain     : the one-field-per-launch path (hvdg_set_batching(ctx, 0)).
  roofline  : the IRLS+CG solver kernel, algorithmic bytes (92 B per active
              px per CG iteration + 80 B per active px per IRLS outer) over
              its event-timed duration, against the measured HBM copy peak.
  cpu_baseline : the reference engine (oracle/_ref, compiled from the
              reference sources) on a bounded sample of the same workload on
              the host cores (one quarter of the fields, counted by solver
              work relative to the workload's mean).
  parity    : outside the timed regions, the e2e call's planes against the
              reference engine's on the cpu_baseline sample and against the
              FP64 oracle on two of its fields: max |dY|, |dC| (IRE) and the
              PSNR deltas against ground truth (the metric's 0.05 dB clause).

--impl reference times the reference engine alone (rank 0), same metric,
one workload quarter per step, rotating through all four.
Multi-GPU (torchrun): each rank decodes its own 64-field batch (fields are
independent; no collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
sys.path.insert(0, str(REPO))

METRIC = "fields/s on 1 B200, batched FP32 vs plain per-field GPU, at <=0.05 dB PSNR delta"
N_NTSC, N_PAL = 40, 24
ALG_BYTES_ITER = 92.0    # per active px per CG iteration
ALG_BYTES_OUTER = 80.0   # per active px per IRLS outer


WORKLOADS = {
    # name: (n_ntsc, n_pal, irls range, CG per outer)
    "mixed64": (N_NTSC, N_PAL, (4, 12), 50),
    # profiling case: same kernels, working set (~260 MB) above L2, short solve
    "small16": (16, 0, (2, 2), 10),
    # profiling case that fills every SM: 32 NTSC fields (~0.6 GB), 2 x 20 CG
    "prof32": (32, 0, (2, 2), 20),
}


WORKLOAD_DESC = {
    "mixed64": "mixed-64: 40 NTSC 910x263 + 24 PAL 1135x313 uint16, irls U{4..12} x 50 CG",
    "small16": "small-16 (profiling): 16 NTSC 910x263 uint16, irls 2 x 10 CG",
    "prof32": "prof-32 (profiling): 32 NTSC 910x263 uint16, irls 2 x 20 CG",
}


def workload(seed: int, name: str = "mixed64"):
    from hvdg import synth
    nn, npal, outer, cg = WORKLOADS[name]
    return synth.mixed_batch(seed, nn, npal, outer_range=outer, cg_per_outer=cg)


def rank_workload(rank: int, name: str = "mixed64"):
    """Each rank decodes its own batch (fields are independent: weak
    scaling, no data-path collective)."""
    return workload(1000 + rank, name)


def max_over_ranks(values, dist, device):
    """Element-wise max of per-rank timings (the slowest rank sets the job
    time)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def throughput(fields_per_rank: int, steps: int, world: int, ms_total: float) -> float:
    """Whole-job fields/s: every rank's fields over the slowest rank's time."""
    return fields_per_rank * steps * world / (ms_total / 1000.0)


def solver_config():
    from hvdg import api
    return api.default_config(fast=0, cg_tol=1e-6, temporal_strength=-1.0)


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """Per-launch DRAM traffic of the solver on the mixed-64 workload, from
    the committed ncu summary (profiles/solver_traffic.json); None for the
    other workloads (not captured) or without the summary."""
    p = REPO / "profiles" / "solver_traffic.json"
    if name == "mixed64" and p.exists():
        try:
            return json.loads(p.read_text()).get("bytes_per_launch")
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"hvdg_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(fields, threads: int, outputs: bool = False):
    """Decode `fields` with the reference engine (OpenMP across fields, as
    parallel_across_fields does); returns seconds (and the decoded planes)."""
    from hvdg import _cabi, synth
    from oracle import ref
    ref.set_threads(threads)
    base = _cabi.config_copy(solver_config())
    geoms = [_cabi.default_geometry(f.standard) for f in fields]
    cfgs = [_cabi.config_copy(base, irls_outer=f.irls_outer, cg_iterations=f.cg_iterations)
            for f in fields]
    ires = [synth.to_ire(f.samples) for f in fields]
    t = time.perf_counter()
    res = ref.decode_fields(ires, [f.parity for f in fields], geoms, cfgs, across_fields=True)
    dt = time.perf_counter() - t
    return (dt, res) if outputs else dt


def field_work(f) -> float:
    """A field's solver work: active pixels x CG iteration budget."""
    from hvdg import _cabi
    g = _cabi.default_geometry(f.standard)
    return float(g.active_lines * g.active_width * f.cg_iterations)


def quarter_samples(fields, n_quarters: int = 4):
    """The workload cut into consecutive quarters; a CPU step decodes one
    quarter, successive steps rotate through them, so steps in multiples of
    four decode the whole workload."""
    q = (len(fields) + n_quarters - 1) // n_quarters
    return [fields[i:i + q] for i in range(0, len(fields), q)]


def field_equivalents(sample, fields) -> float:
    """`sample`'s solver work in units of the workload's mean work per
    field: the fields/s of a sample count the workload's fields it is
    worth, so a heavier or lighter sample does not bias the rate."""
    mean = sum(field_work(f) for f in fields) / len(fields)
    return sum(field_work(f) for f in sample) / mean


def _psnr(a, b, peak=100.0) -> float:
    d = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
    return float(10 * np.log10(peak ** 2 / np.mean(np.abs(d) ** 2)))


def parity_leg(fields, out, sample, ref_y, ref_c, n_oracle: int = 2):
    """Quality of the timed workload's outputs (the e2e call's planes),
    outside every timed region: against the reference engine on the CPU
    sample's fields, and against the FP64 oracle on the `n_oracle` lightest
    fields of that sample (one NTSC, one PAL), in a spawn pool. PSNR deltas
    are |PSNR(ours, truth) - PSNR(theirs, truth)| for luma and chroma."""
    from oracle import jobs

    def compare(ours, y, c, f):
        return (float(np.abs(ours.luma - y).max()), float(np.abs(ours.chroma - c).max()),
                abs(_psnr(ours.luma, f.y_true) - _psnr(y, f.y_true)),
                abs(_psnr(ours.chroma, f.chi_true) - _psnr(c, f.chi_true)))

    res = {}
    rows = [compare(out[i], ref_y[i], ref_c[i], fields[i]) for i in range(len(sample))]
    res["vs_reference"] = {"fields": len(rows), "max_dY_ire": max(r[0] for r in rows),
                           "max_dC_ire": max(r[1] for r in rows),
                           "max_psnr_delta_y_db": max(r[2] for r in rows),
                           "max_psnr_delta_c_db": max(r[3] for r in rows)}
    picks = []
    for std in (0, 1):
        cand = [i for i in range(len(sample)) if fields[i].standard == std]
        if cand:
            picks.append(min(cand, key=lambda i: field_work(fields[i])))
    picks = picks[:n_oracle]
    job_list = [(fields[i].samples, fields[i].standard, fields[i].parity,
                 dict(fast=0, cg_tol=1e-6, temporal_strength=-1.0,
                      irls_outer=fields[i].irls_outer, cg_iterations=fields[i].cg_iterations))
                for i in picks]
    orc = jobs.decode_fields_2d_parallel(job_list)
    rows = [compare(out[i], y, c, fields[i]) for i, (y, c, _) in zip(picks, orc)]
    res["vs_fp64_oracle"] = {"fields": [int(i) for i in picks],
                             "max_dY_ire": max(r[0] for r in rows),
                             "max_dC_ire": max(r[1] for r in rows),
                             "max_psnr_delta_y_db": max(r[2] for r in rows),
                             "max_psnr_delta_c_db": max(r[3] for r in rows)}
    worst = max(res["vs_fp64_oracle"]["max_psnr_delta_y_db"],
                res["vs_fp64_oracle"]["max_psnr_delta_c_db"],
                res["vs_reference"]["max_psnr_delta_y_db"],
                res["vs_reference"]["max_psnr_delta_c_db"])
    res["within_0p05_db"] = bool(worst <= 0.05)
    return res


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    from oracle import ref
    threads = os.cpu_count() or 1
    fields = workload(1000, args.workload)
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference engine library oracle/_ref/libhvdref.so was not built"}))
        return 0
    quarters = quarter_samples(fields)
    for i in range(args.warmup):
        run_reference(quarters[i % len(quarters)][:max(2, threads // 4)], threads)
    total, equiv = 0.0, 0.0
    for i in range(args.steps):
        sample = quarters[i % len(quarters)]
        total += run_reference(sample, threads)
        equiv += field_equivalents(sample, fields)
    v = equiv / total
    desc = (f"per step one quarter ({len(quarters[0])} fields) of the {len(fields)}-field workload, "
            f"rotating (steps in multiples of {len(quarters)} cover every field equally); "
            f"fields counted by solver work (active px x CG budget) relative to the workload's "
            f"mean; OpenMP across fields, {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "fields/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded hvdg.synth mixed NTSC/PAL batch)",
        "config": {"workload": WORKLOAD_DESC[args.workload], "sample": desc},
        "cpu_baseline": {"value": v, "unit": "fields/s", "cores": threads, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": "fields/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# The other configurations of the path (parity cases; measured, not the
# headline): one NTSC field; 16-field NTSC / PAL motion windows (3-D, integer
# SAD motion, 10 x 50); the adjoint on 8 NTSC fields (10 x 50).
CONFIGS = {
    "cfg0-ntsc1": "config 0: 1 NTSC 910x263 uint16 field, 5 IRLS x 30 CG, no motion",
    "cfg1-ntsc16-3d": "config 1: 16 NTSC fields (8 frames), moving rectangles, 3-D window "
                      "(strength 0.5, 1 pass, no anchor / gate / trajectory fit), integer-SAD "
                      "motion 16x16 +-16, 10 IRLS x 50 CG",
    "cfg2-pal16-3d": "config 2: 16 PAL 1135x313 fields, same motion, window and solver as config 1",
    "cfg4-adjoint8": "config 4: forward + adjoint of 8 NTSC fields, 10 IRLS x 50 CG, "
                     "gradients w.r.t. 4 scalars and the samples",
    "frames8-ntsc": "8 NTSC 910x525 int16 composite frames through DecodeFrameBuffer "
                    "(frame-weave 2-D decode, default HvdConfig), one frame per reference call, "
                    "one batch here",
    "yc8-pal": "8 PAL 1135x625 Y/C int16 frame pairs through DecodeYcFrameBuffer "
               "(chroma-only init, default HvdConfig)",
    "window6-ntsc": "DecodeFrameSequenceWindow (the plugin's call): 6 NTSC 910x525 int16 "
                    "composite frames of moving content, core frames 1-4, default HvdConfig "
                    "(adaptive 3-D strength; 2 passes, the second anchored, when it resolves "
                    "above 0; 4 IRLS x 2 CG, fast), host buffers",
}
FRAME_CONFIGS = ("frames8-ntsc", "yc8-pal", "window6-ntsc")


def config_cfg(name):
    from hvdg import api
    if name == "cfg0-ntsc1":
        return api.default_config(irls_outer=5, cg_iterations=150, fast=0, cg_tol=1e-6,
                                  temporal_strength=-1.0)
    if name in ("cfg1-ntsc16-3d", "cfg2-pal16-3d"):
        return api.default_config(irls_outer=10, cg_iterations=500, fast=0, cg_tol=1e-6,
                                  temporal_strength=0.5, passes=1, nr_anchor=0.0,
                                  coherence_gate=0.0, trajectory_fit=0, me_mode=1, me_block=16,
                                  me_range=16)
    return api.default_config(irls_outer=10, cg_iterations=500, fast=0, cg_tol=1e-6,
                              temporal_strength=-1.0)


def config_fields(name):
    from hvdg import _cabi, synth
    if name == "cfg0-ntsc1":
        return [synth.make_field(0, _cabi.STD_NTSC, 0.5)]
    if name == "cfg1-ntsc16-3d":
        return synth.make_sequence(101, _cabi.STD_NTSC, 16, noise_sigma=0.5, moving=True)
    if name == "cfg2-pal16-3d":
        return synth.make_sequence(102, _cabi.STD_PAL, 16, noise_sigma=0.5, moving=True)
    return [synth.make_field(200 + i, _cabi.STD_NTSC, 0.5) for i in range(8)]


def window_arm(args):
    """Core frames/s of the sequence window (DecodeFrameSequenceWindow, the
    call the decode-orc stage makes) through the public API, wall clock of
    the synchronous call with host buffers; or the reference's own call on
    the host cores."""
    from hvdg import _cabi, api, synth
    name = args.workload
    frames, _ = synth.make_frames(302, _cabi.STD_NTSC, 6, noise_sigma=0.5, moving=True)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = api.default_config()
    core = (1, 5)
    ncore = core[1] - core[0]
    npx = fp.frame_width * fp.frame_height
    in_bytes = 2 * api.frame_buffer_size(fp) * len(frames)
    out_bytes = (2 + 2 + 8 + 8) * npx * ncore
    if args.impl == "reference":
        from oracle import ref
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
            return 0
        threads = os.cpu_count() or 1
        ref.set_threads(threads)
        times = []
        for _ in range(max(1, min(args.steps, 3))):
            t = time.perf_counter()
            ref.decode_frame_sequence_window(frames, core[0], core[1], fp, cfg)
            times.append(time.perf_counter() - t)
        v = ncore * len(times) / sum(times)
        print(json.dumps({"impl": "reference", "metric": f"core frames/s ({CONFIGS[name]})",
                          "value": v, "unit": "frames/s", "n_gpus": 1, "steps": len(times),
                          "warmup": 0, "higher_is_better": True, "dtype": "f32",
                          "data": "synthetic (seeded hvdg.synth)",
                          "config": {"workload": CONFIGS[name]},
                          "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads,
                                           "kind": "reference",
                                           "sample": "one 6-frame window per step"},
                          "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return 0
    ctx = api.Context(0)
    for _ in range(args.warmup):
        ctx.decode_frame_sequence_window(frames, core[0], core[1], fp, cfg)
    wall, dev, launches = 0.0, 0.0, 0
    for _ in range(args.steps):
        t = time.perf_counter()
        ctx.decode_frame_sequence_window(frames, core[0], core[1], fp, cfg)
        wall += time.perf_counter() - t
        dev += ctx.last_diag.ms_total
        launches += ctx.last_diag.kernel_launches
    d = ctx.last_diag
    line = {"metric": f"core frames/s ({CONFIGS[name]})", "value": ncore * args.steps / wall,
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * wall / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded hvdg.synth)",
            "config": {"workload": CONFIGS[name], "timing": "wall clock of the synchronous "
                       "host-buffer call (uploads, kernels, host steps, downloads)"},
            "device_ms_per_step": dev / args.steps if dev > 0 else None,
            "resolved_strength": d.resolved_strength, "ambiguity_ire": d.ambiguity_ire,
            "gpu_launches": launches,
            "e2e": {"value": ncore * args.steps / wall, "unit": "frames/s",
                    "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": out_bytes}}
    print(json.dumps(line))
    ctx.close()
    return 0


def frame_arm(args, rank, world):
    """Frames/s of the woven-frame entry points through the public API (host
    int16 frames in, the four YcFrameS16 planes out; wall clock of the
    synchronous call), or of the reference's own per-frame calls."""
    if rank != 0:
        return 0
    from hvdg import _cabi, api, synth
    name = args.workload
    if name == "window6-ntsc":
        return window_arm(args)
    cfg = api.default_config()
    n = 8
    if name == "frames8-ntsc":
        std = _cabi.STD_NTSC
        frames, _ = synth.make_frames(300, std, n, noise_sigma=0.5, moving=True)
        ys = cs = None
    else:
        std = _cabi.STD_PAL
        ys, cs, _ = synth.make_yc_frames(301, std, n, noise_sigma=0.5, moving=True)
    fp = api.frame_params(std)
    if ys is not None:
        fp.chroma_dc = 512.0
    npx = fp.frame_width * fp.frame_height
    in_bytes = (2 if ys is not None else 1) * 2 * api.frame_buffer_size(fp) * n
    out_bytes = (2 + 2 + 8 + 8) * npx * n
    if args.impl == "reference":
        from oracle import ref
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
            return 0
        threads = os.cpu_count() or 1
        ref.set_threads(threads)
        times = []
        for _ in range(max(1, args.steps)):
            t = time.perf_counter()
            for k in range(n):
                if ys is None:
                    ref.decode_frame_buffer(frames[k], fp, cfg)
                else:
                    ref.decode_yc_frame_buffer(ys[k], cs[k], fp, cfg)
            times.append(time.perf_counter() - t)
        v = n * len(times) / sum(times)
        print(json.dumps({"impl": "reference", "metric": f"frames/s ({CONFIGS[name]})",
                          "value": v, "unit": "frames/s", "n_gpus": world, "steps": len(times),
                          "warmup": 0, "higher_is_better": True, "dtype": "f32",
                          "data": "synthetic (seeded hvdg.synth)",
                          "config": {"workload": CONFIGS[name]},
                          "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads,
                                           "kind": "reference",
                                           "sample": f"{n} frames per step, one call each"},
                          "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return 0
    import torch

    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        t.numpy()[...] = a
        return t

    def pinned_zeros(k, dt):
        return torch.zeros(k, dtype=dt, pin_memory=True)

    ctx = api.Context(0)
    keep = []
    if ys is None:
        frames = [pinned(f) for f in frames]
        keep += frames
        frames = [t.numpy() for t in frames]
    else:
        ys = [pinned(a) for a in ys]
        cs = [pinned(a) for a in cs]
        keep += ys + cs
        ys, cs = [t.numpy() for t in ys], [t.numpy() for t in cs]
    outs = []
    for _ in range(n):
        planes = dict(luma=pinned_zeros(npx, torch.int16), chroma=pinned_zeros(npx, torch.int16),
                      u=pinned_zeros(npx, torch.float64), v=pinned_zeros(npx, torch.float64))
        keep += list(planes.values())
        outs.append({k: t.numpy() for k, t in planes.items()})

    def step():
        if ys is None:
            return ctx.decode_frame_buffers(frames, fp, cfg, out=outs)
        return ctx.decode_yc_frame_buffers(ys, cs, fp, cfg, out=outs)

    for _ in range(args.warmup):
        step()
    wall, dev = 0.0, 0.0
    for _ in range(args.steps):
        t = time.perf_counter()
        step()
        wall += time.perf_counter() - t
        dev += ctx.last_diag.ms_total
    launches = ctx.last_diag.kernel_launches
    line = {"metric": f"frames/s ({CONFIGS[name]})", "value": n * args.steps / wall,
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded hvdg.synth)",
            "config": {"workload": CONFIGS[name], "timing": "wall clock of the synchronous "
                       "host-buffer call (uploads, kernels, downloads; pinned host frames and "
                       "output planes)"},
            "device_frames_per_s": n * args.steps / (dev / 1000.0) if dev > 0 else None,
            "device_note": "device time of the kernels (split to re-weave), copies excluded",
            "gpu_launches": launches * args.steps,
            "e2e": {"value": n * args.steps / wall, "unit": "frames/s",
                    "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": out_bytes}}
    print(json.dumps(line))
    ctx.close()
    return 0


def config_arm(args, rank, world):
    """One JSON line for a parity configuration: fields/s through the public
    API (host buffers, wall clock of the synchronous call, copies included)
    and the device time of the same calls from the library's events."""
    if rank != 0:
        return 0
    from hvdg import _cabi, api, synth
    name = args.workload
    cfg = config_cfg(name)
    fields = config_fields(name)
    geoms = [_cabi.default_geometry(f.standard) for f in fields]
    hf = [api.Field(f.samples, g, parity=f.parity) for f, g in zip(fields, geoms)]
    n = len(hf)
    if args.impl == "reference":
        from oracle import ref
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
            return 0
        if name == "cfg4-adjoint8":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no adjoint (no CPU counterpart to time)"}))
            return 0
        threads = os.cpu_count() or 1
        ref.set_threads(threads)
        ires = [synth.to_ire(f.samples) for f in fields]
        times = []
        for _ in range(max(1, args.steps)):
            t = time.perf_counter()
            if name == "cfg0-ntsc1":
                ref.decode_fields(ires, [f.parity for f in fields], geoms, [cfg] * n,
                                  across_fields=False)
            else:
                ref.decode_field_window(ires, [f.parity for f in fields], geoms[0], cfg)
            times.append(time.perf_counter() - t)
        v = n * len(times) / sum(times)
        print(json.dumps({"impl": "reference", "metric": f"fields/s ({CONFIGS[name]})",
                          "value": v, "unit": "fields/s", "n_gpus": world, "steps": len(times),
                          "warmup": 0, "higher_is_better": True, "dtype": "f32",
                          "data": "synthetic (seeded hvdg.synth)",
                          "config": {"workload": CONFIGS[name],
                                     "note": "the reference's float-SSD motion search "
                                             "(it has no integer-SAD mode)" if "3d" in name else ""},
                          "cpu_baseline": {"value": v, "unit": "fields/s", "cores": threads,
                                           "kind": "reference", "sample": f"{n} fields per step"},
                          "e2e": {"value": v, "unit": "fields/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return 0
    ctx = api.Context(0)
    extra = {}

    def step():
        if name == "cfg0-ntsc1":
            out = ctx.decode_fields(hf, cfg)
        elif name == "cfg4-adjoint8":
            out = ctx.decode_fields(hf, cfg)
            yb, cb = [], []
            for d, f in zip(out, fields):
                npx = d.luma.size
                yb.append((2 * (d.luma - f.y_true) / npx).astype(np.float32))
                cb.append((2 * (d.chroma - f.chi_true) / npx).astype(np.complex64))
            ctx.decode_fields_adjoint(hf, cfg, yb, cb, 300)
        else:
            out = ctx.decode_field_window(hf, cfg)
        return out

    for _ in range(args.warmup):
        step()
    wall, dev = 0.0, 0.0
    for _ in range(args.steps):
        t = time.perf_counter()
        out = step()
        wall += time.perf_counter() - t
        dev += ctx.last_diag.ms_total
    psnr = []
    for d, f in zip(out, fields):
        dd = d.luma.astype(np.float64) - f.y_true
        psnr.append(10 * np.log10(100.0 ** 2 / np.mean(dd * dd)))
    line = {"metric": f"fields/s ({CONFIGS[name]})", "value": n * args.steps / wall,
            "unit": "fields/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded hvdg.synth)",
            "config": {"workload": CONFIGS[name], "timing": "wall clock of the synchronous "
                       "host-buffer call (uploads, kernels, downloads)"},
            "device_ms_per_step_last_call": dev / args.steps if name != "cfg4-adjoint8" else None,
            "psnr_y_db_mean": float(np.mean(psnr))}
    line.update(extra)
    print(json.dumps(line))
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--workload", default="mixed64", choices=sorted(WORKLOADS) + sorted(CONFIGS))
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload in FRAME_CONFIGS:
        return frame_arm(args, rank, world)
    if args.workload in CONFIGS:
        return config_arm(args, rank, world)
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)

    from hvdg import _cabi, api
    cfg = solver_config()
    fields = rank_workload(rank, args.workload)
    ctx = api.Context(local)

    # ---- device-resident inputs / outputs ----
    n = len(fields)
    geoms = [_cabi.default_geometry(f.standard) for f in fields]
    d_in = [torch.from_numpy(f.samples.view(np.int16)).cuda() for f in fields]
    d_y = [torch.empty((g.active_lines, g.active_width), dtype=torch.float32, device="cuda")
           for g in geoms]
    d_c = [torch.empty((g.active_lines, g.active_width, 2), dtype=torch.float32, device="cuda")
           for g in geoms]
    fin = (_cabi.FieldIn * n)()
    fout = (_cabi.FieldOut * n)()
    for i, f in enumerate(fields):
        fin[i].samples = d_in[i].data_ptr()
        fin[i].sample_type = _cabi.SAMPLES_U16
        fin[i].parity = f.parity
        fin[i].blanking_level = 16384.0
        fin[i].white_level = 51200.0
        fin[i].geometry = C.pointer(geoms[i])
        fin[i].irls_outer = f.irls_outer
        fin[i].cg_iterations = f.cg_iterations
        fout[i].luma = d_y[i].data_ptr()
        fout[i].chroma = d_c[i].data_ptr()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        ctx.decode_fields_device(fin, fout, n, cfg)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ms_total = ms_solver = 0.0
    pix_iters = pix_outers = 0
    launches = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        d = ctx.decode_fields_device(fin, fout, n, cfg)
        ms_total += d.ms_total
        ms_solver += d.ms_solver
        pix_iters += d.solver_pixel_iters
        pix_outers += d.solver_pixel_outers
        launches += d.kernel_launches
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    if dist is not None:
        ms_total, ms_solver = max_over_ranks([ms_total, ms_solver], dist, "cuda")
        dist.barrier()

    # ---- e2e through the host-buffer API (pinned in/out) ----
    pin_in = []
    for f in fields:
        t = torch.empty(f.samples.shape, dtype=torch.int16, pin_memory=True)
        t.numpy()[...] = f.samples.view(np.int16)
        pin_in.append(t)
    host_fields = [api.Field(pin_in[i].numpy().view(np.uint16), geoms[i], parity=f.parity,
                             irls_outer=f.irls_outer, cg_iterations=f.cg_iterations)
                   for i, f in enumerate(fields)]
    # page-locked output buffers, allocated once and reused every step
    pin_out = []
    for g in geoms:
        ty = torch.empty((g.active_lines, g.active_width), dtype=torch.float32, pin_memory=True)
        tc = torch.empty((g.active_lines, g.active_width, 2), dtype=torch.float32, pin_memory=True)
        pin_out.append((ty, tc))
    host_out = [api.Decoded(ty.numpy(), tc.numpy().view(np.complex64)[..., 0])
                for ty, tc in pin_out]
    ctx.decode_fields(host_fields, cfg, out=host_out)  # warm
    e2e_t = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = ctx.decode_fields(host_fields, cfg, out=host_out)
        e2e_t += time.perf_counter() - t
    h2d = sum(f.samples.nbytes for f in fields)
    d2h = sum(o.luma.nbytes + o.chroma.nbytes for o in out)
    if dist is not None:
        e2e_t = max_over_ranks([e2e_t], dist, "cuda")[0]

    # ---- plain one-field-per-launch path ----
    plain = None
    if not args.no_plain:
        ctx.set_batching(False)
        ctx.decode_fields_device(fin, fout, n, cfg)
        pt = 0.0
        psteps = max(1, min(args.steps, 2))
        for _ in range(psteps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            pt += ctx.decode_fields_device(fin, fout, n, cfg).ms_total
        ctx.set_batching(True)
        if dist is not None:
            pt = max_over_ranks([pt], dist, "cuda")[0]
        plain = {"value": n * psteps * world / (pt / 1000.0), "unit": "fields/s",
                 "ms_per_step": pt / psteps}

    value = throughput(n, args.steps, world, ms_total)
    peak, peak_kind = measured_peaks()
    alg_bytes_per_launch = (ALG_BYTES_ITER * pix_iters + ALG_BYTES_OUTER * pix_outers) / args.steps
    solver_s = ms_solver / 1000.0 / args.steps
    achieved = alg_bytes_per_launch / solver_s / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": profile_traffic(args.workload),
            "traffic_source": "committed one-pass ncu capture of this solver build on this workload "
                              "(profiles/solver_traffic.json), not measured in this run",
            "peak_kind": peak_kind,
            "kernel": "k_solver (persistent IRLS + CG)",
            "alg_bytes_per_launch": alg_bytes_per_launch, "ms_per_launch": 1000 * solver_s}

    line = {
        "metric": METRIC, "value": value, "unit": "fields/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded hvdg.synth mixed NTSC/PAL batch)",
        "config": {"workload": WORKLOAD_DESC[args.workload],
                   "solver": "FP32 planes, FP64 reductions, fixed iterations (cg_tol 1e-6, fast off)",
                   "l2": "flushed between steps (256 MiB write, outside the timed events)",
                   "parallelism": f"fields sharded per rank x{world}, no data-path collective"},
        "e2e": {"value": n * args.steps * world / e2e_t, "unit": "fields/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks,
        "plain": plain,
        "wall_s": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            threads = os.cpu_count() or 1
            sample = quarter_samples(fields)[0]
            run_reference(sample[:2], threads)
            ts, (ry, rc) = run_reference(sample, threads, outputs=True)
            line["cpu_baseline"] = {
                "value": field_equivalents(sample, fields) / ts, "unit": "fields/s",
                "cores": threads, "kind": "reference",
                "sample": f"the first {len(sample)} of the {n} workload fields, reference engine "
                          f"(oracle/_ref) OpenMP across fields, counted by solver work relative "
                          f"to the workload's mean"}
            line["parity"] = parity_leg(fields, out, sample, ry, rc)
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
