"""TEST INFRASTRUCTURE -- oracle decodes as picklable jobs for a process pool.

The FP64 oracle takes ~20 ms (NTSC) / ~30 ms (PAL) per CG iteration on one
host core, so checking a batch at the benchmark's budgets (4-12 IRLS outers
x 50 CG per field) is done field-parallel in a `spawn` process pool (never
forked: a fork after the first CUDA call can hang the child). Only tests/
and bench.py's cpu_baseline leg use this module, as the checker.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor


def decode_field_2d(job):
    """One field through the oracle's 2-D decode (hvd_oracle.decode_fields_2d:
    PrepareFieldObs + HolographicInit + VariationalRefine, sequence.cpp:229-281,
    1076-1114). `job` = (uint16 samples, standard, parity, config kwargs).
    Returns (luma, chroma, solver stats)."""
    samples, standard, parity, cfg_kw = job
    from hvdg import _cabi, api, synth
    from oracle import hvd_oracle as O
    g = _cabi.default_geometry(standard)
    cfg = api.default_config(**cfg_kw)
    stats = []
    (y, chi, _), = O.decode_fields_2d([synth.to_ire(samples)], [parity], g, cfg, stats=stats)
    return y, chi, stats[0]


def pool(n_jobs: int) -> ProcessPoolExecutor:
    """A spawn-context pool sized to the jobs and the host cores."""
    workers = max(1, min(n_jobs, os.cpu_count() or 1))
    return ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"))


def decode_fields_2d_parallel(jobs):
    """decode_field_2d over `jobs` in a spawn pool; results in job order."""
    with pool(len(jobs)) as ex:
        return list(ex.map(decode_field_2d, jobs))


def adjoint_field(job):
    """One field through the FP64 adjoint oracle (hvd_adjoint: the decode's
    forward with its IRLS checkpoints, the implicit-function adjoint of the
    refine, then the init's adjoint). `job` = (uint16 samples, standard,
    parity, config kwargs, luma cotangent, chroma cotangent). Returns
    (d loss / d S on the active picture, {scalar name: gradient})."""
    samples, standard, parity, cfg_kw, yb, cb = job
    from hvdg import _cabi, api, synth
    from oracle import hvd_adjoint as A
    from oracle import hvd_oracle as O
    g = _cabi.default_geometry(standard)
    cfg = api.default_config(**cfg_kw)
    obs = O.prepare_field(synth.to_ire(samples), g, cfg, parity)
    _, _, chi0 = A.init_parts(obs.s, obs.carrier, g)
    aniso = O.resolve_chroma_aniso(chi0, cfg, O.uses_vswitch(g))
    chis = A.refine_forward_budget(obs.s, obs.carrier, chi0, cfg, aniso)
    s_bar, chi0_bar, gl = A.refine_adjoint(obs.s, obs.carrier, chis, cfg, aniso, yb, cb, 1e-8, 3000)
    return s_bar + A.init_adjoint(obs.s, obs.carrier, g, chi0_bar), gl


def adjoint_fields_parallel(jobs):
    """adjoint_field over `jobs` in a spawn pool; results in job order."""
    with pool(len(jobs)) as ex:
        return list(ex.map(adjoint_field, jobs))
