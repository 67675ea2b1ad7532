"""The multi-rank bench path on CPU (gloo, world size 2): every rank gets its
own deterministic batch (disjoint fields), the job time is the maximum over
ranks, and the whole-job throughput counts every rank's fields; the
reference arm runs on rank 0 only."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    fields = bench.rank_workload(rank, "small16")
    digest = [int(np.asarray(f.samples, np.int64).sum()) for f in fields]
    again = [int(np.asarray(f.samples, np.int64).sum()) for f in bench.rank_workload(rank, "small16")]
    digests = [None] * world
    dist.all_gather_object(digests, digest)
    # per-rank timings: rank r reports (10 + r, 3 - r)
    mx = bench.max_over_ranks([10.0 + rank, 3.0 - rank], dist, "cpu")
    # the reference arm on a non-zero rank returns without work
    class A:
        workload = "mixed64"
        steps = 1
        warmup = 0
    rc = bench.reference_arm(A, rank, world) if rank != 0 else 0
    q.put((rank, digest == again, digests, mx, rc))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_reduction():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, deterministic, digests, mx, rc in res:
        assert deterministic
        # disjoint batches: no field of rank 0 equals one of rank 1
        assert not set(digests[0]) & set(digests[1])
        assert mx == [11.0, 3.0]
        assert rc == 0
    sys.path.insert(0, str(REPO))
    import bench
    assert bench.throughput(16, 5, 2, 1000.0) == 160.0


def _chunk_worker(rank, world, port, q):
    """Rank `rank` decodes its share of a 9-frame NTSC sequence's export
    chunks (3-frame cores, 1 frame of context each side) through the
    compiled reference engine's DecodeFrameSequenceWindow -- the decode
    runs on the host here; the sharding, the halo windows and the gather
    are the multi-GPU path's own -- and rank 0 gathers the frames."""
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from hvdg import _cabi, api, sequence, synth
    from oracle import ref
    ref.set_threads(2)
    frames, _ = synth.make_frames(91, _cabi.STD_NTSC, 9, noise_sigma=0.5, moving=True)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = api.default_config(irls_outer=2, cg_iterations=8, fast=1, cg_tol=1e-6,
                             temporal_strength=0.5, passes=1, nr_anchor=0.0)
    chunks = sequence.plan_chunks(0, len(frames) - 1, 3, 1, sequence.is_coupled(cfg))
    mine = sequence.shard(chunks, world, rank)

    def decode(win, cb, ce):
        return ref.decode_frame_sequence_window(win, cb, ce, fp, cfg)

    local = sequence.decode_chunks(decode, frames, mine)
    got = sequence.gather_frames(local, len(chunks), dist)
    q.put((rank, [c.index for c in mine], None if got is None else
           [fr["luma"].tobytes() + fr["chroma"].tobytes() for fr in got]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_chunked_window_sharding():
    """Chunks with their replicated halo frames decode the same on two
    ranks as on one: every core frame comes back exactly once, in order,
    equal to the single-process chunked decode."""
    sys.path.insert(0, str(REPO))
    from oracle import ref
    if not ref.available():
        import pytest
        pytest.skip("reference engine not built")
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_chunk_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=600) for _ in range(world)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res[0][1] == [0, 2] and res[1][1] == [1]
    assert res[1][2] is None
    gathered = res[0][2]
    assert len(gathered) == 9
    from hvdg import _cabi, api, sequence, synth
    frames, _ = synth.make_frames(91, _cabi.STD_NTSC, 9, noise_sigma=0.5, moving=True)
    fp = api.frame_params(_cabi.STD_NTSC)
    cfg = api.default_config(irls_outer=2, cg_iterations=8, fast=1, cg_tol=1e-6,
                             temporal_strength=0.5, passes=1, nr_anchor=0.0)
    ref.set_threads(2)
    chunks = sequence.plan_chunks(0, 8, 3, 1, True)
    single = sequence.gather_frames(sequence.decode_chunks(
        lambda w, cb, ce: ref.decode_frame_sequence_window(w, cb, ce, fp, cfg), frames, chunks),
        len(chunks))
    assert gathered == [fr["luma"].tobytes() + fr["chroma"].tobytes() for fr in single]


def test_chunk_plan_matches_the_stage():
    """The stage's chunk windows (hvd_chroma_decoder_stage.cpp:711-716,
    997-1060): cores tile the range, windows add the overlap clipped to the
    range, no overlap when the fields are decoupled; shards are disjoint
    and cover every chunk."""
    sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
    from hvdg import sequence
    cs = sequence.plan_chunks(10, 23, 6, 1, True)
    assert [(c.first, c.last, c.w0, c.w1) for c in cs] == [(10, 15, 10, 16), (16, 21, 15, 22),
                                                           (22, 23, 21, 23)]
    assert [(c.core_begin, c.core_end) for c in cs] == [(0, 6), (1, 7), (1, 3)]
    cs0 = sequence.plan_chunks(10, 23, 6, 1, False)
    assert all(c.w0 == c.first and c.w1 == c.last for c in cs0)
    for world in (1, 2, 3, 8):
        got = sorted(c.index for r in range(world) for c in sequence.shard(cs, world, r))
        assert got == [c.index for c in cs]
