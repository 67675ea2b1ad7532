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
