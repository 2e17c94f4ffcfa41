"""The N>1 path of bench.py (one independent replica per rank, device timings
reduced with a max over ranks) exercised with world_size 2 on the gloo backend."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # every rank reports its own time; all must see the maximum
    mx = bench.reduce_max(10.0 + rank * 5.0, dist, device="cpu")
    # the reference arm prints on rank 0 only; other ranks return without work
    class A:
        steps, warmup, workload = 3, 3, "layered_vk"
    out = bench.run_reference(A, rank) if rank != 0 else "skip"
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mx, out))


def test_replica_timing_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == 15.0 and res[1][1] == 15.0
    assert res[1][2] is None  # rank 1 does no reference work


def test_single_rank_reduce_is_identity():
    import bench
    assert bench.reduce_max(3.5, None) == 3.5
