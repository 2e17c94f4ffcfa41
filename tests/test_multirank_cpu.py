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


class _FakeParams:
    nx, ny, nz = 4, 3, 2


class _FakeSolver:
    params = _FakeParams()


def _fake_shot(solver, nsteps, shot, nsnap, want_q):
    """A deterministic stand-in for one shot's (misfit, gradients)."""
    import numpy as np
    k = shot  # the shot's index
    g = [np.full((2, 3, 4), float(k + 1) * (q + 1), np.float32) for q in range(5 if want_q else 3)]
    return float(k * k + 0.5), g


def _shots_worker(rank, world, port, q, nshots, want_q):
    import datetime

    import torch.distributed as dist

    from awp_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ran = []

    def shot(solver, nsteps, s, nsnap, wq):
        ran.append(s)
        return _fake_shot(solver, nsteps, s, nsnap, wq)
    J, g = replicas.misfit_gradient_shots(_FakeSolver(), 5, list(range(nshots)), dist=dist,
                                          want_q=want_q, run_shot=shot)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ran, J, [x.tolist() for x in g]))


@pytest.mark.parametrize("nshots,want_q", [(5, False), (1, True)])
def test_shots_dealt_across_ranks_and_summed(nshots, want_q):
    """World size 2 on gloo: every shot runs on exactly one rank, and both
    ranks end with the sum over all shots of the misfit and gradients."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shots_worker, args=(r, 2, port, q, nshots, want_q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ran = sorted(res[0][1] + res[1][1])
    assert ran == list(range(nshots))
    J_all = sum(_fake_shot(None, 5, k, 0, want_q)[0] for k in range(nshots))
    g_all = [sum(_fake_shot(None, 5, k, 0, want_q)[1][q_].astype(np.float64)
                 for k in range(nshots)) for q_ in range(5 if want_q else 3)]
    for rank, _, J, g in res:
        assert J == pytest.approx(J_all, rel=1e-12)
        assert len(g) == len(g_all)
        for a, b in zip(g, g_all):
            assert np.allclose(np.asarray(a), b, rtol=1e-12)


def test_deal_largest_first_round_robin():
    from awp_b200 import replicas
    sizes = [5, 9, 1, 7, 3]
    a = replicas.deal(5, 0, 2, sizes)
    b = replicas.deal(5, 1, 2, sizes)
    # sizes sorted: 9 (1), 7 (3), 5 (0), 3 (4), 1 (2)
    assert a == [1, 0, 2] and b == [3, 4]
    assert sorted(a + b) == list(range(5))
    assert replicas.deal(3, 2, 4) == [2] and replicas.deal(3, 3, 4) == []
    with pytest.raises(ValueError):
        replicas.deal(3, 4, 4)
