"""x-slab decomposition, host side: the part layout, the ownership of point
sources, and the halo trade of SlabRank over torch.distributed with
world_size 2 on gloo (host buffers; a stand-in part holds its fields in host
arrays and packs them as awp_halo_copy does: include/awp_b200.h)."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from awp_b200 import decomp
from awp_b200._lib import HALO_MEDIA, HALO_STRESS, HALO_VELOCITY

NGSL = 8
FIELDS = {HALO_VELOCITY: [0, 1, 2], HALO_STRESS: [3, 4, 5, 6, 7, 8],
          HALO_MEDIA: [15, 16, 17, 18, 19]}


def test_split_x_layout():
    for nx, n in ((24, 2), (31, 3), (100, 4), (64, 1), (50, 6)):
        parts = decomp.split_x(nx, n)
        assert len(parts) == n and parts[0][0] == 0
        assert sum(w for _, w in parts) == nx
        for (x0, w), (x1, _) in zip(parts, parts[1:]):
            assert x1 == x0 + w
        assert all(x0 % 2 == 0 and w >= 4 for x0, w in parts)
    with pytest.raises(ValueError):
        decomp.split_x(10, 4)


def test_part_sources_owner():
    pos = np.array([[0, 3, 2], [1, 3, 2], [12, 5, 5], [13, 5, 5], [24, 1, 1], [26, 1, 1]],
                   np.int32)
    data = np.arange(len(pos) * 2 * 6, dtype=np.float32).reshape(len(pos), 2, 6)
    p0, d0 = decomp.part_sources(pos, data, 0, 12, True, False)
    p1, d1 = decomp.part_sources(pos, data, 12, 12, False, True)
    assert p0[:, 0].tolist() == [0, 1, 12] and p1[:, 0].tolist() == [1, 12, 14]
    assert len(p0) + len(p1) == len(pos)
    assert np.array_equal(np.concatenate([d0, d1]), data)


class FakePart:
    """Fields in host arrays [nx+20][ny_pad][nz_pad]; halo_copy as the library's."""

    def __init__(self, nx, nyp, nzp, seed):
        rng = np.random.default_rng(seed)
        self.nx = nx
        self.shape = (nx + 4 + 2 * NGSL, nyp, nzp)
        self.f = {f: rng.standard_normal(self.shape).astype(np.float32)
                  for fl in FIELDS.values() for f in fl}
        self.hook = None

    def set_exchange(self, fn):
        self.hook = fn

    def synchronize(self):
        pass

    def plane0(self, side, ghost, planes):
        lo, hi = 2 + NGSL, self.nx + 2 + NGSL
        if side == 0:
            return lo - planes if ghost else lo
        return hi if ghost else hi - planes

    def halo_copy(self, unpack, side, hset, planes, addr):
        fids = [f for bit in (HALO_VELOCITY, HALO_STRESS, HALO_MEDIA) if hset & bit
                for f in FIELDS[bit]]
        n = planes * self.shape[1] * self.shape[2]
        p0 = self.plane0(side, unpack, planes)
        for q, f in enumerate(fids):
            view = np.ctypeslib.as_array((ctypes.c_float * n).from_address(addr + q * n * 4))
            if unpack:
                self.f[f][p0:p0 + planes] = view.reshape(planes, *self.shape[1:])
            else:
                view[:] = self.f[f][p0:p0 + planes].ravel()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    widths = [10, 12, 8][:world]
    part = FakePart(widths[rank], 7, 9, seed=rank)
    before = {f: a.copy() for f, a in part.f.items()}
    slab = decomp.SlabRank(part, rank, world, device="cpu")
    assert part.hook == slab.exchange
    slab.exchange(HALO_VELOCITY | HALO_STRESS)
    slab.exchange_media()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, {f: a for f, a in part.f.items()}, before))


@pytest.mark.parametrize("world", [2, 3])
def test_slab_exchange_over_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, after, before = q.get(timeout=120)
        res[r] = (after, before)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    widths = [10, 12, 8][:world]
    H, lo = 4, 2 + NGSL
    for r in range(world):
        after, before = res[r]
        hi = widths[r] + lo
        for f in after:
            # interior and far ghost planes untouched
            assert np.array_equal(after[f][lo:hi], before[f][lo:hi]), (r, f)
            if r > 0:  # low ghost = left neighbour's last interior planes
                nb = res[r - 1][1][f]
                nhi = widths[r - 1] + lo
                assert np.array_equal(after[f][lo - H:lo], nb[nhi - H:nhi]), (r, f)
            else:
                assert np.array_equal(after[f][:lo], before[f][:lo])
            if r < world - 1:  # high ghost = right neighbour's first interior planes
                nb = res[r + 1][1][f]
                assert np.array_equal(after[f][hi:hi + H], nb[lo:lo + H]), (r, f)
            else:
                assert np.array_equal(after[f][hi:], before[f][hi:])
