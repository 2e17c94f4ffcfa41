"""x-slab decomposition on one GPU against the whole grid, every field equal
bit for bit after the run: parts stepped in lockstep by the library
(awp_decomp_*, halos copied in device memory), and parts stepped by one host
thread each whose exchange hooks trade the halos through SlabRank
(awp_set_exchange + awp_halo_copy) with an in-process transport in place of
NCCL.  No kernel waits on another part: the threads meet on the host."""
import queue
import threading
from ctypes import byref, c_void_p

import numpy as np
import pytest

from awp_b200 import Solver, _lib, default_params, scenarios
from awp_b200._lib import check
from awp_b200.decomp import LocalDecomposition, SlabRank, part_media, part_sources, split_x

pytestmark = pytest.mark.gpu

NGSL = 8
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5",
          "r6"]


def plastic_case(nx, seed, steps, ifault=1):
    """NVE 3: low cohesions so that cells near the sources yield."""
    from oracle import refbind
    scn = scenarios.random_small(nx=nx, ny=24, nz=32, q=True, ifault=ifault, steps=steps,
                                 seed=seed, nsrc=4)
    scn.params["nve"] = 3
    pl = refbind.plasticity_inputs(scn, refbind.model_setup(scn))
    return scn, pl


def plast_args(pl):
    return pl["sigma2"], pl["cohes"], pl["phi"], pl["fmajor"], pl["fminor"], pl["strike"], \
        pl["dip"]


def whole_run(scn, steps, pl=None, topo=None):
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    if topo is not None:
        s.topography(topo)
    if pl is not None:
        s.upload_plasticity(*plast_args(pl))
    s.step(steps)
    s.synchronize()
    out = {f: s.field(f) for f in FIELDS + (["yldfac", "neta"] if pl is not None else [])}
    s.close()
    return out


def assemble(parts, layout, name):
    s0 = parts[0]
    nxg = sum(w for _, w in layout)
    out = np.zeros((nxg + 4 + 2 * NGSL,) + s0.shape[1:], np.float32)
    lo = 2 + NGSL
    for q, (s, (x0, w)) in enumerate(zip(parts, layout)):
        f = s.field(name)
        out[x0 + lo:x0 + lo + w] = f[lo:lo + w]
        if q == 0:
            out[:lo] = f[:lo]
        if q == len(parts) - 1:
            out[x0 + lo + w:] = f[lo + w:]
    return out


@pytest.mark.parametrize("nx,nparts,q,ifault", [(31, 3, True, 1), (24, 2, False, 1),
                                                (30, 2, True, 5)])
def test_lockstep_parts_equal_whole_grid(nx, nparts, q, ifault):
    steps = 24
    scn = scenarios.random_small(nx=nx, ny=20, nz=32, q=q, ifault=ifault, steps=steps, seed=37,
                                 nsrc=4)
    want = whole_run(scn, steps)
    assert np.abs(want["xx"]).max() > 0
    with LocalDecomposition(default_params(**scn.params), nparts) as d:
        d.upload_media(scn.media)
        d.upload_sources(scn.src_pos, scn.src_data)
        d.step(steps)
        d.synchronize()
        for f in FIELDS:
            got = d.field(f)
            assert np.array_equal(got, want[f]), (f, float(np.abs(got - want[f]).max()))


@pytest.mark.parametrize("nx,nparts", [(31, 3), (30, 2)])
def test_lockstep_plastic_parts_equal_whole_grid(nx, nparts):
    steps = 20
    scn, pl = plastic_case(nx, 51, steps)
    want = whole_run(scn, steps, pl)
    assert np.any(want["yldfac"] < 1.0)  # cells yield
    with LocalDecomposition(default_params(**scn.params), nparts) as d:
        d.upload_media(scn.media)
        d.upload_sources(scn.src_pos, scn.src_data)
        d.upload_plasticity(*plast_args(pl))
        d.step(steps)
        d.synchronize()
        for f in want:
            got = d.field(f)
            if f == "yldfac":  # the inner ghost planes hold the neighbours' values
                got, w = got[2 + NGSL:-2 - NGSL], want[f][2 + NGSL:-2 - NGSL]
            else:
                w = want[f]
            assert np.array_equal(got, w), (f, float(np.abs(got - w).max()))


@pytest.mark.parametrize("nx,nparts,plastic", [(32, 2, False), (34, 3, True)])
def test_lockstep_topography_parts_equal_whole_grid(tmp_path, nx, nparts, plastic):
    """A curvilinear top grid (Gaussian hill): each part takes its planes of
    the whole grid's metrics and the stress window of the whole grid."""
    steps = 16
    if plastic:
        scn, pl = plastic_case(nx, 57, steps)
    else:
        scn, pl = scenarios.random_small(nx=nx, ny=24, nz=32, q=True, ifault=1, steps=steps,
                                         seed=59, nsrc=4), None
    p = scn.params
    topo = str(tmp_path / "topo.bin")
    depth = p["dh"] * (p["nz"] - 2)
    scenarios.write_topography(topo, p["nx"], p["ny"], p["dh"], amplitude=0.15 * depth,
                               width=5 * p["dh"], rough_rms=0.02 * depth, seed=5)
    want = whole_run(scn, steps, pl, topo)
    with LocalDecomposition(default_params(**p), nparts) as d:
        d.upload_media(scn.media)
        d.upload_sources(scn.src_pos, scn.src_data)
        d.topography(topo)
        if pl is not None:
            d.upload_plasticity(*plast_args(pl))
        d.step(steps)
        d.synchronize()
        for f in want:
            got = d.field(f)
            w = want[f]
            if f == "yldfac":
                got, w = got[2 + NGSL:-2 - NGSL], w[2 + NGSL:-2 - NGSL]
            assert np.array_equal(got, w), (f, float(np.abs(got - w).max()))


class _Sent:
    def wait(self):
        pass


class _Recv:
    def __init__(self, box, t):
        self.box, self.t = box, t

    def wait(self):
        self.t.copy_(self.box.get(timeout=120))


class ThreadComm:
    """isend / irecv between threads of one process (mailboxes keyed by
    source, destination and tag)."""

    def __init__(self, rank, boxes):
        self.rank, self.boxes = rank, boxes

    def isend(self, t, dst, group=None, tag=0):
        self.boxes[(self.rank, dst, tag)].put(t.clone())
        return _Sent()

    def irecv(self, t, src, group=None, tag=0):
        return _Recv(self.boxes[(src, self.rank, tag)], t)


@pytest.mark.parametrize("nx,nparts,plastic", [(28, 2, False), (33, 3, False), (30, 2, True)])
def test_exchange_hook_parts_equal_whole_grid(nx, nparts, plastic):
    steps = 16
    if plastic:
        scn, pl = plastic_case(nx, 53, steps)
    else:
        scn, pl = scenarios.random_small(nx=nx, ny=20, nz=32, q=True, ifault=1, steps=steps,
                                         seed=43, nsrc=4), None
    want = whole_run(scn, steps, pl)
    layout = split_x(nx, nparts)
    boxes = {(a, b, t): queue.Queue() for a in range(nparts) for b in range(nparts)
             for t in (0, 1)}
    parts, slabs = [], []
    for r, (x0, w) in enumerate(layout):
        s = Solver(default_params(**dict(scn.params, nx=w)))
        s.set_subdomain(nx, x0)
        s.upload_media(part_media(scn.media, x0, w))
        p, dat = part_sources(scn.src_pos, scn.src_data, x0, w, r == 0, r == nparts - 1)
        if len(p):
            s.upload_sources(p, dat)
        if pl is not None:
            sl = slice(x0, x0 + w + 4 + 2 * NGSL)
            s.upload_plasticity(*[np.ascontiguousarray(a[sl]) for a in plast_args(pl)[:3]],
                                *plast_args(pl)[3:])
        parts.append(s)
        slabs.append(SlabRank(s, r, nparts, comm=ThreadComm(r, boxes)))
    errors = []

    def run(r):
        try:
            slabs[r].exchange_media()
            parts[r].step(steps)
            parts[r].synchronize()
        except Exception as e:  # noqa: BLE001
            errors.append((r, e))

    threads = [threading.Thread(target=run, args=(r,)) for r in range(nparts)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    assert all(sl.exchanges == (4 if plastic else 2) * steps + 1 for sl in slabs)
    for f in want:
        got = assemble(parts, layout, f)
        w = want[f]
        if f == "yldfac":
            got, w = got[2 + NGSL:-2 - NGSL], w[2 + NGSL:-2 - NGSL]
        assert np.array_equal(got, w), (f, float(np.abs(got - w).max()))
    for s in parts:
        s.close()


def test_subdomain_rules(tmp_path):
    scn = scenarios.random_small(nx=20, ny=16, nz=16, q=False, ifault=1, steps=4, seed=3, nsrc=1)
    p = dict(scn.params, nx=10)
    s = Solver(default_params(**p))
    for args in ((20, 3), (20, 12), (8, 0), (20, -2)):
        with pytest.raises(RuntimeError):
            s.set_subdomain(*args)  # odd offset, past the grid, grid too narrow, negative
    s.set_subdomain(20, 10)
    with pytest.raises(RuntimeError):
        s.receivers(str(tmp_path / "none.txt"), 4)  # point sets are not split
    s.close()
    s = Solver(default_params(**p))
    s.upload_media(part_media(scn.media, 0, 10))
    with pytest.raises(RuntimeError):
        s.set_subdomain(20, 0)  # after the media
    s.close()
    a = Solver(default_params(**p))
    b = Solver(default_params(**p))
    a.set_subdomain(20, 0)
    b.set_subdomain(20, 0)  # overlaps part 0 instead of following it
    arr = (c_void_p * 2)(a.ctx, b.ctx)
    with pytest.raises(RuntimeError, match="starts at"):
        check(_lib.load().awp_decomp_create(arr, 2, byref(c_void_p())), "awp_decomp_create")
    a.close()
    b.close()
