"""GPU parity of the discontinuous mesh (DM): the product's mesh (per-block
velocity / stress kernels plus dvelc2, dstrqc2, intp3d, swap3 and the
checkmesh corrections) against the reference's own CUDA kernels driven in
pmcl3d's single-rank order with ngrids > 1 (refbind.RefMeshSim), every block
set up by the reference's host code (inimesh, init_texture, checkmesh, inicrj).
Tolerance: relative L2 <= 1e-5 per field and block."""
import numpy as np
import pytest

from awp_b200 import Mesh, default_params, scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

REL_REF = 1e-5
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r4", "r6"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def product_mesh(scns):
    m = Mesh([default_params(**s.params) for s in scns])
    for p, s in enumerate(scns):
        g = m.grid(p)
        g.upload_media(s.media)
        if s.src_pos.shape[0]:
            g.upload_sources(s.src_pos, s.src_data)
    return m


@pytest.mark.parametrize("case", [
    dict(nxc=10, nyc=8, nzs=(36, 24), steps=20, q=True),
    dict(nxc=11, nyc=7, nzs=(40, 28), steps=10, q=False),      # odd sizes, elastic media
    dict(nxc=6, nyc=6, nzs=(36, 24, 20), steps=12, q=True),    # three blocks
], ids=["2grids", "2grids-odd-elastic", "3grids"])
def test_mesh_matches_reference(case):
    case = dict(case)
    steps = case.pop("steps")
    scns = scenarios.dm_small(steps=steps, **case)
    setups = refbind.mesh_setup(scns)
    ref = refbind.RefMeshSim(scns, setups)
    ref.step(steps)
    m = product_mesh(scns)
    m.step(steps)
    m.synchronize()
    report = {}
    for p in range(len(scns)):
        g = m.grid(p)
        for f in FIELDS:
            a, r = g.field(f), ref.field(p, f)
            if np.linalg.norm(r) == 0:
                assert np.linalg.norm(a) == 0, (p, f)
                continue
            e = rel_l2(a, r)
            report[(p, f)] = e
            assert e <= REL_REF, (p, f, e)
    # the interface is exercised: the coarse block carries the wavefield
    assert np.linalg.norm(ref.field(len(scns) - 1, "u1")) > 0
    print("\nrel L2 vs reference:", {f"{k[0]}:{k[1]}": f"{v:.1e}" for k, v in report.items()})
    m.close()


def test_mesh_media_checkmesh_matches_reference():
    """checkmesh on the device gives the reference host code's corrected media."""
    scns = scenarios.dm_small(nxc=10, nyc=8, nzs=(36, 24), steps=1)
    setups = refbind.mesh_setup(scns)
    m = product_mesh(scns)
    m.step(1)  # the first step applies the corrections
    m.synchronize()
    g = m.grid(1)
    for k in ("d1", "mu", "lam", "qp", "qs"):
        mine, ref = g.field(k), setups[1]["media"][k]
        bad = mine.view(np.uint32) != ref.view(np.uint32)
        if bad.any():  # isolated 1-ulp differences of the complex division only
            rel = np.abs(mine[bad] - ref[bad]) / np.maximum(np.abs(ref[bad]), 1e-30)
            assert rel.max() < 2e-7 and bad.mean() < 1e-3, (k, int(bad.sum()))
    m.close()


def test_mesh_rejects_bad_stacks():
    from awp_b200 import AwpError
    scns = scenarios.dm_small(nxc=10, nyc=8, nzs=(36, 24), steps=1)
    ps = [default_params(**s.params) for s in scns]
    ps[1].nx = 11  # not a third of the block above
    with pytest.raises(AwpError):
        Mesh(ps)
    ps = [default_params(**s.params) for s in scns]
    ps[1].grid = 0
    with pytest.raises(AwpError):
        Mesh(ps)
