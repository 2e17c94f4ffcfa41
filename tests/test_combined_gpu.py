"""Combined features of the config-3 kind (topography, discontinuous mesh,
plasticity, attenuation) against the reference's own CUDA build.

* a two-block mesh whose top block is curvilinear (NVE 1): refbind.RefMeshSim
  with the reference's topography kernels on block 0;
* a two-block mesh with Drucker-Prager plasticity (NVE 3) on both blocks;
* a curvilinear single grid with NVE 3 in the reference's behaviour (the
  default): at one rank pmcl3d updates only the middle band of grid 0's
  stress, with the Cartesian dstrqc (refbind.RefTopoSim with nve = 3);
* the consistent topography + plasticity path behind its flag
  (awp_set_topo_plasticity): with nothing yielding it equals the NVE 1
  curvilinear run bit for bit.

Tolerances: relative L2 <= 1e-5 (1e-4 with plasticity) per field and block."""
import numpy as np
import pytest

from awp_b200 import Mesh, Solver, default_params, scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r4", "r6"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def check(get_a, get_b, fields, tol, tag):
    rep = {}
    for f in fields:
        a, b = get_a(f), get_b(f)
        if np.linalg.norm(b) == 0:
            assert np.linalg.norm(a) == 0, (tag, f)
            continue
        rep[f] = rel_l2(a, b)
        assert rep[f] <= tol, (tag, f, rep[f])
    return rep


def hill(path, p, scale=0.08):
    depth = p["dh"] * p["nz"]
    scenarios.write_topography(path, p["nx"], p["ny"], p["dh"], amplitude=scale * depth,
                               width=0.3 * p["nx"] * p["dh"], rough_rms=0.004 * depth, seed=4)


def product_mesh(scns, topo=None, plast=None):
    m = Mesh([default_params(**s.params) for s in scns])
    for p, s in enumerate(scns):
        g = m.grid(p)
        g.upload_media(s.media)
        if s.src_pos.shape[0]:
            g.upload_sources(s.src_pos, s.src_data)
        if plast is not None:
            pl = plast[p]
            g.upload_plasticity(pl["sigma2"], pl["cohes"], pl["phi"], pl["fmajor"], pl["fminor"],
                                pl["strike"], pl["dip"])
    if topo:
        m.grid(0).topography(topo)
    return m


def test_topography_on_a_mesh_matches_reference(tmp_path):
    steps = 16
    scns = scenarios.dm_small(nxc=10, nyc=8, nzs=(36, 24), steps=steps, q=True)
    topo = str(tmp_path / "topo.bin")
    hill(topo, scns[0].params)
    setups = refbind.mesh_setup(scns)
    ref = refbind.RefMeshSim(scns, setups, intopo=topo)
    ref.step(steps)
    m = product_mesh(scns, topo=topo)
    m.step(steps)
    m.synchronize()
    for p in range(2):
        rep = check(lambda f: m.grid(p).field(f), lambda f: ref.field(p, f), FIELDS, 1e-5,
                    f"block {p}")
        print(f"\nblock {p} rel L2:", {k: f"{v:.1e}" for k, v in rep.items()})
    assert np.linalg.norm(ref.field(1, "u1")) > 0
    m.close()


def test_plasticity_on_a_mesh_matches_reference():
    steps = 14
    # the reference's NVE 3 strips need every block wider than 2 ngsl + a
    # middle band in y (pmcl3d.c:573-631): coarse block 24 x 32
    scns = scenarios.dm_small(nxc=24, nyc=32, nzs=(36, 24), steps=steps, q=True)
    for s in scns:
        s.params["nve"] = 3
        s.src_data = (s.src_data * 30.0).astype(np.float32)  # strong enough to yield
    setups = refbind.mesh_setup(scns)
    plast = [refbind.plasticity_inputs(s, st) for s, st in zip(scns, setups)]
    for st, pl in zip(setups, plast):
        st["plast"] = pl
    ref = refbind.RefMeshSim(scns, setups)
    ref.step(steps)
    m = product_mesh(scns, plast=plast)
    m.step(steps)
    m.synchronize()
    yielded = sum(int((ref.field(p, "yldfac") < 1).sum()) for p in range(2))
    assert yielded > 100, yielded
    for p in range(2):
        check(lambda f: m.grid(p).field(f), lambda f: ref.field(p, f),
              FIELDS + ["yldfac", "neta"], 1e-4, f"block {p}")
    m.close()


def topo_single(tmp_path, steps, nve, seed=5, consistent=None, cohes=None):
    scn = scenarios.random_small(nx=28, ny=40, nz=36, q=True, ifault=1, steps=steps, seed=seed,
                                 nsrc=3)
    scn.src_data = (scn.src_data * 30.0).astype(np.float32)
    scn.params["nve"] = nve
    topo = str(tmp_path / f"topo_{seed}.bin")
    hill(topo, scn.params)
    setup = refbind.model_setup(scn)
    pl = None
    if nve == 3:
        pl = refbind.plasticity_inputs(scn, setup)
        if cohes is not None:
            pl["cohes"] = np.full_like(pl["cohes"], cohes)
        setup["plast"] = pl
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    if pl is not None:
        s.upload_plasticity(pl["sigma2"], pl["cohes"], pl["phi"], pl["fmajor"], pl["fminor"],
                            pl["strike"], pl["dip"])
    s.topography(topo)
    if consistent is not None:
        s.set_topo_plasticity(consistent)
    s.step(steps)
    s.synchronize()
    return scn, setup, topo, s


def test_topography_plasticity_reference_behaviour(tmp_path):
    steps = 16
    scn, setup, topo, s = topo_single(tmp_path, steps, nve=3)
    ref = refbind.RefTopoSim(scn, setup, topo)
    ref.step(steps)
    assert int((ref.field("yldfac") < 1).sum()) > 50
    check(s.field, ref.field, FIELDS + ["yldfac", "neta"], 1e-4, "topo NVE 3")
    s.close()


def test_topography_plasticity_consistent_flag(tmp_path):
    steps = 12
    # nothing can yield: the consistent path must equal the NVE 1 curvilinear run
    _, _, _, a = topo_single(tmp_path, steps, nve=3, consistent=True, cohes=1e18)
    _, _, _, b = topo_single(tmp_path, steps, nve=1)
    for f in ("u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r6"):
        assert np.array_equal(a.field(f).view(np.uint32), b.field(f).view(np.uint32)), f
    a.close()
    b.close()
    # with yielding it runs, stays finite and differs from the reference behaviour
    _, _, _, c = topo_single(tmp_path, steps, nve=3, consistent=True)
    _, _, _, d = topo_single(tmp_path, steps, nve=3, consistent=False)
    assert c.check_finite()
    assert not np.array_equal(c.field("xx"), d.field("xx"))
    c.close()
    d.close()
