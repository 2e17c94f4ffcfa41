"""The reference's own launch sequence run through libawpb200's reference-named
launchers (the link-time drop-in) against the same sequence through the
reference's CUDA build.

refbind.RefGpuSim / RefMeshSim drive the kernel.cu launchers in pmcl3d's
single-rank order with arrays made by the reference's host code
(init_texture's vx1/vx2/ww/wwo, inicrj, the lam_mu ratio).  Given the path of
libawpb200.so instead of the reference build, the same driver calls
SetDeviceConstValue, SetDeviceFilterParameters, dvelcx_H_opt, dstrqc_H,
addsrc_H, addkinsrc_H, drprecpc_calc_H_opt, drprecpc_app_H, fstr_H, dvelc2_H,
dstrqc2_H, intp3d_H and swap_H of this library.  Tolerance: relative L2
<= 1e-5 per field (1e-4 with plasticity)."""
import numpy as np
import pytest

from awp_b200 import _lib, scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5",
          "r6"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def prod_path():
    lib = _lib.load()
    lib.awp_compat_exit_on_error(0)
    return _lib.LIB_PATH


def compare(get_a, get_b, fields, tol):
    report = {}
    for f in fields:
        a, b = get_a(f), get_b(f)
        if np.linalg.norm(b) == 0:
            assert np.linalg.norm(a) == 0, f
            continue
        report[f] = rel_l2(a, b)
        assert report[f] <= tol, (f, report[f])
    return report


@pytest.mark.parametrize("case", [
    dict(nx=24, ny=20, nz=32, q=True, ifault=1, steps=24, seed=7),
    dict(nx=23, ny=19, nz=36, q=True, ifault=5, steps=20, seed=8, nsrc=3),  # odd, kinematic
    dict(nx=20, ny=22, nz=28, q=False, ifault=1, steps=16, seed=9),          # elastic
], ids=["anelastic-if1", "odd-if5", "elastic"])
def test_single_grid_loop(prod_path, case):
    case = dict(case)
    steps = case.pop("steps")
    scn = scenarios.random_small(steps=steps, **case)
    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    ref.step(steps)
    mine = refbind.RefGpuSim(scn, setup, path=prod_path)
    mine.step(steps)
    assert _lib.load().awp_compat_last_error() == 0
    rep = compare(mine.field, ref.field, FIELDS, 1e-5)
    assert np.linalg.norm(ref.field("u1")) > 0
    print("\nrel L2, launchers of libawpb200 vs the reference build:",
          {k: f"{v:.1e}" for k, v in rep.items()})


def test_plasticity_loop(prod_path):
    steps = 16
    scn = scenarios.random_small(nx=24, ny=32, nz=32, q=True, ifault=1, steps=steps, seed=3)
    scn.params["nve"] = 3
    setup = refbind.model_setup(scn)
    setup["plast"] = refbind.plasticity_inputs(scn, setup)
    ref = refbind.RefGpuSim(scn, setup)
    ref.step(steps)
    mine = refbind.RefGpuSim(scn, setup, path=prod_path)
    mine.step(steps)
    assert _lib.load().awp_compat_last_error() == 0
    assert int((ref.field("yldfac") < 1).sum()) > 1000
    compare(mine.field, ref.field, FIELDS + ["yldfac", "neta"], 1e-4)


def test_mesh_loop(prod_path):
    steps = 16
    scns = scenarios.dm_small(nxc=10, nyc=8, nzs=(36, 24), steps=steps, q=True)
    setups = refbind.mesh_setup(scns)
    ref = refbind.RefMeshSim(scns, setups)
    ref.step(steps)
    mine = refbind.RefMeshSim(scns, setups, path=prod_path)
    mine.step(steps)
    assert _lib.load().awp_compat_last_error() == 0
    for p in range(len(scns)):
        compare(lambda f: mine.field(p, f), lambda f: ref.field(p, f), FIELDS, 1e-5)
    assert np.linalg.norm(ref.field(1, "u1")) > 0
