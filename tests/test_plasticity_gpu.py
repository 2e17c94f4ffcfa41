"""GPU parity of the Drucker-Prager plasticity path (NVE=3).

The product (velocity, stress + memory variables, sources, yield factor and
its application, free-surface imaging) runs against the reference's own CUDA
kernels driven in pmcl3d's NVE=3 order (split stress bands, five yield-factor
strips, drprecpc_app; pmcl3d.c:1858-1879, 2110-2209) and against the FP64
oracle.  Inputs: lithostatic sigma2 from the density (mesh.c:1274-1282),
seeded cohesion and friction angle, principal-stress ratios that leave about
half of the cells at yield.  Tolerance: relative L2 <= 1e-4 (plasticity is a
nonsmooth return, so rounding differences near the yield surface are
amplified more than in the linear path).
"""
import numpy as np
import pytest

from awp_b200 import Solver, default_params, scenarios
from oracle import oracle as orc
from oracle import refbind

pytestmark = pytest.mark.gpu

REL = 1e-4
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r4", "yldfac", "neta"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("case", [
    dict(nx=24, ny=32, nz=32, ifault=1, steps=20, seed=3),
    dict(nx=27, ny=41, nz=36, ifault=5, steps=16, seed=4, nsrc=4),  # odd sizes, kinematic
])
def test_plasticity_parity(case):
    case = dict(case)
    steps = case.pop("steps")
    scn = scenarios.random_small(q=True, steps=steps, **case)
    scn.params["nve"] = 3
    setup = refbind.model_setup(scn)
    pl = refbind.plasticity_inputs(scn, setup)
    setup["plast"] = pl

    ref = refbind.RefGpuSim(scn, setup)
    ref.step(steps)

    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.upload_plasticity(pl["sigma2"], pl["cohes"], pl["phi"], pl["fmajor"], pl["fminor"],
                        pl["strike"], pl["dip"])
    s.step(steps)
    s.synchronize()

    o = orc.OracleSim(scn, setup, 64)
    for k in ("sigma2", "cohes", "phi"):
        o.set_field(k, pl[k])
    o.set_field("yldfac", np.ones(o.shape, np.float32))
    o.set_plasticity(pl["fmajor"], pl["fminor"], pl["Rz"], pl["RzT"])
    o.step(steps)

    y = ref.field("yldfac")
    yielded = int((y < 1).sum())
    assert yielded > 1000, yielded  # the case exercises the return, not only the elastic branch
    report = {}
    for f in FIELDS:
        a = s.field(f)
        r = ref.field(f)
        b = o.field(f, f64=True)
        report[f] = (rel_l2(a, r), rel_l2(a, b), rel_l2(r, b))
        assert report[f][0] <= REL, (f, report[f])
        assert report[f][1] <= REL, (f, report[f])
    print("\nyielded cells:", yielded, "rel L2 (vs ref, vs fp64, ref vs fp64):",
          {k: tuple(f"{x:.2e}" for x in v) for k, v in report.items()})
    s.close()
