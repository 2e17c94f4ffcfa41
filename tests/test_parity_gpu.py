"""GPU parity: product time loop vs the reference's own CUDA build vs the FP64 oracle.

All three runs take identical inputs (refbind.model_setup, the reference's own
host code; the product maps the raw media itself and is checked to agree).
Tolerance: relative L2 <= 1e-5 against the reference build (FP32 both sides),
and <= 1e-4 against the FP64 oracle (single-precision rounding accumulates
over the steps).
"""
import numpy as np
import pytest

from awp_b200 import Solver, default_params, scenarios
from oracle import oracle as orc
from oracle import refbind

pytestmark = pytest.mark.gpu

REL_REF = 1e-5
REL_F64 = 1e-4
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz"]
RFIELDS = ["r1", "r2", "r3", "r4", "r5", "r6"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def product_run(scn, steps):
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.step(steps)
    s.synchronize()
    return s


CASES = [
    dict(nx=24, ny=20, nz=32, q=True, ifault=1, steps=20),
    dict(nx=23, ny=19, nz=28, q=True, ifault=1, steps=15),   # odd nx, ny; nz % 32 != 0
    dict(nx=20, ny=24, nz=32, q=False, ifault=1, steps=20),  # elastic specialisation
    dict(nx=24, ny=20, nz=32, q=True, ifault=5, steps=30, nsrc=4),
    dict(nx=16, ny=18, nz=24, nvar=3, ifault=1, steps=12),   # Q from vs (mesh.c:226-236)
    dict(nx=18, ny=16, nz=20, nvar=8, ifault=1, steps=12),
    dict(nx=41, ny=37, nz=68, q=True, ifault=1, steps=6),    # partial tiles in j, k and i
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_media_matches_reference_host(case):
    case = dict(case)
    steps = case.pop("steps")
    scn = scenarios.random_small(steps=steps, **case)
    setup = refbind.model_setup(scn)
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    m = setup["media"]
    for k in ("d1", "mu", "lam", "qp", "qs"):
        mine = s.field(k)
        ref = m[k]
        bad = mine.view(np.uint32) != ref.view(np.uint32)
        # the complex sums are done in double on both sides; allow isolated 1-ulp
        # differences from the complex division, nothing more
        if bad.any():
            rel = np.abs(mine[bad] - ref[bad]) / np.maximum(np.abs(ref[bad]), 1e-30)
            assert rel.max() < 2e-7, (k, int(bad.sum()), float(rel.max()))
            assert bad.mean() < 1e-3, (k, int(bad.sum()))
    s.close()


@pytest.fixture(params=[1, 0], ids=["tma", "ldg"])
def kernel_family(request):
    """Run the context API on the TMA-pipelined (1) or read-only-path (0) kernels."""
    from awp_b200 import _lib, tune
    lib = _lib.load()
    saved = tune.get_tuning(lib)
    tune.set_tuning(lib, "tma", request.param)
    yield request.param
    for k, v in saved.items():
        tune.set_tuning(lib, k, v)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_time_loop_parity(case, kernel_family):
    case = dict(case)
    steps = case.pop("steps")
    scn = scenarios.random_small(steps=steps, **case)
    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    ref.step(steps)
    prod = product_run(scn, steps)
    o64 = orc.OracleSim(scn, setup, 64)
    o64.step(steps)
    report = {}
    for f in FIELDS + RFIELDS:
        a = prod.field(f)
        r = ref.field(f)
        o = o64.field(f, f64=True)
        e_ref = rel_l2(a, r)
        e_64 = rel_l2(a, o)
        e_ref64 = rel_l2(r, o)
        report[f] = (e_ref, e_64, e_ref64)
        if np.linalg.norm(r) == 0:
            assert np.linalg.norm(a) == 0, f
            continue
        assert e_ref <= REL_REF, (f, report[f])
        assert e_64 <= REL_F64, (f, report[f])
    print("\nrel L2 (vs ref, vs fp64, ref vs fp64):",
          {k: tuple(f"{x:.2e}" for x in v) for k, v in report.items()})
    prod.close()


def test_moment_accumulation_matches_reference():
    scn = scenarios.random_small(nx=24, ny=20, nz=32, ifault=5, nsrc=5, steps=25)
    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    ref.step(25)
    prod = product_run(scn, 25)
    mom = prod.download_moment(scn.src_pos.shape[0])
    rmom = ref.mom.cpu().numpy()[: setup["psrc"].shape[0]]
    assert rel_l2(mom, rmom) < 1e-5
    prod.close()


def test_nonfinite_sentinel():
    scn = scenarios.random_small(steps=2)
    s = product_run(scn, 2)
    assert s.check_finite()
    xx = s.field("xx")
    xx[12, 12, 40] = np.nan
    s.set_field("xx", xx)
    assert not s.check_finite()
    s.close()


def test_state_errors_are_reported():
    from awp_b200 import AwpError
    scn = scenarios.random_small(steps=1)
    s = Solver(default_params(**scn.params))
    with pytest.raises(AwpError) as e:
        s.step(1)  # no media yet
    assert e.value.status == 3
    s.close()
    with pytest.raises(AwpError) as e:
        Solver(default_params(nx=16, ny=16, nz=30))  # nz % 4 != 0 (pmcl3d.c:380)
    assert e.value.status == 1
