"""CPU oracle pinned to the reference's own CUDA build (golden fixtures).

tests/golden/ref_<case>.npz hold the state after N steps of the reference
kernels (src/awp/kernel.cu built unmodified for sm_100a) on seeded inputs;
tests/golden/make_golden.py regenerates them on a GPU machine.  The FP64 and
FP32 oracles, fed the same inputs, must agree with them.
"""
import os

import numpy as np
import pytest

from awp_b200 import scenarios
from oracle import oracle as orc
from oracle import refbind

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
from golden.make_golden import CASES, FIELDS, interior  # noqa: E402

# FP32 accumulation over the steps against the reference's FP32 (fast-math) run
TOL = {64: 1e-5, 32: 1e-5}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb else 1.0))


def load_case(name):
    path = os.path.join(HERE, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated yet")
    return np.load(path)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", [64, 32])
def test_oracle_matches_reference_build(ref_host, name, precision):
    gold = load_case(name)
    case = dict(CASES[name])
    steps = case.pop("steps")
    scn = scenarios.random_small(steps=steps, **case)
    setup = refbind.model_setup(scn, ref_host)
    sim = orc.OracleSim(scn, setup, precision=precision, nthreads=2)
    sim.step(steps)
    p = scn.params
    for f in FIELDS:
        mine = interior(sim.field(f, f64=True), p["nx"], p["ny"], p["nz"])
        ref = gold[f]
        if not np.any(ref):
            assert not np.any(mine), f
            continue
        assert rel_l2(mine, ref) < TOL[precision], (f, rel_l2(mine, ref))
    if "mom" in gold:
        assert rel_l2(sim.moment(len(gold["mom"])), gold["mom"]) < 1e-5


def test_planted_mistake_is_caught(ref_host):
    """A small planted change in the oracle's input (1e-3 relative on every
    inverse Lame modulus) must push it outside the tolerance: the golden
    comparison has teeth."""
    gold = load_case("anelastic_if1")
    case = dict(CASES["anelastic_if1"])
    steps = case.pop("steps")
    scn = scenarios.random_small(steps=steps, **case)
    setup = refbind.model_setup(scn, ref_host)
    lam = setup["media"]["lam"].copy()
    lam *= np.float32(1.001)
    setup["media"]["lam"] = lam
    sim = orc.OracleSim(scn, setup, precision=64, nthreads=2)
    sim.step(steps)
    p = scn.params
    errs = [rel_l2(interior(sim.field(f, f64=True), p["nx"], p["ny"], p["nz"]), gold[f])
            for f in ("xx", "yy", "zz")]
    assert max(errs) > 10 * TOL[64], errs
