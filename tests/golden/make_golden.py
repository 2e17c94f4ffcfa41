"""Generate the golden fixtures of tests/golden/ from the reference's own CUDA build.

Runs on a machine with a GPU and the reference build oracle/_ref/libawpref.so
(oracle/Makefile compiles it from src/awp/kernel.cu).  For each case below the
reference kernels are driven through their own launchers in pmcl3d's
single-rank order (oracle/refbind.py: RefGpuSim) on inputs assembled by the
reference's own host set-up code, and the interior of every state field after
the last step is stored (k range includes the two free-surface image layers).

  python tests/golden/make_golden.py      # writes tests/golden/ref_<case>.npz

The CPU tests (tests/test_oracle_golden.py) pin the CPU oracle to these files.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from awp_b200 import scenarios  # noqa: E402
from oracle import refbind  # noqa: E402

CASES = {
    "anelastic_if1": dict(nx=16, ny=14, nz=16, q=True, ifault=1, steps=24, seed=21),
    "elastic_if1": dict(nx=15, ny=16, nz=16, q=False, ifault=1, steps=24, seed=22),
    "anelastic_if5": dict(nx=16, ny=16, nz=20, q=True, ifault=5, nsrc=3, steps=40, seed=23),
    "nvar3_if1": dict(nx=14, ny=13, nz=12, nvar=3, ifault=1, steps=16, seed=24),
}
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5",
          "r6"]


def interior(a, nx, ny, nz):
    return np.ascontiguousarray(a[10:10 + nx, 10:10 + ny, 32:32 + nz + 2])


def make_case(name, case):
    case = dict(case)
    steps = case.pop("steps")
    scn = scenarios.random_small(steps=steps, **case)
    setup = refbind.model_setup(scn)
    sim = refbind.RefGpuSim(scn, setup)
    sim.step(steps)
    p = scn.params
    out = {f: interior(sim.field(f), p["nx"], p["ny"], p["nz"]) for f in FIELDS}
    out["steps"] = np.array(steps)
    if p["ifault"] == 5:
        out["mom"] = sim.mom.cpu().numpy()[: setup["psrc"].shape[0]]
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **out)
    return out


def main():
    for name, case in CASES.items():
        out = make_case(name, case)
        print(name, {f: float(np.abs(out[f]).max()) for f in ("u1", "xx", "r1")})


if __name__ == "__main__":
    main()
