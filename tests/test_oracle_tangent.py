"""The FP64 oracle on dual numbers (tangent-linear mode) -- the reference the
adjoint gradient is checked against -- pinned by central differences of the
plain FP64 oracle (CPU only)."""
import numpy as np

from awp_b200 import scenarios
from oracle import oracle as orc
from oracle import refbind


def test_dual_oracle_tangent_equals_fp64_differences():
    scn = scenarios.random_small(nx=12, ny=12, nz=12, q=True, ifault=1, steps=10, seed=4,
                                 nsrc=1)
    p = scn.params
    setup = refbind.model_setup(scn)
    m = setup["media"]
    rng = np.random.default_rng(2)
    shape = refbind.padded_shape(p["nx"], p["ny"], p["nz"])
    dirs = {k: rng.standard_normal(shape) * np.abs(np.asarray(m[k], np.float64))
            for k in ("lam", "mu", "d1")}
    probe = (p["nx"] // 2 + 10, p["ny"] // 2 + 10, p["nz"] + 30)

    def run(eps, dual):
        o = orc.OracleSim(scn, setup, precision=65 if dual else 64)
        for k, d in dirs.items():
            base = np.asarray(m[k], np.float64)
            if dual:
                o.set_tangent(k, d)
            else:
                # perturb in double through the float32 interface: the values
                # are exactly representable steps of the base only for eps
                # large enough, so compare to the tolerance below
                o.set_field(k, (base + eps * d).astype(np.float32))
        o.compute_lam_mu()
        o.step(10)
        val = [o.field(f, f64=True)[probe] for f in ("u1", "v1", "w1", "xx")]
        tan = [o.tangent(f)[probe] for f in ("u1", "v1", "w1", "xx")] if dual else None
        o.close()
        return val, tan

    _, tan = run(0.0, True)
    eps = 1e-3
    vp, _ = run(eps, False)
    vm, _ = run(-eps, False)
    for t, a, b in zip(tan, vp, vm):
        fd = (a - b) / (2 * eps)
        assert abs(t - fd) <= 2e-3 * max(abs(fd), 1e-30), (t, fd)
