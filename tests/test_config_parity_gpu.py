"""Parity at the sizes of the benchmark configurations, not only on small grids.

* Elastic half-space, 128^3, h = 100 m, dt = 5 ms, Mxy Ricker' source at the
  centre, 16 surface receivers on a seeded layout, the whole 500-step run:
  the product, the reference's own CUDA build driven in pmcl3d's single-rank
  order (refbind.RefGpuSim) and the FP64 oracle; every wavefield component at
  the end and every seismogram sample.
* Anelastic layered + von Karman model, 512 x 512 x 256, h = 50 m, 200
  kinematic subfaults, 256 surface receivers, 160 steps (of the run's 2000):
  the product against the reference build on the final wavefield and the
  seismograms, and against the FP64 oracle on the final wavefield.
* The misfit gradient on a 64^3 anelastic model over 200 steps against the
  FP64 dual-number oracle's exact derivative and against central differences.

Tolerances: relative L2 <= 1e-5 against the reference build, <= 1e-4 against
the FP64 oracle (FP32 rounding accumulated over the steps), 1e-3 for the
gradient.  Each test prints the errors it measured."""
import numpy as np
import pytest
import torch

from awp_b200 import Solver, adjoint, default_params, scenarios
from oracle import oracle as orc
from oracle import refbind

pytestmark = pytest.mark.gpu

REL_REF = 1e-5
REL_F64 = 1e-4
WAVE = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz"]
NAMES = ["u1", "v1", "w1"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


class _Dev:
    """A raw device float32 array seen by torch without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3}


def surface_receivers(rng, n, nx, ny, margin):
    x = rng.integers(margin, nx - margin, n)
    y = rng.integers(margin, ny - margin, n)
    return np.stack([x, y, np.zeros(n, np.int64)], 1)


def padded_index(xyz, p):
    """Linear index of interior cell (x, y, z from the surface) in the padded layout."""
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    sl, yl = (ny + 20) * (nz + 64), nz + 64
    return np.array([(x + 10) * sl + (y + 10) * yl + (nz + 31 - z) for x, y, z in xyz],
                    np.int64)


def product_run(scn, steps, idx):
    """Steps the product one at a time and samples u, v, w at idx after each."""
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    n = int(np.prod(refbind.padded_shape(scn.params["nx"], scn.params["ny"], scn.params["nz"])))
    views = [torch.as_tensor(_Dev(s.device_ptr(f), n), device="cuda") for f in NAMES]
    ti = torch.as_tensor(idx, device="cuda")
    seis = []
    for _ in range(steps):
        s.step(1)
        s.synchronize()
        seis.append(torch.stack([v[ti] for v in views]).cpu().numpy())
    return s, np.stack(seis)  # [steps][3][nrec]


def reference_run(scn, setup, steps, idx):
    ref = refbind.RefGpuSim(scn, setup)
    ti = torch.as_tensor(idx, device="cuda")
    seis = []
    ref.after_step.append(
        lambda sim, n: seis.append(torch.stack([sim.f[f].view(-1)[ti] for f in NAMES])
                                   .cpu().numpy()))
    ref.step(steps)
    return ref, np.stack(seis)


def test_config1_elastic_halfspace_128_full_run():
    steps = 500
    scn = scenarios.halfspace(steps=steps)
    p = scn.params
    rng = np.random.default_rng(1)
    xyz = surface_receivers(rng, 16, p["nx"], p["ny"], 21)
    idx = padded_index(xyz, p)
    setup = refbind.model_setup(scn)

    s, seis = product_run(scn, steps, idx)
    ref, seis_ref = reference_run(scn, setup, steps, idx)

    o = orc.OracleSim(scn, setup, precision=64)
    seis_64 = []
    for _ in range(steps):
        o.step(1)
        seis_64.append(np.stack([o.field(f, f64=True).reshape(-1)[idx] for f in NAMES]))
    seis_64 = np.stack(seis_64)

    assert np.abs(seis_ref).max() > 0
    report = {"seismograms": (rel_l2(seis, seis_ref), rel_l2(seis, seis_64),
                              rel_l2(seis_ref, seis_64))}
    for f in WAVE:
        a, r, b = s.field(f), ref.field(f), o.field(f, f64=True)
        report[f] = (rel_l2(a, r), rel_l2(a, b), rel_l2(r, b))
    for k, (vs_ref, vs_64, _) in report.items():
        assert vs_ref <= REL_REF, (k, report[k])
        assert vs_64 <= REL_F64, (k, report[k])
    print("\n128^3 half-space, 500 steps: rel L2 (product vs reference build, product vs FP64, "
          "reference build vs FP64):",
          {k: tuple(f"{x:.1e}" for x in v) for k, v in report.items()})
    s.close()
    o.close()


def test_config2_layered_512_reduced_steps():
    steps = 160
    scn = scenarios.layered_vk(steps=steps)
    p = scn.params
    rng = np.random.default_rng(2)
    xyz = surface_receivers(rng, 256, p["nx"], p["ny"], 21)
    idx = padded_index(xyz, p)
    setup = refbind.model_setup(scn)

    s, seis = product_run(scn, steps, idx)
    mine = {f: s.field(f) for f in WAVE}
    s.close()
    torch.cuda.empty_cache()
    ref, seis_ref = reference_run(scn, setup, steps, idx)
    report = {"seismograms": rel_l2(seis, seis_ref)}
    for f in WAVE:
        report[f] = rel_l2(mine[f], ref.field(f))
    del ref
    torch.cuda.empty_cache()
    assert np.abs(seis_ref).max() > 0
    for k, v in report.items():
        assert v <= REL_REF, (k, v)

    o = orc.OracleSim(scn, setup, precision=64)
    del setup
    o.step(steps)
    f64 = {f: rel_l2(mine[f], o.field(f, f64=True)) for f in WAVE}
    o.close()
    for k, v in f64.items():
        assert v <= REL_F64, (k, v)
    print("\n512x512x256 layered model, 160 steps: rel L2 vs reference build",
          {k: f"{v:.1e}" for k, v in report.items()}, "vs FP64",
          {k: f"{v:.1e}" for k, v in f64.items()})


def test_config4_gradient_64cube():
    from test_adjoint_gpu import J_at, moduli, oracle_directional
    steps = 200
    scn = scenarios.random_small(nx=64, ny=64, nz=64, h=100.0, dt=0.005, q=True, ifault=1,
                                 steps=steps, seed=5, nsrc=1)
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    lam, mu, rho = moduli(scn)
    rng = np.random.default_rng(6)
    xyz = np.concatenate([surface_receivers(rng, 12, 64, 64, 4),
                          np.stack([rng.integers(4, 60, 4), rng.integers(4, 60, 4),
                                    rng.integers(2, 40, 4)], 1)]).astype(np.int32)
    comp = (np.arange(16) % 3).astype(np.int32)
    pert = [(1 + 0.03 * rng.standard_normal(lam.shape)).astype(np.float32) for _ in range(3)]
    s.set_moduli(lam * pert[0], mu * pert[1], rho * pert[2])
    s.reset()
    d_obs = adjoint.seismograms(s, steps, xyz, comp)
    m = (lam, mu, rho)
    s.set_moduli(*m)
    s.reset()
    J, _, gl, gm, gr = adjoint.misfit_gradient(s, steps, xyz, comp, d_obs, nsnap=14)
    assert J > 0
    eps = 1e-3
    rows = []
    for d in range(2):
        dm = tuple((x * rng.standard_normal(x.shape)).astype(np.float64) for x in m)
        adj = float(np.sum(gl * dm[0]) + np.sum(gm * dm[1]) + np.sum(gr * dm[2]))
        tan = oracle_directional(scn, m, dm, steps, xyz, comp, d_obs)
        mp = tuple((x + eps * y).astype(np.float32) for x, y in zip(m, dm))
        mm = tuple((x - eps * y).astype(np.float32) for x, y in zip(m, dm))
        fd = (J_at(s, mp, steps, xyz, comp, d_obs) - J_at(s, mm, steps, xyz, comp, d_obs)) / (
            2 * eps)
        rows.append((adj, tan, fd))
        assert abs(adj - tan) <= 1e-3 * abs(tan), (d, adj, tan)
        assert abs(adj - fd) <= 1e-3 * abs(adj), (d, adj, fd)
    print("\n64^3, 200 steps: (adjoint, FP64 tangent, central difference) per direction:",
          [tuple(f"{x:.6e}" for x in r) for r in rows])
    s.close()
