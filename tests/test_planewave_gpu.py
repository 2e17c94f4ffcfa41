"""Plane-wave input (IFAULT=6: ini_plane_wave, source.c:797-833; addplanesrc_H
on level align + ND + 1 of the bottom grid while cur_step < NST,
pmcl3d.c:2035-2041, kernel.cu:3860-3925) against the reference's own CUDA
build driven in pmcl3d's single-rank order and against the FP64 oracle, then
through the pmcl3d driver (INSRC text file of NST lines "vx vy vz").

Tolerances: relative L2 <= 1e-5 against the reference build, <= 1e-4 against
the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

from awp_b200 import Solver, default_params, scenarios
from oracle import oracle as orc
from oracle import refbind

pytestmark = pytest.mark.gpu

FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r4"]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def plane_series(nst, dt, seed=5):
    """A Ricker-like velocity history per component, seeded amplitudes."""
    rng = np.random.default_rng(seed)
    t = np.arange(nst) * dt
    t0, f0 = 8 * dt, 1.0 / (6 * dt)
    a = (np.pi * f0 * (t - t0)) ** 2
    w = (1 - 2 * a) * np.exp(-a)
    return [(rng.uniform(0.5, 1.5) * 1e-2 * w).astype(np.float32) for _ in range(3)]


def case(steps=30, q=True, nz=32):
    """A homogeneous medium (constant Q where q): the plane enters rows 4 .. 3 +
    nx of the padded grid, six of them in the ghost region, where both builds
    read the media as they are; the tests fill the whole padded arrays as
    MEDIASTART 0 does (mesh.c:80-87).  With the ghost media left zero, as the
    reference's inimesh leaves them for MEDIASTART >= 1 at one rank, its
    division by mu there gives inf in both builds."""
    scn = scenarios.random_small(nx=24, ny=20, nz=nz, q=q, ifault=1, steps=steps, seed=17,
                                 nsrc=1)
    # vp, vs, rho, then qp, qs where the run is anelastic
    for col, v in enumerate((3400.0, 2000.0, 2500.0, 150.0, 75.0)[: 5 if q else 3]):
        scn.media[..., col] = v
    scn.params.update(ifault=6, nst=steps, read_step=steps, nd=6)
    return scn


def fill_padding(s, ref=None, oracle=None):
    """The product's interior d1 / 1/mu / 1/lambda (homogeneous) over the whole
    padded arrays, in the product, the reference binding and the oracle."""
    full = {}
    for f in ("d1", "mu", "lam"):
        a = s.field(f)
        v = a[a.shape[0] // 2, a.shape[1] // 2, a.shape[2] // 2]
        full[f] = np.full(a.shape, v, np.float32)
        s.set_field(f, full[f])
        if ref is not None:
            assert ref.f[f][a.shape[0] // 2, a.shape[1] // 2, a.shape[2] // 2].item() == v
            ref.f[f].fill_(float(v))
        if oracle is not None:
            oracle.set_field(f, full[f])
    return full


@pytest.mark.parametrize("q", [True, False])
def test_plane_wave_matches_reference_and_oracle(q):
    steps = 30
    scn = case(steps, q)
    p = scn.params
    vx, vy, vz = plane_series(p["nst"], p["dt"])
    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    ref.set_plane_wave(vx, vy, vz)
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    o = orc.OracleSim(scn, setup, 64)
    fill_padding(s, ref, o)
    ref.step(steps)
    s.upload_plane_wave(vx, vy, vz)
    s.step(steps)
    s.synchronize()
    o.set_plane_wave(vx, vy, vz)
    o.step(steps)
    assert np.abs(ref.field("xx")).max() > 0
    rep = {}
    for f in FIELDS:
        a, r, b = s.field(f), ref.field(f), o.field(f, f64=True)
        rep[f] = (rel_l2(a, r), rel_l2(a, b))
        if np.linalg.norm(r) == 0:
            assert np.linalg.norm(a) == 0, f
            continue
        assert rep[f][0] <= 1e-5, (f, rep[f])
        assert rep[f][1] <= 1e-4, (f, rep[f])
    print("\\nplane wave rel L2 (vs reference build, vs FP64):",
          {k: tuple(f"{x:.1e}" for x in v) for k, v in rep.items()})
    s.close()


def test_plane_wave_rules():
    scn = case()
    p = scn.params
    vx, vy, vz = plane_series(p["nst"], p["dt"])
    s = Solver(default_params(**p))
    with pytest.raises(RuntimeError):
        s.upload_plane_wave(vx[:-1], vy[:-1], vz[:-1])  # NST samples wanted
    s.close()
    p1 = dict(p, ifault=1)
    s = Solver(default_params(**p1))
    with pytest.raises(RuntimeError):
        s.upload_plane_wave(vx, vy, vz)  # only an IFAULT=6 run takes it
    s.close()


def test_driver_plane_wave_run(tmp_path):
    """pmcl3d -I 6 with the series in an INSRC text file: its surface output
    files equal the library run's gathered frames bit for bit."""
    nt = 48  # the plane enters 7 levels above the bottom of 16: ~30 steps to the surface
    scn = case(nt, nz=16)
    p = scn.params
    vx, vy, vz = plane_series(p["nst"], p["dt"])
    scn.media.astype(np.float32).tofile(os.path.join(tmp_path, "media_0"))
    # nine decimals: every float32 sample reads back exactly through fscanf "%e"
    with open(os.path.join(tmp_path, "planewave.txt"), "w") as fh:
        for a, b, c in zip(vx, vy, vz):
            fh.write(f"{a:.9e} {b:.9e} {c:.9e}\n")
    ntiskp, wstep = 2, 4
    tmax = (nt - 1) * p["dt"] + p["dt"] * 0.5
    args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
            "-T", tmax, "-D", p["nd"], "-A", p["arbc"], "-V", 1, "-B", 0, "-n", 5,
            "-I", 6, "-S", 0, "-N", p["nst"], "-R", p["nst"],
            "--INVEL", "media", "--INSRC", "planewave.txt", "-o", "out", "-c", "chk",
            "-r", ntiskp, "-W", wstep, "--NBGX", 1, "--NEDX", p["nx"], "--NSKPX", 1,
            "--NBGY", 1, "--NSKPY", 1, "--NBGZ", 1, "--NEDZ", 1, "--NSKPZ", 1]
    exe = os.path.join(ROOT, "awp_b200", "bin", "pmcl3d")
    r = subprocess.run([exe] + [str(x) for x in args], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    assert "Using plane wave input" in r.stdout
    import torch
    s = Solver(default_params(**p))
    # MEDIASTART 0 (mesh.c:80-87, the driver's homogeneous fill): vp 1500, vs 500,
    # rho 2000 over the whole padded grid
    shape = s.field("d1").shape
    vp, vs, dd = 1500.0, 500.0, 2000.0
    s.set_field("d1", np.full(shape, dd, np.float32))
    s.set_field("mu", np.full(shape, np.float32(1.0 / (dd * vs * vs)), np.float32))
    s.set_field("lam", np.full(shape, np.float32(1.0 / (dd * (vp * vp - 2.0 * vs * vs))),
                               np.float32))
    s.upload_plane_wave(vx, vy, vz)
    rec = p["nx"] * p["ny"]
    bufs = [torch.zeros(rec, device="cuda") for _ in range(3)]
    frames = {c: [] for c in "XYZ"}
    for step in range(1, nt + 1):
        s.step(1)
        if step % ntiskp == 0:
            s.gather(0, p["nx"] - 1, 1, 0, p["ny"] - 1, 1, 0, 0, 1, *[b.data_ptr() for b in bufs])
            s.synchronize()
            for c, b in zip("XYZ", bufs):
                frames[c].append(b.cpu().numpy().copy())
    s.close()
    assert max(np.abs(f).max() for f in frames["Z"]) > 0
    for step in range(ntiskp * wstep, nt + 1, ntiskp * wstep):
        n0 = step // ntiskp - wstep
        for c in "XYZ":
            got = np.fromfile(os.path.join(tmp_path, "out", f"S{c}_0_{step:07d}"), np.float32)
            want = np.concatenate(frames[c][n0:n0 + wstep])
            assert got.shape == want.shape, (c, got.shape, want.shape)
            assert np.array_equal(got, want), (c, step)
