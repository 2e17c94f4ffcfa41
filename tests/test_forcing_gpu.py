"""IFAULT=4 prescribed velocities (frcvel_cu, kernel.cu:1836-1934) through the
context API against the reference's own frcvel_H driven in pmcl3d's
single-rank order (pmcl3d.c:714-722, 792-805, 1175, 1821-1826, 2442-2486):
windows of frames with a carry slot, linear interpolation over tskp steps,
the restoring force of the last prescribed step applied every later step.
Then through the pmcl3d driver, whose INSRC parameters and sub-volume reads
(read_src_ifault_4 and read_awp_subvolume, source.c:377-680) are restated
below.  Tolerance: relative L2 <= 1e-5 against the reference build; the
driver's files equal the library run's frames bit for bit."""
import os
import subprocess
from ctypes import c_int, c_void_p

import numpy as np
import pytest
import torch

from awp_b200 import Solver, default_params, scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r4"]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def box_points(i0, i1, j0, j1, k0, k1, nz, seismio=0):
    """read_src_ifault_4's point order (source.c:571-596): k outermost (from
    the bottom up with SEISM-IO output), then j, then i; z = NZ - k + 1."""
    ks = range(k1, k0 - 1, -1) if seismio else range(k0, k1 + 1)
    return np.array([(i, j, nz - k + 1) for k in ks for j in range(j0, j1 + 1)
                     for i in range(i0, i1 + 1)], np.int32)


@pytest.mark.parametrize("tskp,window,nframes", [(3, 4, 8), (1, 5, 10)])
def test_prescribed_velocities_match_reference(tskp, window, nframes):
    steps = nframes * tskp + 6  # six steps of the static force after the last frame
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=True, ifault=1, steps=steps, seed=31,
                                 nsrc=1)
    p = scn.params
    p.update(ifault=4, nst=nframes, read_step=window)
    pos = box_points(6, 9, 5, 7, 3, 5, p["nz"])
    npsrc = pos.shape[0]
    rng = np.random.default_rng(8)
    frames = [(rng.standard_normal((nframes, npsrc)) * 1e-2).astype(np.float32)
              for _ in range(3)]

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.velocity_forcing(pos, *frames, tskp=tskp, window=window)
    s.step(steps)
    s.synchronize()

    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    lib = ref.lib
    V = c_void_p
    lib.frcvel_H.argtypes = [c_int, c_int, c_int, V, c_int, c_int, V] + [V] * 9 + [c_int] * 3
    d_pos = torch.from_numpy(pos.reshape(-1)).cuda()
    d_a = [torch.zeros((window + 1) * npsrc, device="cuda") for _ in range(3)]
    for q in range(3):  # the first window, carry slot zero (pmcl3d.c:792-805)
        d_a[q][npsrc:] = torch.from_numpy(frames[q][:window].reshape(-1)).cuda()
    state = {"step": 1, "next": 1}  # source_step = 1 before the loop (pmcl3d.c:1175)

    def forcing(sim, cur):
        state["step"] += 1
        lib.frcvel_H(state["step"], window, 3, V(d_pos.data_ptr()), npsrc, tskp, None,
                     *[V(a.data_ptr()) for a in d_a], None, None, None,
                     *[V(sim.f[f].data_ptr()) for f in ("u1", "v1", "w1")], -1, -1, 0)

    def refresh(sim, cur):
        if cur < nframes * tskp - 1 and (cur + 1) % (window * tskp) == 0:
            w = state["next"]
            for q in range(3):
                d_a[q][npsrc:] = torch.from_numpy(
                    frames[q][w * window:(w + 1) * window].reshape(-1)).cuda()
            state["next"] += 1
            state["step"] = 0

    ref.after_velocity.append(forcing)
    ref.after_step.append(refresh)
    ref.step(steps)
    assert state["next"] == nframes // window
    rep = {}
    for f in FIELDS:
        rep[f] = rel_l2(s.field(f), ref.field(f))
        assert rep[f] <= 1e-5, (f, rep[f])
    assert float(torch.abs(ref.f["xx"]).max()) > 0
    print("\nIFAULT 4 rel L2 vs reference build:", {k: f"{v:.1e}" for k, v in rep.items()})
    s.close()


def test_forcing_rules():
    scn = scenarios.random_small(nx=16, ny=16, nz=16, q=False, ifault=1, steps=4, seed=3,
                                 nsrc=1)
    p = dict(scn.params, ifault=4, nst=4, read_step=2)
    pos = box_points(3, 4, 3, 4, 2, 2, p["nz"])
    fr = [np.zeros((4, 4), np.float32)] * 3
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    with pytest.raises(RuntimeError):
        s.velocity_forcing(pos, *[a[:3] for a in fr], tskp=1, window=2)  # 3 frames, window 2
    with pytest.raises(RuntimeError):
        s.velocity_forcing(np.array([[40, 3, 3]], np.int32), *[a[:, :1] for a in fr], tskp=1,
                           window=2)  # outside the padded grid
    s.close()
    s = Solver(default_params(**dict(p, ifault=1)))
    with pytest.raises(RuntimeError):
        s.velocity_forcing(pos, *fr, tskp=1, window=2)  # only an IFAULT=4 run takes them
    s.close()


def subvolume(files, dim, extg, t0, t1, seismio):
    """read_awp_subvolume (source.c:377-461): frames t0..t1-1 of the
    sub-volume, [t][points] in the reading order."""
    nx, ny, nz = dim
    x0, x1, y0, y1, z0, z1 = extg
    out = []
    for name in files:
        a = np.fromfile(name, np.float32).reshape(-1, nz, ny, nx)
        ks = list(range(z0, z1)) if seismio else [nz - k - 1 for k in range(z1 - 1, z0 - 1, -1)]
        out.append(np.stack([a[t0:t1, k, y0:y1, x0:x1] for k in ks], 1).reshape(t1 - t0, -1))
    return out


@pytest.mark.parametrize("seismio", [0, 1])
def test_driver_prescribed_velocities(tmp_path, seismio):
    """pmcl3d -I 4: the INSRC parameter file and the previous run's volume
    output files; surface output equal to the library run bit for bit."""
    nt, tskp, window, nframes = 30, 2, 4, 12
    scn = scenarios.random_small(nx=16, ny=16, nz=16, q=True, ifault=1, steps=nt, seed=41,
                                 nsrc=1)
    p = dict(scn.params, ifault=4, nst=nframes, read_step=window)
    scn.media.astype(np.float32).tofile(tmp_path / "media_0")
    dim = (30, 28, 20)
    off = (3, 2, 4)
    ext = (4, 9, 5, 8, 2, 4)  # x, y, z extents of the prescribed volume
    os.makedirs(tmp_path / "dyn")
    rng = np.random.default_rng(5)
    for c in "XYZ":
        (rng.standard_normal((nframes,) + dim[::-1]) * 1e-2).astype(np.float32).tofile(
            tmp_path / "dyn" / f"S{c}")
    with open(tmp_path / "frc.txt", "w") as fh:
        fh.write(f"{ext[0]} {ext[1]}\n{ext[2]} {ext[3]}\n{ext[4]} {ext[5]}\n")
        fh.write(f"{dim[0]} {dim[1]} {dim[2]}\n{off[0]} {off[1]} {off[2]}\n")
        fh.write(f"dyn/S%c\n{seismio}\n{tskp}\n")
    ntiskp, wstep = 2, 3
    args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
            "-T", (nt - 1) * p["dt"] + 0.5 * p["dt"], "-D", p["nd"], "-A", p["arbc"],
            "-V", 1, "-B", 1, "-n", 5, "-I", 4, "-S", 1, "-N", nframes, "-R", window,
            "--INVEL", "media", "--INSRC", "frc.txt", "-o", "out", "-c", "chk",
            "-r", ntiskp, "-W", wstep, "--NBGX", 1, "--NEDX", p["nx"], "--NSKPX", 1,
            "--NBGY", 1, "--NSKPY", 1, "--NBGZ", 1, "--NEDZ", 1, "--NSKPZ", 1]
    exe = os.path.join(ROOT, "awp_b200", "bin", "pmcl3d")
    r = subprocess.run([exe] + [str(a) for a in args], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]

    pos = box_points(ext[0], ext[1], ext[2], ext[3], ext[4], ext[5], p["nz"], seismio)
    extg = (ext[0] + off[0] - 1, ext[1] + off[0], ext[2] + off[1] - 1, ext[3] + off[1],
            ext[4] + off[2] - 1, ext[5] + off[2])
    frames = subvolume([tmp_path / "dyn" / f"S{c}" for c in "XYZ"], dim, extg, 0, nframes,
                       seismio)
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.velocity_forcing(pos, *frames, tskp=tskp, window=window)
    rec = p["nx"] * p["ny"]
    bufs = [torch.zeros(rec, device="cuda") for _ in range(3)]
    got = {c: [] for c in "XYZ"}
    for step in range(1, nt + 1):
        s.step(1)
        if step % ntiskp == 0:
            s.gather(0, p["nx"] - 1, 1, 0, p["ny"] - 1, 1, 0, 0, 1, *[b.data_ptr() for b in bufs])
            s.synchronize()
            for c, b in zip("XYZ", bufs):
                got[c].append(b.cpu().numpy().copy())
    s.close()
    assert max(np.abs(f).max() for f in got["X"]) > 0
    for step in range(ntiskp * wstep, nt + 1, ntiskp * wstep):
        n0 = step // ntiskp - wstep
        for c in "XYZ":
            out = np.fromfile(tmp_path / "out" / f"S{c}_0_{step:07d}", np.float32)
            want = np.concatenate(got[c][n0:n0 + wstep])
            assert np.array_equal(out, want), (c, step)
