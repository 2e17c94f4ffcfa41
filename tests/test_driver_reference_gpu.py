"""The pmcl3d executable against the reference: surface / volume output files
(SX, SY, SZ) of a single-grid run and of a two-block discontinuous mesh.

The reference side runs the reference's own CUDA kernels in pmcl3d's
single-rank order (refbind.RefGpuSim, RefMeshSim) and gathers every NTISKP
steps with the reference's own velbuffer_H (kernel.cu:3927-4011, the w
component one cell below the surface on grid 0), at the recording points of
calcRecordingPoints (calc.c:9-72) restated below; the frames are laid out as
the single-rank file view of pmcl3d.c:489-521 (WRITE_STEP x rec_NZ x rec_NY x
rec_NX floats, x fastest).  Tolerance: relative L2 <= 1e-5 per file."""
import ctypes
import os
import subprocess
from ctypes import c_int, c_void_p

import numpy as np
import pytest
import torch

from awp_b200 import scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PMCL3D = os.path.join(ROOT, "awp_b200", "bin", "pmcl3d")
REL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def recording(n, nbg, ned, nskp, nz_axis=False):
    """NED made a record point (pmcl3d.c:438-440), then calcRecordingPoints at
    coordinate 0 (calc.c:9-72): (first, last, skip, count) of this rank,
    0-based, and the count of the whole file axis."""
    ned = ned - (ned - nbg) % nskp
    full = (ned - nbg) // nskp + 1
    if nz_axis:
        return (nbg - 1, ned - 1, nskp, full), full
    b = nbg - 1
    e = ((n + nbg - 1) % nskp - nskp + n) if n <= ned else ned - 1
    return (b, e, nskp, (e - b) // nskp + 1), full


def write_block(scn, d, p):
    scn.media.astype(np.float32).tofile(os.path.join(d, f"media_{p}"))
    with open(os.path.join(d, f"src_{p}"), "wb") as fh:
        for s in range(scn.src_pos.shape[0]):
            np.asarray(scn.src_pos[s], np.int32).tofile(fh)
            np.asarray(scn.src_data[s], np.float32).tofile(fh)


def velbuffer_frames(lib, sims, axes, nt, ntiskp, bathy=None):
    """Per grid, the reference's velbuffer_H gathered every ntiskp steps
    (FOLLOWBATHY=1 on grid 0 with `bathy`, a device int32 tensor)."""
    V = c_void_p
    lib.velbuffer_H.argtypes = [V] * 8 + [c_int] * 13 + [V, c_int, V, c_int]
    frames = {p: {c: [] for c in "XYZ"} for p in axes}

    def grab(step):
        for p, ax in axes.items():
            sim = sims[p]
            (bx, ex, sx, nxr), (by, ey, sy, nyr), (bz, ez, sz, nzr) = ax
            rec = nxr * nyr * nzr
            bufs = [torch.zeros(rec, device="cuda") for _ in range(4)]
            lib.velbuffer_H(*[c_void_p(sim.f[f].data_ptr()) for f in ("u1", "v1", "w1", "neta")],
                            *[c_void_p(b.data_ptr()) for b in bufs], 1, bx, ex, sx, by, ey, sy,
                            bz, ez, sz, nxr, nyr, nzr, None,
                            1 if (bathy is not None and p == 0) else 0,
                            c_void_p(bathy.data_ptr()) if (bathy is not None and p == 0)
                            else None, p)
            torch.cuda.synchronize()
            for c, b in zip("XYZ", bufs):
                frames[p][c].append(b.cpu().numpy().reshape(nzr, nyr, nxr))
    return frames, grab


def compare_files(out, frames, axes, full, nt, ntiskp, wstep):
    """Each output file against the reference frames; the error of a file is
    its L2 difference over the largest L2 norm of that component's files in
    the run (the first arrivals are orders of magnitude below the later
    wavefield, so their own norm would weigh rounding far beyond its share)."""
    checked = 0
    errs = {}
    files = {}
    for p, ax in axes.items():
        nX, nY, nZ = full[p]
        for step in range(ntiskp * wstep, nt + 1, ntiskp * wstep):
            n0 = step // ntiskp - wstep
            for c in "XYZ":
                got = np.fromfile(os.path.join(out, f"S{c}_{p}_{step:07d}"), np.float32)
                want = np.zeros((wstep, nZ, nY, nX), np.float32)
                for t in range(wstep):
                    fr = frames[p][c][n0 + t]
                    want[t, :fr.shape[0], :fr.shape[1], :fr.shape[2]] = fr
                assert got.size == want.size, (p, c, got.size, want.size)
                files[(p, c, step)] = (got.astype(np.float64), want.ravel().astype(np.float64))
    scale = {}
    for (p, c, step), (_, want) in files.items():
        scale[(p, c)] = max(scale.get((p, c), 0.0), float(np.linalg.norm(want)))
    for (p, c, step), (got, want) in files.items():
        if scale[(p, c)] == 0.0:
            assert not np.any(got), (p, c, step)
            continue
        errs[(p, c, step)] = float(np.linalg.norm(got - want)) / scale[(p, c)]
        checked += 1
    assert checked > 0
    print("\nrel L2 per output file:", {f"{k[1]}_{k[0]}_{k[2]}": f"{v:.1e}" for k, v in errs.items()})
    for k, e in errs.items():
        assert e <= REL, (k, e)
    return checked


def run_driver(args, cwd):
    r = subprocess.run([PMCL3D] + [str(a) for a in args], cwd=cwd, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    return r


def test_single_grid_output_matches_reference(tmp_path):
    nt, ntiskp, wstep = 40, 2, 4
    scn = scenarios.random_small(nx=24, ny=20, nz=32, steps=nt, seed=19, ifault=1, nsrc=2)
    p = scn.params
    write_block(scn, tmp_path, 0)
    tmax = (nt - 1) * p["dt"] + p["dt"] * 0.5
    run_driver(["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
                "-T", tmax, "-D", p["nd"], "-A", p["arbc"], "-V", 1, "-B", 1, "-n", 5,
                "-I", 1, "-S", scn.src_pos.shape[0], "-N", p["nst"], "-R", p["nst"],
                "--INVEL", "media", "--INSRC", "src", "-o", "out", "-c", "chk", "-r", ntiskp,
                "-W", wstep, "--NBGX", 2, "--NEDX", p["nx"], "--NSKPX", 3, "--NBGY", 1,
                "--NEDY", p["ny"] - 1, "--NSKPY", 2, "--NBGZ", 1, "--NEDZ", 5, "--NSKPZ", 2],
               tmp_path)
    ax = (recording(p["nx"], 2, p["nx"], 3), recording(p["ny"], 1, p["ny"] - 1, 2),
          recording(p["nz"], 1, 5, 2, nz_axis=True))
    axes = {0: [a[0] for a in ax]}
    full = {0: tuple(a[1] for a in ax)}
    ref = refbind.RefGpuSim(scn, refbind.model_setup(scn))
    frames, grab = velbuffer_frames(ref.lib, [ref], axes, nt, ntiskp)
    ref.after_step.append(lambda sim, n: grab(n) if n % ntiskp == 0 else None)
    ref.step(nt)
    compare_files(os.path.join(tmp_path, "out"), frames, axes, full, nt, ntiskp, wstep)


def test_two_block_mesh_run_matches_reference(tmp_path):
    """pmcl3d -G 2 (a 3x finer block over a coarse one) against RefMeshSim:
    output of the top block's surface and of a plane of the coarse block."""
    nt, ntiskp, wstep = 36, 2, 3
    scns = scenarios.dm_small(nxc=10, nyc=8, nzs=(36, 24), steps=nt, q=True)
    for p, s in enumerate(scns):
        write_block(s, tmp_path, p)
    p0, p1 = scns[0].params, scns[1].params
    tmax = (nt - 1) * p0["dt"] + p0["dt"] * 0.5
    nsrc = ",".join(str(s.src_pos.shape[0]) for s in scns)
    run_driver(["-G", 2, "-X", p1["nx"], "-Y", p1["ny"], "-Z", f"{p0['nz']},{p1['nz']}",
                "-H", p1["dh"], "-t", p0["dt"], "-T", tmax, "-D", p1["nd"], "-A", p0["arbc"],
                "-V", 1, "-B", 1, "-n", 5, "-I", 1, "-S", nsrc, "-N", p0["nst"],
                "-R", p0["nst"], "--INVEL", "media", "--INSRC", "src", "-o", "out",
                "-c", "chk", "-r", ntiskp, "-W", wstep,
                "--NBGX", "1,2", "--NEDX", f"{p0['nx']},{p1['nx']}", "--NSKPX", "2,2",
                "--NBGY", "1,1", "--NEDY", f"{p0['ny']},{p1['ny']}", "--NSKPY", "3,1",
                "--NBGZ", "1,3", "--NEDZ", "3,3", "--NSKPZ", "1,1"], tmp_path)
    ax0 = (recording(p0["nx"], 1, p0["nx"], 2), recording(p0["ny"], 1, p0["ny"], 3),
           recording(p0["nz"], 1, 3, 1, nz_axis=True))
    ax1 = (recording(p1["nx"], 2, p1["nx"], 2), recording(p1["ny"], 1, p1["ny"], 1),
           recording(p1["nz"], 3, 3, 1, nz_axis=True))
    axes = {0: [a[0] for a in ax0], 1: [a[0] for a in ax1]}
    full = {0: tuple(a[1] for a in ax0), 1: tuple(a[1] for a in ax1)}
    ref = refbind.RefMeshSim(scns, refbind.mesh_setup(scns))
    frames, grab = velbuffer_frames(ref.lib, ref.sims, axes, nt, ntiskp)
    for n in range(1, nt + 1):
        ref.step(1)
        if n % ntiskp == 0:
            grab(n)
    compare_files(os.path.join(tmp_path, "out"), frames, axes, full, nt, ntiskp, wstep)
    chk = open(os.path.join(tmp_path, "chk")).read()
    assert chk.count("GRID NUMBER:") == 2 and chk.strip().endswith("END")


def reference_bathymetry(mu, d1):
    """pmcl3d.c:909-925 restated: per padded column the highest level
    k > align from the top down with sqrt(1/(mu*d1)) > 0.001 (float product,
    double reciprocal and root, float compare), 0 where none; [j][i]."""
    align = refbind.ALIGN
    nxp, nyp, nzp = mu.shape
    top = nzp - align - 1
    out = np.zeros((nyp, nxp), np.int32)
    vs = np.sqrt(1.0 / (mu * d1).astype(np.float64)).astype(np.float32)
    for k in range(top, align, -1):
        hit = (vs[:, :, k] > np.float32(0.001)).T & (out == 0)
        out[hit] = k
    return out


def test_followbathy_output_matches_reference(tmp_path):
    """FOLLOWBATHY=1: a near-fluid top layer (vs 0.5 mm/s, three cells thick)
    over half of the surface; the driver's output files against the
    reference's velbuffer_H with the surface levels pmcl3d derives, and the
    library's levels against that derivation."""
    nt, ntiskp, wstep = 32, 2, 4
    scn = scenarios.random_small(nx=24, ny=20, nz=32, steps=nt, seed=29, ifault=1, nsrc=2)
    p = scn.params
    scn.media[:3, :, : p["nx"] // 2, 1] = 0.0005
    write_block(scn, tmp_path, 0)
    tmax = (nt - 1) * p["dt"] + p["dt"] * 0.5
    r = run_driver(["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
                    "-T", tmax, "-D", p["nd"], "-A", p["arbc"], "-V", 1, "-B", 1, "-n", 5,
                    "-I", 1, "-S", scn.src_pos.shape[0], "-N", p["nst"], "-R", p["nst"],
                    "--INVEL", "media", "--INSRC", "src", "-o", "out", "-c", "chk", "-r",
                    ntiskp, "-W", wstep, "--NBGX", 1, "--NEDX", p["nx"], "--NSKPX", 1,
                    "--NBGY", 1, "--NEDY", p["ny"], "--NSKPY", 1, "--NBGZ", 1, "--NEDZ", 3,
                    "--NSKPZ", 1, "--FOLLOWBATHY", 1], tmp_path)
    assert os.path.getsize(os.path.join(tmp_path, "debug", "bathy.0000")) > 0, r.stdout
    ax = (recording(p["nx"], 1, p["nx"], 1), recording(p["ny"], 1, p["ny"], 1),
          recording(p["nz"], 1, 3, 1, nz_axis=True))
    axes = {0: [a[0] for a in ax]}
    full = {0: tuple(a[1] for a in ax)}
    ref = refbind.RefGpuSim(scn, refbind.model_setup(scn))
    bathy = reference_bathymetry(ref.f["mu"].cpu().numpy(), ref.f["d1"].cpu().numpy())
    top = ref.f["mu"].shape[2] - refbind.ALIGN - 1
    inner = bathy[refbind.NGSL + 2: refbind.NGSL + 2 + p["ny"],
                  refbind.NGSL + 2: refbind.NGSL + 2 + p["nx"]]
    assert (inner[:, : p["nx"] // 2] == top - 3).all() and (inner[:, p["nx"] // 2:] == top).all()

    from awp_b200 import Solver, default_params
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    assert np.array_equal(s.bathymetry(), bathy)
    s.close()

    dev = torch.from_numpy(bathy).cuda()
    frames, grab = velbuffer_frames(ref.lib, [ref], axes, nt, ntiskp, bathy=dev)
    ref.after_step.append(lambda sim, n: grab(n) if n % ntiskp == 0 else None)
    ref.step(nt)
    compare_files(os.path.join(tmp_path, "out"), frames, axes, full, nt, ntiskp, wstep)
