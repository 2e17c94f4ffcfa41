"""SGTFILE output (topography/receivers/sgt.c: receivers of the six stresses
on their staggered grids, and the material on the node grid written once)
against the reference's own point-set device code (cuinterp_interp_H through
ref_points_shim.c) hooked into the reference's CUDA kernels run in pmcl3d's
single-rank order, and through the pmcl3d driver.  Tolerance: relative L2
<= 1e-5 against the reference build."""
import os
import subprocess

import numpy as np
import pytest
import torch

from awp_b200 import Solver, default_params, pointfiles, scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

GT = {"Gxx": 3, "Gyy": 4, "Gzz": 5, "Gxy": 6, "Gxz": 7, "Gyz": 8}
FIELD = {"Gxx": "xx", "Gyy": "yy", "Gzz": "zz", "Gxy": "xy", "Gxz": "xz", "Gyz": "yz"}
NODE = 9
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def layout(rng, n, nx, ny, nz, h):
    x = rng.uniform(2 * h, (nx - 3) * h, n)
    y = rng.uniform(2 * h, (ny - 3) * h, n)
    z = -rng.uniform(0.0, (nz - 4) * h, n)
    # volume coordinates: a surface coordinate lies above the top stress node of
    # the normal-stress and xy grids, which the reference refuses (error 701)
    t = np.zeros(n, np.int32)
    return np.stack([x, y, z], 1), t


def test_sgt_files_match_reference(tmp_path):
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=True, ifault=1, steps=24, seed=23)
    p = scn.params
    nx, ny, nz, h = p["nx"], p["ny"], p["nz"], p["dh"]
    gpu, cpu, nw, stride = 2, 2, 2, 2
    nsteps = gpu * cpu * nw * stride
    nt = nsteps + 1
    rng = np.random.default_rng(7)
    coords, types = layout(rng, 10, nx, ny, nz, h)
    base = str(tmp_path / "sgt")
    path = str(tmp_path / "sgt.txt")
    pointfiles.write_input(path, base, coords, types, degree=3, gpu_buffer_size=gpu,
                           cpu_buffer_size=cpu, num_writes=nw, stride=stride, steps=1)

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.sgt(path, nt)
    s.step(nsteps)
    s.synchronize()
    got = pointfiles.read_receiver_series(base, 10, nt, gpu, cpu, nw, stride,
                                          components=pointfiles.COMPONENTS_SGT)
    s.close()

    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    pts = {c: refbind.RefPoints(path, GT[c], nx, ny, nz, h) for c in GT}
    samples = {c: [] for c in GT}
    out = torch.zeros(64, device="cuda")

    def record(sim, step):
        if step % stride:
            return
        for c, rp in pts.items():
            out.zero_()
            rp.interp(out.data_ptr(), sim.f[FIELD[c]].data_ptr())
            samples[c].append(out[: rp.count].cpu().numpy().copy())

    record(ref, 0)
    ref.after_step.append(record)
    ref.step(nsteps)
    host = refbind.RefHost()
    nsamp = nsteps // stride
    for c in GT:
        idx = host.point_coefs(path, GT[c], nx, ny, nz, h)["indices"]
        mine = got[c][idx][:, :nsamp]
        want = np.stack(samples[c][:nsamp], 1)
        assert mine.shape == want.shape, (c, mine.shape, want.shape)
        assert np.abs(want).max() > 0, c
        assert rel_l2(mine, want) <= 1e-5, (c, rel_l2(mine, want))

    # the material on the node grid, one sample per point; "_d1" holds 1/lambda
    # as the reference writes it
    node = refbind.RefPoints(path, NODE, nx, ny, nz, h)
    idx = host.point_coefs(path, NODE, nx, ny, nz, h)["indices"]
    for suffix, fld in (("d1", "lam"), ("lami", "lam"), ("mui", "mu")):
        out.zero_()
        node.interp(out.data_ptr(), ref.f[fld].data_ptr())
        want = out[: node.count].cpu().numpy()
        mine = np.fromfile(f"{base}_{suffix}", np.float32)[idx]
        assert rel_l2(mine, want) <= 1e-6, (suffix, rel_l2(mine, want))


def test_driver_writes_sgt_files(tmp_path):
    scn = scenarios.random_small(nx=16, ny=16, nz=16, q=False, ifault=1, steps=8, seed=5, nsrc=1)
    p = scn.params
    scn.media.astype(np.float32).tofile(os.path.join(tmp_path, "media_0"))
    with open(os.path.join(tmp_path, "src_0"), "wb") as fh:
        for k in range(scn.src_pos.shape[0]):
            np.asarray(scn.src_pos[k], np.int32).tofile(fh)
            np.asarray(scn.src_data[k], np.float32).tofile(fh)
    coords = np.array([[5 * p["dh"], 6 * p["dh"], -3 * p["dh"]],
                       [7 * p["dh"], 7 * p["dh"], -5.5 * p["dh"]]])
    pointfiles.write_input(str(tmp_path / "sgt.txt"), "sgt", coords, [0, 0], degree=1)
    nt = 8
    args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
            "-T", (nt - 1) * p["dt"] + 0.5 * p["dt"], "-D", p["nd"], "-V", 1, "-B", 1, "-n", 5,
            "-I", 1, "-S", 1, "-N", p["nst"], "-R", p["nst"], "--INVEL", "media",
            "--INSRC", "src", "--SGTFILE", "sgt.txt"]
    exe = os.path.join(ROOT, "awp_b200", "bin", "pmcl3d")
    r = subprocess.run([exe] + [str(a) for a in args], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    for suffix in ("d1", "lami", "mui"):
        assert os.path.getsize(os.path.join(tmp_path, f"sgt_{suffix}")) == 2 * 4
    files = [f for f in os.listdir(tmp_path) if f.startswith("sgt_Gxx_")]
    assert files, os.listdir(tmp_path)
