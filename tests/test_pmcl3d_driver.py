"""The pmcl3d command-line drop-in: argument handling (CPU) and a full run with
the reference's input and output files (GPU)."""
import os
import subprocess

import numpy as np
import pytest

from awp_b200 import Solver, default_params, scenarios

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PMCL3D = os.path.join(ROOT, "awp_b200", "bin", "pmcl3d")


def run(args, cwd, timeout=300):
    return subprocess.run([PMCL3D] + [str(a) for a in args], cwd=cwd, capture_output=True,
                          text=True, timeout=timeout)


def test_binary_exists():
    assert os.access(PMCL3D, os.X_OK)


def test_rejects_multi_rank(tmp_path):
    r = run(["-x", "2"], tmp_path)
    assert r.returncode == 1 and "one rank" in r.stderr


def test_nz_block_rule(tmp_path):
    # pmcl3d.c:380-391: NZ must be divisible by BLOCK_SIZE_Z (4); the reference
    # prints the message and returns 0
    r = run(["-Z", "30"], tmp_path)
    assert r.returncode == 0 and "not divisble by BLOCK_SIZE_Z" in r.stderr


def test_plane_wave_needs_read_step_equal_nst(tmp_path):
    # pmcl3d.c:751-761: IFAULT=6 reads NST samples and wants READ_STEP == NST
    r = run(["-X", 16, "-Y", 16, "-Z", 16, "-I", 6, "-N", 20, "-R", 10], tmp_path)
    assert r.returncode == 1 and "READ_STEP should be equal NST" in r.stderr
    r = run(["-X", 16, "-Y", 16, "-Z", 16, "-I", 6, "-N", 0, "-R", 0], tmp_path)
    assert r.returncode == 1 and "should be > 0 for IFAULT=6" in r.stderr


def test_unknown_option_prints_usage(tmp_path):
    r = run(["--BOGUS", "1"], tmp_path)
    assert r.returncode != 0


def write_inputs(scn, d):
    scn.media.astype(np.float32).tofile(os.path.join(d, "media_0"))
    with open(os.path.join(d, "src_0"), "wb") as fh:
        for s in range(scn.src_pos.shape[0]):
            np.asarray(scn.src_pos[s], np.int32).tofile(fh)
            np.asarray(scn.src_data[s], np.float32).tofile(fh)


@pytest.mark.gpu
def test_full_run_matches_library(tmp_path):
    scn = scenarios.random_small(nx=24, ny=20, nz=32, steps=12, seed=9, ifault=1, nsrc=2)
    p = scn.params
    write_inputs(scn, tmp_path)
    ntiskp, wstep, nt = 2, 3, 12
    tmax = (nt - 1) * p["dt"] + p["dt"] * 0.5
    args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
            "-T", tmax, "-D", p["nd"], "-A", p["arbc"], "-V", 1, "-B", 1, "-n", 5,
            "-I", 1, "-S", scn.src_pos.shape[0], "-N", p["nst"], "-R", p["nst"],
            "--INVEL", "media", "--INSRC", "src", "-o", "out", "-c", "chk",
            "-r", ntiskp, "-W", wstep, "--NBGX", 1, "--NEDX", p["nx"], "--NSKPX", 2,
            "--NBGY", 1, "--NSKPY", 3, "--NBGZ", 1, "--NEDZ", 3, "--NSKPZ", 1]
    r = run(args, tmp_path)
    assert r.returncode == 0, r.stderr + r.stdout
    # the same run through the library
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    import torch
    rnx = (p["nx"] - 1) // 2 + 1
    nedy = p["ny"] - (p["ny"] - 1) % 3
    rny = (nedy - 1) // 3 + 1
    rnz = 3
    rec = rnx * rny * rnz
    bufs = [torch.zeros(rec, device="cuda") for _ in range(3)]
    frames = {c: [] for c in "XYZ"}
    nedx = p["nx"] - (p["nx"] - 1) % 2
    for step in range(1, nt + 1):
        s.step(1)
        if step % ntiskp == 0:
            s.gather(0, nedx - 1, 2, 0, nedy - 1, 3, 0, 2, 1, *[b.data_ptr() for b in bufs])
            s.synchronize()  # the gather runs on the context's stream
            for c, b in zip("XYZ", bufs):
                frames[c].append(b.cpu().numpy().copy())
    s.close()
    for step in range(ntiskp * wstep, nt + 1, ntiskp * wstep):
        n0 = step // ntiskp - wstep
        for c in "XYZ":
            f = os.path.join(tmp_path, "out", f"S{c}_0_{step:07d}")
            got = np.fromfile(f, np.float32)
            want = np.concatenate(frames[c][n0:n0 + wstep])
            assert got.shape == want.shape, (c, got.shape, want.shape)
            assert np.array_equal(got, want), (c, step)
    chk = open(os.path.join(tmp_path, "chk")).read()
    assert "STABILITY CRITERIA" in chk and chk.strip().endswith("END")


def test_recvfile_needs_readable_file(tmp_path):
    scn = scenarios.random_small(nx=16, ny=16, nz=16, steps=2, seed=9, ifault=1, nsrc=1)
    write_inputs(scn, tmp_path)
    r = run(["-X", 16, "-Y", 16, "-Z", 16, "-T", 0.01, "-B", 1, "-n", 5, "--INVEL", "media",
             "--INSRC", "src", "--RECVFILE", "missing.txt"], tmp_path)
    assert r.returncode != 0


@pytest.mark.gpu
@pytest.mark.parametrize("topo", [False, True])
def test_point_sets_match_library(tmp_path, topo):
    """--SOURCEFILE and --RECVFILE (and --INTOPO) through the executable give the
    same receiver files as the same run through the library."""
    from awp_b200 import pointfiles
    scn = scenarios.random_small(nx=24, ny=20, nz=32, steps=12, seed=9, ifault=1, nsrc=2)
    p = scn.params
    write_inputs(scn, tmp_path)
    topo_args = []
    if topo:
        scenarios.write_topography(str(tmp_path / "topo.bin"), p["nx"], p["ny"], p["dh"],
                                   amplitude=0.1 * p["dh"] * p["nz"], width=5 * p["dh"],
                                   rough_rms=0.0)
        topo_args = ["--INTOPO", str(tmp_path / "topo.bin")]
    nt = 12
    tmax = (nt - 1) * p["dt"] + p["dt"] * 0.5
    h = p["dh"]
    os.makedirs(tmp_path / "lib", exist_ok=True)
    for d in (tmp_path, tmp_path / "lib"):
        pointfiles.write_input(str(d / "src.txt"), str(d / "msrc"), [[8 * h, 9 * h, -12 * h]],
                               degree=3, gpu_buffer_size=2, cpu_buffer_size=3, steps=18)
        # the ring is refilled at steps 0, 6 and 12: three blocks of 6 samples
        rates = np.linspace(0, 1, 18 * 6, dtype=np.float32).reshape(1, 18, 6) * 1e14
        pointfiles.write_source_rates(str(d / "msrc"), rates)
        pointfiles.write_input(str(d / "recv.txt"), str(d / "rcv"),
                               [[5 * h, 6 * h, 0.0], [9.5 * h, 7 * h, -3 * h]], [1, 0],
                               degree=3, gpu_buffer_size=3, cpu_buffer_size=2, num_writes=2)
    args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
            "-T", tmax, "-D", p["nd"], "-A", p["arbc"], "-V", 1, "-B", 1, "-n", 5,
            "-I", 1, "-S", scn.src_pos.shape[0], "-N", p["nst"], "-R", p["nst"],
            "--INVEL", "media", "--INSRC", "src", "-o", "out", "-c", "chk",
            "--SOURCEFILE", str(tmp_path / "src.txt"), "--RECVFILE", str(tmp_path / "recv.txt")]
    r = run(args + topo_args, tmp_path)
    assert r.returncode == 0, r.stderr + r.stdout
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    if topo:
        s.topography(str(tmp_path / "topo.bin"))
    s.sourcefile(str(tmp_path / "lib" / "src.txt"))
    s.receivers(str(tmp_path / "lib" / "recv.txt"), nt)
    s.step(nt)
    s.synchronize()
    s.close()
    got = pointfiles.read_receiver_series(str(tmp_path / "rcv"), 2, nt, 3, 2, 2, 1)
    want = pointfiles.read_receiver_series(str(tmp_path / "lib" / "rcv"), 2, nt, 3, 2, 2, 1)
    for c in "xyz":
        assert got[c].shape == (2, 12) and np.any(got[c] != 0)
        assert np.array_equal(got[c], want[c]), c


@pytest.mark.gpu
def test_partitioned_media_file(tmp_path):
    """MEDIASTART=3 reads rank 0's partition, input_rst/mediapart/media0000000.bin
    (mesh.c:138-141), with the layout of MEDIASTART 1: both runs write the same
    surface files."""
    scn = scenarios.random_small(nx=16, ny=16, nz=16, steps=6, seed=13, ifault=1, nsrc=1)
    p = scn.params
    outs = {}
    for ms in (1, 3):
        d = tmp_path / f"ms{ms}"
        d.mkdir()
        write_inputs(scn, d)
        if ms == 3:
            os.makedirs(d / "input_rst" / "mediapart")
            os.rename(d / "media_0", d / "input_rst" / "mediapart" / "media0000000.bin")
        args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
                "-T", 5.5 * p["dt"], "-D", p["nd"], "-V", 1, "-B", ms, "-n", 5,
                "-I", 1, "-S", 1, "-N", p["nst"], "-R", p["nst"], "--INVEL", "media",
                "--INSRC", "src", "-o", "out", "-c", "chk", "-r", 1, "-W", 2]
        r = run(args, d)
        assert r.returncode == 0, r.stderr + r.stdout
        outs[ms] = sorted(os.listdir(d / "out"))
        assert outs[ms]
        for f in outs[ms]:
            outs[(ms, f)] = np.fromfile(d / "out" / f, np.float32)
    assert outs[1] == outs[3]
    for f in outs[1]:
        assert np.array_equal(outs[(1, f)], outs[(3, f)]), f
    assert any(np.abs(outs[(1, f)]).max() > 0 for f in outs[1])


@pytest.mark.gpu
def test_split_sources_equal_point_sources(tmp_path):
    """IFAULT=2 (read_src_ifault_2, source.c:15-128), READ_STEP < NST as the
    files intend it (the reference's own window refresh has no defined result
    there, swap.c:345-353): the header
    "<INSRC>_0" + rank and the READ_STEP windows "<INSRC_I2>_0" + rank +
    "_<idx>" hold the same series as an IFAULT=1 file; both runs write the
    same surface files bit for bit (the last window partly past NST)."""
    scn = scenarios.random_small(nx=16, ny=16, nz=16, steps=10, seed=17, ifault=1, nsrc=3)
    p = scn.params
    nst, rs = p["nst"], 5
    np_ = scn.src_pos.shape[0]
    data = np.asarray(scn.src_data, np.float32).reshape(np_, -1, 6)[:, :nst]
    outs = {}
    for ifault in (1, 2):
        d = tmp_path / f"if{ifault}"
        d.mkdir()
        write_inputs(scn, d)
        if ifault == 2:
            with open(d / "tpsrc_00000000", "wb") as fh:
                np.array([np_, 0, 0], np.int32).tofile(fh)
                np.asarray(scn.src_pos, np.int32).reshape(-1).tofile(fh)
            for idx in range(1, -(-nst // rs) + 1):
                win = np.zeros((6, rs, np_), np.float32)
                t0 = (idx - 1) * rs
                n = min(rs, nst - t0)
                win[:, :n, :] = data[:, t0:t0 + n, :].transpose(2, 1, 0)
                win.tofile(d / f"fault_0{0:07d}_{idx:03d}")
        args = ["-X", p["nx"], "-Y", p["ny"], "-Z", p["nz"], "-H", p["dh"], "-t", p["dt"],
                "-T", 9.5 * p["dt"], "-D", p["nd"], "-V", 1, "-B", 1, "-n", 5,
                "-I", ifault, "-S", np_, "-N", nst, "-R", nst if ifault == 1 else rs,
                "--INVEL", "media", "--INSRC", "src" if ifault == 1 else "tpsrc",
                "--INSRC_I2", "fault", "-o", "out", "-c", "chk", "-r", 1, "-W", 2]
        r = run(args, d)
        assert r.returncode == 0, r.stderr + r.stdout
        outs[ifault] = sorted(os.listdir(d / "out"))
        for f in outs[ifault]:
            outs[(ifault, f)] = np.fromfile(d / "out" / f, np.float32)
    assert outs[1] == outs[2] and outs[1]
    for f in outs[1]:
        assert np.array_equal(outs[(1, f)], outs[(2, f)]), f
    assert any(np.abs(outs[(1, f)]).max() > 0 for f in outs[1])
