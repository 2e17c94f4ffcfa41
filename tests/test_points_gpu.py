"""GPU parity of the RECVFILE receivers and SOURCEFILE sources.

The product runs the whole time loop with the point sets and writes the
receiver files itself.  The reference side runs the reference's own CUDA
kernels in pmcl3d's single-rank order (refbind.RefGpuSim) with the
reference's own point-set device code hooked in where pmcl3d calls it
(cuinterp_interp_H after the free-surface imaging, cusource_add_cartesian_H
after the stress update; ref_points_shim.c).  The FP64 oracle runs the same
schedule on the CPU.  Tolerances: relative L2 <= 1e-5 against the reference
build, <= 1e-4 against the FP64 oracle.
"""
import numpy as np
import pytest
import torch

from awp_b200 import Solver, default_params, pointfiles, scenarios
from oracle import oracle as orc
from oracle import refbind

pytestmark = pytest.mark.gpu

REL_REF = 1e-5
REL_F64 = 1e-4
GT = {"x": 0, "y": 1, "z": 2, "xx": 3, "yy": 4, "zz": 5, "xy": 6, "xz": 7, "yz": 8}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def receiver_layout(rng, n, nx, ny, nz, h):
    x = rng.uniform(2 * h, (nx - 3) * h, n)
    y = rng.uniform(2 * h, (ny - 3) * h, n)
    z = -rng.uniform(0.0, (nz - 4) * h, n)
    t = np.zeros(n, np.int32)
    t[: n // 3] = 1          # surface receivers
    z[-1] = -0.4 * nz * h    # the last one in the volume (see test_points_cpu)
    x[2] = -4 * h            # one outside the domain: never written
    return np.stack([x, y, z], 1), t


@pytest.mark.parametrize("degree,gpu,cpu,nw,stride", [(3, 2, 3, 2, 2), (1, 4, 1, 1, 1)])
def test_receivers_match_reference(tmp_path, degree, gpu, cpu, nw, stride):
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=True, ifault=1, steps=24, seed=21)
    p = scn.params
    nx, ny, nz, h = p["nx"], p["ny"], p["nz"], p["dh"]
    nsteps = gpu * cpu * nw * stride  # exactly one file per component
    nt = nsteps + 1
    rng = np.random.default_rng(3)
    coords, types = receiver_layout(rng, 12, nx, ny, nz, h)
    base = str(tmp_path / "recv")
    path = str(tmp_path / "recv.txt")
    pointfiles.write_input(path, base, coords, types, degree=degree, gpu_buffer_size=gpu,
                           cpu_buffer_size=cpu, num_writes=nw, stride=stride, steps=1)

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.receivers(path, nt)
    assert s.receiver_counts() == (11, 11, 11)
    s.step(nsteps)
    s.synchronize()
    got = pointfiles.read_receiver_series(base, 12, nt, gpu, cpu, nw, stride)

    # reference kernels + the reference's receiver gather, sampled every `stride` steps
    setup = refbind.model_setup(scn)
    ref = refbind.RefGpuSim(scn, setup)
    pts = {c: refbind.RefPoints(path, GT[c], nx, ny, nz, h) for c in ("x", "y", "z")}
    fld = {"x": "u1", "y": "v1", "z": "w1"}
    samples = {c: [] for c in pts}
    out = torch.zeros(64, device="cuda")

    def record(sim, step):
        if step % stride:
            return
        for c, rp in pts.items():
            out.zero_()
            rp.interp(out.data_ptr(), sim.f[fld[c]].data_ptr())
            samples[c].append(out[: rp.count].cpu().numpy().copy())

    record(ref, 0)
    ref.after_step.append(record)
    ref.step(nsteps)

    # FP64 oracle fields interpolated with the reference's weights
    o = orc.OracleSim(scn, setup, 64)
    host = refbind.RefHost()
    coefs = {c: host.point_coefs(path, GT[c], nx, ny, nz, h) for c in pts}
    o_samples = {c: [] for c in pts}

    def o_record():
        for c, cf in coefs.items():
            F = o.field(fld[c], f64=True)
            vals = np.zeros(len(cf["ix"]))
            nb = cf["lx"].shape[1]
            for q in range(len(cf["ix"])):
                blk = F[2 + cf["ix"][q]: 2 + cf["ix"][q] + nb, 2 + cf["iy"][q]: 2 + cf["iy"][q] + nb,
                        32 + cf["iz"][q]: 32 + cf["iz"][q] + nb]
                vals[q] = np.einsum("i,j,k,ijk->", cf["lx"][q].astype(np.float64),
                                    cf["ly"][q].astype(np.float64),
                                    cf["lz"][q].astype(np.float64), blk)
            o_samples[c].append(vals)

    o_record()
    for step in range(1, nsteps + 1):
        o.step(1)
        if step % stride == 0:
            o_record()

    nsamp = nsteps // stride  # samples of the complete file (step 0 .. nsteps - stride)
    for c in pts:
        idx = coefs[c]["indices"]
        mine = got[c][idx]                                # [owned][samples], file order
        r = np.stack(samples[c][:nsamp], axis=1)          # reference gather
        b = np.stack(o_samples[c][:nsamp], axis=1)
        assert mine.shape == r.shape, (mine.shape, r.shape)
        assert np.all(got[c][2] == 0)                     # the receiver outside the domain
        e_ref, e_64 = rel_l2(mine, r), rel_l2(mine, b)
        assert e_ref <= REL_REF, (c, e_ref)
        assert e_64 <= REL_F64, (c, e_64)
    for rp in pts.values():
        rp.close()
    s.close()


def source_layout(n, nx, ny, nz, h, spacing):
    xs = 4 * h + spacing * h * np.arange(n)
    return np.stack([xs % ((nx - 8) * h) + 4 * h,
                     np.full(n, 0.5 * ny * h) + 0.37 * h * np.arange(n),
                     -(0.3 * nz * h + 0.61 * h * np.arange(n))], 1)


@pytest.mark.parametrize("spacing,with_ref", [(6.3, True), (1.0, False)])
def test_sourcefile_matches_reference(tmp_path, spacing, with_ref):
    """Well separated sources against the reference build and the oracle;
    overlapping sources (their Lagrange stencils share cells, where the
    reference's threads race on the read-modify-write) against the oracle only."""
    steps = 24
    scn = scenarios.random_small(nx=28, ny=24, nz=32, q=True, ifault=1, steps=steps, seed=8,
                                 nsrc=1)
    p = scn.params
    nx, ny, nz, h, dt = p["nx"], p["ny"], p["nz"], p["dh"], p["dt"]
    gpu, cpu, nsamples, degree = 2, 3, 30, 3
    coords = source_layout(3, nx, ny, nz, h, spacing)
    base = str(tmp_path / "src")
    path = str(tmp_path / "src.txt")
    pointfiles.write_input(path, base, coords, degree=degree, gpu_buffer_size=gpu,
                           cpu_buffer_size=cpu, steps=nsamples)
    rng = np.random.default_rng(9)
    rates = (rng.standard_normal((3, nsamples, 6)) * 3e13).astype(np.float32)
    pointfiles.write_source_rates(base, rates)

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.sourcefile(path)
    s.step(steps)
    s.synchronize()

    setup = refbind.model_setup(scn)
    host = refbind.RefHost()
    comps = ["xx", "yy", "zz", "xy", "xz", "yz"]
    coefs = {c: host.point_coefs(path, GT[c], nx, ny, nz, h) for c in comps}
    o = orc.OracleSim(scn, setup, 64)
    for ci, c in enumerate(comps):
        vals = rates[coefs[c]["indices"], :, ci].T  # [samples][owned]
        o.add_point_sources(c, coefs[c], vals, 1)
    o.step(steps)

    ref = None
    if with_ref:
        ref = refbind.RefGpuSim(scn, setup)
        pts = {c: refbind.RefPoints(path, GT[c], nx, ny, nz, h) for c in comps}
        dev_rates = torch.from_numpy(rates).cuda()

        def add(sim, step):
            for ci, c in enumerate(comps):
                v = dev_rates[torch.as_tensor(coefs[c]["indices"], device="cuda").long(), step,
                              ci].contiguous()
                pts[c].srcadd(sim.f[c].data_ptr(), v.data_ptr(), h, dt)

        ref.after_stress.append(add)
        ref.step(steps)

    for f in ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r5"]:
        a = s.field(f)
        e_64 = rel_l2(a, o.field(f, f64=True))
        assert e_64 <= REL_F64, (f, e_64)
        if ref is not None:
            e_ref = rel_l2(a, ref.field(f))
            assert e_ref <= REL_REF, (f, e_ref)
    if ref is not None:
        for rp in pts.values():
            rp.close()
    s.close()


def test_sourcefile_past_end_of_file_is_reported(tmp_path):
    """Reading past the samples the rate files hold is an I/O error."""
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=True, ifault=1, steps=8, seed=8, nsrc=1)
    p = scn.params
    base = str(tmp_path / "src")
    path = str(tmp_path / "src.txt")
    pointfiles.write_input(path, base, [[500.0, 500.0, -400.0]], degree=1, gpu_buffer_size=2,
                           cpu_buffer_size=2, steps=4)
    pointfiles.write_source_rates(base, np.ones((1, 4, 6), np.float32))
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.sourcefile(path)
    s.step(3)
    from awp_b200 import AwpError
    with pytest.raises(AwpError) as e:
        s.step(1)  # step 4 needs samples 4..7
    assert e.value.status == 4
    s.close()
