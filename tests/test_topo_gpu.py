"""GPU parity of the curvilinear topography path.

The product steps with awp_topography_init; the reference side is the
reference's own topography code (topo_init ... topo_set_constants and the
topo_velocity_interior_H / topo_stress_*_H launchers of src/topography,
oracle/_ref/libawpref_topo.so) in place of dvelcx / dstrqc inside the
single-rank pmcl3d order of refbind.RefGpuSim, exactly as pmcl3d.c:1661-1924
swaps them.  The two builds round differently (the reference's compiler
contracts the generated sums into FMAs at will), so the bar is relative
L2 <= 1e-5 per field, the bar of the Cartesian path.
"""
import numpy as np
import pytest
import torch

from awp_b200 import Solver, default_params, pointfiles, scenarios
from oracle import refbind

pytestmark = pytest.mark.gpu

REL_REF = 1e-5
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz"]
GT = {"x": 0, "y": 1, "z": 2, "xx": 3, "yy": 4, "zz": 5, "xy": 6, "xz": 7, "yz": 8}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def hill(path, p, amp=0.15, rough=0.02, seed=5):
    depth = p["dh"] * (p["nz"] - 2)
    return scenarios.write_topography(path, p["nx"], p["ny"], p["dh"], amplitude=amp * depth,
                                      width=5 * p["dh"], rough_rms=rough * depth, seed=seed)


def random_state(p, seed, scale=1e-3):
    """Seeded wavefield over the whole padded block (exercises every operator,
    the six boundary rows included, from the first step)."""
    rng = np.random.default_rng(seed)
    shp = refbind.padded_shape(p["nx"], p["ny"], p["nz"])
    st = {f: (rng.standard_normal(shp) * (scale if f in ("u1", "v1", "w1") else 1e5))
          .astype(np.float32) for f in FIELDS}
    return st


@pytest.mark.parametrize("q,amp", [(True, 0.15), (False, 0.15), (True, 0.0)])
def test_half_steps_match_reference(tmp_path, q, amp):
    """Three steps from a random state: velocity and stress operators in the
    interior and in the top six rows, memory variables, sponge, Q(f)."""
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=q, ifault=1, steps=4, seed=31, nsrc=1)
    p = scn.params
    path = str(tmp_path / "topo.bin")
    hill(path, p, amp=amp, rough=0.02 if amp else 0.0)
    st = random_state(p, 3)

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.topography(path)
    for f, a in st.items():
        s.set_field(f, a)
    s.step(3)
    s.synchronize()

    setup = refbind.model_setup(scn)
    ref = refbind.RefTopoSim(scn, setup, path)
    for f, a in st.items():
        ref.f[f].copy_(torch.from_numpy(a))
    ref.npsrc = 0  # the random state only
    ref.step(3)

    for f in FIELDS + (["r1", "r4", "r6"] if q else []):
        e = rel_l2(s.field(f), ref.field(f))
        assert e <= REL_REF, (f, e)
    ref.close()
    s.close()


@pytest.mark.parametrize("q", [True, False])
def test_source_run_matches_reference(tmp_path, q):
    """Twenty steps of a point-source run (one source on the free-surface
    row) over a hill with roughness."""
    steps = 20
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=q, ifault=1, steps=steps, seed=12)
    p = scn.params
    path = str(tmp_path / "topo.bin")
    hill(path, p)

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.topography(path)
    s.step(steps)
    s.synchronize()

    setup = refbind.model_setup(scn)
    ref = refbind.RefTopoSim(scn, setup, path)
    ref.step(steps)
    for f in FIELDS:
        e = rel_l2(s.field(f), ref.field(f))
        assert e <= REL_REF, (f, e)
    ref.close()
    s.close()


def test_sourcefile_and_receivers_match_reference(tmp_path):
    """SOURCEFILE moments added through the cell Jacobian and receivers placed
    through the surface function (sources_add_curvilinear, source.c:283-340)
    against the reference's own point-set code on its topography metrics."""
    steps = 12
    scn = scenarios.random_small(nx=28, ny=24, nz=32, q=True, ifault=1, steps=steps, seed=8,
                                 nsrc=1)
    p = scn.params
    nx, ny, nz, h, dt = p["nx"], p["ny"], p["nz"], p["dh"], p["dt"]
    tpath = str(tmp_path / "topo.bin")
    hill(tpath, p)
    gpu, cpu, nsamples, degree = 2, 3, 18, 3
    xs = np.array([6.2, 13.7, 20.1]) * h
    coords = np.stack([xs, np.array([7.3, 12.9, 15.4]) * h,
                       -np.array([6.4, 11.1, 3.7]) * h], 1)
    base = str(tmp_path / "src")
    spath = str(tmp_path / "src.txt")
    pointfiles.write_input(spath, base, coords, degree=degree, gpu_buffer_size=gpu,
                           cpu_buffer_size=cpu, steps=nsamples)
    rng = np.random.default_rng(9)
    rates = (rng.standard_normal((3, nsamples, 6)) * 3e13).astype(np.float32)
    pointfiles.write_source_rates(base, rates)
    rbase = str(tmp_path / "recv")
    rpath = str(tmp_path / "recv.txt")
    rc = np.stack([rng.uniform(3 * h, (nx - 4) * h, 9), rng.uniform(3 * h, (ny - 4) * h, 9),
                   -rng.uniform(0.0, 0.6 * nz * h, 9)], 1)
    rt = np.zeros(9, np.int32)
    rt[:3] = 1
    nt = steps + 1
    pointfiles.write_input(rpath, rbase, rc, rt, degree=degree, gpu_buffer_size=steps,
                           cpu_buffer_size=1, num_writes=1, stride=1, steps=1)

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.topography(tpath)
    s.sourcefile(spath)
    s.receivers(rpath, nt)
    s.step(steps)
    s.synchronize()
    got = pointfiles.read_receiver_series(rbase, 9, nt, steps, 1, 1, 1)

    setup = refbind.model_setup(scn)
    ref = refbind.RefTopoSim(scn, setup, tpath)
    (d_f, d_f1, d_f2, d_fc, d_g3, d_g3c), _ = ref.metric_ptrs()
    fnorm = metrics_f(tpath, nx, ny, nz, h)
    comps = ["xx", "yy", "zz", "xy", "xz", "yz"]
    jac = {"xx": (d_fc, d_g3c), "yy": (d_fc, d_g3c), "zz": (d_fc, d_g3c), "xy": (d_f, d_g3c),
           "xz": (d_f1, d_g3), "yz": (d_f2, d_g3)}
    spts = {c: refbind.RefPoints(spath, GT[c], nx, ny, nz, h, ftopo=fnorm) for c in comps}
    rpts = {c: refbind.RefPoints(rpath, GT[c], nx, ny, nz, h, ftopo=fnorm) for c in "xyz"}
    dev_rates = torch.from_numpy(rates).cuda()
    host = refbind.RefHost()
    own = {c: host.point_coefs(spath, GT[c], nx, ny, nz, h)["indices"] for c in comps}

    def add(sim, step):
        for ci, c in enumerate(comps):
            v = dev_rates[torch.as_tensor(own[c], device="cuda").long(), step, ci].contiguous()
            spts[c].srcadd_curv(sim.f[c].data_ptr(), v.data_ptr(), h, dt, jac[c][0], jac[c][1])

    fld = {"x": "u1", "y": "v1", "z": "w1"}
    samples = {c: [] for c in rpts}
    out = torch.zeros(64, device="cuda")

    def record(sim, step):
        for c, rp in rpts.items():
            out.zero_()
            rp.interp(out.data_ptr(), sim.f[fld[c]].data_ptr())
            samples[c].append(out[: rp.count].cpu().numpy().copy())

    record(ref, 0)
    ref.after_stress.append(add)
    ref.after_step.append(record)
    ref.step(steps)

    for f in FIELDS + ["r1", "r5"]:
        e = rel_l2(s.field(f), ref.field(f))
        assert e <= REL_REF, (f, e)
    for c in rpts:
        r = np.stack(samples[c][:steps], axis=1)
        mine = got[c]
        assert mine.shape[0] == r.shape[0] == rpts[c].count == 9, (mine.shape, r.shape)
        e = rel_l2(mine, r)
        assert e <= REL_REF, (c, e)
    for rp in list(spts.values()) + list(rpts.values()):
        rp.close()
    ref.close()
    s.close()


def test_forcefile_matches_reference(tmp_path):
    """FORCEFILE boundary forces on the curvilinear block (forces_add,
    forces.c:67-96; cusource_add_force, source.cu:118-157) against the
    reference's own device code on its topography metrics, hooked after the
    stress update as pmcl3d.c:1989-1994 places it."""
    steps = 12
    scn = scenarios.random_small(nx=28, ny=24, nz=32, q=True, ifault=1, steps=steps, seed=12,
                                 nsrc=1)
    p = scn.params
    nx, ny, nz, h, dt = p["nx"], p["ny"], p["nz"], p["dh"], p["dt"]
    tpath = str(tmp_path / "topo.bin")
    hill(tpath, p)
    gpu, cpu, nsamples, degree = 2, 3, 18, 3
    coords = np.stack([np.array([6.2, 13.7, 17.4]) * h, np.array([7.3, 12.9, 9.6]) * h,
                       np.zeros(3)], 1)
    base = str(tmp_path / "force")
    fpath = str(tmp_path / "force.txt")
    pointfiles.write_input(fpath, base, coords, [1, 1, 1], degree=degree, gpu_buffer_size=gpu,
                           cpu_buffer_size=cpu, steps=nsamples)
    rng = np.random.default_rng(21)
    rates = (rng.standard_normal((3, nsamples, 3)) * 1e9).astype(np.float32)
    for c, name in enumerate(("fx", "fy", "fz")):
        np.ascontiguousarray(rates[:, :, c]).tofile(f"{base}_{name}")

    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    with pytest.raises(RuntimeError):
        s.forcefile(fpath)  # the topography comes first
    s.topography(tpath)
    s.forcefile(fpath)
    s.step(steps)
    s.synchronize()

    setup = refbind.model_setup(scn)
    ref = refbind.RefTopoSim(scn, setup, tpath)
    (d_f, d_f1, d_f2, d_fc, d_g3, d_g3c), _ = ref.metric_ptrs()
    fnorm = metrics_f(tpath, nx, ny, nz, h)
    fpts = {c: refbind.RefPoints(fpath, GT[c], nx, ny, nz, h, ftopo=fnorm) for c in "xyz"}
    host = refbind.RefHost()
    own = {c: torch.as_tensor(host.point_coefs(fpath, GT[c], nx, ny, nz, h)["indices"],
                              device="cuda").long() for c in "xyz"}
    assert all(len(v) == 3 for v in own.values())
    dev_rates = torch.from_numpy(rates).cuda()
    fld = {"x": "u1", "y": "v1", "z": "w1"}
    # forces.c:84-96: metric and SBP weight per component
    met = {"x": (d_f1, d_g3c, 2.9022824945274315), "y": (d_f2, d_g3c, 2.9022824945274315),
           "z": (d_fc, d_g3, 3.55599789310935)}

    def add(sim, step):
        for ci, c in enumerate("xyz"):
            v = dev_rates[own[c], step, ci].contiguous()
            fm, dg, q = met[c]
            fpts[c].force(sim.f[fld[c]].data_ptr(), v.data_ptr(), sim.f["d1"].data_ptr(), h, dt,
                          q, fm, nx, nz, dg)

    ref.after_stress.append(add)
    ref.step(steps)
    assert float(torch.abs(ref.f["w1"]).max()) > 0
    rep = {}
    for f in FIELDS:
        rep[f] = rel_l2(s.field(f), ref.field(f))
        assert rep[f] <= REL_REF, (f, rep[f])
    print("\nFORCEFILE rel L2 vs reference build:", {k: f"{v:.1e}" for k, v in rep.items()})
    for rp in fpts.values():
        rp.close()
    ref.close()
    s.close()


def test_forcefile_rules(tmp_path):
    """Volume (type 0) points are refused as forces_boundary_check refuses them."""
    scn = scenarios.random_small(nx=28, ny=24, nz=32, q=False, ifault=1, steps=4, seed=3,
                                 nsrc=1)
    p = scn.params
    tpath = str(tmp_path / "topo.bin")
    hill(tpath, p)
    coords = np.array([[6.2 * p["dh"], 7.3 * p["dh"], -2.0 * p["dh"]]])
    fpath = str(tmp_path / "force.txt")
    pointfiles.write_input(fpath, str(tmp_path / "force"), coords, [0], degree=1, steps=4)
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.topography(tpath)
    with pytest.raises(RuntimeError, match="boundary"):
        s.forcefile(fpath)
    s.close()


def metrics_f(path, nx, ny, nz, h):
    """The normalised surface function of the product's metric set-up (pinned
    bit for bit to the reference's host code by the CPU tests)."""
    import ctypes
    from awp_b200 import _lib
    out = np.zeros(10 * (nx + 20) * (ny + 84) + 4 * (nz + 64), np.float32)
    err = _lib.load().awp_topo_metrics(path.encode(), nx, ny, nz, h,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert err == 0
    return out[: (nx + 20) * (ny + 84)].copy()


def test_topography_state_errors(tmp_path):
    """Topography after receivers, twice, or on a lower grid is refused."""
    from awp_b200 import AwpError
    scn = scenarios.random_small(nx=24, ny=20, nz=32, q=False, steps=2)
    p = scn.params
    path = str(tmp_path / "topo.bin")
    hill(path, p)
    s = Solver(default_params(**p))
    s.upload_media(scn.media)
    s.topography(path)
    with pytest.raises(AwpError) as e:
        s.topography(path)
    assert e.value.status == 3
    s.close()
    s = Solver(default_params(**p))
    with pytest.raises(AwpError) as e:
        s.topography(str(tmp_path / "missing.bin"))
    assert e.value.status == 4
    bad = str(tmp_path / "bad.bin")
    scenarios.write_topography(bad, p["nx"] + 1, p["ny"], p["dh"])
    with pytest.raises(AwpError) as e:
        s.topography(bad)
    assert e.value.status == 1
    s.close()
