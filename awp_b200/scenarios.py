"""Seeded synthetic inputs for the benchmark and test workloads.

No public dataset is involved: each workload is generated from its seed with
the shapes, sizes and value distributions of the corresponding run.

* ``halfspace``   -- homogeneous elastic half-space with a point moment-tensor
  source (Mxy, Ricker derivative) at the grid centre (IFAULT=1).
* ``layered_vk``  -- 1-D vs gradient with depth, vp = 1.73 vs, Gardner rho,
  von Karman perturbation, Qs = 50 vs[km/s], Qp = 2 Qs, and a kinematic
  finite fault of random subfaults (IFAULT=5, Brune source time function).
* ``random_small`` -- small random heterogeneous media for parity tests.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Scenario:
    name: str
    params: dict          # awp_params fields
    media: np.ndarray     # float32 [nz][ny][nx][nvar], surface first
    src_pos: np.ndarray   # int32 [nsrc][3] INSRC coordinates (1-based, z from surface)
    src_data: np.ndarray  # float32 [nsrc][read_step][6]
    steps: int
    description: str = ""


def ricker_derivative(nt: int, dt: float, f0: float, t0: float | None = None) -> np.ndarray:
    """Time derivative of a Ricker wavelet (the moment-rate of a Ricker moment)."""
    t0 = 1.2 / f0 if t0 is None else t0
    t = np.arange(nt) * dt - t0
    a = (math.pi * f0 * t) ** 2
    # d/dt [(1 - 2a) exp(-a)] with a = (pi f0 t)^2
    dadt = 2.0 * (math.pi * f0) ** 2 * t
    return ((-2.0 * dadt) * np.exp(-a) - (1.0 - 2.0 * a) * np.exp(-a) * dadt).astype(np.float64)


def workload_meta(name: str, nx=None, ny=None, nz=None) -> tuple[dict, str]:
    """Solver parameters and description of a named benchmark workload
    (``layered_vk``, ``halfspace``) at its default or given size, without
    generating its medium."""
    if name == "layered_vk":
        nx, ny, nz = nx or 512, ny or 512, nz or 256
        h, dt, nsub = 50.0, 0.0035, 200
        params = dict(nx=nx, ny=ny, nz=nz, dh=h, dt=dt, nd=20, arbc=0.92, npc=0, nve=1,
                      ifault=5, nst=2, read_step=2, socalq=1)
        return params, (f"anelastic 1-D gradient + von Karman {nx}x{ny}x{nz}, h={h}, dt={dt}, "
                        f"{nsub} kinematic subfaults")
    if name == "halfspace":
        nx, ny, nz = nx or 128, ny or 128, nz or 128
        h, dt, f0, steps = 100.0, 0.005, 2.0, 500
        params = dict(nx=nx, ny=ny, nz=nz, dh=h, dt=dt, nd=20, arbc=0.92, npc=0, nve=1,
                      ifault=1, nst=steps, read_step=steps, socalq=1)
        return params, f"elastic half-space {nx}x{ny}x{nz}, h={h}, dt={dt}, Mxy Ricker' {f0} Hz"
    raise ValueError(f"unknown workload {name}")


def halfspace(nx=128, ny=128, nz=128, h=100.0, dt=0.005, steps=500, f0=2.0, m0=1e15,
              vp=6000.0, vs=3464.0, rho=2700.0, nd=20, seed=1) -> Scenario:
    media = np.empty((nz, ny, nx, 5), np.float32)
    media[..., 0] = vp
    media[..., 1] = vs
    media[..., 2] = rho
    media[..., 3] = 0.0  # Qp <= 0: elastic (mesh.c:434-438)
    media[..., 4] = 0.0
    nst = steps
    stf = ricker_derivative(nst, dt, f0) * m0
    data = np.zeros((1, nst, 6), np.float32)
    data[0, :, 5] = stf  # Mxy
    pos = np.array([[nx // 2, ny // 2, nz // 2]], np.int32)
    params = dict(nx=nx, ny=ny, nz=nz, dh=h, dt=dt, nd=nd, arbc=0.92, npc=0, nve=1,
                  ifault=1, nst=nst, read_step=nst, socalq=1)
    return Scenario("halfspace", params, media, pos, data, steps,
                    f"elastic half-space {nx}x{ny}x{nz}, h={h}, dt={dt}, Mxy Ricker' {f0} Hz")


def von_karman(shape, dh, corr_len, hurst, std, seed) -> np.ndarray:
    """Von Karman random field, generated spectrally, unit-free with given std."""
    import scipy.fft as sfft
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    kz = np.fft.fftfreq(nz, d=dh) * 2 * math.pi
    ky = np.fft.fftfreq(ny, d=dh) * 2 * math.pi
    kx = np.fft.rfftfreq(nx, d=dh) * 2 * math.pi
    k2 = (kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    # 3-D von Karman power spectrum ~ (1 + k^2 a^2)^-(H + 3/2); amplitude = sqrt
    amp = (1.0 + k2 * corr_len * corr_len) ** (-(hurst + 1.5) / 2.0)
    amp = amp.astype(np.float32)
    del k2
    noise = rng.standard_normal(shape, dtype=np.float32)
    spec = sfft.rfftn(noise, workers=-1)
    del noise
    spec *= amp
    del amp
    field = sfft.irfftn(spec, s=shape, workers=-1).astype(np.float32)
    del spec
    field -= field.mean()
    field *= std / max(float(field.std()), 1e-30)
    return field


def layered_vk(nx=512, ny=512, nz=256, h=50.0, dt=0.0035, steps=2000, nsub=200,
               vs_top=1000.0, vs_bot=3500.0, std=0.05, corr=500.0, hurst=0.1,
               seed_medium=2, seed_src=3, vp_cap=6300.0, nd=20) -> Scenario:
    depth = (np.arange(nz, dtype=np.float32) + 0.5) / nz  # 0 = surface (file k=0)
    vs1d = vs_top + (vs_bot - vs_top) * depth
    pert = von_karman((nz, ny, nx), h, corr, hurst, std, seed_medium)
    pert = np.clip(pert, -3 * std, 3 * std)
    vs = vs1d[:, None, None] * (1.0 + pert)
    del pert
    vp = np.minimum(1.73 * vs, vp_cap).astype(np.float32)
    vs = (vp / 1.73).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)  # Gardner, kg/m^3 with vp in m/s
    qs = (50.0 * vs / 1000.0).astype(np.float32)
    qp = (2.0 * qs).astype(np.float32)
    media = np.stack([vp, vs, rho, qp, qs], axis=-1).astype(np.float32)
    del vp, vs, rho, qp, qs
    src_pos, src_data = kinematic_fault(nx, ny, nz, h, nsub, seed_src)
    params = dict(nx=nx, ny=ny, nz=nz, dh=h, dt=dt, nd=nd, arbc=0.92, npc=0, nve=1,
                  ifault=5, nst=2, read_step=2, socalq=1)
    return Scenario("layered_vk", params, media, src_pos, src_data, steps,
                    f"anelastic 1-D gradient + von Karman {nx}x{ny}x{nz}, h={h}, dt={dt}, "
                    f"{nsub} kinematic subfaults")


def adjoint_case(nx=256, ny=256, nz=128, h=100.0, dt=0.005, steps=1500, nrec=64, seed=5,
                 smooth_m=1000.0, f0=2.0, m0=1e15):
    """Misfit-gradient workload: true model = the anelastic 1-D gradient + von
    Karman medium (seeded), start model = the same smoothed by a Gaussian of
    `smooth_m` metres; a moment-tensor point source (IFAULT 1, Mxy Ricker') at
    a quarter depth and `nrec` surface receivers on a seeded random layout.
    Returns (scenario of the start model, (lam, mu, rho) true, (lam, mu, rho)
    start, rec_xyz, rec_comp); moduli arrays [nz][ny][nx], surface first."""
    import scipy.ndimage as ndi
    true = layered_vk(nx=nx, ny=ny, nz=nz, h=h, dt=dt, steps=steps, nsub=1, seed_medium=seed,
                      seed_src=seed + 1)
    med = true.media
    sig = smooth_m / h
    start_media = med.copy()
    for q in range(3):
        start_media[..., q] = ndi.gaussian_filter(med[..., q], sig, mode="nearest")

    def moduli(m):
        vp, vs, rho = (m[..., q].astype(np.float64) for q in range(3))
        return ((rho * (vp * vp - 2 * vs * vs)).astype(np.float32),
                (rho * vs * vs).astype(np.float32), rho.astype(np.float32))

    nst = steps + 1
    data = np.zeros((1, nst, 6), np.float32)
    data[0, :, 5] = ricker_derivative(nst, dt, f0) * m0
    pos = np.array([[nx // 2, ny // 2, nz - nz // 4]], np.int32)
    params = dict(true.params, ifault=1, nst=nst, read_step=nst)
    scn = Scenario("adjoint_case", params, start_media, pos, data, steps,
                   f"misfit gradient {nx}x{ny}x{nz}, h={h}, dt={dt}, {steps} steps, "
                   f"{nrec} surface receivers, start model smoothed by {smooth_m:g} m")
    rng = np.random.default_rng(seed + 2)
    xyz = np.stack([rng.integers(nx // 8, nx - nx // 8, nrec), rng.integers(ny // 8, ny - ny // 8, nrec),
                    np.zeros(nrec, np.int64)], 1).astype(np.int32)
    comp = rng.integers(0, 3, nrec).astype(np.int32)
    return scn, moduli(med), moduli(start_media), xyz, comp


def kinematic_fault(nx, ny, nz, h, nsub, seed, strike=0.0, dip=90.0, rake=180.0):
    """Random subfaults on a vertical plane x = nx/2 (IFAULT=5 layout, source.c:165-181)."""
    rng = np.random.default_rng(seed)
    ny0, ny1 = ny // 4, 3 * ny // 4
    nz0, nz1 = max(3, nz // 16), nz // 2
    cells = set()
    pos = []
    while len(pos) < nsub:
        y = int(rng.integers(ny0, ny1))
        z = int(rng.integers(nz0, nz1))
        if (y, z) in cells:
            continue
        cells.add((y, z))
        pos.append((nx // 2, y, z))
    pos = np.array(pos, np.int32)
    data = np.zeros((nsub, 2, 6), np.float32)
    data[:, 0, 0] = 1.0                                  # Brune
    data[:, 0, 1] = rng.uniform(0.5, 1.5, nsub)          # slip (m)
    data[:, 0, 2] = rng.uniform(0.0, 3.0, nsub)          # rupture time (s)
    data[:, 0, 3] = rng.uniform(0.3, 1.0, nsub)          # rise time (s)
    data[:, 0, 4] = h * h                                # subfault area (m^2)
    data[:, 1, 0] = strike + rng.uniform(-10, 10, nsub)  # strike (deg)
    data[:, 1, 1] = dip
    data[:, 1, 2] = rake + rng.uniform(-15, 15, nsub)
    return pos, data


def random_small(nx=24, ny=20, nz=32, h=100.0, dt=0.004, steps=20, seed=7, nvar=5,
                 q=True, ifault=1, nsrc=3, nst=None) -> Scenario:
    """Small random heterogeneous model for parity tests (any nx, ny; nz % 4 == 0)."""
    rng = np.random.default_rng(seed)
    vs = rng.uniform(1500.0, 3000.0, (nz, ny, nx)).astype(np.float32)
    vp = (vs * rng.uniform(1.6, 1.9, (nz, ny, nx))).astype(np.float32)
    rho = rng.uniform(2200.0, 2800.0, (nz, ny, nx)).astype(np.float32)
    cols = [vp, vs, rho]
    if nvar >= 5:
        if q:
            qs = rng.uniform(20.0, 400.0, (nz, ny, nx)).astype(np.float32)
            qp = (qs * rng.uniform(1.5, 2.5, (nz, ny, nx))).astype(np.float32)
        else:
            qs = np.zeros_like(vs)
            qp = np.zeros_like(vs)
        cols += [qp, qs]
    if nvar == 8:
        cols = [np.zeros_like(vs)] * 3 + cols
    media = np.stack(cols, axis=-1).astype(np.float32)
    nst = nst or steps + 2
    if ifault == 5:
        pos, data = kinematic_fault(nx, ny, nz, h, nsrc, seed + 1)
        data[:, 0, 2] = rng.uniform(0.0, steps * dt * 0.3, nsrc)
        data[:, 0, 3] = rng.uniform(5 * dt, 10 * dt, nsrc)
        nst = 2
    else:
        pos = np.stack([rng.integers(3, nx - 2, nsrc), rng.integers(3, ny - 2, nsrc),
                        rng.integers(1, nz - 2, nsrc)], axis=1).astype(np.int32)
        pos[0, 2] = 1  # one source on the free surface row
        data = (rng.standard_normal((nsrc, nst, 6)) * 1e13).astype(np.float32)
    params = dict(nx=nx, ny=ny, nz=nz, dh=h, dt=dt, nd=min(6, nx // 4), arbc=0.92,
                  npc=0, nve=1, ifault=ifault, nst=nst, read_step=nst, socalq=1)
    return Scenario("random_small", params, media, pos, data, steps,
                    f"random {nx}x{ny}x{nz} nvar={nvar} q={q} ifault={ifault}")


def batch_ensemble(n=96, seed=6, steps=1000, lo=(64, 64, 64), hi=(256, 256, 128), h=100.0,
                   dt=0.004):
    """An ensemble of independent simulations of uneven sizes for the batched
    path: grid sizes drawn from `seed` uniformly between `lo` and `hi` (nz a
    multiple of 4), each with its own seeded random anelastic medium and a
    random moment-tensor point source (IFAULT 1, seeded moment-rate samples)."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        nx = int(rng.integers(lo[0], hi[0] + 1))
        ny = int(rng.integers(lo[1], hi[1] + 1))
        nz = int(rng.integers(lo[2] // 4, hi[2] // 4 + 1)) * 4
        sc = random_small(nx=nx, ny=ny, nz=nz, h=h, dt=dt, steps=steps, seed=seed * 1000 + q,
                          q=True, ifault=1, nsrc=1)
        sc.name = f"batch_{q}"
        out.append(sc)
    return out


def dm_small(nxc=10, nyc=8, nzs=(36, 24), h_coarse=150.0, dt=0.004, steps=12, q=True, seed=31,
             nsrc=1):
    """A discontinuous mesh of len(nzs) blocks for parity tests: block p has
    (3^(n-1-p) nxc) x (3^(n-1-p) nyc) x nzs[p] cells at h_coarse / 3^(n-1-p),
    random media per block, point sources next to every interface.  Returns one
    Scenario per block (params carry grid / ngrids, ND scaled like
    pmcl3d.c:1026 does)."""
    n = len(nzs)
    out = []
    for p in range(n):
        f = 3 ** (n - 1 - p)
        sub = random_small(nx=nxc * f, ny=nyc * f, nz=nzs[p], q=q, ifault=1, steps=steps,
                           seed=seed + p, nsrc=nsrc if p == 0 else 1)
        sub.params.update(dh=h_coarse / f, dt=dt, nd=2 * f, grid=p, ngrids=n)
        # one source a few cells above each interface and one below it, so the
        # wavefield crosses the interfaces in both directions within a few steps
        nxp, nyp, nzp = sub.params["nx"], sub.params["ny"], sub.params["nz"]
        pos = []
        if p < n - 1:
            pos.append([nxp // 2, nyp // 2, nzp - 4])  # 4 cells above the block's bottom
        if p > 0:
            pos.append([nxp // 2 + 1, nyp // 2, 4])    # 4 cells below the block's top
        k = len(pos)
        sub.src_pos = np.asarray(pos, np.int32).reshape(k, 3)
        sub.src_data = sub.src_data[:1].repeat(k, 0)[:k]
        sub.name = f"dm_small_{p}"
        out.append(sub)
    return out


def write_topography(path, nx, ny, h, amplitude=1000.0, width=5000.0, rough_rms=100.0,
                     seed=4, padding=8):
    """Topography file of the reference format (serial_reader.c:9-62): int32
    nx, ny, padding, then float32 elevation (m) [nx + 2 padding][ny + 2 padding]
    with y fastest.  A Gaussian hill at the centre plus seeded smooth
    roughness (rms `rough_rms`)."""
    rng = np.random.default_rng(seed)
    gx = (np.arange(nx + 2 * padding) - padding) * h
    gy = (np.arange(ny + 2 * padding) - padding) * h
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    xc, yc = 0.5 * (nx - 1) * h, 0.5 * (ny - 1) * h
    elev = amplitude * np.exp(-((X - xc) ** 2 + (Y - yc) ** 2) / (2.0 * width ** 2))
    if rough_rms > 0:
        noise = rng.standard_normal(X.shape)
        # smooth with a 5-point box twice (fractal-like small-scale relief)
        for _ in range(2):
            noise = (noise + np.roll(noise, 1, 0) + np.roll(noise, -1, 0) +
                     np.roll(noise, 1, 1) + np.roll(noise, -1, 1)) / 5.0
        noise *= rough_rms / max(noise.std(), 1e-30)
        elev = elev + noise
    with open(path, "wb") as fh:
        np.asarray([nx, ny, padding], np.int32).tofile(fh)
        elev.astype(np.float32).tofile(fh)
    return elev.astype(np.float32)


def lithostatic_sigma2(d1_padded, nx, ny, nz, dh):
    """Vertical lithostatic stress on the padded grid from the padded density,
    as pmcl3d's Drucker-Prager set-up forms it (mesh.c:1274-1282): -dh/2 rho g
    in the surface cell and the image above it, then rho g dh more per cell
    downwards, accumulated in double and stored as float cell by cell."""
    top = nz + 31
    s2 = np.zeros_like(d1_padded, dtype=np.float32)
    sl = (slice(2, nx + 18), slice(2, ny + 18))
    d = d1_padded[sl[0], sl[1], :].astype(np.float64)
    cur = (-dh / 2.0 * d[:, :, top] * 9.81).astype(np.float32)
    s2[sl[0], sl[1], top] = cur
    s2[sl[0], sl[1], top + 1] = cur
    for k in range(top - 1, 29, -1):
        cur = (cur.astype(np.float64) - dh * d[:, :, k] * 9.81).astype(np.float32)
        s2[sl[0], sl[1], k] = cur
    return s2


def config3_blocks(nxc=213, nyc=213, nz_fine=320, nz_coarse=96, h_fine=40.0, dt=0.0028,
                   steps=3000, src_depth_m=8000.0, f0=2.0, m0=1e16, seed=4, vp_cap=6300.0):
    """Topography + discontinuous mesh + plasticity + attenuation workload: a
    fine block of (3 nxc) x (3 nyc) x nz_fine cells at h_fine over a 3x coarser
    block of nxc x nyc x nz_coarse (the fine block must be a multiple of 3 in x
    and y, so 640 becomes 639); each block carries the anelastic 1-D gradient
    (vs 1000..3500 m/s over the whole depth, vp = 1.73 vs, Gardner density,
    Qs = 50 vs[km/s], Qp = 2 Qs) with its own seeded von Karman perturbation;
    a moment-tensor point source (Mxy Ricker', IFAULT 1) at src_depth_m in the
    fine block.  dt keeps vp dt / h below 0.45 on the fine block.  Returns the
    two block Scenarios (params carry grid / ngrids)."""
    h_coarse = 3 * h_fine
    depth_total = nz_fine * h_fine + nz_coarse * h_coarse
    blocks = []
    for p, (nx, ny, nz, h, z0) in enumerate([(3 * nxc, 3 * nyc, nz_fine, h_fine, 0.0),
                                             (nxc, nyc, nz_coarse, h_coarse,
                                              nz_fine * h_fine)]):
        zc = z0 + (np.arange(nz, dtype=np.float32) + 0.5) * h  # file k = 0 is the top
        vs1d = 1000.0 + 2500.0 * zc / depth_total
        pert = np.clip(von_karman((nz, ny, nx), h, 500.0, 0.1, 0.05, seed + 10 * p), -0.15, 0.15)
        vs = vs1d[:, None, None] * (1.0 + pert)
        del pert
        vp = np.minimum(1.73 * vs, vp_cap).astype(np.float32)
        vs = (vp / 1.73).astype(np.float32)
        rho = (310.0 * vp ** 0.25).astype(np.float32)
        qs = (50.0 * vs / 1000.0).astype(np.float32)
        media = np.stack([vp, vs, rho, (2.0 * qs).astype(np.float32), qs], axis=-1)
        del vp, vs, rho, qs
        nst = steps + 2
        if p == 0:
            pos = np.array([[nx // 2, ny // 2, int(round(src_depth_m / h))]], np.int32)
            data = np.zeros((1, nst, 6), np.float32)
            data[0, :, 5] = ricker_derivative(nst, dt, f0) * m0
        else:
            pos = np.zeros((0, 3), np.int32)
            data = np.zeros((0, nst, 6), np.float32)
        params = dict(nx=nx, ny=ny, nz=nz, dh=h, dt=dt, nd=20 * (3 if p == 0 else 1),
                      arbc=0.92, npc=0, nve=3, ifault=1, nst=nst, read_step=nst, socalq=1,
                      grid=p, ngrids=2)
        blocks.append(Scenario(f"config3_{p}", params, media, pos, data, steps,
                               f"block {p}: {nx}x{ny}x{nz} at h={h}"))
    return blocks
