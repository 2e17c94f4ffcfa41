"""ctypes bindings to the reference builds under oracle/_ref -- TEST INFRASTRUCTURE.

* ``RefHost``  -> oracle/_ref/libawpref_host.so: the reference's own host set-up
  code (src/awp/mesh.c, cerjan.c, grid.c) compiled on the CPU.
* ``RefGpuSim`` -> oracle/_ref/libawpref.so: the reference's own CUDA kernels
  (src/awp/kernel.cu) driven through its launchers in the order of the
  single-rank pmcl3d time loop (src/awp/pmcl3d.c:1628-2487).

``model_setup`` assembles every per-run array the time loop needs (media,
memory-variable arrays, sponge, Q(f) table, surface Lame ratio) with the
reference's own host code, so the oracle, the reference GPU build and the
product can all be fed identical inputs.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from ctypes import POINTER, byref, c_double, c_float, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
NGSL, ALIGN = 8, 32

_F = POINTER(c_float)
_I = POINTER(c_int)


def fptr(a):
    return a.ctypes.data_as(_F)


def padded_shape(nx, ny, nz):
    return (nx + 4 + 2 * NGSL, ny + 4 + 2 * NGSL, nz + 2 * ALIGN)


class RefHost:
    def __init__(self, path=None):
        path = path or os.path.join(REF_DIR, "libawpref_host.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        lib.ref_tausub.argtypes = [c_float, c_float, _F]
        lib.ref_weights_sub.argtypes = [c_float, c_float, _F, _F]
        lib.ref_inimesh.argtypes = ([ctypes.c_char_p, c_int, c_float, c_float, c_float, c_float,
                                     c_int, c_int, c_int, c_int, c_int] + [_F] * 5 + [_F] * 8)
        lib.ref_init_texture.argtypes = ([c_int] * 3 + [_F] * 3 + [c_int] * 4 +
                                         [_F, _F, _I, _F])
        lib.ref_inicrj.argtypes = [c_float] + [c_int] * 8 + [_F] * 3
        lib.ref_hoek_brown.argtypes = [c_float] * 5 + [c_int, _F, _F]
        lib.ref_rotation_matrix.argtypes = [_F, _F, _F, _F]
        lib.ref_checkmesh.argtypes = [c_int] * 6 + [_F, _F]
        lib.ref_checkmesh_ww.argtypes = [c_int] * 6 + [_I, _I]
        lib.ref_input_read.argtypes = [ctypes.c_char_p, POINTER(ctypes.c_longlong),
                                       ctypes.c_char_p, c_int]
        lib.ref_input_data.argtypes = [_F, _F, _F, _I]
        lib.ref_point_coefs.argtypes = [c_int, c_int, c_int, c_int, c_float] + [_I] * 4 + [_F] * 3
        self.lib = lib

    def tausub(self, taumin, taumax):
        out = np.zeros(8, np.float32)
        self.lib.ref_tausub(taumin, taumax, fptr(out))
        return out

    def weights_sub(self, ex, fac):
        w = np.zeros(8, np.float32)
        c = np.zeros(16, np.float32)
        self.lib.ref_weights_sub(ex, fac, fptr(w), fptr(c))
        return w, c

    def inimesh(self, media, fp=2.5, fac=0.005, q0=5.0, ex=0.0, nve=1, socalq=1):
        """Run inimesh on `media` ([nz][ny][nx][nvar] float32) via a temp file."""
        nz, ny, nx, nvar = media.shape
        shp = padded_shape(nx, ny, nz)
        out = {k: np.zeros(shp, np.float32) for k in ("d1", "mu", "lam", "qp", "qs")}
        taumax = c_float()
        taumin = c_float()
        tau8 = np.zeros(8, np.float32)
        w8 = np.zeros(8, np.float32)
        coeff = np.zeros(16, np.float32)
        vse = np.zeros(2, np.float32)
        vpe = np.zeros(2, np.float32)
        dde = np.zeros(2, np.float32)
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "media.bin")
            np.ascontiguousarray(media, np.float32).tofile(path)
            self.lib.ref_inimesh(path.encode(), nvar, fp, fac, q0, ex, nx, ny, nz, nve, socalq,
                                 fptr(out["d1"]), fptr(out["mu"]), fptr(out["lam"]),
                                 fptr(out["qp"]), fptr(out["qs"]), byref(taumax), byref(taumin),
                                 fptr(tau8), fptr(w8), fptr(coeff), fptr(vse), fptr(vpe),
                                 fptr(dde))
        out.update(taumax=taumax.value, taumin=taumin.value, tau8=tau8, w8=w8, coeff=coeff,
                   vse=vse, vpe=vpe, dde=dde)
        return out

    def init_texture(self, nx, ny, nz, tau1, tau2, w8, xls, xre, yls, yre):
        shp = padded_shape(nx, ny, nz)
        vx1 = np.zeros(shp, np.float32)
        vx2 = np.zeros(shp, np.float32)
        wwo = np.zeros(shp, np.float32)
        ww = np.zeros(shp, np.int32)
        self.lib.ref_init_texture(nx, ny, nz, fptr(np.ascontiguousarray(tau1, np.float32)),
                                  fptr(np.ascontiguousarray(tau2, np.float32)),
                                  fptr(np.ascontiguousarray(w8, np.float32)), xls, xre, yls, yre,
                                  fptr(vx1), fptr(vx2), ww.ctypes.data_as(_I), fptr(wwo))
        return vx1, vx2, ww, wwo

    def inicrj(self, arbc, nx, ny, nz, nd, islowest=1, npc=0):
        dx = np.ones(nx + 4 + 2 * NGSL, np.float32)
        dy = np.ones(ny + 4 + 2 * NGSL, np.float32)
        dz = np.ones(nz + 2 * ALIGN, np.float32)
        self.lib.ref_inicrj(arbc, nx, ny, nz, nx, ny, nd, islowest, npc, fptr(dx), fptr(dy),
                            fptr(dz))
        return dx, dy, dz

    def hoek_brown(self, sigma_0, sigma_ci, gsi, mi, d, tunnel):
        phi = c_float()
        cohes = c_float()
        self.lib.ref_hoek_brown(sigma_0, sigma_ci, gsi, mi, d, tunnel, byref(phi), byref(cohes))
        return phi.value, cohes.value


    def checkmesh(self, lo, hi, nl, nh):
        """checkmesh (mesh.c:1404-1443): lo (coarse, padded) corrected in place
        from hi (fine) at the coarse grid's top three levels; nl/nh = (nx, ny, nz)."""
        if lo.dtype == np.int32:
            return self.lib.ref_checkmesh_ww(*nl, *nh, lo.ctypes.data_as(_I),
                                             np.ascontiguousarray(hi).ctypes.data_as(_I))
        return self.lib.ref_checkmesh(*nl, *nh, fptr(lo), fptr(np.ascontiguousarray(hi)))

    def rotation_matrix(self, strike, dip):
        """rotation_matrix (mesh.c:1370-1401): Rz, RzT from strike/dip in degrees."""
        st = np.ascontiguousarray(strike, np.float32)
        dp = np.ascontiguousarray(dip, np.float32)
        rz = np.zeros(9, np.float32)
        rzt = np.zeros(9, np.float32)
        self.lib.ref_rotation_matrix(fptr(st), fptr(dp), fptr(rz), fptr(rzt))
        return rz, rzt


    def input_read(self, path):
        """input_init (readers/input.c:35-42): (status, header dict, x, y, z, type)."""
        hdr = (ctypes.c_longlong * 8)()
        fname = ctypes.create_string_buffer(2048)
        err = self.lib.ref_input_read(path.encode(), hdr, fname, 2048)
        if err:
            return err, None, None, None, None, None
        n = int(hdr[0])
        x = np.zeros(n, np.float32)
        y = np.zeros(n, np.float32)
        z = np.zeros(n, np.float32)
        t = np.zeros(n, np.int32)
        self.lib.ref_input_data(fptr(x), fptr(y), fptr(z), t.ctypes.data_as(_I))
        keys = ["length", "gpu_buffer_size", "cpu_buffer_size", "steps", "num_writes", "stride",
                "degree", "major"]
        h = {k: int(v) for k, v in zip(keys, hdr)}
        h["file"] = fname.value.decode()
        return 0, h, x, y, z, t

    def point_coefs(self, path, grid_type, nx, ny, nz, h, ftopo=None):
        """The interpolation set-up of source_init_common for one component,
        built from the reference's own routines (see ref_host_shim.c); with
        `ftopo` (the normalised surface function) on the curvilinear block."""
        err, hdr, *_ = self.input_read(path)
        assert err == 0, err
        n = hdr["length"]
        nb = hdr["degree"] + 1
        idx = np.zeros(n, np.int32)
        ix = np.zeros(n, np.int32)
        iy = np.zeros(n, np.int32)
        iz = np.zeros(n, np.int32)
        lx = np.zeros(n * nb, np.float32)
        ly = np.zeros(n * nb, np.float32)
        lz = np.zeros(n * nb, np.float32)
        I = lambda a: a.ctypes.data_as(_I)  # noqa: E731
        if ftopo is None:
            cnt = self.lib.ref_point_coefs(grid_type, nx, ny, nz, h, I(idx), I(ix), I(iy), I(iz),
                                           fptr(lx), fptr(ly), fptr(lz))
        else:
            f = np.ascontiguousarray(ftopo, np.float32)
            self.lib.ref_point_coefs_topo.argtypes = [c_int, c_int, c_int, c_int, c_float, _F] + \
                [_I] * 4 + [_F] * 3
            cnt = self.lib.ref_point_coefs_topo(grid_type, nx, ny, nz, h, fptr(f), I(idx), I(ix),
                                                I(iy), I(iz), fptr(lx), fptr(ly), fptr(lz))
        assert cnt >= 0, cnt
        return dict(indices=idx[:cnt], ix=ix[:cnt], iy=iy[:cnt], iz=iz[:cnt],
                    lx=lx[:cnt * nb].reshape(cnt, nb), ly=ly[:cnt * nb].reshape(cnt, nb),
                    lz=lz[:cnt * nb].reshape(cnt, nb))


def mesh_setup(scns, host: RefHost | None = None):
    """Per-block set-up of a discontinuous mesh at one rank from the
    reference's host code: inimesh per block, then checkmesh of every coarser
    block's media against the block above (pmcl3d.c:879-901), init_texture per
    block and checkmesh of the texture arrays (pmcl3d.c:1049-1059), inicrj with
    the bottom sponge on the lowest block only (pmcl3d.c:1014-1033)."""
    host = host or RefHost()
    setups = []
    for p, scn in enumerate(scns):
        st = model_setup(scn, host)
        q = scn.params
        n = q["ngrids"]
        dx, dy, dz = host.inicrj(q.get("arbc", 0.92), q["nx"], q["ny"], q["nz"], q["nd"],
                                 1 if p == n - 1 else 0, q.get("npc", 0))
        st.update(dcrjx=dx, dcrjy=dy, dcrjz=dz)
        setups.append(st)
    for p in range(1, len(scns)):
        nl = tuple(scns[p].params[k] for k in ("nx", "ny", "nz"))
        nh = tuple(scns[p - 1].params[k] for k in ("nx", "ny", "nz"))
        for k in ("d1", "mu", "lam", "qp", "qs"):
            host.checkmesh(setups[p]["media"][k], setups[p - 1]["media"][k], nl, nh)
        for k in ("vx1", "vx2", "wwo", "ww"):
            host.checkmesh(setups[p][k], setups[p - 1][k], nl, nh)
    return setups


class RefMeshSim:
    """The reference CUDA kernels on a discontinuous mesh, driven in pmcl3d's
    single-rank order with ngrids > 1 (pmcl3d.c:1628-2490): dvelcx per block,
    dvelc2, intp3d, swap3 (swap-area exchanges are no-ops at one rank), dstrqc
    per block, dstrqc2, sources, intp3d, swap3, fstr on block 0."""

    def __init__(self, scns, setups, path=None, intopo=None):
        import torch
        self.torch = torch
        self.n = len(scns)
        self.sims = [RefGpuSim(s, st, path=path, defer_consts=True)
                     if (p > 0 or intopo is None) else
                     RefTopoSim(s, st, intopo, path=path, defer_consts=True)
                     for p, (s, st) in enumerate(zip(scns, setups))]
        self.nve = scns[0].params.get("nve", 1)
        lib = self.sims[0].lib
        self.lib = lib
        V = c_void_p
        lib.dvelc2_H.argtypes = [V] * 13 + [c_int, c_int, V, c_int]
        lib.dstrqc2_H.argtypes = [V] * 22 + [c_int, c_int, V] + [V] * 5 + [c_int] * 5
        lib.intp3d_H.argtypes = [V] * 18 + [c_int, c_int, c_int, V, c_int]
        lib.swap_H.argtypes = [V] * 18 + [c_int, c_int] + [V] * 4 + [c_int, V, c_int]
        DH = np.array([s.params["dh"] for s in scns], np.float32)
        nxt = np.array([s.params["nx"] for s in scns], np.int32)
        nyt = np.array([s.params["ny"] for s in scns], np.int32)
        nzt = np.array([s.params["nz"] for s in scns], np.int32)
        z9 = np.zeros(9, np.float32)
        Rz, RzT, fmajor, fminor = z9, z9, 0.0, 0.0
        if self.nve == 3:  # one principal-stress frame for every block (nonlinear.dat)
            pl = setups[0]["plast"]
            Rz = np.ascontiguousarray(pl["Rz"], np.float32)
            RzT = np.ascontiguousarray(pl["RzT"], np.float32)
            fmajor, fminor = float(pl["fmajor"]), float(pl["fminor"])
        lib.SetDeviceConstValue(fptr(DH), c_float(scns[0].params["dt"]), nxt.ctypes.data_as(_I),
                                nyt.ctypes.data_as(_I), nzt.ctypes.data_as(_I), self.n,
                                c_float(fmajor), c_float(fminor), fptr(Rz), fptr(RzT))
        # zeroed swap-area buffers (never read at one rank, pmcl3d.c:1434-1508)
        self.zbuf = torch.zeros(1 << 16, device="cuda")
        for p, sim in enumerate(self.sims):
            sim.grid = p
            sim.ngrids = self.n
            # the initial sample goes into every block with sources (pmcl3d.c:1175-1187)
            if sim.p["ifault"] == 1 and sim.npsrc:
                sim._addsrc(1)
        torch.cuda.synchronize()

    def _fields(self, sim, order):
        return [c_void_p(sim.f[k].data_ptr()) for k in order]

    def _interfaces(self):
        V9 = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz"]
        S9 = ["xx", "yy", "zz", "xy", "xz", "yz", "u1", "v1", "w1"]
        for p in range(1, self.n):
            lo, hi = self.sims[p], self.sims[p - 1]
            self.lib.intp3d_H(*self._fields(lo, V9), *self._fields(hi, V9), lo.nx, lo.ny, 0,
                              None, p)
        zb = c_void_p(self.zbuf.data_ptr())
        for p in range(self.n - 1):
            lo, hi = self.sims[p + 1], self.sims[p]
            self.lib.swap_H(*self._fields(lo, S9), *self._fields(hi, S9), lo.nx, lo.ny,
                            zb, zb, zb, zb, 0, None, p)

    def step(self, n=1):
        lib = self.lib
        for _ in range(n):
            for sim in self.sims:
                sim.cur += 1
                sim.velocity()
            for p in range(self.n - 1):
                sim = self.sims[p]
                f = sim.f
                P = sim.ptr
                lib.dvelc2_H(P(f["u1"]), P(f["v1"]), P(f["w1"]), P(f["xx"]), P(f["yy"]),
                             P(f["zz"]), P(f["xy"]), P(f["xz"]), P(f["yz"]), P(sim.dcrjx),
                             P(sim.dcrjy), P(sim.dcrjz), P(f["d1"]), sim.nx, sim.ny, None, p)
            self._interfaces()
            for sim in self.sims:
                sim.stress_all()
            for p in range(self.n - 1):
                sim = self.sims[p]
                f = sim.f
                P = sim.ptr
                xls, xre, yls, yre = 2 + NGSL, sim.nx + NGSL + 1, 2 + NGSL, sim.ny + NGSL + 1
                lib.dstrqc2_H(*[P(f[k]) for k in ("xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2",
                                                  "r3", "r4", "r5", "r6", "u1", "v1", "w1",
                                                  "lam", "mu", "qp", "qs")],
                              P(sim.dcrjx), P(sim.dcrjy), P(sim.dcrjz), sim.nx, sim.ny, None,
                              P(sim.coeff), P(sim.vx1), P(sim.vx2), P(sim.ww), P(sim.wwo),
                              xls, xre, yls, yre, p)
            for sim in self.sims:
                sim.sources()
            self._interfaces()
            if self.nve == 3:  # yield factor and return per grid (pmcl3d.c:2108-2209)
                for sim in self.sims:
                    sim.plasticity()
            sim0 = self.sims[0]
            nx, ny = sim0.nx, sim0.ny
            P = sim0.ptr
            f = sim0.f
            lib.fstr_H(P(f["zz"]), P(f["xz"]), P(f["yz"]), None, 2 + NGSL, nx + NGSL + 1,
                       2 + NGSL, ny + NGSL + 1)
        self.torch.cuda.synchronize()

    def field(self, p, name):
        return self.sims[p].field(name)


class RefPoints:
    """The reference's own point-set device code for one component
    (interpolation.cu cuinterp_interp_H, source.cu cusource_add_cartesian_H),
    set up from an ASCII v2 file by ref_points_shim.c."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            path = os.path.join(REF_DIR, "libawpref_points.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
            lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
            lib.ref_pts_create.restype = c_void_p
            lib.ref_pts_create.argtypes = [ctypes.c_char_p, c_int, c_int, c_int, c_int, c_float,
                                           _I]
            lib.ref_pts_create_topo.restype = c_void_p
            lib.ref_pts_create_topo.argtypes = [ctypes.c_char_p, c_int, c_int, c_int, c_int,
                                                c_float, _F, _I]
            lib.ref_pts_srcadd_curv.argtypes = [c_void_p, c_void_p, c_void_p, c_float, c_float,
                                                c_void_p, c_int, c_void_p]
            lib.ref_pts_interp.argtypes = [c_void_p, c_void_p, c_void_p]
            lib.ref_pts_srcadd.argtypes = [c_void_p, c_void_p, c_void_p, c_float, c_float]
            lib.ref_pts_force.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_float,
                                          c_float, c_float, c_void_p, c_int, c_int, c_int,
                                          c_void_p]
            lib.ref_pts_destroy.argtypes = [c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, path, grid_type, nx, ny, nz, h, ftopo=None):
        """`ftopo`: the normalised surface function (the first f array of
        awp_topo_metrics) for a curvilinear block, else None."""
        lib = self.lib()
        n = c_int(0)
        if ftopo is None:
            self.h = lib.ref_pts_create(path.encode(), grid_type, nx, ny, nz, h, byref(n))
        else:
            self._f = np.ascontiguousarray(ftopo, np.float32)
            self.h = lib.ref_pts_create_topo(path.encode(), grid_type, nx, ny, nz, h,
                                             fptr(self._f), byref(n))
        self.ny = ny
        if not self.h:
            raise RuntimeError("reference point-set set-up failed")
        self.count = n.value

    def interp(self, d_out_ptr, d_in_ptr):
        self.lib().ref_pts_interp(self.h, c_void_p(d_out_ptr), c_void_p(d_in_ptr))

    def srcadd(self, d_field_ptr, d_values_ptr, h, dt):
        self.lib().ref_pts_srcadd(self.h, c_void_p(d_field_ptr), c_void_p(d_values_ptr), h, dt)

    def srcadd_curv(self, d_field_ptr, d_values_ptr, h, dt, d_f_ptr, d_dg_ptr):
        self.lib().ref_pts_srcadd_curv(self.h, c_void_p(d_field_ptr), c_void_p(d_values_ptr), h,
                                       dt, c_void_p(d_f_ptr), self.ny, c_void_p(d_dg_ptr))

    def force(self, d_field_ptr, d_values_ptr, d_d1_ptr, h, dt, quad_weight, d_f_ptr, nx, nz,
              d_dg_ptr):
        """cusource_add_force_H on a velocity component (forces.c:74-94)."""
        self.lib().ref_pts_force(self.h, c_void_p(d_field_ptr), c_void_p(d_values_ptr),
                                 c_void_p(d_d1_ptr), h, dt, quad_weight, c_void_p(d_f_ptr), nx,
                                 self.ny, nz, c_void_p(d_dg_ptr))

    def close(self):
        if self.h:
            self.lib().ref_pts_destroy(self.h)
            self.h = None


def lithostatic_sigma2(d1, nx, ny, nz, dh):
    """Vertical lithostatic stress of inidrpr_hoekbrown_light (mesh.c:1274-1282):
    -dh/2 rho g at the surface cell (and the image above it), then one cell of
    rho g dh more per cell downwards, evaluated in double and stored as float
    at every step like the reference."""
    shp = padded_shape(nx, ny, nz)
    s2 = np.zeros(shp, np.float32)
    top = nz + ALIGN - 1
    sl = (slice(2, nx + 2 + 2 * NGSL), slice(2, ny + 2 + 2 * NGSL))
    d = d1[sl[0], sl[1], :].astype(np.float64)
    cur = (-dh / 2.0 * d[:, :, top] * 9.81).astype(np.float32)
    s2[sl[0], sl[1], top] = cur
    s2[sl[0], sl[1], top + 1] = cur
    for k in range(top - 1, ALIGN - 3, -1):
        cur = (cur.astype(np.float64) - dh * d[:, :, k] * 9.81).astype(np.float32)
        s2[sl[0], sl[1], k] = cur
    return s2


def plasticity_inputs(scn, setup, seed=7, cohes=(2e4, 2e5), phi=(25.0, 35.0),
                      strike=(40.0, 0.0, 130.0), fmajor=1.6, fminor=0.5, host=None):
    """Drucker-Prager inputs on the padded grid: lithostatic sigma2 from the
    density, seeded cohesion and friction angle per cell, the principal-stress
    ratios and the rotation of nonlinear.dat (dip fixed to 0/90/0 as in
    mesh.c:1199-1204).  Low cohesions make cells near the sources yield."""
    host = host or RefHost()
    p = scn.params
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    shp = padded_shape(nx, ny, nz)
    rng = np.random.default_rng(seed)
    sigma2 = lithostatic_sigma2(setup["media"]["d1"], nx, ny, nz, p["dh"])
    coh = rng.uniform(cohes[0], cohes[1], shp).astype(np.float32)
    ph = rng.uniform(phi[0], phi[1], shp).astype(np.float32)
    dip = np.array([0.0, 90.0, 0.0], np.float32)
    st = np.array(strike, np.float32)
    rz, rzt = host.rotation_matrix(st, dip)
    return dict(sigma2=sigma2, cohes=coh, phi=ph, fmajor=np.float32(fmajor),
                fminor=np.float32(fminor), strike=st, dip=dip, Rz=rz, RzT=rzt)


def tau12(tau8, dt):
    """tau1/tau2 of pmcl3d.c:1036-1049 (float division, double exp)."""
    tau8 = np.asarray(tau8, np.float32)
    arg = (np.float32(-dt) / tau8).astype(np.float32)
    tau2 = np.exp(arg.astype(np.float64)).astype(np.float32)
    tau1 = (0.5 * (1.0 - tau2.astype(np.float64))).astype(np.float32)
    return tau1, tau2


def lam_mu_ref(lam, mu, nx, ny, nz):
    """pmcl3d.c:944-951 at one rank (double divisions, float ratio)."""
    shp = padded_shape(nx, ny, nz)
    out = np.zeros((shp[0], shp[1]), np.float32)
    ktop = nz + ALIGN - 1
    sl = (slice(2 + NGSL, nx + NGSL + 2), slice(2 + NGSL, ny + NGSL + 2))
    t_xl = (1.0 / lam[sl[0], sl[1], ktop].astype(np.float64)).astype(np.float32)
    t_xl2m = (2.0 / mu[sl[0], sl[1], ktop].astype(np.float64) +
              t_xl.astype(np.float64)).astype(np.float32)
    out[sl] = t_xl / t_xl2m
    return out


def map_sources(scn):
    """inisource at one rank (source.c:131-264): file (x, y, z-from-surface) ->
    the psrc triple addsrc_cu indexes with, keeping only in-window sources."""
    p = scn.params
    nz = p["nz"]
    pos = np.asarray(scn.src_pos, np.int64)
    z = nz + 1 - pos[:, 2]
    keep = ((pos[:, 0] >= -1) & (pos[:, 0] <= p["nx"] + 2) & (pos[:, 1] >= -1) &
            (pos[:, 1] <= p["ny"] + 2) & (z >= 1) & (z <= nz))
    psrc = np.stack([pos[:, 0], pos[:, 1], z], axis=1)[keep].astype(np.int32)
    data = np.asarray(scn.src_data, np.float32)[keep]
    rs = p["read_step"] if p["ifault"] != 5 else 2
    comps = [np.ascontiguousarray(data[:, :rs, q]) for q in range(6)]  # xx yy zz xz yz xy
    return psrc, comps, rs


def model_setup(scn, host: RefHost | None = None, fp=2.5, fac=0.005, q0=5.0, ex=0.0):
    """Every per-run array of the single-rank time loop, from the reference's host code."""
    host = host or RefHost()
    p = scn.params
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    m = host.inimesh(scn.media, fp=fp, fac=fac, q0=q0, ex=ex, nve=p.get("nve", 1),
                     socalq=p.get("socalq", 1))
    tau1, tau2 = tau12(m["tau8"], p["dt"])
    xls, xre = 2 + NGSL, nx + NGSL + 1
    yls, yre = 2 + NGSL, ny + NGSL + 1
    vx1, vx2, ww, wwo = host.init_texture(nx, ny, nz, tau1, tau2, m["w8"], xls, xre, yls, yre)
    dcrjx, dcrjy, dcrjz = host.inicrj(p.get("arbc", 0.92), nx, ny, nz, p.get("nd", 20), 1,
                                      p.get("npc", 0))
    lm = lam_mu_ref(m["lam"], m["mu"], nx, ny, nz)
    psrc, comps, rs = map_sources(scn)
    return dict(media=m, vx1=vx1, vx2=vx2, ww=ww, wwo=wwo, dcrjx=dcrjx, dcrjy=dcrjy,
                dcrjz=dcrjz, lam_mu=lm, coeff=m["coeff"], psrc=psrc, src=comps,
                src_stride=rs, tau1=tau1, tau2=tau2)


class RefGpuSim:
    """The reference CUDA kernels driven in pmcl3d's single-rank order."""

    FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz",
              "r1", "r2", "r3", "r4", "r5", "r6"]

    def __init__(self, scn, setup, path=None, defer_consts=False):
        import torch
        self.grid, self.ngrids = 0, 1
        path = path or os.path.join(REF_DIR, "libawpref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.torch = torch
        lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        V = c_void_p
        lib.SetDeviceConstValue.argtypes = [_F, c_float, _I, _I, _I, c_int, c_float, c_float,
                                            _F, _F]
        lib.SetDeviceFilterParameters.argtypes = [c_int, POINTER(c_double), POINTER(c_double)]
        lib.dvelcx_H_opt.argtypes = [V] * 13 + [c_int, c_int, V] + [c_int] * 4
        lib.dstrqc_H.argtypes = [V] * 23 + [c_int, c_int, V] + [V] * 5 + [c_int] * 9
        lib.fstr_H.argtypes = [V] * 4 + [c_int] * 4
        lib.addsrc_H.argtypes = [c_int, c_int, c_int, V, c_int, V] + [V] * 12 + [c_int]
        lib.addkinsrc_H.argtypes = [c_int, c_int, V, c_int, V] + [V] * 15 + [c_int]
        lib.drprecpc_calc_H_opt.argtypes = [V] * 13 + [c_int] * 5 + [V, c_int]
        lib.drprecpc_app_H.argtypes = [V] * 9 + [c_int] * 5 + [V, c_int]
        lib.addplanesrc_H.argtypes = [c_int, c_int, c_int, V, V, V, c_int, c_int, c_int] + \
            [V] * 9 + [c_int]
        self.lib = lib
        self.plane = None
        self.scn = scn
        p = scn.params
        self.p = p
        self.nx, self.ny, self.nz = p["nx"], p["ny"], p["nz"]
        dev = torch.device("cuda")
        m = setup["media"]

        def T(a, dtype=torch.float32):
            return torch.as_tensor(np.ascontiguousarray(a)).to(dev, dtype)

        shp = padded_shape(self.nx, self.ny, self.nz)
        self.f = {k: torch.zeros(shp, dtype=torch.float32, device=dev) for k in self.FIELDS}
        self.f.update(d1=T(m["d1"]), mu=T(m["mu"]), lam=T(m["lam"]), qp=T(m["qp"]),
                      qs=T(m["qs"]))
        self.vx1 = T(setup["vx1"])
        self.vx2 = T(setup["vx2"])
        self.ww = T(setup["ww"], torch.int32)
        self.wwo = T(setup["wwo"])
        self.dcrjx, self.dcrjy, self.dcrjz = (T(setup["dcrjx"]), T(setup["dcrjy"]),
                                              T(setup["dcrjz"]))
        self.lam_mu = T(setup["lam_mu"])
        self.coeff = T(setup["coeff"])
        self.psrc = T(setup["psrc"], torch.int32)
        self.npsrc = int(setup["psrc"].shape[0])
        self.src = [T(c) for c in setup["src"]]
        self.stride = setup["src_stride"]
        self.mom = torch.zeros(max(self.npsrc, 1), dtype=torch.float32, device=dev)
        self.filt = None
        DH = np.array([p["dh"]], np.float32)
        nxt = np.array([self.nx], np.int32)
        nyt = np.array([self.ny], np.int32)
        nzt = np.array([self.nz], np.int32)
        Rz = np.zeros(9, np.float32)
        RzT = np.zeros(9, np.float32)
        fmajor = fminor = 0.0
        self.nve = p.get("nve", 1)
        if self.nve == 3:
            pl = setup["plast"]
            Rz = np.ascontiguousarray(pl["Rz"], np.float32)
            RzT = np.ascontiguousarray(pl["RzT"], np.float32)
            fmajor, fminor = float(pl["fmajor"]), float(pl["fminor"])
            self.f.update(sigma2=T(pl["sigma2"]), cohes=T(pl["cohes"]), phi=T(pl["phi"]))
            self.f["yldfac"] = torch.ones(shp, dtype=torch.float32, device=dev)
        self.f["neta"] = torch.zeros(shp, dtype=torch.float32, device=dev)
        if not defer_consts:
            lib.SetDeviceConstValue(fptr(DH), c_float(p["dt"]), nxt.ctypes.data_as(_I),
                                    nyt.ctypes.data_as(_I), nzt.ctypes.data_as(_I), 1,
                                    c_float(fmajor), c_float(fminor), fptr(Rz), fptr(RzT))
        fz = np.zeros(20, np.float64)
        lib.SetDeviceFilterParameters(0, fz.ctypes.data_as(POINTER(c_double)),
                                      fz.ctypes.data_as(POINTER(c_double)))
        self._fz = fz
        self.cur = 0
        self.source_step = 1
        # callables(sim, step): after the velocity update (IFAULT 4 frcvel,
        # pmcl3d.c:1821-1826), after the stress update (SOURCEFILE adds,
        # pmcl3d.c:1987-2004) and after the free-surface imaging (receivers,
        # pmcl3d.c:2246-2247)
        self.after_velocity = []
        self.after_stress = []
        self.after_step = []
        if p["ifault"] == 1 and self.npsrc and not defer_consts:
            # initial sample added on the host before the copy (pmcl3d.c:1175-1187)
            self._addsrc(1)
        torch.cuda.synchronize()

    def ptr(self, t):
        return c_void_p(t.data_ptr())

    def _addsrc(self, i):
        f = self.f
        s = self.src
        self.lib.addsrc_H(i, self.stride, 3, self.ptr(self.psrc), self.npsrc, None,
                          *[self.ptr(t) for t in s],
                          self.ptr(f["xx"]), self.ptr(f["yy"]), self.ptr(f["zz"]),
                          self.ptr(f["xy"]), self.ptr(f["yz"]), self.ptr(f["xz"]), self.grid)

    def _stress(self, s_i, e_i, s_j, e_j):
        f = self.f
        P = self.ptr
        self.lib.dstrqc_H(P(f["xx"]), P(f["yy"]), P(f["zz"]), P(f["xy"]), P(f["xz"]), P(f["yz"]),
                          P(f["r1"]), P(f["r2"]), P(f["r3"]), P(f["r4"]), P(f["r5"]), P(f["r6"]),
                          P(f["u1"]), P(f["v1"]), P(f["w1"]), P(f["lam"]), P(f["mu"]),
                          P(f["qp"]), P(self.coeff), P(f["qs"]), P(self.dcrjx), P(self.dcrjy),
                          P(self.dcrjz), self.ny, self.nz, None, P(self.lam_mu), P(self.vx1),
                          P(self.vx2), P(self.ww), P(self.wwo), self.nx, self.p.get("npc", 0),
                          0, 0, s_i, e_i, s_j, e_j, self.grid)

    def _calc(self, s_i, e_i, s_j, e_j):
        f = self.f
        P = self.ptr
        self.lib.drprecpc_calc_H_opt(P(f["xx"]), P(f["yy"]), P(f["zz"]), P(f["xy"]), P(f["xz"]),
                                     P(f["yz"]), P(f["mu"]), P(f["d1"]), P(f["sigma2"]),
                                     P(f["yldfac"]), P(f["cohes"]), P(f["phi"]), P(f["neta"]),
                                     self.nz, s_i, e_i, s_j, e_j, None, self.grid)

    def margins(self):
        """yls2/yre2 of pmcl3d.c:621-627 at one rank (ylsp = yls, yrep = yre)."""
        yls, yre = 2 + NGSL, self.ny + NGSL + 1
        yls2 = int(yls + int(yre - yls) * 0.25)
        if yls2 % 2 != 0:
            yls2 += 1
        yre2 = int(yls + int(yre - yls) * 0.75)
        if yre2 % 2 == 0:
            yre2 -= 1
        return max(yls2, yls + NGSL + 2), min(yre2, yre - NGSL - 2)

    def velocity(self):
        f = self.f
        P = self.ptr
        self.lib.dvelcx_H_opt(P(f["u1"]), P(f["v1"]), P(f["w1"]), P(f["xx"]), P(f["yy"]),
                              P(f["zz"]), P(f["xy"]), P(f["xz"]), P(f["yz"]), P(self.dcrjx),
                              P(self.dcrjy), P(self.dcrjz), P(f["d1"]), self.ny, self.nz, None,
                              2 + NGSL, self.nx + NGSL + 1, self.grid, self.ngrids)

    def stress_all(self):
        """Stress in pmcl3d's launch order (pmcl3d.c:1841-1924); NVE=3 leaves
        the middle y band of xss2..xse2 for later (pmcl3d.c:1858-1879)."""
        nx = self.nx
        yls, yre = 2 + NGSL, self.ny + NGSL + 1
        xls, xre = 2 + NGSL, nx + NGSL + 1
        if self.nve == 3:
            yls2, yre2 = self.margins()
            self._stress(NGSL + 4, nx + NGSL - 1, yls, yls2 - 1)
            self._stress(NGSL + 4, nx + NGSL - 1, yre2 + 1, yre)
        else:
            # dstrqc over xss2..xse2, then the xss1 and xss3 strips (pmcl3d.c:1845-1919)
            self._stress(NGSL + 4, nx + NGSL - 1, yls, yre)
        self._stress(xls, NGSL + 3, yls, yre)
        self._stress(nx + NGSL, xre, yls, yre)
        for hook in self.after_stress:
            hook(self, self.cur)

    def set_plane_wave(self, vx, vy, vz):
        """IFAULT 6 input series (ini_plane_wave, source.c:797-833) on the device."""
        self.plane = [self.torch.as_tensor(np.ascontiguousarray(v, np.float32)).cuda()
                      for v in (vx, vy, vz)]

    def sources(self):
        f = self.f
        P = self.ptr
        if self.p["ifault"] == 6:
            # addplanesrc_H while cur_step < NST (pmcl3d.c:2035-2041)
            if self.plane is not None and self.cur < self.p["nst"]:
                self.lib.addplanesrc_H(self.cur, 3, self.p["nst"], None, P(f["mu"]), P(f["lam"]),
                                       self.p["nd"], self.nx, self.ny,
                                       *[P(t) for t in self.plane], P(f["xx"]), P(f["yy"]),
                                       P(f["zz"]), P(f["xy"]), P(f["yz"]), P(f["xz"]), self.grid)
            return
        if self.p["ifault"] < 4 and self.cur < self.p["nst"]:
            self.source_step += 1
            if self.npsrc:
                self._addsrc(self.source_step)
        elif self.p["ifault"] == 5 and self.npsrc:
            fdp = None if self.filt is None else P(self.filt)
            self.lib.addkinsrc_H(self.cur, 3, P(self.psrc), self.npsrc, None, P(f["mu"]),
                                 *[P(t) for t in self.src], P(f["xx"]), P(f["yy"]),
                                 P(f["zz"]), P(f["xy"]), P(f["yz"]), P(f["xz"]),
                                 P(self.mom), fdp, self.grid)

    def plasticity(self):
        f = self.f
        P = self.ptr
        nx = self.nx
        xls, xre, yls, yre = 2 + NGSL, nx + NGSL + 1, 2 + NGSL, self.ny + NGSL + 1
        yls2, yre2 = self.margins()
        # pmcl3d.c:2110-2209 at one rank (xlsp = xls, ...)
        self._calc(xls, xre, yls, yls + NGSL)
        self._calc(xls, xre, yre - NGSL, yre)
        self._stress(NGSL + 4, nx + NGSL - 1, yls2, yre2)
        self._calc(xls, xls + NGSL, yls, yre)
        self._calc(xre - NGSL, xre, yls, yre)
        self._calc(xls + NGSL, xre - NGSL, yls + NGSL, yre - NGSL)
        self.lib.drprecpc_app_H(P(f["xx"]), P(f["yy"]), P(f["zz"]), P(f["xy"]),
                                P(f["xz"]), P(f["yz"]), P(f["mu"]), P(f["sigma2"]),
                                P(f["yldfac"]), self.nz, xls, xre, yls, yre, None, self.grid)

    def step(self, n=1):
        f = self.f
        P = self.ptr
        nx, ny = self.nx, self.ny
        xls, xre, yls, yre = 2 + NGSL, nx + NGSL + 1, 2 + NGSL, ny + NGSL + 1
        yls2, yre2 = self.margins()
        if self.nve == 3 and yre2 < yls2:
            raise ValueError("NVE=3 needs a non-empty middle stress region (pmcl3d.c:621-627)")
        for _ in range(n):
            self.cur += 1
            self.velocity()
            for hook in self.after_velocity:
                hook(self, self.cur)
            self.stress_all()
            self.sources()
            if self.nve == 3:
                self.plasticity()
            self.lib.fstr_H(P(f["zz"]), P(f["xz"]), P(f["yz"]), None, xls, xre, yls, yre)
            for hook in self.after_step:
                hook(self, self.cur)
        self.torch.cuda.synchronize()

    def field(self, name):
        return self.f[name].cpu().numpy()


class RefTopoSim(RefGpuSim):
    """RefGpuSim with the reference's curvilinear topography on its grid
    (oracle/_ref/libawpref_topo.so: topo_init ... topo_set_constants, then
    topo_velocity_interior_H and topo_stress_{interior,left,right}_H in place of
    dvelcx / dstrqc, pmcl3d.c:1522-1548, 1661-1698, 1841-1924).  The
    free-surface imaging, sources and receivers stay the Cartesian ones, as in
    pmcl3d.  With NVE=3 the reference at one rank runs no curvilinear stress on
    grid 0 (the interior launch belongs to the NVE < 3 branch, pmcl3d.c:1841-1857,
    and topo_stress_left/right_H return without neighbour ranks): the stress
    of grid 0 is the Cartesian dstrqc_H over the middle band of the plasticity
    section (RefGpuSim.plasticity)."""

    def __init__(self, scn, setup, intopo, path=None, topo_path=None, defer_consts=False):
        super().__init__(scn, setup, path=path, defer_consts=defer_consts)
        topo_path = topo_path or os.path.join(REF_DIR, "libawpref_topo.so")
        if not os.path.exists(topo_path):
            raise FileNotFoundError(f"{topo_path} missing: run `make -C oracle ref`")
        tl = ctypes.CDLL(topo_path, mode=ctypes.RTLD_LOCAL)
        tl.ref_topo_create.restype = c_void_p
        tl.ref_topo_create.argtypes = [ctypes.c_char_p, c_int, c_int, c_int, c_float, c_float,
                                       POINTER(c_void_p)]
        tl.ref_topo_velocity.argtypes = [c_void_p]
        tl.ref_topo_stress.argtypes = [c_void_p]
        tl.ref_topo_destroy.argtypes = [c_void_p]
        tl.ref_topo_metric_ptrs.argtypes = [c_void_p, POINTER(c_void_p), POINTER(c_int)]
        self.tl = tl
        f = self.f
        order = [f["d1"], f["lam"], f["mu"], f["qp"], self.coeff, f["qs"], self.vx1, self.vx2,
                 self.ww, self.wwo, f["xx"], f["yy"], f["zz"], f["xy"], f["xz"], f["yz"],
                 f["r1"], f["r2"], f["r3"], f["r4"], f["r5"], f["r6"], f["u1"], f["v1"], f["w1"],
                 self.dcrjx, self.dcrjy, self.dcrjz]
        arr = (c_void_p * len(order))(*[t.data_ptr() for t in order])
        p = self.p
        self.T = tl.ref_topo_create(intopo.encode(), self.nx, self.ny, self.nz, c_float(p["dt"]),
                                    c_float(p["dh"]), arr)
        self._keep = (order, arr)

    def metric_ptrs(self):
        out = (c_void_p * 6)()
        ld = c_int(0)
        self.tl.ref_topo_metric_ptrs(self.T, out, byref(ld))
        return list(out), ld.value

    def velocity(self):
        self.tl.ref_topo_velocity(self.T)

    def stress_all(self):
        if self.nve != 3:
            self.tl.ref_topo_stress(self.T)
        for hook in self.after_stress:
            hook(self, self.cur)

    def close(self):
        if getattr(self, "T", None):
            self.tl.ref_topo_destroy(self.T)
            self.T = None
