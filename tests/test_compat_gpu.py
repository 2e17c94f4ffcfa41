"""The reference-named launchers of libawpb200 (drop-in ABI) against the
reference's own launchers, one call each on identical random device state."""
import ctypes
import os
from ctypes import c_float, c_int, c_void_p

import numpy as np
import pytest

from awp_b200 import _lib
from oracle import refbind

pytestmark = pytest.mark.gpu

F = ctypes.POINTER(c_float)
I = ctypes.POINTER(c_int)


@pytest.fixture(scope="module")
def libs():
    import torch  # noqa: F401
    prod = _lib.load()
    prod.awp_compat_exit_on_error(0)
    ref = ctypes.CDLL(os.path.join(refbind.REF_DIR, "libawpref.so"), mode=ctypes.RTLD_LOCAL)
    for lib in (prod, ref):
        lib.SetDeviceConstValue.argtypes = [F, c_float, I, I, I, c_int, c_float, c_float, F, F]
        lib.dvelcx_H_opt.argtypes = [c_void_p] * 13 + [c_int, c_int, c_void_p] + [c_int] * 4
        lib.dstrqc_H.argtypes = [c_void_p] * 23 + [c_int, c_int, c_void_p] + [c_void_p] * 5 + [c_int] * 9
        lib.fstr_H.argtypes = [c_void_p] * 4 + [c_int] * 4
        lib.addsrc_H.argtypes = [c_int, c_int, c_int, c_void_p, c_int, c_void_p] + [c_void_p] * 12 + [c_int]
    return prod, ref


def setconst(lib, nx, ny, nz, dh, dt):
    DH = np.array([dh], np.float32)
    n = [np.array([v], np.int32) for v in (nx, ny, nz)]
    z9 = np.zeros(9, np.float32)
    lib.SetDeviceConstValue(DH.ctypes.data_as(F), dt, *[a.ctypes.data_as(I) for a in n], 1,
                            0.0, 0.0, z9.ctypes.data_as(F), z9.ctypes.data_as(F))


def state(nx, ny, nz, seed, positive=()):
    import torch
    rng = np.random.default_rng(seed)
    shp = refbind.padded_shape(nx, ny, nz)
    out = {}
    for name in ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4",
                 "r5", "r6", "d1", "mu", "lam", "qp", "qs"]:
        a = rng.standard_normal(shp).astype(np.float32)
        if name in ("d1",):
            a = rng.uniform(2000, 3000, shp).astype(np.float32)
        if name in ("mu", "lam"):
            a = rng.uniform(1e-11, 5e-11, shp).astype(np.float32)
        if name in ("qp", "qs"):
            a = rng.uniform(0.0, 0.02, shp).astype(np.float32)
        out[name] = torch.as_tensor(a).cuda()
    return out


def clone(st):
    return {k: v.clone() for k, v in st.items()}


def P(t):
    return c_void_p(t.data_ptr())


@pytest.mark.parametrize("dims", [(24, 20, 32), (23, 19, 28)])
def test_dvelcx_H_opt(libs, dims):
    import torch
    prod, ref = libs
    nx, ny, nz = dims
    a = state(nx, ny, nz, 1)
    b = clone(a)
    dcx = torch.rand(nx + 20, device="cuda") * 0.2 + 0.8
    dcy = torch.rand(ny + 20, device="cuda") * 0.2 + 0.8
    dcz = torch.rand(nz + 64, device="cuda") * 0.2 + 0.8
    for lib, s in ((ref, a), (prod, b)):
        setconst(lib, nx, ny, nz, 100.0, 0.004)
        lib.dvelcx_H_opt(P(s["u1"]), P(s["v1"]), P(s["w1"]), P(s["xx"]), P(s["yy"]), P(s["zz"]),
                         P(s["xy"]), P(s["xz"]), P(s["yz"]), P(dcx), P(dcy), P(dcz), P(s["d1"]),
                         ny, nz, None, 10, nx + 9, 0, 1)
        torch.cuda.synchronize()
    assert prod.awp_compat_last_error() == 0
    for f in ("u1", "v1", "w1"):
        assert torch.equal(a[f], b[f]) or torch.allclose(a[f], b[f], rtol=1e-6, atol=1e-6), f


@pytest.mark.parametrize("dims", [(24, 20, 32), (23, 19, 28)])
def test_dstrqc_H(libs, dims):
    import torch
    prod, ref = libs
    nx, ny, nz = dims
    a = state(nx, ny, nz, 2)
    b = clone(a)
    rng = np.random.default_rng(3)
    tau1, tau2 = refbind.tau12(np.linspace(0.01, 1.0, 8), 0.004)
    w8 = np.linspace(0.1, 1.7, 8).astype(np.float32)
    host = refbind.RefHost()
    vx1, vx2, ww, wwo = host.init_texture(nx, ny, nz, tau1, tau2, w8, 10, nx + 9, 10, ny + 9)
    tex = [torch.as_tensor(x).cuda() for x in (vx1, vx2, ww, wwo)]
    coeff = torch.as_tensor(rng.standard_normal(16).astype(np.float32) * 20).cuda()
    lam_mu = torch.as_tensor(rng.uniform(0.2, 0.4, (nx + 20, ny + 20)).astype(np.float32)).cuda()
    dcx = torch.rand(nx + 20, device="cuda") * 0.2 + 0.8
    dcy = torch.rand(ny + 20, device="cuda") * 0.2 + 0.8
    dcz = torch.rand(nz + 64, device="cuda") * 0.2 + 0.8
    for lib, s in ((ref, a), (prod, b)):
        setconst(lib, nx, ny, nz, 100.0, 0.004)
        lib.dstrqc_H(P(s["xx"]), P(s["yy"]), P(s["zz"]), P(s["xy"]), P(s["xz"]), P(s["yz"]),
                     P(s["r1"]), P(s["r2"]), P(s["r3"]), P(s["r4"]), P(s["r5"]), P(s["r6"]),
                     P(s["u1"]), P(s["v1"]), P(s["w1"]), P(s["lam"]), P(s["mu"]), P(s["qp"]),
                     P(coeff), P(s["qs"]), P(dcx), P(dcy), P(dcz), ny, nz, None, P(lam_mu),
                     P(tex[0]), P(tex[1]), P(tex[2]), P(tex[3]), nx, 0, 0, 0, 10, nx + 9, 10,
                     ny + 9, 0)
        torch.cuda.synchronize()
    assert prod.awp_compat_last_error() == 0
    for f in ("xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5", "r6", "u1", "v1",
              "w1"):
        d = (a[f] - b[f]).abs().max().item()
        scale = a[f].abs().max().item()
        assert d <= 1e-5 * scale, (f, d, scale)


def test_fstr_and_addsrc_H(libs):
    import torch
    prod, ref = libs
    nx, ny, nz = 23, 19, 28
    a = state(nx, ny, nz, 4)
    b = clone(a)
    nsrc, rs = 5, 7
    psrc = torch.as_tensor(np.array([[3, 4, 5], [10, 11, 1], [20, 2, 27], [5, 5, 5], [1, 1, 1]],
                                    np.int32)).cuda()
    comps = [torch.randn(nsrc * rs, device="cuda") * 1e10 for _ in range(6)]
    for lib, s in ((ref, a), (prod, b)):
        setconst(lib, nx, ny, nz, 100.0, 0.004)
        lib.fstr_H(P(s["zz"]), P(s["xz"]), P(s["yz"]), None, 10, nx + 9, 10, ny + 9)
        lib.addsrc_H(3, rs, 3, P(psrc), nsrc, None, *[P(c) for c in comps], P(s["xx"]),
                     P(s["yy"]), P(s["zz"]), P(s["xy"]), P(s["yz"]), P(s["xz"]), 0)
        torch.cuda.synchronize()
    for f in ("xx", "yy", "zz", "xy", "xz", "yz"):
        assert torch.equal(a[f], b[f]), f


def _argtypes(lib):
    V = c_void_p
    lib.frcvel_H.argtypes = [c_int, c_int, c_int, V, c_int, c_int, V] + [V] * 9 + [c_int] * 3
    lib.addplanesrc_H.argtypes = [c_int, c_int, c_int, V, V, V, c_int, c_int, c_int] + [V] * 9 + \
        [c_int]
    lib.fvel_H.argtypes = [V] * 5 + [c_int] * 7
    lib.velbuffer_H.argtypes = [V] * 8 + [c_int] * 13 + [V, c_int, V, c_int]


def test_frcvel_H(libs):
    """Prescribed velocities (IFAULT 4): interpolated steps, the last
    prescribed step (restoring force stored in the source arrays) and the
    static force after it, with and without the x window."""
    import torch
    prod, ref = libs
    nx, ny, nz = 23, 19, 28
    a = state(nx, ny, nz, 5)
    b = clone(a)
    npsrc, rs, tskp = 6, 4, 3
    psrc = torch.as_tensor(np.array([[3, 4, 5], [10, 11, 1], [20, 2, 27], [5, 5, 5], [1, 1, 1],
                                     [22, 18, 3]], np.int32)).cuda()
    srcs = {}
    for lib, s in ((ref, a), (prod, b)):
        _argtypes(lib)
        setconst(lib, nx, ny, nz, 100.0, 0.004)
        g = torch.Generator(device="cpu").manual_seed(11)
        comps = [(torch.randn((rs + 1) * npsrc, generator=g) * 0.1).cuda() for _ in range(6)]
        for window in ((-1, -1), (12, 28)):
            for i in range(1, rs * tskp + 4):
                lib.frcvel_H(i, rs, 3, P(psrc), npsrc, tskp, None, *[P(c) for c in comps],
                             P(s["u1"]), P(s["v1"]), P(s["w1"]), window[0], window[1], 0)
        torch.cuda.synchronize()
        srcs[id(lib)] = comps
    assert prod.awp_compat_last_error() == 0
    for f in ("u1", "v1", "w1"):
        assert torch.allclose(a[f], b[f], rtol=1e-6, atol=1e-7), f
    for ca, cb in zip(srcs[id(ref)], srcs[id(prod)]):
        assert torch.allclose(ca, cb, rtol=1e-6, atol=1e-6)


def test_addplanesrc_H(libs):
    import torch
    prod, ref = libs
    for nx, ny in ((23, 19), (24, 20)):
        nz = 32
        a = state(nx, ny, nz, 6)
        b = clone(a)
        n_src = 7
        comps = [torch.randn(n_src, device="cuda") * 1e3 for _ in range(3)]
        for lib, s in ((ref, a), (prod, b)):
            _argtypes(lib)
            setconst(lib, nx, ny, nz, 100.0, 0.004)
            for step in (0, 3, 6):
                lib.addplanesrc_H(step, 3, n_src, None, P(s["mu"]), P(s["lam"]), 5, nx, ny,
                                  *[P(c) for c in comps], P(s["xx"]), P(s["yy"]), P(s["zz"]),
                                  P(s["xy"]), P(s["yz"]), P(s["xz"]), 0)
            torch.cuda.synchronize()
        assert prod.awp_compat_last_error() == 0
        for f in ("xx", "yy", "zz", "xy", "xz", "yz"):
            assert torch.equal(a[f], b[f]), (f, (a[f] - b[f]).abs().max().item())


def test_fvel_H(libs):
    import torch
    prod, ref = libs
    rng = np.random.default_rng(9)
    for nx, ny in ((23, 19), (24, 20)):
        nz = 28
        a = state(nx, ny, nz, 7)
        b = clone(a)
        lam_mu = torch.as_tensor(rng.uniform(0.2, 0.4, (nx + 20, ny + 20)).astype(np.float32))
        lam_mu = lam_mu.cuda()
        for lib, s in ((ref, a), (prod, b)):
            _argtypes(lib)
            setconst(lib, nx, ny, nz, 100.0, 0.004)
            lib.fvel_H(P(s["u1"]), P(s["v1"]), P(s["w1"]), None, P(lam_mu), nx, 0, 0, 10, nx + 9,
                       10, ny + 9)
            torch.cuda.synchronize()
        assert prod.awp_compat_last_error() == 0
        for f in ("u1", "v1", "w1"):
            assert torch.equal(a[f], b[f]), (f, (a[f] - b[f]).abs().max().item())


@pytest.mark.parametrize("nve,bathy", [(1, False), (3, False), (1, True)])
def test_velbuffer_H(libs, nve, bathy):
    import torch
    prod, ref = libs
    nx, ny, nz = 23, 19, 28
    s = state(nx, ny, nz, 8)
    s["neta"] = torch.randn_like(s["u1"])
    nb = (2, nx - 1, 3, 1, ny - 2, 2, 0, 4, 2)
    rec = [(nb[3 * q + 1] - nb[3 * q]) // nb[3 * q + 2] + 1 for q in range(3)]
    ktop = nz + 31
    bt = np.full((ny + 20, nx + 20), ktop, np.int32)
    bt[::3, ::2] = ktop - 2
    bt_d = torch.as_tensor(bt).cuda()
    out = {}
    for lib in (ref, prod):
        _argtypes(lib)
        setconst(lib, nx, ny, nz, 100.0, 0.004)
        bufs = [torch.full((int(np.prod(rec)),), -7.0, device="cuda") for _ in range(4)]
        lib.velbuffer_H(P(s["u1"]), P(s["v1"]), P(s["w1"]), P(s["neta"]), *[P(t) for t in bufs],
                        nve, *nb, *rec, None, 1 if bathy else 0,
                        P(bt_d) if bathy else None, 0)
        torch.cuda.synchronize()
        out[id(lib)] = bufs
    assert prod.awp_compat_last_error() == 0
    for x, y in zip(out[id(ref)], out[id(prod)]):
        assert torch.equal(x, y)


def test_single_rank_exchanges_and_printing(libs):
    """At world size 1 the halo exchanges return at once (both neighbour ranks
    -1); a real neighbour is refused with the launchers' error behaviour.  The
    debug printers print nothing, as in the reference."""
    prod, _ = libs
    V = c_void_p
    prod.update_bound_y_H.argtypes = [V] * 9 + [c_int, c_int, V, V, c_int, c_int, c_int]
    prod.update_yldfac_data_x_H.argtypes = [V] * 3 + [c_int, c_int, V, V, c_int, c_int, c_int]
    prod.update_swapzone_buffer_y_H.argtypes = [V] * 11 + [c_int, V, V] + [c_int] * 5
    prod.print_const_H.argtypes = [c_int]
    prod.awp_compat_last_error()
    prod.update_bound_y_H(*([None] * 9), 10, 10, None, None, -1, -1, 0)
    prod.update_yldfac_data_x_H(None, None, None, 10, 10, None, None, -1, -1, 0)
    prod.update_swapzone_buffer_y_H(*([None] * 11), 10, None, None, -1, -1, 34, 39, 0)
    prod.print_const_H(2)
    assert prod.awp_compat_last_error() == 0
    prod.update_bound_y_H(*([None] * 9), 10, 10, None, None, 1, -1, 0)
    assert prod.awp_compat_last_error() != 0
