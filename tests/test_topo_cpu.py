"""Topography metrics on the CPU: the product's reader, geom_custom, and the
f / g interpolants and derivatives against the reference's own code
(readers/serial_reader.c, geometry/geometry.c, metrics/metrics.c,
metrics/kernel.c compiled into oracle/_ref/libawpref_host.so), bit for bit."""
import ctypes

import numpy as np
import pytest

from awp_b200 import _lib, scenarios

F = ctypes.POINTER(ctypes.c_float)
NAMES = ["f", "f_1", "f_2", "f_c", "f1_1", "f1_2", "f1_c", "f2_1", "f2_2", "f2_c",
         "g", "g_c", "g3", "g3_c"]


def split(out, nx, ny, nz):
    nf = (nx + 20) * (ny + 84)
    ng = nz + 64
    d = {}
    for q, n in enumerate(NAMES[:10]):
        d[n] = out[q * nf:(q + 1) * nf].reshape(nx + 20, ny + 84)
    for q, n in enumerate(NAMES[10:]):
        d[n] = out[10 * nf + q * ng:10 * nf + (q + 1) * ng]
    return d


def product(path, nx, ny, nz, h):
    out = np.zeros(10 * (nx + 20) * (ny + 84) + 4 * (nz + 64), np.float32)
    err = _lib.load().awp_topo_metrics(path.encode(), nx, ny, nz, h, out.ctypes.data_as(F))
    return err, split(out, nx, ny, nz)


def reference(ref_host, path, nx, ny, nz, h):
    lib = ref_host.lib
    lib.ref_topo_metrics.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, F]
    out = np.zeros(10 * (nx + 20) * (ny + 84) + 4 * (nz + 64), np.float32)
    err = lib.ref_topo_metrics(path.encode(), nx, ny, nz, h, out.ctypes.data_as(F))
    return err, split(out, nx, ny, nz)


@pytest.mark.parametrize("dims", [(24, 20, 32, 50.0), (31, 17, 48, 37.5), (16, 16, 13, 100.0)])
@pytest.mark.parametrize("padding", [8, 11])
def test_metrics_match_reference(ref_host, tmp_path, dims, padding):
    nx, ny, nz, h = dims
    path = str(tmp_path / "topo.bin")
    scenarios.write_topography(path, nx, ny, h, amplitude=300.0, width=6 * h, rough_rms=20.0,
                               seed=nx + padding, padding=padding)
    e1, mine = product(path, nx, ny, nz, h)
    e2, ref = reference(ref_host, path, nx, ny, nz, h)
    assert e1 == e2 == 0
    for n in NAMES:
        assert np.array_equal(mine[n].view(np.uint32), ref[n].view(np.uint32)), n


def test_flat_topography_metrics():
    """With f = 1 the x / y derivatives vanish and the interpolants are 1
    (the premise of the flat-topography = Cartesian check)."""
    import tempfile, os
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "flat.bin")
        scenarios.write_topography(path, 24, 20, 50.0, amplitude=0.0, rough_rms=0.0)
        err, m = product(path, 24, 20, 32, 50.0)
        assert err == 0
        # derivatives of interpolants are valid two cells inside the window
        # the interpolants are computed on (relative -6 .. n + 6)
        core = (slice(10 - 2, 10 + 24 + 2), slice(42 - 2, 42 + 20 + 2))
        for n in ("f", "f_1", "f_2", "f_c"):
            assert np.all(m[n][core] == 1.0), n
        for n in ("f1_1", "f1_2", "f1_c", "f2_1", "f2_2", "f2_c"):
            # the float D4 weights do not sum to exactly 0: a constant's
            # derivative is a few ulp of 1/h, not 0
            assert np.all(np.abs(m[n][core]) < 1e-6 / 50.0 * 10), n


def test_bad_topography_files(tmp_path):
    path = str(tmp_path / "t.bin")
    scenarios.write_topography(path, 24, 20, 50.0, padding=8)
    assert product(path, 25, 20, 32, 50.0)[0] == 902          # wrong nx
    scenarios.write_topography(path, 24, 20, 50.0, padding=4)
    assert product(path, 24, 20, 32, 50.0)[0] == 902          # padding < ngsl
    assert product(str(tmp_path / "none.bin"), 24, 20, 32, 50.0)[0] == 101


def product_coefs_topo(path, intopo, grid_type, nx, ny, nz, h, degree):
    lib = _lib.load()
    n = 4096
    nb = degree + 1
    cnt = ctypes.c_int()
    I = ctypes.POINTER(ctypes.c_int)
    arrs = [np.zeros(n, np.int32) for _ in range(4)]
    ls = [np.zeros(n * nb, np.float32) for _ in range(3)]
    err = lib.awp_point_coefs_topo(path.encode(), intopo.encode(), grid_type, nx, ny, nz, h, n,
                                   ctypes.byref(cnt), *[a.ctypes.data_as(I) for a in arrs],
                                   *[a.ctypes.data_as(F) for a in ls])
    c = cnt.value
    return err, dict(indices=arrs[0][:c], ix=arrs[1][:c], iy=arrs[2][:c], iz=arrs[3][:c],
                     lx=ls[0][:c * nb].reshape(c, nb), ly=ls[1][:c * nb].reshape(c, nb),
                     lz=ls[2][:c * nb].reshape(c, nb))


@pytest.mark.parametrize("degree", [1, 3])
@pytest.mark.parametrize("grid_type", range(9))
def test_curvilinear_point_coefs_match_reference(ref_host, tmp_path, degree, grid_type):
    """Receivers / SOURCEFILE points on the curvilinear block: the vertical
    coordinate through the surface function interpolated at the point
    (metrics_interpolate_f_point, source.c:283-340), then the usual Lagrange
    set-up -- against the reference's own routines, bit for bit."""
    from awp_b200 import pointfiles
    nx, ny, nz, h = 28, 24, 32, 100.0
    intopo = str(tmp_path / "topo.bin")
    depth = h * (nz - 2)
    scenarios.write_topography(intopo, nx, ny, h, amplitude=0.15 * depth, width=5 * h,
                               rough_rms=0.02 * depth, seed=5)
    rng = np.random.default_rng(11 + grid_type)
    n = 14
    coords = np.stack([rng.uniform(2 * h, (nx - 3) * h, n), rng.uniform(2 * h, (ny - 3) * h, n),
                       -rng.uniform(0.0, 0.7 * nz * h, n)], 1)
    types = np.zeros(n, np.int32)
    types[:4] = 1
    path = str(tmp_path / "pts.txt")
    pointfiles.write_input(path, str(tmp_path / "out"), coords, types, degree=degree)
    e1, mine = product_coefs_topo(path, intopo, grid_type, nx, ny, nz, h, degree)
    assert e1 == 0
    _, f = product(intopo, nx, ny, nz, h)
    ref = ref_host.point_coefs(path, grid_type, nx, ny, nz, h, ftopo=f["f"])
    assert len(mine["ix"]) == len(ref["ix"]) == n
    for k in ("indices", "ix", "iy", "iz"):
        assert np.array_equal(mine[k], ref[k]), k
    for k in ("lx", "ly", "lz"):
        assert np.array_equal(mine[k].view(np.uint32), ref[k].view(np.uint32)), k
