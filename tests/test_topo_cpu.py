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
