"""Point sets (RECVFILE / SOURCEFILE) on the CPU: the product's ASCII v2 reader
and its Lagrange interpolation set-up against the reference's own code
(readers/input.c, grid/grid_3d.c, interpolation/*.c, mpi/distribute.c compiled
into oracle/_ref/libawpref_host.so), bit for bit."""
import ctypes
import os

import numpy as np
import pytest

from awp_b200 import _lib, pointfiles

F = ctypes.POINTER(ctypes.c_float)
I = ctypes.POINTER(ctypes.c_int)


def product_read(path):
    lib = _lib.load()
    hdr = (ctypes.c_longlong * 8)()
    fname = ctypes.create_string_buffer(2048)
    n = 4096
    x = np.zeros(n, np.float32)
    y = np.zeros(n, np.float32)
    z = np.zeros(n, np.float32)
    t = np.zeros(n, np.int32)
    err = lib.awp_input_read(path.encode(), hdr, fname, 2048, x.ctypes.data_as(F),
                             y.ctypes.data_as(F), z.ctypes.data_as(F), t.ctypes.data_as(I), n)
    if err:
        return err, None, None, None, None, None
    keys = ["length", "gpu_buffer_size", "cpu_buffer_size", "steps", "num_writes", "stride",
            "degree", "major"]
    h = {k: int(v) for k, v in zip(keys, hdr)}
    h["file"] = fname.value.decode()
    m = h["length"]
    return 0, h, x[:m], y[:m], z[:m], t[:m]


def product_coefs(path, grid_type, nx, ny, nz, h, degree):
    lib = _lib.load()
    n = 4096
    nb = degree + 1
    cnt = ctypes.c_int()
    arrs = [np.zeros(n, np.int32) for _ in range(4)]
    ls = [np.zeros(n * nb, np.float32) for _ in range(3)]
    err = lib.awp_point_coefs(path.encode(), grid_type, nx, ny, nz, h, n, ctypes.byref(cnt),
                              *[a.ctypes.data_as(I) for a in arrs],
                              *[a.ctypes.data_as(F) for a in ls])
    c = cnt.value
    return err, dict(indices=arrs[0][:c], ix=arrs[1][:c], iy=arrs[2][:c], iz=arrs[3][:c],
                     lx=ls[0][:c * nb].reshape(c, nb), ly=ls[1][:c * nb].reshape(c, nb),
                     lz=ls[2][:c * nb].reshape(c, nb))


HEADER_CASES = {
    "plain": "2.0.0\nfile={out}\nlength=3\nsteps=1e3\nstride=10\ndegree=3\n"
             "gpu_buffer_size=10\ncpu_buffer_size=10\n\ncoordinates\n"
             "0 0.0 0.0 0.0\n0 1.5 0.0 -2.5\n1 0.0 1.5 0.0\n",
    "comments": "2.1.0\n# a comment line\nfile={out}\nlength=2 \n#another\nnum_writes=4\n"
                "steps=600\nstride=1\ndegree=1\ngpu_buffer_size=2\ncpu_buffer_size=3\n"
                "coordinates\n0 10 20 -30\n0 11.25 22.5 -33.75\n",
    "defaults": "2.0.0\nfile={out}\nlength=1\ncoordinates\n0 1 2 3\n",
    "unknown_key": "2.0.0\nfile={out}\nlength=1\nbogus=3\ncoordinates\n0 1 2 3\n",
    "no_equals": "2.0.0\nfile={out}\nlength\ncoordinates\n0 1 2 3\n",
    "not_divisible": "2.0.0\nfile={out}\nlength=1\nsteps=7\ngpu_buffer_size=2\n"
                     "cpu_buffer_size=2\ncoordinates\n0 1 2 3\n",
    "short_body": "2.0.0\nfile={out}\nlength=3\ncoordinates\n0 1 2 3\n0 1 2\n",
}


@pytest.mark.parametrize("case", sorted(HEADER_CASES))
def test_reader_matches_reference(ref_host, tmp_path, case):
    path = str(tmp_path / "in.txt")
    with open(path, "w") as fh:
        fh.write(HEADER_CASES[case].format(out=str(tmp_path / "out")))
    mine = product_read(path)
    ref = ref_host.input_read(path)
    assert mine[0] == ref[0], (mine[0], ref[0])
    if ref[0]:
        return
    assert mine[1] == ref[1]
    for a, b in zip(mine[2:], ref[2:]):
        assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_wrong_major_version(tmp_path):
    """A major version other than 2 is refused with ERR_WRONG_VERSION (201).
    (The reference's reader reaches the same code but then closes the file a
    second time -- _read_header closes it before returning the error and
    _input_read closes it again, readers/input.c:258-260, 293-296 -- which
    aborts the process, so the reference is not run on this case.)"""
    path = str(tmp_path / "in.txt")
    with open(path, "w") as fh:
        fh.write(f"1.0.0\nfile={tmp_path / 'out'}\nlength=1\ncoordinates\n0 1 2 3\n")
    assert product_read(path)[0] == 201


def random_points(rng, n, nx, ny, nz, h, surface_frac=0.3):
    x = rng.uniform(-0.3 * h, (nx - 0.7) * h, n)
    y = rng.uniform(-0.3 * h, (ny - 0.7) * h, n)
    z = -rng.uniform(0.0, (nz - 3) * h, n)
    t = (rng.uniform(0, 1, n) < surface_frac).astype(np.int32)
    # a few points exactly on grid nodes and half nodes (ties in argnearest)
    k = max(1, n // 8)
    x[:k] = np.round(x[:k] / (0.5 * h)) * 0.5 * h
    y[:k] = np.round(y[:k] / (0.5 * h)) * 0.5 * h
    z[:k] = np.round(z[:k] / (0.5 * h)) * 0.5 * h
    t[-1] = 0
    z[-1] = -0.5 * (nz // 2) * h  # the reference checks only the last point's z status
    # points outside the domain are dropped by dist_indices
    x[1] = -5 * h
    return np.stack([x, y, z], 1), t


@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("grid_type", range(10))  # 9: the material node grid
def test_interpolation_matches_reference(ref_host, tmp_path, degree, grid_type):
    nx, ny, nz, h = 24, 20, 32, 50.0
    rng = np.random.default_rng(100 + 10 * degree + grid_type)
    coords, types = random_points(rng, 40, nx, ny, nz, h)
    path = str(tmp_path / "pts.txt")
    pointfiles.write_input(path, str(tmp_path / "pts"), coords, types, degree=degree)
    err, mine = product_coefs(path, grid_type, nx, ny, nz, h, degree)
    assert err == 0, err
    ref = ref_host.point_coefs(path, grid_type, nx, ny, nz, h)
    assert len(mine["indices"]) == len(ref["indices"]) > 0
    assert 1 not in mine["indices"]
    for k in ("indices", "ix", "iy", "iz"):
        assert np.array_equal(mine[k], ref[k]), k
    for k in ("lx", "ly", "lz"):
        assert np.array_equal(mine[k].view(np.uint32), ref[k].view(np.uint32)), k


def test_last_point_out_of_bounds_is_an_error(tmp_path):
    """The reference aborts (AWPCHK) when the last query's vertical weights
    were clamped: a surface point of the x component lies half a cell above
    its top node (source.c:383 via interpolation.cu:60-63)."""
    path = str(tmp_path / "pts.txt")
    pointfiles.write_input(path, str(tmp_path / "pts"), [[100.0, 100.0, 0.0]], [1], degree=3)
    err, _ = product_coefs(path, 0, 24, 20, 32, 50.0, 3)
    assert err == 701
    err, _ = product_coefs(path, 2, 24, 20, 32, 50.0, 3)  # w sits on the surface node
    assert err == 0


def test_lagrange_weights_reproduce_polynomials(tmp_path):
    """Degree-n Lagrange weights are exact for polynomials of degree <= n
    (tests/interpolation/test_lagrange.c:74 of the reference)."""
    nx, ny, nz, h = 24, 20, 32, 10.0
    rng = np.random.default_rng(5)
    coords, types = random_points(rng, 30, nx, ny, nz, h, surface_frac=0.0)
    path = str(tmp_path / "pts.txt")
    for degree in (1, 2, 3):
        pointfiles.write_input(path, str(tmp_path / "pts"), coords, types, degree=degree)
        err, c = product_coefs(path, 0, nx, ny, nz, h, degree)
        assert err == 0
        for lw in (c["lx"], c["ly"], c["lz"]):
            nodes = np.arange(lw.shape[1], dtype=np.float64)
            for p in range(degree + 1):
                vals = (lw.astype(np.float64) * nodes ** p).sum(1)
                q = (lw.astype(np.float64) * nodes).sum(1)
                assert np.allclose(vals, q ** p, rtol=1e-4, atol=1e-4)
