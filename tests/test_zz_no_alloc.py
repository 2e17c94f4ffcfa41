"""awp_check_finite_noalloc -- the allocation-free non-finite check.

It exists for callers that own all their device memory and cannot ask the
CUDA allocator for more (a host code running the wavefield in its own
pre-reserved pool, a watchdog thread checking a running simulation between
steps).  Called through the C ABI on a context's fields, it must agree with
the context's own awp_check_finite on two calls in a row, and reject more
fields than its fixed scratch holds.  Collected last (file name) so a failure
here stops a -x run only after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from awp_b200 import Solver, _lib, default_params, scenarios

pytestmark = pytest.mark.gpu

WAVEFIELD = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz"]


def noalloc(lib, solver, names):
    ptrs = (ctypes.c_void_p * len(names))(*[solver.device_ptr(n) for n in names])
    ok = (ctypes.c_int * len(names))()
    n = int(np.prod(solver.shape))
    st = lib.awp_check_finite_noalloc(ptrs, len(names), ctypes.c_longlong(n), ok, None)
    return st, [int(v) for v in ok]


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.awp_check_finite_noalloc.restype = ctypes.c_int
    lib.awp_check_finite_noalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                             ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                                             ctypes.c_void_p]
    return lib


def test_matches_check_finite_on_two_calls(lib):
    scn = scenarios.random_small(nx=24, ny=20, nz=32, steps=3, seed=31)
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.step(3)
    s.synchronize()
    # call 1: finite wavefield
    st, ok = noalloc(lib, s, WAVEFIELD)
    assert st == 0, lib.awp_last_error()
    assert all(ok) and s.check_finite()
    # call 2: one planted NaN in xy -- only that field is flagged
    xy = s.field("xy")
    xy[15, 14, 40] = np.nan
    s.set_field("xy", xy)
    st, ok = noalloc(lib, s, WAVEFIELD)
    assert st == 0
    assert ok == [0 if n == "xy" else 1 for n in WAVEFIELD]
    assert all(ok) == s.check_finite()
    # call 3: repaired -- the flags of call 2 must not linger in the shared scratch
    xy[15, 14, 40] = 0.0
    s.set_field("xy", xy)
    st, ok = noalloc(lib, s, WAVEFIELD)
    assert st == 0 and all(ok) and s.check_finite()
    s.close()


def test_rejects_more_fields_than_scratch(lib):
    scn = scenarios.random_small(nx=8, ny=8, nz=8, steps=1, seed=32)
    s = Solver(default_params(**scn.params))
    st, ok = noalloc(lib, s, ["u1"] * 33)
    assert st == 1  # AWP_ERR_ARG
    assert b"AWP_NOALLOC_MAX_FIELDS" in lib.awp_last_error()
    st, ok = noalloc(lib, s, ["u1"] * 32)
    assert st == 0 and all(ok)
    s.close()
