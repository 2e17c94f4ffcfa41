"""Launch shapes never change results: every tuning gives bit-identical fields."""
import itertools

import numpy as np
import pytest

from awp_b200 import Solver, _lib, default_params, scenarios, tune

pytestmark = pytest.mark.gpu


def run(scn, steps):
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    s.step(steps)
    out = {f: s.field(f) for f in ("u1", "v1", "w1", "xx", "yz", "r1", "r6")}
    s.close()
    return out


@pytest.mark.parametrize("q", [True, False])
def test_tuning_is_bitwise_neutral(q):
    lib = _lib.load()
    saved = tune.get_tuning(lib)
    # odd sizes: partial tiles in j and k, chunk remainders in i
    scn = scenarios.random_small(nx=41, ny=37, nz=68, q=q, steps=6, seed=5)
    base = None
    try:
        for tv, ts, ich in itertools.product((1, 0), (1, 0), (16, 64, 512)):
            tune.set_tuning(lib, "tma_vel", tv)
            tune.set_tuning(lib, "tma_str", ts)
            tune.set_tuning(lib, "ichunk", ich)
            out = run(scn, 6)
            if base is None:
                base = out
                continue
            for f in out:
                assert np.array_equal(out[f].view(np.uint32), base[f].view(np.uint32)), \
                    (f, tv, ts, ich)
    finally:
        for k, v in saved.items():
            tune.set_tuning(lib, k, v)


def test_promotion_change_on_a_live_context_is_bitwise_neutral():
    """A context re-encodes its tensor maps when the L2 promotion changes
    between steps; the fields equal those of a run at one promotion."""
    lib = _lib.load()
    saved = tune.get_tuning(lib)
    scn = scenarios.random_small(nx=41, ny=37, nz=68, q=True, steps=8, seed=7)
    try:
        tune.set_tuning(lib, "tma", 1)
        tune.set_tuning(lib, "ichunk", 16)
        tune.set_tuning(lib, "l2_promotion", 3)
        base = run(scn, 8)
        s = Solver(default_params(**scn.params))
        s.upload_media(scn.media)
        s.upload_sources(scn.src_pos, scn.src_data)
        for pr in (0, 1, 2, 3):
            tune.set_tuning(lib, "l2_promotion", pr)
            assert lib.awp_get_tuning(b"l2_promotion") == pr
            s.step(2)
        out = {f: s.field(f) for f in base}
        s.close()
        for f in base:
            assert np.array_equal(out[f].view(np.uint32), base[f].view(np.uint32)), f
    finally:
        for k, v in saved.items():
            tune.set_tuning(lib, k, v)


def test_bad_tuning_rejected():
    lib = _lib.load()
    assert lib.awp_set_tuning(b"ichunk", 2) != 0
    assert lib.awp_set_tuning(b"tma", 2) != 0
    assert lib.awp_set_tuning(b"nonsense", 8) != 0
    assert lib.awp_get_tuning(b"nonsense") == -1
    assert lib.awp_set_tuning(b"l2_promotion", 4) != 0
