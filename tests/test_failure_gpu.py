"""Failure detection of the TMA pipeline waits, without a GPU fault.

Every mbarrier wait of the TMA-pipelined kernels polls a bounded number of
times.  With the poll limit set to 0 every wait gives up at once: the CTA must
drain the copies it already issued, leave its march, set the context's error
word, and the next awp_synchronize must report AWP_ERR_CUDA (once).  With the
limit back at its default the same context and a fresh one run on, and a
fresh run matches a run that never saw the failure bit for bit."""
import numpy as np
import pytest

from awp_b200 import AwpError, Solver, _lib, default_params, scenarios, tune

pytestmark = pytest.mark.gpu

FIELDS = ("u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1")


def make(scn):
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    return s


def test_pipeline_wait_limit_reports_and_recovers():
    lib = _lib.load()
    saved = tune.get_tuning(lib)
    default_limit = lib.awp_get_tuning(b"spin_limit")
    assert default_limit == 1 << 26
    scn = scenarios.random_small(nx=40, ny=24, nz=64, q=True, steps=6, seed=21)
    try:
        tune.set_tuning(lib, "tma", 1)  # both half-steps on the TMA kernels
        ref = make(scn)
        ref.step(6)
        ref.synchronize()
        want = {f: ref.field(f) for f in FIELDS}
        ref.close()

        s = make(scn)
        assert lib.awp_set_tuning(b"spin_limit", 0) == 0
        s.step(2)
        with pytest.raises(AwpError) as e:
            s.synchronize()
        assert e.value.status == 2  # AWP_ERR_CUDA
        assert "iteration limit" in str(e.value)
        assert lib.awp_set_tuning(b"spin_limit", default_limit) == 0
        # reported once; the context keeps working
        s.synchronize()
        s.step(1)
        s.synchronize()
        s.close()

        again = make(scn)
        again.step(6)
        again.synchronize()
        for f in FIELDS:
            assert np.array_equal(again.field(f).view(np.uint32), want[f].view(np.uint32)), f
        again.close()
    finally:
        lib.awp_set_tuning(b"spin_limit", default_limit)
        for k, v in saved.items():
            tune.set_tuning(lib, k, v)

