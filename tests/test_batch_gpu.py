"""Batched instances (awp_batch_*): many independent simulations of uneven
sizes advanced by persistent tile-queue launches replayed as a CUDA graph.
The batch leaves each instance's arithmetic unchanged, so every field of
every instance must equal, bit for bit, the same run through awp_step."""
import numpy as np
import pytest

from awp_b200 import AwpError, Batch, Solver, default_params, pointfiles, scenarios

pytestmark = pytest.mark.gpu

FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5",
          "r6"]

# (nx, ny, nz, q, ifault, seed): uneven sizes, anelastic and elastic, point
# and kinematic sources
INSTANCES = [(24, 20, 32, True, 1, 3), (40, 28, 16, True, 5, 4), (16, 16, 32, False, 1, 5),
             (32, 24, 24, True, 1, 6), (20, 36, 20, False, 5, 7)]


def make(spec, steps):
    nx, ny, nz, q, ifault, seed = spec
    scn = scenarios.random_small(nx=nx, ny=ny, nz=nz, q=q, ifault=ifault, steps=steps,
                                 seed=seed, nsrc=2)
    s = Solver(default_params(**scn.params))
    s.upload_media(scn.media)
    s.upload_sources(scn.src_pos, scn.src_data)
    return s


@pytest.mark.parametrize("mode,ty,ichunk,graph,branches",
                         [(0, 8, 16, True, 0), (0, 4, 8, True, 0), (0, 8, 32, False, 0),
                          (1, 8, 16, True, 0), (1, 8, 16, True, 2), (1, 8, 16, True, 1)])
def test_batch_equals_plain_runs(mode, ty, ichunk, graph, branches):
    steps = 12
    plain = [make(sp, steps) for sp in INSTANCES]
    for s in plain:
        s.step(steps)
        s.synchronize()
    want = [{f: s.field(f) for f in FIELDS} for s in plain]
    for s in plain:
        s.close()

    solvers = [make(sp, steps) for sp in INSTANCES]
    b = Batch(solvers)
    b.set_mode(mode)
    b.set_shape(ty, ichunk)
    b.set_graph(graph)
    # mode 1 with fewer branches than instances deals several instances'
    # launches onto one captured branch
    b.set_branches(branches)
    info = b.info()
    assert info["instances"] == len(INSTANCES)
    b.step(5)
    b.step(steps - 5)  # a second replay of the same graph
    b.synchronize()
    for n, s in enumerate(solvers):
        assert s.current_step == steps
        for f in FIELDS:
            got = s.field(f)
            assert np.array_equal(got.view(np.uint32), want[n][f].view(np.uint32)), (n, f)
    b.close()
    for s in solvers:
        s.close()


def test_batch_then_plain_steps_continue():
    """Steps through the batch and then through awp_step on an instance agree
    with a run through awp_step alone."""
    spec = INSTANCES[0]
    ref = make(spec, 8)
    ref.step(8)
    ref.synchronize()
    want = ref.field("xx")
    ref.close()
    s = make(spec, 8)
    b = Batch([s])
    b.step(5)
    b.close()
    s.step(3)
    s.synchronize()
    assert np.array_equal(s.field("xx").view(np.uint32), want.view(np.uint32))
    s.close()


def test_batch_refusals(tmp_path):
    a = make(INSTANCES[0], 4)
    c = make(INSTANCES[2], 4)
    path = str(tmp_path / "recv.txt")
    pointfiles.write_input(path, str(tmp_path / "r"), [[800.0, 800.0, -400.0]], [0], degree=1)
    c.receivers(path, 5)
    with pytest.raises(AwpError) as e:
        Batch([a, c])
    assert e.value.status == 7  # AWP_ERR_UNSUPPORTED
    with pytest.raises(AwpError) as e:
        Batch([a, a])
    assert e.value.status == 1
    b = Batch([a])
    a.step(1)  # stepped outside the batch
    with pytest.raises(AwpError) as e:
        b.step(1)
    assert e.value.status == 3
    b.close()
    a.close()
    c.close()
