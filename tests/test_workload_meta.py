"""The reference arm's workload config (scenarios.workload_meta) names the same
model and parameters as the scenario the GPU arm generates."""
from awp_b200 import scenarios


def test_workload_meta_matches_scenarios():
    for name, kw in (("halfspace", dict(nx=32, ny=24, nz=16)),
                     ("layered_vk", dict(nx=128, ny=96, nz=64))):
        sc = getattr(scenarios, name)(**kw)
        params, desc = scenarios.workload_meta(name, kw["nx"], kw["ny"], kw["nz"])
        assert desc == sc.description
        for k, v in params.items():
            assert sc.params[k] == v, (name, k)
