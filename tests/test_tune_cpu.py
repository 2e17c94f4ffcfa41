"""Host logic of the launch-shape autotuner, on a fake library and solver.

The fake solver reports per-phase times that depend on the tuning in force,
so the test knows which candidate the tuner must install; no GPU is used."""
from awp_b200 import tune


class FakeLib:
    KEYS = {"tma": 1, "tma_vel": 1, "tma_str": 1, "ichunk": 64, "l2_promotion": 3,
            "spin_limit": 1 << 26}

    def __init__(self):
        self.v = dict(self.KEYS)

    def awp_set_tuning(self, key, value):
        k = key.decode()
        if k not in self.v:
            return 1
        if k == "tma":
            self.v["tma_vel"] = self.v["tma_str"] = value
        self.v[k] = value
        return 0

    def awp_get_tuning(self, key):
        return self.v.get(key.decode(), -1)


class FakeSolver:
    """velocity: the read-only family is fastest at ichunk 32; stress: TMA at
    ichunk 64; the promotion granule 1 shaves the TMA stress time."""

    def __init__(self, lib):
        self.lib = lib
        self.acc = {"velocity": [0.0, 0], "stress": [0.0, 0]}
        self.steps = 0

    def profile_phases(self, on):
        pass

    def phase_times(self):
        out = {k: tuple(v) for k, v in self.acc.items()}
        self.acc = {"velocity": [0.0, 0], "stress": [0.0, 0]}
        return out

    def step(self, n):
        v = self.lib.v
        ich = v["ichunk"]
        vel = (0.80 if v["tma_vel"] else 0.70) + (0.0 if ich == 32 else 0.05)
        st = (1.70 if v["tma_str"] else 1.90) + (0.0 if ich == 64 else 0.06)
        if v["tma_str"] and v["l2_promotion"] == 1:
            st -= 0.02
        for _ in range(n):
            self.acc["velocity"][0] += vel
            self.acc["velocity"][1] += 1
            self.acc["stress"][0] += st
            self.acc["stress"][1] += 1
        self.steps += n


def test_autotune_installs_the_fastest_choice():
    lib = FakeLib()
    s = FakeSolver(lib)
    res = tune.autotune(s, steps=3)
    ch = res["chosen"]
    # velocity 0.70 + 0.05 and stress 1.70 at ichunk 64 (2.45) beat
    # 0.70 + 1.76 at ichunk 32 (2.46)
    assert ch == {"tma_vel": 0, "tma_str": 1, "ichunk": 64, "l2_promotion": 1}
    for k in ("tma_vel", "tma_str", "ichunk", "l2_promotion"):
        assert lib.v[k] == ch[k]
    assert tune.get_tuning(lib) == ch
    # every family x chunk row, then one row per promotion granule
    n = len(tune.CANDIDATES["tma"]) * len(tune.CANDIDATES["ichunk"])
    assert len(res["table"]) == n + len(tune.PROMOTIONS)
    assert sorted(r["l2_promotion"] for r in res["table"][n:]) == sorted(tune.PROMOTIONS)


def test_autotune_keeps_the_promotion_without_a_tma_kernel():
    lib = FakeLib()
    lib.v["l2_promotion"] = 2

    class ReadOnlyWins(FakeSolver):
        def step(self, n):
            v = self.lib.v
            vel = 0.9 if v["tma_vel"] else 0.7
            st = 2.0 if v["tma_str"] else 1.8
            for _ in range(n):
                self.acc["velocity"][0] += vel
                self.acc["velocity"][1] += 1
                self.acc["stress"][0] += st
                self.acc["stress"][1] += 1

    res = tune.autotune(ReadOnlyWins(lib), steps=2)
    assert res["chosen"]["tma_vel"] == 0 and res["chosen"]["tma_str"] == 0
    assert res["chosen"]["l2_promotion"] == 2
    assert len(res["table"]) == len(tune.CANDIDATES["tma"]) * len(tune.CANDIDATES["ichunk"])
