"""The autotuner's search logic without a GPU: a stand-in engine whose run
time is a known function of the launch parameters.

* the coordinate search finds the optimum of a separable cost and leaves
  the engine at it;
* a move must beat the best so far by more than 2 % (run-to-run spread);
* the start point is DEFAULT projected onto the searched values;
* load/save round-trip the cache file under the cache key."""
from ompmc_b200 import autotune as T


class FakeEngine:
    """run_beam takes `cost(cfg)` seconds per 10^6 histories."""

    def __init__(self, cost):
        self.cost = cost
        self.cfg = {}
        self.runs = 0

    def event_params(self, **kw):
        self.cfg.update(kw)

    def run_beam(self, nhist, nbatch, seed=0, mode=0, **kw):
        self.runs += 1
        return None, None, {"seconds": self.cost(self.cfg) * nhist / 1e6}


def test_finds_optimum_of_separable_cost():
    best = {"electron_tsteps": 2, "tail_boost": 8, "electron_chsteps": 2}
    space = {"electron_tsteps": [1, 2, 4], "tail_boost": [1, 8, 32], "electron_chsteps": [1, 2, 4, 8]}

    def cost(c):
        return 1.0 + sum(0.2 * abs(space[k].index(c[k]) - space[k].index(v)) for k, v in best.items())

    eng = FakeEngine(cost)
    cfg, rate, trials = T.tune_beam(eng, nhist=1_000_000, space=space, repeats=1)
    assert {k: cfg[k] for k in best} == best
    assert {k: eng.cfg[k] for k in best} == best            # the engine is left at the best
    assert abs(rate - 1e6 / 1.0) < 1e-6
    assert len(trials) == len({tuple(sorted(c.items())) for c, _ in trials})


def test_small_gains_do_not_move_and_start_is_projected():
    space = {"electron_tsteps": [1, 2], "tail_boost": [4, 8]}   # DEFAULT tail_boost 32 is not searched

    def cost(c):
        return 1.0 - (0.01 if c["electron_tsteps"] == 2 else 0.0)   # 1 % better: below the 2 % bar

    eng = FakeEngine(cost)
    cfg, _, _ = T.tune_beam(eng, nhist=1_000_000, space=space, repeats=1)
    assert cfg["electron_tsteps"] == T.DEFAULT["electron_tsteps"]
    assert cfg["tail_boost"] == 4                               # projected onto the first searched value
    for k in ("inflight", "block", "electron_split", "electron_chsteps", "drain_particles"):
        assert cfg[k] == T.DEFAULT[k]


def test_cache_roundtrip(tmp_path):
    import numpy as np
    key = T.cache_key("B200", np.zeros((64, 64, 64)), ["H2O521ICRU", "LUNG521ICRU"], "6mv 5x5")
    assert key == "B200|64x64x64|H2O521ICRU,LUNG521ICRU|6mv 5x5"
    path = tmp_path / "tuned.json"
    assert T.load(path, key) is None
    T.save(path, key, {"electron_tsteps": 1, "tail_boost": 8}, 4.4e7)
    got = T.load(path, key)
    assert got == {"electron_tsteps": 1, "tail_boost": 8, "hist_per_s": 4.4e7}
