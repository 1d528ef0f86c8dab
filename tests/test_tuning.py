"""Autotuner bookkeeping (no GPU): the fastest candidate is kept, the
context's options are restored after tuning, the choice is cached per key in
a JSON file and reused without timing."""
import json

import pytest

from msolve_b200.tuning import TUNABLE, Autotuner, static_candidates, tuning_key


class FakeCtx:
    def __init__(self):
        self.opts = {"multigrid": 1.0, "multigrid_packed": 1.0, "multigrid_levels": 6.0}
        self.device = 0
        self.history = []

    def get_option(self, k):
        return self.opts[k]

    def set_option(self, k, v):
        self.opts[k] = float(v)
        self.history.append((k, float(v)))


def fake_cost(ctx):
    """Seconds as a function of the options in force when measure() runs."""
    o = ctx.opts
    return 1.0 + (0.0 if o["multigrid_packed"] else 0.2) + (0.0 if o["multigrid"] else 5.0) + \
        (0.0 if o["multigrid_levels"] >= 5 else 0.3)


def test_picks_fastest_and_restores(tmp_path):
    ctx = FakeCtx()
    ctx.opts["multigrid_levels"] = 4.0  # a non-default value to be restored
    t = Autotuner(ctx, str(tmp_path / "tune.json"))
    seen = []
    best = t.tune("k", lambda c: seen.append(dict(ctx.opts)) or fake_cost(ctx), static_candidates())
    assert best == {"multigrid": 1, "multigrid_packed": 1, "multigrid_levels": 6}
    assert len(seen) == 4 and seen[1]["multigrid_packed"] == 0.0  # each candidate measured with its options
    assert ctx.opts == {"multigrid": 1.0, "multigrid_packed": 1.0, "multigrid_levels": 4.0}
    t.apply(best)
    assert ctx.opts["multigrid_levels"] == 6.0


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    ctx = FakeCtx()
    Autotuner(ctx, path).tune("k", lambda c: fake_cost(ctx), static_candidates())
    data = json.load(open(path))
    assert set(data["k"]) == {"options", "seconds", "candidates"} and len(data["k"]["candidates"]) == 4

    def fail(_c):
        raise AssertionError("a cached key is not timed again")
    assert Autotuner(FakeCtx(), path).tune("k", fail, static_candidates())["multigrid_packed"] == 1


def test_options_restored_when_a_candidate_fails():
    ctx = FakeCtx()

    def measure(c):
        if c["multigrid"] == 0:
            raise RuntimeError("candidate failed")
        return fake_cost(ctx)
    with pytest.raises(RuntimeError):
        Autotuner(ctx).tune("k", measure, static_candidates())
    assert ctx.opts == {"multigrid": 1.0, "multigrid_packed": 1.0, "multigrid_levels": 6.0}
    assert set(TUNABLE) == set(ctx.opts)


def test_key_pads_the_batch():
    assert tuning_key("B200", 32, 32, 32, 1000, False) == tuning_key("B200", 32, 32, 32, 1024, False)
    assert tuning_key("B200", 32, 32, 32, 1025, False) != tuning_key("B200", 32, 32, 32, 1024, False)
    assert tuning_key("B200", 24, 24, 24, 256, True).endswith("|mass")
