"""The autotuner on a real batch: it returns one of its candidates, leaves
the context's options as they were, and the tuned configuration solves the
batch to the same tolerance."""
import numpy as np
import pytest

import msolve_b200 as M
from msolve_b200.tuning import TUNABLE, static_candidates

pytestmark = pytest.mark.gpu


def test_tune_mc_small_batch(ctx, tmp_path):
    n, R = 8, 64
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(3).standard_normal((R, 12))
    mesh = M.GpuMesh(ctx, model)
    before = {k: ctx.get_option(k) for k in TUNABLE}
    tuner = M.Autotuner(ctx, str(tmp_path / "tune.json"))
    opts = tuner.tune_mc(mesh, kl, xi, tol=1e-10)
    assert opts in static_candidates()
    assert {k: ctx.get_option(k) for k in TUNABLE} == before
    rec = tuner.cache[tuner.last_key]
    assert len(rec["candidates"]) == 4 and all(c["seconds"] > 0 for c in rec["candidates"])
    tuner.apply(opts)
    try:
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=12, simulations=R,
                                                        tolerance=1e-10)
        mc.RandomNumbers = xi
        mc.Solve()
        assert (mc.Residuals < 1e-10).all()
    finally:
        for k, v in before.items():
            ctx.set_option(k, v)


def test_analyzer_autotune(ctx):
    n, R = 8, 40
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(8).standard_normal((R, 12))
    before = {k: ctx.get_option(k) for k in TUNABLE}
    ref = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=12, simulations=R,
                                                     tolerance=1e-10)
    ref.RandomNumbers = xi
    ref.Solve()
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=12, simulations=R,
                                                    tolerance=1e-10, autotune=True)
    mc.RandomNumbers = xi
    mc.Solve()
    assert mc.TunedOptions in static_candidates()
    assert {k: ctx.get_option(k) for k in TUNABLE} == before
    assert (mc.Residuals < 1e-10).all()
    assert np.abs(mc.Solutions - ref.Solutions).max() <= 1e-8 * np.abs(ref.Solutions).max()
