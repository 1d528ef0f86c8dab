"""Failure detection without a GPU fault: the bounded device waits expire into
MSG_ERR_TIMEOUT and leave the context usable; a realization with a NaN
modulus (injected through its xi row) ends in MSG_ERR_BREAKDOWN on its own
while the rest of its batch converges; a context's memory budget turns an
allocation beyond it into MSG_ERR_OUT_OF_MEMORY."""
import numpy as np
import pytest

import msolve_b200 as M
from msolve_b200 import _native as N

pytestmark = pytest.mark.gpu


def small_batch(ctx, n, R, mode="mixed", xi=None, max_iterations=2000):
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    if xi is None:
        xi = np.random.default_rng(4).standard_normal((R, 12))
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=12, simulations=R, mode=mode,
                                                    tolerance=1e-10, max_iterations=max_iterations)
    mc.RandomNumbers = xi
    return mc


def test_bounded_wait_expires_and_context_survives(ctx):
    assert N.lib().MSG_WAIT_SELFTEST(ctx.handle, 1 << 14) == N.MSG_ERR_TIMEOUT
    assert b"expired" in N.lib().MSG_LAST_ERROR(ctx.handle)
    assert N.lib().MSG_WAIT_SELFTEST(ctx.handle, 0) == N.MSG_ERR_INVALID_ARGUMENT
    mc = small_batch(ctx, 6, 8)  # the context still solves
    mc.Solve()
    assert (mc.Residuals < 1e-10).all()


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_nan_realization_breaks_down_alone(ctx, mode):
    R, bad = 8, 3
    xi = np.random.default_rng(6).standard_normal((R, 12))
    xi[bad, 2] = np.nan
    mc = small_batch(ctx, 6, R, mode=mode, xi=xi)
    with pytest.raises(M.InvalidOperationError) as e:
        mc.Solve()
    assert e.value.code == N.MSG_ERR_BREAKDOWN
    good = np.arange(R) != bad
    assert (mc.Residuals[good] < 1e-10).all()
    assert np.isfinite(mc.Solutions[good]).all()
    ref = small_batch(ctx, 6, R - 1, mode=mode, xi=xi[good])
    ref.Solve()
    assert np.abs(mc.Solutions[good] - ref.Solutions).max() <= 1e-8 * np.abs(ref.Solutions).max()


def test_memory_budget_is_enforced():
    small = M.Context(0, mem_budget_bytes=1 << 20)
    with pytest.raises(M.MSolveError) as e:
        mc = small_batch(small, 8, 64)
        mc.Solve()
    assert e.value.code == N.MSG_ERR_OUT_OF_MEMORY
    assert b"budget" in N.lib().MSG_LAST_ERROR(small.handle)
