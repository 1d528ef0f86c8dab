"""GPU parity of the batched Newmark path (MSG_NEWMARK_BATCH) against the
oracle's restatement of NewmarkDynamicAnalyzer with a direct (skyline) solve
per step, realization by realization, on the same KL fields. Each GPU step is
solved to an FP64 true relative residual of 1e-11 (started from the Newmark
predictor, or from the last displacement). Step errors
propagate through the velocity and acceleration updates (a0 = 1/(alpha dt^2)
amplifies them), so the bound is 1e-8 of the maximum on the tip history and
1e-7 on the final displacement field."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def predictor(ctx, request):
    """newmark_predictor option: each step starts from the Newmark predictor (1)
    or from the last displacement (0)."""
    ctx.set_option("newmark_predictor", request.param)
    yield request.param
    ctx.set_option("newmark_predictor", 1)


@pytest.mark.parametrize("predictor", [0, 1], indirect=True)
@pytest.mark.parametrize("n,R,steps", [(4, 3, 30), (6, 33, 20)])
def test_newmark_batch_matches_oracle(ctx, n, R, steps, predictor):
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(n).standard_normal((R, 12))
    dt = 0.01
    load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * steps, 0.1, dof=0)
    corner = int(np.argmax(model.xyz.sum(1)))
    nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * steps, load, expansion_order=12,
                                  simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                  tolerance=1e-11, tip_dof=int(model.dof[corner, 0]))
    nm.RandomNumbers = xi
    hist = nm.Solve()
    assert hist.shape == (R, steps) and (nm.Iterations > 0).all()
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field(cen, [n, n, n], kl.table(), xi, mean=kl.mean, sigma=kl.sigma, mean_correction=kl.mean_correction)
    cons = (model.dof < 0).astype(np.uint8)
    for r in sorted({0, R // 2, R - 1}):
        t, u, info = O.block_newmark(n, n, n, cons, E[r], model.poisson, 1.0, 0.01, 0.001, 0.25, 0.5, dt, steps, 0.1,
                                     1.0, 0, model.n_dofs, tip_dof=nm.tip_dof)
        assert info["status"] == 0
        scale = np.abs(t).max()
        assert scale > 0
        assert np.abs(hist[r] - t).max() <= 1e-8 * scale, (r, np.abs(hist[r] - t).max() / scale)
        assert np.abs(nm.Solutions[r] - u).max() <= 1e-7 * np.abs(u).max()


def test_predictor_start_takes_fewer_iterations(ctx):
    """Started from the Newmark predictor, the steps of an 8^3 batch converge in
    fewer iterations than from the last displacement, to the same results
    within the bounds of the oracle comparison (tip history 1e-8, final field
    1e-7 of the maximum: a0 = 1/(alpha dt^2) amplifies the step residuals)."""
    n, R, steps, dt = 8, 40, 30, 0.01
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(3).standard_normal((R, 12))
    corner = int(np.argmax(model.xyz.sum(1)))
    out = {}
    for p in (1, 0):
        ctx.set_option("newmark_predictor", p)
        try:
            load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * steps, 0.1, dof=0)
            nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * steps, load, expansion_order=12,
                                          simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                          tolerance=1e-12, tip_dof=int(model.dof[corner, 0]))
            nm.RandomNumbers = xi
            out[p] = (nm.Solve(), nm.Solutions.copy(), nm.Iterations.copy())
        finally:
            ctx.set_option("newmark_predictor", 1)
    assert out[1][2].sum() < out[0][2].sum()
    for k, bound in ((0, 1e-8), (1, 1e-7)):
        scale = np.abs(out[0][k]).max()
        assert np.abs(out[1][k] - out[0][k]).max() <= bound * scale


def test_newmark_rejects_bad_coefficients(ctx):
    model = M.clamped_block_model(3)
    kl = M.LognormalStochasticCoefficientsProvider([3, 3, 3], 0.6, 4, 3)
    load = M.MassAccelerationSinusoidalLoad(1.0, 0.01, 0.05, 0.1)
    nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.4, 0.01, 0.05, load, expansion_order=4, simulations=2)
    with pytest.raises(M.InvalidOperationError):
        nm.Solve()
