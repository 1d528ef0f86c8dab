"""GPU parity of the Gaussian-field Monte Carlo (MSG_KL gaussian = 1,
MonteCarloAnalyzer): the field against the oracle's GetCoefficient restatement
(1e-13 relative), batched mixed-precision and FP64 drop-in solutions against
FP64 oracle solves of the composed matrix K_0 + sum_k xi_k K_k (the stiffness
of that field), 1e-8 relative in the max norm."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def _setup(n, R, seed):
    model = M.clamped_block_model(n)
    kl = M.GaussianStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 8, mean=1.0, covariance=0.15)
    xi = np.random.default_rng(seed).standard_normal((R, 12))
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field_gaussian(cen, [n, n, n], kl.table(), xi, kl.mean, kl.covariance)
    assert E.min() > 0
    return model, kl, xi, E


def test_gaussian_field_matches_oracle(ctx):
    model, kl, xi, E = _setup(8, 40, 1)
    mesh = M.GpuMesh(ctx, model)
    Eg = kl.field(mesh, xi)
    assert np.abs(Eg - E).max() <= 1e-13 * np.abs(E).max()


@pytest.mark.parametrize("mode,n,R", [("mixed", 8, 24), ("mixed", 12, 16), ("fp64", 6, 3)])
def test_gaussian_monte_carlo_matches_oracle(ctx, mode, n, R):
    model, kl, xi, E = _setup(n, R, n)
    tol = 1e-10 if mode == "mixed" else 1e-12
    mc = M.MonteCarloAnalyzer(ctx, model, kl, expansion_order=12, simulations=R, mode=mode, tolerance=tol)
    mc.RandomNumbers = xi
    mc.Solve()
    cons = (model.dof < 0).astype(np.uint8)
    for r in sorted({0, R // 2, R - 1}):
        xo, info = O.block_solve_pcg(n, n, n, cons, E[r], model.poisson, model.subdomains[0].RHS, tol=1e-13,
                                     max_it=100000)
        assert info["status"] == 0
        err = np.abs(mc.Solutions[r] - xo).max() / np.abs(xo).max()
        assert err <= 1e-8, (r, err)


def test_monte_carlo_analyzer_needs_gaussian_provider(ctx):
    model = M.clamped_block_model(4)
    kl = M.LognormalStochasticCoefficientsProvider([4, 4, 4], 0.8, 4, 4)
    with pytest.raises(TypeError):
        M.MonteCarloAnalyzer(ctx, model, kl, expansion_order=4, simulations=2)
