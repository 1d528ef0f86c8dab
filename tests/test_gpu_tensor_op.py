"""GPU parity of the tensor-core element product (option "tensor_operator" = 1:
the multigrid loop's level-0 search-direction launch computes E_e Khat u_e
with tcgen05.mma in TF32 with a three-term split, k_lvl_tc). The batched
Monte Carlo solve must still meet the FP64 bound: displacements within 1e-8
(max norm, relative) of FP64 oracle solves converged to 1e-13, with the FP32
rounding of the product close enough to the Walsh-mode kernel's that the
iteration counts stay within two of the default path on the same batch
(Hexa8WithStochasticMaterial.cs:61-110: K_e = E_e Khat for unit cubes)."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def _solve(ctx, model, kl, xi, K, tensor):
    ctx.set_option("tensor_operator", tensor)
    try:
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=xi.shape[0],
                                                        mode="mixed", tolerance=1e-10)
        mc.RandomNumbers = xi
        mc.Solve()
    finally:
        ctx.set_option("tensor_operator", 0)
    return mc


@pytest.mark.parametrize("n,R", [(8, 32), (16, 64), (32, 64)])
def test_tensor_core_product_matches_oracle_and_walsh_path(ctx, n, R):
    K = 20
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 8)
    xi = np.random.default_rng(100 + n).standard_normal((R, K))
    tc = _solve(ctx, model, kl, xi, K, 1)
    ref = _solve(ctx, model, kl, xi, K, 0)
    assert (tc.Residuals < 1e-10).all()
    assert np.abs(tc.Iterations - ref.Iterations).max() <= 2, (tc.Iterations, ref.Iterations)
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field(cen, [n, n, n], kl.table(), xi, sigma=kl.sigma)
    cons = (model.dof < 0).astype(np.uint8)
    for r in sorted({0, R // 2, R - 1}):
        xo, info = O.block_solve_pcg(n, n, n, cons, E[r], model.poisson, model.subdomains[0].RHS, tol=1e-13,
                                     max_it=100000)
        assert info["status"] == 0
        err = np.abs(tc.Solutions[r] - xo).max() / np.abs(xo).max()
        assert err <= 1e-8, (r, err)


def test_tensor_core_product_on_the_cantilever(ctx):
    """Non-cubic lattice (10 x 4 x 4, x = 0 clamped, partial tiles in y and z)."""
    model = M.cantilever_model()
    kl = M.LognormalStochasticCoefficientsProvider([10, 4, 4], 2.0, 10, 6)
    xi = np.random.default_rng(5).standard_normal((32, 10))
    tc = _solve(ctx, model, kl, xi, 10, 1)
    ref = _solve(ctx, model, kl, xi, 10, 0)
    assert (tc.Residuals < 1e-10).all()
    assert np.abs(tc.Solutions - ref.Solutions).max() <= 1e-8 * np.abs(ref.Solutions).max()
