"""GPU parity of the stochastic Galerkin product (MSG_PC_BASIS,
MSG_PC_GALERKIN_MATVEC) against the oracle's restatement of
PolynomialChaosSolverPCGMatrixCalculator.MultiplyWithMatrix over assembled FP64
matrices K_0 (mean modulus) and K_i (modulus mean * i-th KL term).
Tolerance 1e-12 relative (max norm): the same FP64 products summed in another
order (element by element on the device, CSR rows in the oracle)."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def test_basis_matches_oracle():
    for m, p in ((1, 3), (2, 2), (3, 3), (4, 2)):
        b, n = M.pc_basis(m, p)
        bo, no = O.pc_basis(m, p)
        assert np.array_equal(b, bo) and np.array_equal(n, no)


@pytest.mark.parametrize("n,m,p", [(4, 2, 2), (6, 3, 2), (5, 2, 3)])
def test_galerkin_product_matches_oracle(ctx, n, m, p):
    model = M.clamped_block_model(n)
    kl = M.GaussianStochasticCoefficientsProvider([n, n, n], 0.3 * n, max(m, 4), 8, mean=2.0, covariance=0.15)
    mesh = M.GpuMesh(ctx, model)
    op = M.PolynomialChaosSolverPCGMatrixCalculator(mesh, kl, m, p)
    P = op.PsiSize
    u = np.random.default_rng(n + m + p).standard_normal((P, model.n_dofs))
    y = op.MultiplyWithMatrix(u)
    # the oracle's matrices: E_0 = mean, E_{i+1} = mean * term_i (Gaussian field of a unit germ minus the mean)
    cen = O.centroids(model.xyz, model.conn)
    K = kl.n_terms
    fields = [np.full(model.n_elems, kl.mean)]
    for i in range(m):
        unit = np.zeros((1, K))
        unit[0, i] = 1.0
        fields.append(O.kl_field_gaussian(cen, [n, n, n], kl.table(), unit, kl.mean, kl.covariance)[0] - kl.mean)
    csr = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
    X = model.xyz[model.conn].reshape(-1, 24)
    vals = []
    for E in fields:
        Ke, st = O.h8_stiffness_batch(X, E, model.poisson)
        assert st == 0
        csr.assemble(Ke)
        vals.append(csr.val.copy())
    yo = O.pc_gaussian_matvec(csr, np.array(vals), m, p, u)
    assert np.abs(y - yo).max() <= 1e-12 * np.abs(yo).max()


def test_galerkin_product_needs_gaussian_field(ctx):
    model = M.clamped_block_model(3)
    kl = M.LognormalStochasticCoefficientsProvider([3, 3, 3], 0.9, 4, 4)
    mesh = M.GpuMesh(ctx, model)
    with pytest.raises(TypeError):
        M.PolynomialChaosSolverPCGMatrixCalculator(mesh, kl, 2, 2)
