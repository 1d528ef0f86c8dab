"""Oracle Gaussian-field Monte Carlo (GaussianFileStochasticCoefficientsProvider
+ MonteCarloAnalyzer): the field restates GetCoefficient term by term, and the
matrix the analyzer composes, K_0 + sum_k xi_k K_k with K_0 built at
coefficient 1 and K_k at the k-th term, equals the stiffness of that field."""
import numpy as np

import oracle as O


def _setup(n=3, K=6, R=3, mean=2.0, cov=0.15):
    xyz, conn = O.block_mesh(n, n, n, 1.0)
    cen = O.centroids(xyz, conn)
    tab = O.kl_table([n, n, n], 0.2 * n, K, 8)
    xi = np.random.default_rng(4).standard_normal((R, K))
    return xyz, conn, cen, tab, xi, mean, cov


def test_field_restates_get_coefficient():
    xyz, conn, cen, tab, xi, mean, cov = _setup()
    E = O.kl_field_gaussian(cen, [3, 3, 3], tab, xi, mean, cov)
    L = np.array([3.0, 3.0, 3.0])
    for r in range(xi.shape[0]):
        for e in (0, 7, 26):
            result = 1.0
            for k in range(xi.shape[1]):
                f = cov * np.sqrt(tab["eig"][k])
                for a in range(3):
                    x = cen[e, a] - L[a] / 2
                    w, amp, idx = tab["w"][k, a], tab["amp"][k, a], tab["idx"][k, a]
                    f *= amp * np.sin(w * x) if idx % 2 == 0 else amp * np.cos(w * x)
                result += xi[r, k] * f
            assert abs(E[r, e] - mean * result) <= 1e-14 * mean


def test_composed_matrix_equals_stiffness_of_the_field():
    xyz, conn, cen, tab, xi, mean, cov = _setup()
    K = xi.shape[1]
    ne = conn.shape[0]
    X = O.element_xyz(xyz, conn)
    nd = 3 * xyz.shape[0]

    def assemble(E):
        Ke, st = O.h8_stiffness_batch(X, E, 0.3)
        assert st == 0
        A = np.zeros((nd, nd))
        full = O.unpack300(Ke)
        for e in range(ne):
            d = (conn[e][:, None] * 3 + np.arange(3)[None, :]).ravel()
            A[np.ix_(d, d)] += full[e]
        return A

    K0 = assemble(np.full(ne, mean))
    Kk = []
    for k in range(K):
        unit = np.zeros((1, K))
        unit[0, k] = 1.0
        coef = O.kl_field_gaussian(cen, [3, 3, 3], tab, unit, mean, cov)[0] - mean  # mean * term k
        Kk.append(assemble(coef))
    E = O.kl_field_gaussian(cen, [3, 3, 3], tab, xi, mean, cov)
    for r in range(xi.shape[0]):
        composed = K0 + sum(xi[r, k] * Kk[k] for k in range(K))
        direct = assemble(E[r])
        assert np.abs(composed - direct).max() <= 1e-12 * np.abs(direct).max()
