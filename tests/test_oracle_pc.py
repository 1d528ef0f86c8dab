"""Oracle polynomial-chaos restatement (PolynomialChaosCoefficientsCalculator,
Gaussian branch of MultiplyWithMatrix), pinned independently: the basis is
every multi-index of total degree <= p exactly once, in increasing degree, with
norms prod alpha!; the Galerkin weights equal <psi_j psi_k> and
<xi_v psi_j psi_k> computed by Gauss-Hermite quadrature of probabilists'
Hermite products."""
import itertools
import math

import numpy as np
from numpy.polynomial import hermite_e as He

import oracle as O


def test_basis_is_every_multi_index_once_by_degree():
    for m, p in ((2, 3), (3, 2), (4, 3)):
        b, n = O.pc_basis(m, p)
        expect = {a for a in itertools.product(range(p + 1), repeat=m) if sum(a) <= p}
        got = [tuple(r) for r in b]
        assert len(got) == len(expect) == len(set(got)) and set(got) == expect
        deg = [sum(r) for r in got]
        assert deg == sorted(deg)
        assert all(n[i] == np.prod([math.factorial(a) for a in got[i]]) for i in range(len(got)))


def _galerkin_blocks(m, p):
    """G_pos [P][P] of the oracle product: scalar 'matrices' K_pos = delta(pos)."""
    P = O.pc_basis(m, p)[0].shape[0]

    class One:
        n = 1
        rp = np.array([0, 1], dtype=np.int64)
        ci = np.array([0], dtype=np.int32)

    G = np.zeros((m + 1, P, P))
    for pos in range(m + 1):
        vals = np.zeros((m + 1, 1))
        vals[pos, 0] = 1.0
        for k in range(P):
            u = np.zeros((P, 1))
            u[k, 0] = 1.0
            G[pos, :, k] = O.pc_gaussian_matvec(One, vals, m, p, u)[:, 0]
    return G


def test_galerkin_weights_are_hermite_expectations():
    m, p = 2, 3
    basis, _ = O.pc_basis(m, p)
    P = basis.shape[0]
    G = _galerkin_blocks(m, p)
    x, w = He.hermegauss(12)
    w = w / w.sum()  # standard normal weights

    def psi(a, xs):  # product of He_{a_l}(xi_l)
        out = 1.0
        for l, al in enumerate(a):
            c = np.zeros(al + 1)
            c[al] = 1.0
            out = out * He.hermeval(xs[l], c)
        return out

    grid = np.meshgrid(*([x] * m), indexing="ij")
    W = np.prod(np.meshgrid(*([w] * m), indexing="ij"), axis=0)
    for j in range(P):
        for k in range(P):
            pj, pk = psi(basis[j], grid), psi(basis[k], grid)
            assert abs(G[0, j, k] - np.sum(W * pj * pk)) <= 1e-9 * max(1.0, abs(G[0, j, k]))
            for v in range(m):
                e = np.sum(W * grid[v] * pj * pk)
                assert abs(G[v + 1, j, k] - e) <= 1e-9 * max(1.0, abs(e)), (v, j, k, G[v + 1, j, k], e)
