"""Oracle re-orthogonalised PCG (SolverPCG + SearchVectors): with an empty
store it is the plain Jacobi-PCG in exact arithmetic (same iteration count,
same solution); a load already in the span of the stored directions is solved
from the starting vector with almost no iterations; a full store is reported."""
import numpy as np

import msolve_b200 as M
import oracle as O


def _csr(model, E):
    csr = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
    Ke, _ = O.h8_stiffness_batch(model.xyz[model.conn].reshape(-1, 24), E, model.poisson)
    csr.assemble(Ke)
    return csr


def test_empty_store_is_plain_pcg_and_recycling_pays():
    model = M.cantilever_model()
    csr = _csr(model, np.ones(model.n_elems))
    b = model.subdomains[0].RHS
    store = O.SearchVectorStore(model.n_dofs, 400)
    x, info = O.pcg_reorth(csr, store, b, tol=1e-10)
    xj, ij = csr.pcg_jacobi(b, tol=1e-10)
    assert info["status"] == 0 and abs(info["iterations"] - ij["iterations"]) <= 1
    assert np.abs(x - xj).max() <= 1e-10 * np.abs(xj).max()
    assert store.count == info["iterations"] + 1
    # the same load scaled: the starting vector (all pairs but the last) nearly solves it
    x2, info2 = O.pcg_reorth(csr, store, 2.0 * b, start=1, tol=1e-10)
    assert info2["status"] == 0 and info2["iterations"] <= 3
    assert np.abs(x2 - 2.0 * xj).max() <= 1e-9 * np.abs(xj).max()


def test_full_store_is_reported():
    model = M.cantilever_model()
    csr = _csr(model, np.ones(model.n_elems))
    store = O.SearchVectorStore(model.n_dofs, 5)
    _, info = O.pcg_reorth(csr, store, model.subdomains[0].RHS, tol=1e-10)
    assert info["status"] == -1 and store.count == 5
