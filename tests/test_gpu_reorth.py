"""GPU parity of the re-orthogonalised PCG with search vectors kept across solves
(MSG_SVS_*, MSG_PCG_SOLVE_REORTH) against the oracle's restatement of SolverPCG
with SolverPCGReorthogonalizationSearchVectorCalculator, on the 10 x 4 x 4
cantilever: a sequence of solves with one matrix and changing loads (the store
grows and later solves start from it), then a changed matrix started from the
store with a fresh store. Same stopping rule: iteration counts within 1 of the
oracle's, store sizes equal, displacements within 1e-10 (max norm) of the
oracle's."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def _csr(model, E):
    csr = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
    Ke, st = O.h8_stiffness_batch(model.xyz[model.conn].reshape(-1, 24), E, model.poisson)
    assert st == 0
    csr.assemble(Ke)
    return csr


def test_reorthogonalized_sequence_matches_oracle(ctx):
    model = M.cantilever_model()
    mesh = M.GpuMesh(ctx, model)
    rng = np.random.default_rng(11)
    b0 = model.subdomains[0].RHS.copy()
    loads = [b0, 1.3 * b0 + 0.01 * rng.standard_normal(model.n_dofs), 1.6 * b0 + 0.01 * rng.standard_normal(model.n_dofs)]
    E1 = np.ones(model.n_elems)
    E2 = np.exp(0.3 * rng.standard_normal(model.n_elems))
    search = M.SolverPCGReorthogonalizationSearchVectorCalculator(mesh, 600)
    store = O.SearchVectorStore(model.n_dofs, 600)
    csr = _csr(model, E1)
    solver = M.SolverPCGReorthogonalized(ctx, model, search, tolerance=1e-10)
    solver.matrix = mesh.assemble(E1, model.poisson)
    its = []
    for k, b in enumerate(loads):
        model.subdomains[0].Forces = b
        start = 0 if k == 0 else 1
        x = solver.Solve(start_from_store=start)
        xo, info = O.pcg_reorth(csr, store, b, start=start, tol=1e-10)
        assert info["status"] == 0
        assert abs(solver.iterations - info["iterations"]) <= 1, (k, solver.iterations, info["iterations"])
        assert search.count == store.count
        assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()
        its.append(solver.iterations)
    assert its[2] < its[0]  # the recycled directions pay off for a load in their span
    # a changed matrix: starting vector from the store, then a fresh store
    solver.matrix = mesh.assemble(E2, model.poisson)
    csr2 = _csr(model, E2)
    model.subdomains[0].Forces = b0
    x = solver.Solve(start_from_store=2)
    xo, info = O.pcg_reorth(csr2, store, b0, start=2, tol=1e-10)
    assert info["status"] == 0 and abs(solver.iterations - info["iterations"]) <= 1
    assert search.count == store.count
    assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()
    model.subdomains[0].Forces = b0
    search.ClearSearchVectors(5)
    assert search.count == 5
    search.ClearSearchVectors(0)
    assert search.count == 0
    search.close()


def test_full_store_is_reported(ctx):
    model = M.cantilever_model()
    mesh = M.GpuMesh(ctx, model)
    search = M.SolverPCGReorthogonalizationSearchVectorCalculator(mesh, 10)
    solver = M.SolverPCGReorthogonalized(ctx, model, search, tolerance=1e-10)
    solver.matrix = mesh.assemble(np.ones(model.n_elems), model.poisson)
    with pytest.raises(M.MSolveError) as e:
        solver.Solve()
    assert e.value.code == -100  # MSG_ERR_OUT_OF_MEMORY
    assert search.count == 10
    search.close()
