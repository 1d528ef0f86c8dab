"""GPU parity of the assembled FP64 path: BSR assembly and product against the
oracle's CSR/skyline, and the device Jacobi-PCG against the oracle's
SolverPCG restatement and the skyline LDL^T direct solve."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def oracle_csr(model, E):
    Ke, _ = O.h8_stiffness_batch(model.element_xyz(), E, model.poisson)
    C = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
    C.assemble(Ke)
    return C, Ke


def test_bsr_product_and_diagonal_match_oracle(ctx):
    for model in (M.cantilever_model(), M.clamped_block_model(7)):
        rng = np.random.default_rng(7)
        E = np.exp(0.3 * rng.standard_normal(model.n_elems))
        mesh = M.GpuMesh(ctx, model)
        A = mesh.assemble(E, model.poisson)
        C, _ = oracle_csr(model, E)
        for _ in range(3):
            x = rng.standard_normal(model.n_dofs)
            y, yo = A.Multiply(x), C.multiply(x)
            assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()
        assert np.abs(A.Diagonal() - C.diagonal()).max() <= 1e-14 * np.abs(C.diagonal()).max()


def test_assembly_from_element_matrices_equals_assembly_from_E(ctx):
    model = M.clamped_block_model(4)
    E = np.linspace(0.5, 2.0, model.n_elems)
    mesh = M.GpuMesh(ctx, model)
    Ke = M.h8_stiffness_batch(ctx, model.element_xyz(), E, 0.3)
    A1, A2 = mesh.assemble(E, 0.3), mesh.assemble_from_element_matrices(Ke)
    x = np.random.default_rng(0).standard_normal(model.n_dofs)
    assert np.array_equal(A1.Multiply(x), A2.Multiply(x))


def test_mesh_info(ctx):
    info = M.GpuMesh(ctx, M.clamped_block_model(32)).info()
    assert info["structured"] and info["n_dofs"] == 104544 and (info["nx"], info["ny"], info["nz"]) == (32, 32, 32)
    assert not M.GpuMesh(ctx, M.Model(np.random.default_rng(0).random((8, 3)), np.arange(8)[None])
                         .ConnectDataStructures()).info()["structured"]
    # true 3x3 blocks over all nodes (incl. clamped) of a 33^3 lattice
    n = 33
    expect = sum((3 - (i in (0, n - 1))) * (3 - (j in (0, n - 1))) * (3 - (k in (0, n - 1)))
                 for i in range(n) for j in range(n) for k in range(n))
    assert info["nnzb"] == expect and info["n_block_rows"] == n ** 3


def test_cantilever_static_analyzer_matches_skyline_and_oracle_pcg(ctx):
    """Config 1: 10x4x4 cantilever, E=1, nu=0.3, x=0 clamped, -1 in z over the tip face."""
    model = M.cantilever_model()
    solver = M.SolverPCG(ctx, model, max_iterations=20000, tolerance=1e-10)
    static = M.StaticAnalyzer(M.ProblemStructural(ctx, model), M.LinearAnalyzer(solver))
    static.BuildMatrices()
    static.Initialize()
    static.Solve()
    u = model.subdomains[0].Solution
    C, Ke = oracle_csr(model, model.E_elem)
    S = O.Skyline(model.conn, model.dof, model.n_dofs)
    S.assemble(Ke)
    F, _ = S.factorized()
    us = S.solve(F, model.subdomains[0].RHS)
    up, info = C.pcg_jacobi(model.subdomains[0].RHS, tol=1e-10)
    assert abs(solver.iterations - info["iterations"]) <= 1
    assert np.abs(u - up).max() <= 1e-8 * np.abs(up).max()
    assert np.abs(u - us).max() <= 1e-8 * np.abs(us).max()


def test_pcg_reference_iteration_semantics(ctx):
    model = M.clamped_block_model(6)
    mesh = M.GpuMesh(ctx, model)
    rng = np.random.default_rng(9)
    E = np.exp(0.3 * rng.standard_normal(model.n_elems))
    A = mesh.assemble(E, 0.3)
    solver = M.SolverPCG(ctx, model)
    solver.matrix = A
    x = solver.Solve(20000, 1e-8)
    C, _ = oracle_csr(model, E)
    xo, info = C.pcg_jacobi(model.subdomains[0].RHS, tol=1e-8)
    assert solver.iterations == info["iterations"]
    # same stopping iteration; the last recursive residuals agree to summation-order noise
    assert solver.rel_res < 1e-8 and info["rel_res"] < 1e-8
    assert abs(solver.rel_res - info["rel_res"]) <= 0.25 * info["rel_res"]
    # at a 1e-8 stop the two iterates differ by rounding amplified through the Krylov recurrence
    assert np.abs(x - xo).max() <= 1e-6 * np.abs(xo).max()
    x = solver.Solve(20000, 1e-12)
    xo, info = C.pcg_jacobi(model.subdomains[0].RHS, tol=1e-12)
    assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()


def test_pcg_zero_rhs_and_not_converged(ctx):
    model = M.clamped_block_model(4)
    A = M.GpuMesh(ctx, model).assemble(model.E_elem, 0.3)
    solver = M.SolverPCG(ctx, model)
    solver.matrix = A
    model.subdomains[0].Forces = np.zeros(model.n_dofs)
    x = solver.Solve(100, 1e-8)
    assert solver.iterations == 0 and not x.any()
    model.ConnectDataStructures()
    with pytest.raises(M.InvalidOperationError) as e:
        solver.Solve(5, 1e-12)
    assert e.value.code == -2001 and solver.iterations == 5


def test_mixed_assembled_solve_reaches_fp64_true_residual(ctx):
    """FP32 values in the loop, FP64 refinement: the FP64 true residual meets the
    tolerance and the field agrees with an FP64 oracle solve; repeated calls on
    the same matrix reuse the captured loop and give identical answers."""
    n = 12
    model = M.clamped_block_model(n)
    E = np.exp(0.3 * np.random.default_rng(8).standard_normal(model.n_elems))
    mesh = M.GpuMesh(ctx, model)
    A = mesh.assemble(E, model.poisson)
    b = model.subdomains[0].RHS
    fp64 = M.SolverPCG(ctx, model, tolerance=1e-10)
    fp64.matrix = A
    x64 = fp64.Solve()
    mixed = M.SolverPCG(ctx, model, tolerance=1e-10, precision="mixed")
    mixed.matrix = A
    xm = mixed.Solve()
    xm2 = mixed.Solve()
    assert np.array_equal(xm, xm2)
    C, _ = oracle_csr(model, E)
    xo, _ = C.pcg_jacobi(b, tol=1e-13)
    r = b - C.multiply(xm)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    assert abs(mixed.rel_res - np.linalg.norm(r) / np.linalg.norm(b)) <= 1e-3 * mixed.rel_res + 1e-16
    assert np.abs(xm - xo).max() <= 1e-8 * np.abs(xo).max()
    assert mixed.iterations <= 1.3 * fp64.iterations + 16


def test_mixed_zero_rhs_and_not_converged(ctx):
    """The mixed loop keeps SolverPCG's guards: a zero right-hand side returns
    x = 0 after no iteration; an iteration limit below what the tolerance needs
    raises not-converged (-2001) with iterations = the limit, and the iterate it
    leaves (the FP32 correction folded into the FP64 x) is the one the same
    limit gives on a second call, and is closer to the solution than x = 0."""
    model = M.clamped_block_model(6)
    A = M.GpuMesh(ctx, model).assemble(model.E_elem, 0.3)
    solver = M.SolverPCG(ctx, model, precision="mixed")
    solver.matrix = A
    model.subdomains[0].Forces = np.zeros(model.n_dofs)
    x = solver.Solve(100, 1e-8)
    assert solver.iterations == 0 and not x.any()
    model.ConnectDataStructures()
    b = model.subdomains[0].RHS
    xs = []
    for _ in range(2):
        with pytest.raises(M.InvalidOperationError) as e:
            solver.Solve(7, 1e-12)
        assert e.value.code == -2001 and solver.iterations == 7
        xs.append(model.subdomains[0].Solution.copy())
    assert np.array_equal(xs[0], xs[1]) and np.abs(xs[0]).max() > 0
    C, _ = oracle_csr(model, model.E_elem)
    r = b - C.multiply(xs[0])
    assert np.linalg.norm(r) < np.linalg.norm(b)
