"""GPU parity at the full sizes of the benchmark configurations, against FP64
oracle solves of the same inputs (the oracle restates SolverPCG and
NewmarkDynamicAnalyzer; ISAAR.MSolve.Solvers/PCG/SolverPCG.cs:105-149,
ISAAR.MSolve.Analyzers/NewmarkDynamicAnalyzer.cs:280-315).

* Monte Carlo, 1024 realizations of the 32^3 block (50-term KL, sigma 0.3),
  each to the benchmark's FP64 true relative residual of 1e-9: eight
  realizations spread over the batch within 1e-8 (max norm, relative to the
  oracle's maximum) of oracle solves converged to 1e-12.
* Single 64^3 static solve: the FP64 drop-in at the reference's stopping rule
  (1e-8) equals the oracle's PCG at the same rule to 1e-10 with the same
  iteration count (+-1); FP32 values + FP64 refinement to a 1e-10 relative
  residual is within 1e-8 of the oracle converged to 1e-12.
* Newmark, 256 realizations of the 24^3 block, 200 steps: four of them, tip
  histories and final fields within 1e-8 of the oracle's FP64 integration
  (each step converged to 1e-14). Each GPU step is solved to a 1e-13 true
  relative residual: the integration carries step errors forward
  (a0 = 1/(beta dt^2) = 4e4), so looser steps drift further from the oracle
  (1e-8 steps end 6e-4 away).
* Serving, one 48^3 request through MSG_SERVE_*: within 1e-8 of the oracle.
"""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def _fields(P, xi):
    return O.kl_field(P["centroids"], P["domain"], P["table"], np.atleast_2d(xi), sigma=0.3)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_mc_1024_realizations_32cube_against_oracle(ctx):
    n, R, K = 32, 1024, 50
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 16)
    xi = np.random.default_rng(31).standard_normal((R, K))
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=R, mode="mixed",
                                                    tolerance=1e-9)
    mc.RandomNumbers = xi
    mc.Solve()
    assert (mc.Residuals < 1e-9).all()
    P = O.block_problem(n, K, 16)
    assert np.array_equal(P["b"], model.subdomains[0].RHS)
    rows = np.linspace(0, R - 1, 8).astype(int)
    E = _fields(P, xi[rows])
    for i, r in enumerate(rows):
        xo, info = O.block_solve_pcg(n, n, n, P["constrained"], E[i], 0.3, P["b"], tol=1e-12, max_it=100000)
        assert info["status"] == 0
        err = _rel(mc.Solutions[r], xo)
        assert err <= 1e-8, (int(r), err)
        assert mc.TipValues[r] == mc.Solutions[r][mc.tip_dof]


def test_single_64cube_fp64_and_mixed_against_oracle(ctx):
    n = 64
    model = M.clamped_block_model(n)
    P = O.block_problem(n, 1, 4)
    A = M.GpuMesh(ctx, model).assemble(np.ones(model.n_elems), model.poisson)
    s64 = M.SolverPCG(ctx, model, max_iterations=100000, tolerance=1e-8, precision="fp64")
    s64.matrix = A
    x64 = s64.Solve().copy()
    xo8, info8 = O.block_solve_pcg(n, n, n, P["constrained"], np.ones(n ** 3), 0.3, P["b"], tol=1e-8,
                                   max_it=100000)
    assert info8["status"] == 0
    assert abs(s64.iterations - info8["iterations"]) <= 1, (s64.iterations, info8["iterations"])
    assert _rel(x64, xo8) <= 1e-10
    smx = M.SolverPCG(ctx, model, max_iterations=100000, tolerance=1e-10, precision="mixed")
    smx.matrix = A
    xmx = smx.Solve().copy()
    assert smx.rel_res < 1e-10
    xo, info = O.block_solve_pcg(n, n, n, P["constrained"], np.ones(n ** 3), 0.3, P["b"], tol=1e-12, max_it=100000)
    assert info["status"] == 0
    assert _rel(xmx, xo) <= 1e-8
    A.close()


def test_newmark_24cube_200_steps_against_oracle(ctx):
    n, R, K, steps, dt = 24, 256, 50, 200, 0.01
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 12)
    xi = np.random.default_rng(24).standard_normal((R, K))
    load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * steps, 0.1, dof=0)
    corner = int(np.argmax(model.xyz.sum(1)))
    nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * steps, load, expansion_order=K,
                                  simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                  tolerance=1e-13, tip_dof=int(model.dof[corner, 0]))
    nm.RandomNumbers = xi
    hist = nm.Solve()
    assert hist.shape == (R, steps)
    P = O.block_problem(n, K, 12)
    rows = np.linspace(0, R - 1, 4).astype(int)
    E = _fields(P, xi[rows])
    for i, r in enumerate(rows):
        t, u, info = O.block_newmark(n, n, n, P["constrained"], E[i], model.poisson, 1.0, 0.01, 0.001, 0.25, 0.5, dt,
                                     steps, 0.1, 1.0, 0, model.n_dofs, solver=2, tol=1e-14, tip_dof=nm.tip_dof)
        assert info["status"] == 0
        assert _rel(hist[r], t) <= 1e-8, (int(r), _rel(hist[r], t))
        assert _rel(nm.Solutions[r], u) <= 1e-8, (int(r), _rel(nm.Solutions[r], u))


def test_serving_48cube_request_against_oracle(ctx):
    from msolve_b200.serving import Server
    n, K = 48, 50
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 12)
    xi = np.random.default_rng(48).standard_normal(K)
    srv = Server(ctx, max_batch=64)
    try:
        mid = srv.add_model(model, kl, tol=1e-10)
        out = srv.poll(srv.submit(mid, xi), timeout_ms=-1)
    finally:
        srv.stop()
    assert out["rel_res"] < 1e-10
    P = O.block_problem(n, K, 12)
    E = _fields(P, xi)
    xo, info = O.block_solve_pcg(n, n, n, P["constrained"], E[0], 0.3, P["b"], tol=1e-12, max_it=100000)
    assert info["status"] == 0
    assert _rel(out["X"], xo) <= 1e-8
