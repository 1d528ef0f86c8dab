"""GPU parity of the multigrid-preconditioned batched solve (the default;
MSG_SET_OPTION "multigrid" = 0 selects the Jacobi-preconditioned loop):
geometric V-cycle on the padded lattice, FP32 inner loop, FP64 true-residual
replacement, per-realization convergence to the same FP64 relative residual as
the Jacobi loop.

Tolerances: displacements 1e-8 relative (max-norm) to an FP64 oracle solve
converged to 1e-13, for solves to a true relative residual of 1e-10 (the bound
of the Jacobi-preconditioned batched path); Newmark histories as the Jacobi
Newmark test (1e-8 of the maximum on the tip history, 1e-7 on the final field)."""
import contextlib

import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


DEFAULTS = {"multigrid": 1, "fixed_updates": 0, "multigrid_levels": 6, "multigrid_sweeps": 20, "multigrid_packed": 1,
            "multigrid_fused_coarse": 1}


@contextlib.contextmanager
def options(ctx, **kw):
    for k, v in kw.items():
        ctx.set_option(k, v)
    try:
        yield
    finally:
        for k, v in DEFAULTS.items():
            ctx.set_option(k, v)


def problem(model, dims, R, seed, n_terms=20):
    kl = M.LognormalStochasticCoefficientsProvider(list(dims), 0.2 * max(dims), n_terms, 8)
    xi = np.random.default_rng(seed).standard_normal((R, n_terms))
    return kl, xi


def oracle_fields(model, kl, xi, dims):
    cen = O.centroids(model.xyz, model.conn)
    return O.kl_field(cen, list(dims), kl.table(), xi, mean=kl.mean, sigma=kl.sigma,
                      mean_correction=kl.mean_correction)


def mixed_solve(ctx, model, kl, xi, tol):
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=xi.shape[1],
                                                    simulations=xi.shape[0], mode="mixed", tolerance=tol)
    mc.RandomNumbers = xi
    mc.Solve()
    return mc


@pytest.mark.parametrize("n,R,mg,levels,packed", [(4, 5, 1, 6, 1), (8, 40, 1, 6, 1), (16, 64, 1, 6, 1),
                                                  (16, 64, 1, 3, 1), (16, 70, 1, 6, 0), (8, 40, 0, 6, 1)])
def test_multigrid_matches_fp64_oracle(ctx, n, R, mg, levels, packed):
    """packed = 0: the level-0 operator with one realization per lane."""
    model = M.clamped_block_model(n)
    kl, xi = problem(model, (n, n, n), R, seed=n)
    with options(ctx, multigrid=mg, multigrid_levels=levels, multigrid_packed=packed):
        mc = mixed_solve(ctx, model, kl, xi, 1e-10)
    assert (mc.Residuals < 1e-10).all()
    E = oracle_fields(model, kl, xi, (n, n, n))
    cons = (model.dof < 0).astype(np.uint8)
    for r in sorted({0, R // 2, R - 1}):
        xo, info = O.block_solve_pcg(n, n, n, cons, E[r], model.poisson, model.subdomains[0].RHS, tol=1e-13,
                                     max_it=100000)
        assert info["status"] == 0
        err = np.abs(mc.Solutions[r] - xo).max() / np.abs(xo).max()
        assert err <= 1e-8, (r, err)


def test_multigrid_cantilever_two_levels(ctx):
    """10 x 4 x 4 cantilever (x = 0 clamped): one coarse level of 5 x 2 x 2."""
    model = M.cantilever_model()
    kl, xi = problem(model, (10, 4, 4), 12, seed=3)
    mc = mixed_solve(ctx, model, kl, xi, 1e-10)
    assert (mc.Residuals < 1e-10).all()
    E = oracle_fields(model, kl, xi, (10, 4, 4))
    cons = (model.dof < 0).astype(np.uint8)
    for r in (0, 11):
        xo, info = O.block_solve_pcg(10, 4, 4, cons, E[r], model.poisson, model.subdomains[0].RHS, tol=1e-13,
                                     max_it=100000)
        err = np.abs(mc.Solutions[r] - xo).max() / np.abs(xo).max()
        assert err <= 1e-8, (r, err)


def test_multigrid_cuts_iterations(ctx):
    n, R = 16, 32
    model = M.clamped_block_model(n)
    kl, xi = problem(model, (n, n, n), R, seed=5)
    with options(ctx, multigrid=0):
        jac = mixed_solve(ctx, model, kl, xi, 1e-8)
    mg = mixed_solve(ctx, model, kl, xi, 1e-8)
    with options(ctx, multigrid_levels=2):
        mg2 = mixed_solve(ctx, model, kl, xi, 1e-8)
    assert (mg.Residuals < 1e-8).all() and (mg2.Residuals < 1e-8).all()
    assert mg.Iterations.max() * 5 < jac.Iterations.min(), (mg.Iterations.max(), jac.Iterations.min())
    assert mg.Iterations.mean() <= mg2.Iterations.mean()


def test_multigrid_batch_invariant_with_fixed_updates(ctx):
    """Per-realization arithmetic does not depend on the batch: a realization
    solved inside a batch of 40 and in a batch of its own agrees bit for bit."""
    n, R = 8, 40
    model = M.clamped_block_model(n)
    kl, xi = problem(model, (n, n, n), R, seed=9)
    with options(ctx, fixed_updates=1):
        full = mixed_solve(ctx, model, kl, xi, 1e-10)
        for r in (0, 17, 39):
            one = mixed_solve(ctx, model, kl, xi[r:r + 1], 1e-10)
            assert np.array_equal(one.Solutions[0], full.Solutions[r]), r
            assert one.Iterations[0] == full.Iterations[r]


@pytest.mark.parametrize("case", ["cube16", "cantilever"])
def test_fused_coarsest_sweeps_identical(ctx, case):
    """All coarsest-level sweeps in one launch (multigrid_fused_coarse = 1)
    return bit for bit what one launch per sweep returns: 2 x 2 x 2 coarsest
    elements of a 16^3 cube and 5 x 2 x 2 of the 10 x 4 x 4 cantilever."""
    if case == "cube16":
        model, dims, R = M.clamped_block_model(16), (16, 16, 16), 70
    else:
        model, dims, R = M.cantilever_model(), (10, 4, 4), 12
    kl, xi = problem(model, dims, R, seed=31)
    with options(ctx, multigrid_fused_coarse=0):
        ref = mixed_solve(ctx, model, kl, xi, 1e-10)
    fused = mixed_solve(ctx, model, kl, xi, 1e-10)
    assert np.array_equal(fused.Solutions, ref.Solutions)
    assert np.array_equal(fused.Iterations, ref.Iterations)


def test_fused_coarsest_sweeps_identical_with_mass(ctx):
    """The same with a mass term (Newmark on the V-cycle loop)."""
    n, R, steps, dt = 8, 33, 5, 0.01
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(7).standard_normal((R, 12))
    load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * steps, 0.1, dof=0)
    out = []
    for fused in (0, 1):
        with options(ctx, multigrid=2, multigrid_fused_coarse=fused):
            nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * steps, load, expansion_order=12,
                                          simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                          tolerance=1e-10)
            nm.RandomNumbers = xi
            out.append((nm.Solve(), nm.Solutions.copy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("n,R,steps,mg", [(4, 3, 30, 2), (8, 33, 20, 2), (8, 33, 20, 1)])
def test_multigrid_newmark_matches_oracle(ctx, n, R, steps, mg):
    """multigrid = 2 puts the mass-term systems on the V-cycle loop too (1, the
    default, keeps them on the Jacobi loop). Steps are solved to 1e-12 here so
    that the step errors stay below the history bound with either loop."""
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(n).standard_normal((R, 12))
    dt = 0.01
    load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * steps, 0.1, dof=0)
    corner = int(np.argmax(model.xyz.sum(1)))
    with options(ctx, multigrid=mg):
        nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * steps, load, expansion_order=12,
                                      simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                      tolerance=1e-12, tip_dof=int(model.dof[corner, 0]))
        nm.RandomNumbers = xi
        hist = nm.Solve()
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field(cen, [n, n, n], kl.table(), xi, mean=kl.mean, sigma=kl.sigma, mean_correction=kl.mean_correction)
    cons = (model.dof < 0).astype(np.uint8)
    for r in sorted({0, R // 2, R - 1}):
        t, u, info = O.block_newmark(n, n, n, cons, E[r], model.poisson, 1.0, 0.01, 0.001, 0.25, 0.5, dt, steps, 0.1,
                                     1.0, 0, model.n_dofs, tip_dof=nm.tip_dof)
        assert info["status"] == 0
        scale = np.abs(t).max()
        assert np.abs(hist[r] - t).max() <= 1e-8 * scale, (r, np.abs(hist[r] - t).max() / scale)
        assert np.abs(nm.Solutions[r] - u).max() <= 1e-7 * np.abs(u).max()
