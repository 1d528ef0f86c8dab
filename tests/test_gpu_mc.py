"""GPU parity of the Monte Carlo path: KL field, the plain FP64 drop-in
(realization by realization, assembled BSR + Jacobi-PCG) and the batched
mixed-precision matrix-free solve, against per-realization FP64 oracle solves.

Tolerances: E field 1e-13 relative; FP64 drop-in displacements 1e-10 relative
to the oracle at the same stopping rule; mixed-precision displacements 1e-8
relative (max-norm) to an FP64 oracle solve converged to 1e-13."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def setup(n, R, seed=1, n_terms=20):
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, n_terms, 8)
    xi = np.random.default_rng(seed).standard_normal((R, n_terms))
    return model, kl, xi


def oracle_fields(model, kl, xi, n):
    cen = O.centroids(model.xyz, model.conn)
    return O.kl_field(cen, [n, n, n], kl.table(), xi, mean=kl.mean, sigma=kl.sigma,
                      mean_correction=kl.mean_correction)


def oracle_solve(model, n, E, tol=1e-13):
    cons = (model.dof < 0).astype(np.uint8)
    x, info = O.block_solve_pcg(n, n, n, cons, E, model.poisson, model.subdomains[0].RHS, tol=tol, max_it=100000)
    assert info["status"] == 0
    return x, info


def test_kl_field_matches_oracle(ctx):
    for mc in (False, True):
        model, kl, xi = setup(8, 70, n_terms=30)
        kl.mean_correction = mc
        mesh = M.GpuMesh(ctx, model)
        E = kl.field(mesh, xi)
        Eo = oracle_fields(model, kl, xi, 8)
        assert np.abs(E - Eo).max() <= 1e-13 * np.abs(Eo).max()


def test_fp64_dropin_matches_oracle_pcg(ctx):
    """Same stopping rule -> same iteration count (+-1 from summation order);
    tightly converged -> same displacements to 1e-10."""
    n, R = 6, 3
    model, kl, xi = setup(n, R)
    E = oracle_fields(model, kl, xi, n)
    for tol in (1e-8, 1e-12):
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=20, simulations=R,
                                                        mode="fp64", tolerance=tol)
        mc.RandomNumbers = xi
        mc.Solve()
        for r in range(R):
            xo, info = oracle_solve(model, n, E[r], tol=tol)
            assert abs(mc.Iterations[r] - info["iterations"] - 1) <= 1
            assert mc.TipValues[r] == mc.Solutions[r][mc.tip_dof]
            if tol == 1e-12:
                assert np.abs(mc.Solutions[r] - xo).max() <= 1e-10 * np.abs(xo).max()
            else:
                assert np.abs(mc.Solutions[r] - xo).max() <= 1e-6 * np.abs(xo).max()


@pytest.mark.parametrize("n,R", [(4, 5), (8, 40), (12, 64)])
def test_mixed_batched_matches_fp64_oracle(ctx, n, R):
    model, kl, xi = setup(n, R, seed=n)
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=20, simulations=R, mode="mixed",
                                                    tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    assert (mc.Residuals < 1e-10).all()
    E = oracle_fields(model, kl, xi, n)
    for r in sorted({0, R // 2, R - 1}):
        xo, _ = oracle_solve(model, n, E[r])
        err = np.abs(mc.Solutions[r] - xo).max() / np.abs(xo).max()
        assert err <= 1e-8, (r, err)
        # residual reported by the GPU is the FP64 true residual of the returned x
        C = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
        C.assemble(O.h8_stiffness_batch(model.element_xyz(), E[r], 0.3)[0])
        b = model.subdomains[0].RHS
        rr = np.linalg.norm(b - C.multiply(mc.Solutions[r])) / np.linalg.norm(b)
        assert abs(rr - mc.Residuals[r]) <= 1e-3 * mc.Residuals[r] + 1e-15


def test_mixed_result_is_independent_of_the_batch(ctx):
    """A realization solved alone and inside a batch gives the same answer
    (realization-innermost layout: no cross-realization arithmetic)."""
    n, R = 6, 33
    model, kl, xi = setup(n, R, seed=3)
    runs = []
    for rows in (slice(0, R), slice(5, 6)):
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=20,
                                                        simulations=xi[rows].shape[0], mode="mixed", tolerance=1e-10)
        mc.RandomNumbers = xi[rows]
        mc.Solve()
        runs.append(mc)
    a, b = runs[0].Solutions[5], runs[1].Solutions[0]
    assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()


def distorted_model(n, seed=12, amp=0.15):
    """n^3 clamped block whose interior nodes are moved by up to amp in each axis."""
    model = M.clamped_block_model(n)
    rng = np.random.default_rng(seed)
    inner = (model.xyz > 0.5).all(axis=1) & (model.xyz < n - 0.5).all(axis=1)
    model.xyz[inner] += amp * rng.uniform(-1, 1, (int(inner.sum()), 3))
    return model


def oracle_csr_solve(model, E_r):
    Cs = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
    Cs.assemble(O.h8_stiffness_batch(model.element_xyz(), E_r, model.poisson)[0])
    xo, info = Cs.pcg_jacobi(model.subdomains[0].RHS, tol=1e-13)
    assert info["status"] == 0
    return xo, Cs


@pytest.mark.parametrize("element_batch", [1, 0])
def test_mixed_on_a_distorted_mesh_matches_oracle(ctx, element_batch):
    """A mesh that is not a cube lattice (interior nodes moved) takes the mixed
    mode through the batched element-by-element loop (element_batch = 1) or
    realization by realization through the assembled FP32-value PCG with FP64
    refinement (0): within 1e-8 of FP64 oracle solves of the same geometry."""
    n, R, K = 4, 3, 5
    model = distorted_model(n)
    rng = np.random.default_rng(12)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 4)
    xi = rng.standard_normal((R, K))
    ctx.set_option("element_batch", element_batch)
    try:
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=R,
                                                        mode="mixed", tolerance=1e-10)
        mc.RandomNumbers = xi
        mc.Solve()
    finally:
        ctx.set_option("element_batch", 1)
    assert (mc.Residuals < 1e-10).all()
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field(cen, [n, n, n], kl.table(), xi, sigma=kl.sigma)
    for r in range(R):
        xo, _ = oracle_csr_solve(model, E[r])
        assert np.abs(mc.Solutions[r] - xo).max() <= 1e-8 * np.abs(xo).max()
        assert mc.TipValues[r] == mc.Solutions[r][mc.tip_dof]


@pytest.mark.parametrize("mode,element_batch", [("fp64", 1), ("mixed", 0)])
def test_per_realization_path_on_a_larger_second_mesh(mode, element_batch):
    """The per-realization path keeps its element-matrix buffer in the context
    across calls; a call on a mesh with more elements than the previous one
    grows it (fresh context: 3^3, then 5^3 distorted meshes, oracle parity on
    both)."""
    c = M.Context(0)
    c.set_option("element_batch", element_batch)
    K, R = 4, 2
    for n in (3, 5):
        model = distorted_model(n, seed=n)
        kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 4)
        xi = np.random.default_rng(n).standard_normal((R, K))
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(c, model, kl, expansion_order=K, simulations=R, mode=mode,
                                                        tolerance=1e-12 if mode == "fp64" else 1e-10)
        mc.RandomNumbers = xi
        mc.Solve()
        E = O.kl_field(O.centroids(model.xyz, model.conn), [n, n, n], kl.table(), xi, sigma=kl.sigma)
        for r in range(R):
            xo, _ = oracle_csr_solve(model, E[r])
            assert np.abs(mc.Solutions[r] - xo).max() <= 1e-8 * np.abs(xo).max(), (n, r)


def test_multigrid_on_a_distorted_lattice(ctx):
    """A mesh with the lattice's topology and moved interior nodes (8^3, 40
    realizations) takes PCG over the element-by-element operator with the cube
    lattice's V-cycle as preconditioner: within 1e-8 of FP64 oracle solves of
    the distorted geometry, with at least 3x fewer operator products than the
    same loop with the diagonal preconditioner (multigrid 0)."""
    n, R, K = 8, 40, 10
    model = distorted_model(n, seed=21, amp=0.2)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 8)
    xi = np.random.default_rng(22).standard_normal((R, K))
    runs = {}
    for mg in (1, 0):
        ctx.set_option("multigrid", mg)
        try:
            mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=R,
                                                            mode="mixed", tolerance=1e-10)
            mc.RandomNumbers = xi
            mc.Solve()
        finally:
            ctx.set_option("multigrid", 1)
        assert (mc.Residuals < 1e-10).all()
        runs[mg] = mc
    assert 3 * runs[1].Iterations.mean() < runs[0].Iterations.mean(), (runs[1].Iterations.mean(),
                                                                         runs[0].Iterations.mean())
    E = O.kl_field(O.centroids(model.xyz, model.conn), [n, n, n], kl.table(), xi, sigma=kl.sigma)
    for r in (0, R - 1):
        xo, _ = oracle_csr_solve(model, E[r])
        for mc in runs.values():
            assert np.abs(mc.Solutions[r] - xo).max() <= 1e-8 * np.abs(xo).max(), r


def test_element_batch_on_a_distorted_mesh_sample(ctx):
    """Batched element-by-element loop on a distorted 10^3 mesh, 70 realizations
    (three 32-wide groups, the last one partly padding): sampled realizations
    within 1e-8 of FP64 oracle solves; the reported residual is the FP64 true
    residual of the returned displacements; a realization solved alone agrees
    with its batched solve to 1e-9."""
    n, R, K = 10, 70, 12
    model = distorted_model(n, seed=5, amp=0.2)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 8)
    xi = np.random.default_rng(8).standard_normal((R, K))
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=R, mode="mixed",
                                                    tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    assert (mc.Residuals < 1e-10).all()
    assert (mc.Iterations > 0).all()
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field(cen, [n, n, n], kl.table(), xi, sigma=kl.sigma)
    b = model.subdomains[0].RHS
    for r in (0, 37, R - 1):
        xo, Cs = oracle_csr_solve(model, E[r])
        assert np.abs(mc.Solutions[r] - xo).max() <= 1e-8 * np.abs(xo).max(), r
        rr = np.linalg.norm(b - Cs.multiply(mc.Solutions[r])) / np.linalg.norm(b)
        assert abs(rr - mc.Residuals[r]) <= 1e-3 * mc.Residuals[r] + 1e-15
    one = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=1, mode="mixed",
                                                     tolerance=1e-10)
    one.RandomNumbers = xi[37:38]
    one.Solve()
    a = mc.Solutions[37]
    assert np.abs(one.Solutions[0] - a).max() <= 1e-9 * np.abs(a).max()


def test_element_batch_on_a_renumbered_lattice_matches_the_lattice_path(ctx):
    """The cube lattice with its nodes and elements renumbered at random is not
    recognised as a lattice and goes through the element-by-element loop; its
    displacements, mapped back, agree with the lattice path's to 1e-8."""
    n, R, K = 6, 9, 10
    base = M.clamped_block_model(n)
    rng = np.random.default_rng(4)
    perm = rng.permutation(base.n_nodes)          # new id of old node i: perm[i]
    eperm = rng.permutation(base.n_elems)
    xyz = np.empty_like(base.xyz)
    xyz[perm] = base.xyz
    conn = perm[base.conn][eperm]
    ren = M.Model(xyz, conn, base.young, base.poisson)
    ren.constrain(np.nonzero(np.isclose(xyz[:, 2], 0.0))[0])
    for node, d, amount in base.loads:
        ren.add_load(perm[node], d, amount)
    ren.ConnectDataStructures()
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 8)
    xi = rng.standard_normal((R, K))
    runs = []
    for model in (base, ren):
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=K, simulations=R,
                                                        mode="mixed", tolerance=1e-11)
        mc.RandomNumbers = xi
        mc.Solve()
        assert (mc.Residuals < 1e-11).all()
        runs.append(mc)
    assert M.GpuMesh(ctx, base).info()["structured"] and not M.GpuMesh(ctx, ren).info()["structured"]
    for r in range(R):
        xb, xr = runs[0].Solutions[r], runs[1].Solutions[r]
        # DOF (node i, component c) of the base model is DOF (perm[i], c) of the renumbered one
        nodes, comps = np.nonzero(base.dof >= 0)
        assert np.abs(xr[ren.dof[perm[nodes], comps]] - xb[base.dof[nodes, comps]]).max() <= 1e-8 * np.abs(xb).max()


def test_mixed_32cube_sample_against_oracle(ctx):
    """Config 3 geometry (32^3, 50-term KL, l = 6.4, sigma = 0.3), a 64-realization batch."""
    n, R = 32, 64
    model, kl, xi = setup(n, R, seed=2024, n_terms=50)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 50, 16)
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=50, simulations=R, mode="mixed",
                                                    tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    assert (mc.Residuals < 1e-10).all()
    E = oracle_fields(model, kl, xi, n)
    xo, _ = oracle_solve(model, n, E[7], tol=1e-12)
    err = np.abs(mc.Solutions[7] - xo).max() / np.abs(xo).max()
    assert err <= 1e-8, err


def test_batches_and_resume_match_one_call(ctx, tmp_path):
    """batch_size splits and a checkpointed resume return, bit for bit, what one
    call over all realizations returns (fixed_updates = 1: per-realization
    arithmetic independent of the batch)."""
    n, R = 8, 45
    model, kl, xi = setup(n, R, seed=11)
    ctx.set_option("fixed_updates", 1)
    try:
        one = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=20, simulations=R,
                                                         tolerance=1e-10)
        one.RandomNumbers = xi
        one.Solve()
        ck = str(tmp_path / "mc.npz")
        split = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=20, simulations=R,
                                                           tolerance=1e-10, batch_size=16, checkpoint=ck)
        split.RandomNumbers = xi
        split.Solve()
        assert np.array_equal(split.Solutions, one.Solutions)
        assert np.array_equal(split.TipValues, one.TipValues) and np.array_equal(split.Iterations, one.Iterations)
        # a second analyzer on the finished checkpoint solves nothing and reports the same values
        again = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=20, simulations=R,
                                                           tolerance=1e-10, batch_size=16, checkpoint=ck)
        again.RandomNumbers = xi
        again.Solve()
        assert np.isnan(again.Solutions).all() and np.array_equal(again.TipValues, one.TipValues)
    finally:
        ctx.set_option("fixed_updates", 0)
