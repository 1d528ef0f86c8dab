"""GPU parity of the ragged batch (MSG_MC_SOLVE_RAGGED): systems of uneven mesh
size and shape solved in the same launches, each realization against an FP64
oracle solve of its own geometry and field (1e-8 relative, max-norm), and the
same bits for a system alone and in the mix."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def distorted_model(n, seed, amp=0.15):
    model = M.clamped_block_model(n)
    rng = np.random.default_rng(seed)
    inner = (model.xyz > 0.5).all(axis=1) & (model.xyz < n - 0.5).all(axis=1)
    model.xyz[inner] += amp * rng.uniform(-1, 1, (int(inner.sum()), 3))
    return model


def systems():
    """(model, kl, xi) of three systems: a distorted 4^3 with 3 realizations, the
    6^3 lattice with 40 (two 32-wide groups, the second mostly padding) and a
    distorted 5^3 with one."""
    out = []
    for n, R, K, distort, seed in ((4, 3, 5, True, 1), (6, 40, 8, False, 2), (5, 1, 6, True, 3)):
        model = distorted_model(n, seed) if distort else M.clamped_block_model(n)
        kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 4)
        xi = np.random.default_rng(10 + seed).standard_normal((R, K))
        out.append((model, kl, xi))
    return out


def solve(ctx, syss, tol=1e-10):
    batch = M.RaggedMonteCarloBatch(ctx, tolerance=tol)
    for model, kl, xi in syss:
        batch.add(model, kl, xi)
    return batch.Solve()


def oracle_solution(model, kl, xi_r, n):
    E = O.kl_field(O.centroids(model.xyz, model.conn), [n, n, n], kl.table(), xi_r[None, :], sigma=kl.sigma)[0]
    Cs = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
    Cs.assemble(O.h8_stiffness_batch(model.element_xyz(), E, model.poisson)[0])
    xo, info = Cs.pcg_jacobi(model.subdomains[0].RHS, tol=1e-13)
    assert info["status"] == 0
    return xo, Cs


@pytest.fixture
def lattice_loop(ctx, request):
    """ragged_lattice_loop option: cube lattices through the lattice loop (1) or
    the shared element-by-element batch (0)."""
    ctx.set_option("ragged_lattice_loop", request.param)
    yield request.param
    ctx.set_option("ragged_lattice_loop", 1)


@pytest.mark.parametrize("lattice_loop", [0, 1], indirect=True)
def test_ragged_batch_matches_oracle(ctx, lattice_loop):
    syss = systems()
    res = solve(ctx, syss)
    for (model, kl, xi), r in zip(syss, res):
        n = round(model.xyz[:, 0].max())
        assert (r["Residuals"] < 1e-10).all()
        assert (r["Iterations"] > 0).all()
        b = model.subdomains[0].RHS
        for k in sorted({0, xi.shape[0] - 1}):
            xo, Cs = oracle_solution(model, kl, xi[k], n)
            x = r["Solutions"][k]
            assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max(), (n, k)
            rr = np.linalg.norm(b - Cs.multiply(x)) / np.linalg.norm(b)
            assert abs(rr - r["Residuals"][k]) <= 1e-3 * r["Residuals"][k] + 1e-15
            assert r["TipValues"][k] == x[M.tip_dof(model)]


@pytest.fixture
def multigrid(ctx, request):
    ctx.set_option("multigrid", request.param)
    yield request.param
    ctx.set_option("multigrid", 1)


@pytest.mark.parametrize("lattice_loop", [0, 1], indirect=True)
@pytest.mark.parametrize("multigrid", [0, 1], indirect=True)
def test_system_alone_equals_the_mix(ctx, multigrid, lattice_loop):
    """A system's arithmetic is independent of the other systems: each system
    solved alone gives the same bits as in the ragged mix. With the multigrid
    option on, the two even lattices (the distorted 4^3 and the 6^3) take the
    V-cycle of their cube lattice and the 5^3 the diagonal inside the same
    loop; alone, the 5^3 takes the fused Jacobi loop, which differs from the
    standard PCG only in rounding (1e-8). One realization solved alone agrees
    with its batched solve to 1e-9 (the true-residual steps of a system are
    shared by its realizations)."""
    syss = systems()
    mix = solve(ctx, syss)
    for i, s in enumerate(syss):
        alone = solve(ctx, [s])[0]
        if multigrid and i == 2:
            a, m = alone["Solutions"], mix[i]["Solutions"]
            assert np.abs(a - m).max() <= 1e-8 * np.abs(m).max()
            assert (alone["Residuals"] < 1e-10).all() and (mix[i]["Residuals"] < 1e-10).all()
            continue
        for key in ("Solutions", "TipValues", "Iterations", "Residuals"):
            assert np.array_equal(alone[key], mix[i][key]), (i, key)
    model, kl, xi = syss[1]
    one = solve(ctx, [(model, kl, xi[17:18])])[0]
    a = mix[1]["Solutions"][17]
    assert np.abs(one["Solutions"][0] - a).max() <= 1e-9 * np.abs(a).max()


def test_lattice_system_equals_its_own_batch_call(ctx):
    """With the ragged_lattice_loop option on (default), a structured cube
    lattice of a ragged batch is solved by the lattice loop of
    MSG_MC_SOLVE_BATCH: the same bits as the analyzer's own mixed-mode call."""
    model, kl, xi = systems()[1]
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=kl.n_terms,
                                                    simulations=xi.shape[0], mode="mixed", tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    r = solve(ctx, systems())[1]
    for key, ref in (("Solutions", mc.Solutions), ("TipValues", mc.TipValues), ("Iterations", mc.Iterations),
                     ("Residuals", mc.Residuals)):
        assert np.array_equal(r[key], ref), key


@pytest.mark.parametrize("lattice_loop", [0], indirect=True)
def test_lattice_systems_take_the_vcycle(ctx, lattice_loop):
    """Two 8^3 systems, one a cube lattice and one with moved interior nodes:
    with the multigrid option each converges in a fraction of the Jacobi
    iterations, to the same 1e-10 residual and within 1e-8 of the Jacobi
    solution."""
    syss = []
    for distort, seed in ((False, 4), (True, 5)):
        model = distorted_model(8, seed) if distort else M.clamped_block_model(8)
        kl = M.LognormalStochasticCoefficientsProvider([8, 8, 8], 1.6, 10, 4)
        syss.append((model, kl, np.random.default_rng(seed).standard_normal((37, 10))))
    vc = solve(ctx, syss)
    ctx.set_option("multigrid", 0)
    try:
        jac = solve(ctx, syss)
    finally:
        ctx.set_option("multigrid", 1)
    for v, j in zip(vc, jac):
        assert (v["Residuals"] < 1e-10).all() and (j["Residuals"] < 1e-10).all()
        assert v["Iterations"].max() * 2 < j["Iterations"].min()
        assert np.abs(v["Solutions"] - j["Solutions"]).max() <= 1e-8 * np.abs(j["Solutions"]).max()


@pytest.mark.parametrize("multigrid", [0, 1], indirect=True)
def test_analyzer_on_a_distorted_mesh_is_the_one_system_batch(ctx, multigrid):
    """MSG_MC_SOLVE_BATCH in mixed mode on a mesh that is not a cube lattice
    runs the same loop as the ragged batch of that one system (the Jacobi loop
    with multigrid 0, the V-cycle-preconditioned one with multigrid 1):
    bit-identical results."""
    model, kl, xi = systems()[0]
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=kl.n_terms,
                                                    simulations=xi.shape[0], mode="mixed", tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    r = solve(ctx, [(model, kl, xi)])[0]
    assert np.array_equal(mc.Solutions, r["Solutions"]) and np.array_equal(mc.Iterations, r["Iterations"])


def test_ragged_batch_rejects_invalid_systems(ctx):
    model, kl, xi = systems()[0]
    other = M.Context(0)
    batch = M.RaggedMonteCarloBatch(other, tolerance=1e-10)
    batch.systems.append(dict(model=model, kl=kl, xi=xi, tip_dof=0, keep=False, mesh=M.GpuMesh(ctx, model)))
    with pytest.raises(M.ArgumentError):
        batch.Solve()  # mesh of another context
    with pytest.raises(M.ArgumentError):
        M.RaggedMonteCarloBatch(ctx).Solve()  # no systems


MIX = ((4, 3, 5, False, 4), (6, 40, 8, False, 5), (5, 2, 6, True, 6), (8, 70, 10, False, 7))
MIX_SIDES = [row[0] for row in MIX]


def lattice_mix():
    """Three cube lattices (4^3 with 3 realizations, 6^3 with 40, 8^3 with 70:
    two 64-wide groups, the second mostly padding) and a distorted 5^3 block."""
    out = []
    for n, R, K, distort, seed in MIX:
        model = distorted_model(n, seed) if distort else M.clamped_block_model(n)
        kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 4)
        xi = np.random.default_rng(20 + seed).standard_normal((R, K))
        out.append((model, kl, xi))
    return out


@pytest.fixture
def side_by_side(ctx):
    yield
    ctx.set_option("ragged_side_by_side", 1)


def test_lattices_side_by_side_equal_one_after_another(ctx, side_by_side):
    """The ragged_side_by_side option (default 1) steps the loops of a batch's
    cube lattices side by side, each on its own stream: every lattice takes the
    steps it takes alone, so the results are the same bits as with the lattices
    solved one after another, call after call, and as the analyzer's own call."""
    syss = lattice_mix()
    ctx.set_option("ragged_side_by_side", 0)
    ref = solve(ctx, syss)
    ctx.set_option("ragged_side_by_side", 1)
    for _ in range(2):  # the second call reuses the streams, buffers and loop graphs
        got = solve(ctx, syss)
        for a, b in zip(got, ref):
            for key in ("Solutions", "TipValues", "Iterations", "Residuals"):
                assert np.array_equal(a[key], b[key]), key
    model, kl, xi = syss[3]
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=kl.n_terms,
                                                    simulations=xi.shape[0], mode="mixed", tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    assert np.array_equal(got[3]["Solutions"], mc.Solutions)
    assert np.array_equal(got[3]["Iterations"], mc.Iterations)
    for k, ((model, kl, xi), n) in enumerate(zip(syss, MIX_SIDES)):
        assert got[k]["Residuals"].max() < 1e-10
        xo, _ = oracle_solution(model, kl, xi[-1], n)
        assert np.abs(got[k]["Solutions"][-1] - xo).max() <= 1e-8 * np.abs(xo).max()


def test_lattices_side_by_side_not_converged(ctx, side_by_side):
    """An iteration limit that stops every lattice: the same outcome (not
    converged), iteration counts and partial solutions either way."""
    syss = lattice_mix()
    outs = []
    for opt in (0, 1):
        ctx.set_option("ragged_side_by_side", opt)
        batch = M.RaggedMonteCarloBatch(ctx, max_iterations=2, tolerance=1e-12)
        for model, kl, xi in syss:
            batch.add(model, kl, xi)
        with pytest.raises(M.InvalidOperationError) as e:
            batch.Solve()
        outs.append((e.value.code, batch.Results))
    assert outs[0][0] == outs[1][0]
    for a, b in zip(outs[0][1], outs[1][1]):
        for key in ("Solutions", "Iterations", "Residuals"):
            assert np.array_equal(a[key], b[key]), key
