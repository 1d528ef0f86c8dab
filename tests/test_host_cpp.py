"""The C++ host mirror (msolve_b200/host/msolve.hpp) and its driver, which
replays the reference's analyzer call sequences against the C ABI. On the CPU:
the header compiles warning-free and its model (generator order, DOF
numbering, assigned loads) equals the Python mirror's exactly. On the GPU:
the StaticAnalyzer -> LinearAnalyzer -> SolverPCG chain, the Monte Carlo
analyzer, the Newmark analyzer and the serving loop return the same bits as the Python mirror
(same ABI calls on the same inputs), the static solve matches the oracle's
skyline LDL^T to 1e-8, and the Newmark guard raises InvalidOperationException."""
import os
import subprocess

import numpy as np
import pytest

import msolve_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("host") / "msolve_driver")
    lib = os.path.join(ROOT, "msolve_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(lib, "host"), os.path.join(lib, "host", "msolve_driver.cpp"), "-L" + lib,
           "-lmsolve_gpu", "-Wl,-rpath," + lib, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def run(driver, *args):
    r = subprocess.run([driver, *map(str, args)], capture_output=True, text=True, timeout=600)
    return r.returncode, r.stderr


@pytest.mark.parametrize("kind,n", [("cantilever", 0), ("block", 4), ("block", 7)])
def test_model_matches_python_mirror(driver, tmp_path, kind, n):
    out = tmp_path / "model.bin"
    rc, err = run(driver, "model", kind, n, out)
    assert rc == 0, err
    model = M.cantilever_model() if kind == "cantilever" else M.clamped_block_model(n)
    raw = out.read_bytes()
    nd = int(np.frombuffer(raw[:4], dtype=np.int32)[0])
    dof = np.frombuffer(raw[4:4 + 12 * model.n_nodes], dtype=np.int32).reshape(-1, 3)
    forces = np.frombuffer(raw[4 + 12 * model.n_nodes:], dtype=np.float64)
    assert nd == model.n_dofs
    assert np.array_equal(dof, model.dof)
    assert np.array_equal(forces, model.subdomains[0].RHS)


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_static_chain_matches_python_and_skyline(ctx, driver, tmp_path, mixed):
    import oracle as O
    out = tmp_path / "static.bin"
    rc, err = run(driver, "static", "cantilever", 0, out, "mixed" if mixed else "fp64")
    assert rc == 0, err
    raw = out.read_bytes()
    its = int(np.frombuffer(raw[:4], dtype=np.int32)[0])
    u = np.frombuffer(raw[12:], dtype=np.float64)
    model = M.cantilever_model()
    solver = M.SolverPCG(ctx, model, max_iterations=20000, tolerance=1e-10, precision="mixed" if mixed else "fp64")
    static = M.StaticAnalyzer(M.ProblemStructural(ctx, model), M.LinearAnalyzer(solver))
    static.BuildMatrices()
    static.Initialize()
    static.Solve()
    assert its == solver.iterations
    assert np.array_equal(u, model.subdomains[0].Solution)
    X = model.xyz[model.conn].reshape(-1, 24)
    Ke, st = O.h8_stiffness_batch(X, model.E_elem, model.poisson)
    assert st == 0
    S = O.Skyline(model.conn, model.dof, model.n_dofs)
    S.assemble(Ke)
    F, _ = S.factorized()
    us = S.solve(F, model.subdomains[0].RHS)
    assert np.abs(u - us).max() <= 1e-8 * np.abs(us).max()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_monte_carlo_matches_python_mirror(ctx, driver, tmp_path, mode):
    n, R, terms = 6, 8, 12
    xi = np.random.default_rng(17).standard_normal((R, terms))
    xi_path = tmp_path / "xi.bin"
    xi_path.write_bytes(xi.tobytes())
    out = tmp_path / "mc.bin"
    rc, err = run(driver, "mc", n, R, terms, xi_path, out, mode)
    assert rc == 0, err
    raw = np.frombuffer(out.read_bytes(), dtype=np.uint8)
    tip = raw[:8 * R].view(np.float64)
    res = raw[8 * R:16 * R].view(np.float64)
    its = raw[16 * R:20 * R].view(np.int32)
    X = raw[20 * R:].view(np.float64).reshape(R, -1)
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, terms, 6)
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=terms, simulations=R, mode=mode,
                                                    tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    assert np.array_equal(tip, mc.TipValues) and np.array_equal(res, mc.Residuals)
    assert np.array_equal(its, mc.Iterations) and np.array_equal(X, mc.Solutions)


@pytest.mark.gpu
def test_ragged_batch_matches_python_mirror(ctx, driver, tmp_path):
    """C++ RaggedMonteCarloBatch (a lattice and a block with moved interior
    nodes) returns the same bits as the Python mirror's batch."""
    n1, n2, R, terms = 5, 4, 3, 6
    xi = np.random.default_rng(31).standard_normal((2, R, terms))
    xi_path = tmp_path / "xi.bin"
    xi_path.write_bytes(xi.tobytes())
    out = tmp_path / "rg.bin"
    rc, err = run(driver, "ragged", n1, n2, R, terms, xi_path, out)
    assert rc == 0, err
    m1, m2 = M.clamped_block_model(n1), M.clamped_block_model(n2)
    hi = m2.xyz.max()
    inner = np.flatnonzero(((m2.xyz > 0.5) & (m2.xyz < hi - 0.5)).all(axis=1))
    for i in inner:  # the driver's move_interior: exact binary fractions
        m2.xyz[i] += 0.0625 * (((7 * i + 3 * np.arange(3)) % 5) - 2)
    batch = M.RaggedMonteCarloBatch(ctx, tolerance=1e-10)
    for m, n, x in ((m1, n1, xi[0]), (m2, n2, xi[1])):
        batch.add(m, M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, terms, 6), x)
    res = batch.Solve()
    raw = out.read_bytes()
    off = 0
    for m, r in zip((m1, m2), res):
        tip = np.frombuffer(raw, np.float64, R, off); off += 8 * R
        rel = np.frombuffer(raw, np.float64, R, off); off += 8 * R
        its = np.frombuffer(raw, np.int32, R, off); off += 4 * R
        X = np.frombuffer(raw, np.float64, R * m.n_dofs, off).reshape(R, -1); off += 8 * R * m.n_dofs
        assert np.array_equal(tip, r["TipValues"]) and np.array_equal(rel, r["Residuals"])
        assert np.array_equal(its, r["Iterations"]) and np.array_equal(X, r["Solutions"])
    assert off == len(raw)


@pytest.mark.gpu
def test_newmark_matches_python_mirror(ctx, driver, tmp_path):
    n, R, terms, steps = 4, 3, 12, 10
    xi = np.random.default_rng(23).standard_normal((R, terms))
    xi_path = tmp_path / "xi.bin"
    xi_path.write_bytes(xi.tobytes())
    out = tmp_path / "nm.bin"
    rc, err = run(driver, "newmark", n, R, terms, xi_path, steps, out)
    assert rc == 0, err
    raw = np.frombuffer(out.read_bytes(), dtype=np.float64)
    hist, U = raw[:R * steps].reshape(R, steps), raw[R * steps:].reshape(R, -1)
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, terms, 6)
    dt = 0.01
    load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * steps, 0.1, dof=0)
    nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * steps, load, expansion_order=terms,
                                  simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                  tolerance=1e-10)
    nm.RandomNumbers = xi
    h = nm.Solve()
    assert np.array_equal(hist, h) and np.array_equal(U, nm.Solutions)


@pytest.mark.gpu
def test_newmark_guard_raises_invalid_operation(driver):
    rc, err = run(driver, "guard")
    assert rc == 3 and "Newmark alpha has to be bigger than 0.25" in err, err


@pytest.mark.gpu
def test_server_matches_python_mirror(ctx, driver, tmp_path):
    """Two models served side by side through the C++ Server: every request
    returns the bits the Python server returns for the same realization (a
    request's arithmetic does not depend on the mix)."""
    from msolve_b200.serving import Server
    n1, n2, R, terms = 6, 10, 5, 12
    xi = np.random.default_rng(29).standard_normal((2, R, terms))
    xi_path = tmp_path / "xi.bin"
    xi_path.write_bytes(xi.tobytes())
    out = tmp_path / "serve.bin"
    rc, err = run(driver, "serve", n1, n2, R, terms, xi_path, out)
    assert rc == 0, err
    raw = out.read_bytes()
    srv = Server(ctx, max_batch=32)
    try:
        off = 0
        for k, n in enumerate((n1, n2)):
            model = M.clamped_block_model(n)
            kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, terms, 6)
            m = srv.add_model(model, kl, tol=1e-10)
            for r in range(R):
                its = int(np.frombuffer(raw[off:off + 4], dtype=np.int32)[0])
                res = float(np.frombuffer(raw[off + 4:off + 12], dtype=np.float64)[0])
                X = np.frombuffer(raw[off + 12:off + 12 + 8 * model.n_dofs], dtype=np.float64)
                off += 12 + 8 * model.n_dofs
                py = srv.poll(srv.submit(m, xi[k, r]), timeout_ms=-1)
                assert its == py["iterations"] and res == py["rel_res"] and np.array_equal(X, py["X"])
        assert off == len(raw)
    finally:
        srv.stop()


def test_status_codes_map_to_reference_exceptions(driver):
    r = subprocess.run([driver, "errors"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    kinds = dict(line.split() for line in r.stdout.splitlines())
    inv, arg, other = "InvalidOperationException", "ArgumentException", "MSolveException"
    assert kinds == {"-2001": inv, "-2002": inv, "-1001": inv, "-2007": inv, "-2005": arg, "-100": other,
                     "-2003": other, "-2006": other}


def test_kl_table_matches_python_provider(driver, tmp_path):
    n, terms = 8, 20
    out = tmp_path / "kl.bin"
    rc, err = run(driver, "kl", n, terms, out)
    assert rc == 0, err
    raw = out.read_bytes()
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, terms, 6)
    o = 0
    for arr, dt in ((kl.w, np.float64), (kl.amp, np.float64), (kl.idx, np.int32), (kl.eig, np.float64)):
        nb = arr.size * np.dtype(dt).itemsize
        got = np.frombuffer(raw[o:o + nb], dtype=dt).reshape(arr.shape)
        assert np.array_equal(got, arr)
        o += nb
    assert o == len(raw)


@pytest.mark.gpu
def test_reorthogonalized_solver_matches_python_mirror(ctx, driver, tmp_path):
    model = M.cantilever_model()
    b0 = model.subdomains[0].RHS.copy()
    rng = np.random.default_rng(31)
    loads = np.stack([b0, 2.0 * b0, b0 + 0.01 * np.abs(b0).max() * rng.standard_normal(model.n_dofs)])
    b_path = tmp_path / "b.bin"
    b_path.write_bytes(loads.tobytes())
    out = tmp_path / "reorth.bin"
    rc, err = run(driver, "reorth", b_path, out)
    assert rc == 0, err
    raw = out.read_bytes()
    provider = M.ProblemStructural(ctx, model)
    K = provider.CalculateMatrix()
    search = M.SolverPCGReorthogonalizationSearchVectorCalculator(provider.mesh, 400)
    solver = M.SolverPCGReorthogonalized(ctx, model, search, tolerance=1e-10)
    solver.matrix = K
    off = 0
    for k in range(3):
        its, count = np.frombuffer(raw[off:off + 8], dtype=np.int32)
        x = np.frombuffer(raw[off + 8:off + 8 + 8 * model.n_dofs], dtype=np.float64)
        off += 8 + 8 * model.n_dofs
        model.subdomains[0].Forces = loads[k]
        xp = solver.Solve(start_from_store=0 if k == 0 else 1)
        assert its == solver.iterations and count == search.count and np.array_equal(x, xp)
    assert off == len(raw)


@pytest.mark.gpu
def test_stress_batch_matches_python_mirror(ctx, driver, tmp_path):
    model = M.cantilever_model()
    u = np.random.default_rng(37).standard_normal((model.n_elems, 24))
    u_path = tmp_path / "u.bin"
    u_path.write_bytes(u.tobytes())
    out = tmp_path / "stress.bin"
    rc, err = run(driver, "stress", u_path, out)
    assert rc == 0, err
    raw = np.frombuffer(out.read_bytes(), dtype=np.float64)
    ne = model.n_elems
    eps, sig, f = raw[:ne * 48], raw[ne * 48:ne * 96], raw[ne * 96:]
    e2, s2, f2 = M.h8_stress_batch(ctx, model.xyz[model.conn], model.E_elem, model.poisson, u)
    assert np.array_equal(eps, e2.ravel()) and np.array_equal(sig, s2.ravel()) and np.array_equal(f, f2.ravel())


@pytest.mark.gpu
def test_galerkin_product_matches_python_mirror(ctx, driver, tmp_path):
    n, m, p = 4, 2, 2
    model = M.clamped_block_model(n)
    kl = M.GaussianStochasticCoefficientsProvider([n, n, n], 0.3 * n, max(m, 4), 8, mean=2.0, covariance=0.15)
    op = M.PolynomialChaosSolverPCGMatrixCalculator(M.GpuMesh(ctx, model), kl, m, p)
    u = np.random.default_rng(41).standard_normal((op.PsiSize, model.n_dofs))
    u_path = tmp_path / "u.bin"
    u_path.write_bytes(u.tobytes())
    out = tmp_path / "pc.bin"
    rc, err = run(driver, "pc", n, m, p, u_path, out)
    assert rc == 0, err
    y = np.frombuffer(out.read_bytes(), dtype=np.float64).reshape(op.PsiSize, -1)
    assert np.array_equal(y, op.MultiplyWithMatrix(u))
