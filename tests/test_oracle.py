"""CPU tests of the oracle (the C++ restatement of the reference): pinned to
closed-form known answers and cross-checked between its independent paths."""
import numpy as np
import pytest

import oracle as O


def test_golden_exact_stiffness_pins_both_restatements(golden):
    for key in ("unit_cube", "parallelepiped"):
        d = golden[key]
        K = np.array(d["K300"])
        for path in ("fortran", "csharp"):
            Ko, st = O.h8_stiffness(np.array(d["xyz"]), d["E"], d["nu"], path)
            assert st == 0
            # 13-digit Gauss literal of the reference -> ~5e-14 relative
            assert np.abs(Ko - K).max() <= 1e-12 * np.abs(K).max(), (key, path)


def random_hexa(rng, amp=0.15):
    c = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], float)
    return c * rng.uniform(0.5, 2.0, 3) + rng.uniform(-amp, amp, (8, 3))


def test_fortran_and_csharp_paths_agree_on_distorted_elements():
    rng = np.random.default_rng(1)
    for _ in range(50):
        x = random_hexa(rng)
        E, nu = rng.uniform(0.5, 5.0), rng.uniform(0.0, 0.45)
        Kf, s1 = O.h8_stiffness(x, E, nu, "fortran")
        Kc, s2 = O.h8_stiffness(x, E, nu, "csharp")
        assert s1 == 0 and s2 == 0
        assert np.abs(Kf - Kc).max() <= 1e-13 * np.abs(Kf).max()


def test_rigid_body_null_space_and_spd():
    rng = np.random.default_rng(2)
    for _ in range(10):
        x = random_hexa(rng)
        K = O.unpack300(O.h8_stiffness(x, 1.0, 0.3)[0])
        modes = []
        for c in range(3):
            v = np.zeros((8, 3)); v[:, c] = 1; modes.append(v.ravel())
        for a, b in ((0, 1), (1, 2), (2, 0)):
            v = np.zeros((8, 3)); v[:, a] = -x[:, b]; v[:, b] = x[:, a]; modes.append(v.ravel())
        for m in modes:
            assert np.abs(K @ m).max() <= 1e-12 * np.abs(K).max() * np.abs(m).max()
        ev = np.linalg.eigvalsh(K)
        assert (ev[6:] > 1e-8 * ev[-1]).all()


def test_negative_determinant_is_reported():
    x = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], float)
    x = x[[1, 0, 3, 2, 5, 4, 7, 6]]  # mirrored node order -> negative Jacobian
    assert O.h8_stiffness(x, 1.0, 0.3, "fortran")[1] == -1001
    assert O.h8_stiffness(x, 1.0, 0.3, "csharp")[1] == -1001


def test_patch_test_uniform_strain():
    """A linear displacement field gives element forces that cancel at shared nodes."""
    xyz, conn = O.block_mesh(2, 2, 2)
    Ke, st = O.h8_stiffness_batch(O.element_xyz(xyz, conn), 1.0, 0.3)
    dof = np.arange(3 * xyz.shape[0], dtype=np.int32).reshape(-1, 3)
    C = O.CSR(xyz.shape[0], conn, dof, 3 * xyz.shape[0])
    C.assemble(Ke)
    G = np.array([[1e-3, 2e-4, 0], [0, -5e-4, 1e-4], [3e-4, 0, 2e-3]])
    u = (xyz @ G.T).ravel()
    f = C.multiply(u).reshape(-1, 3)
    interior = np.all((xyz > 0) & (xyz < 2), axis=1)
    assert np.abs(f[interior]).max() < 1e-14


def test_consistent_mass_total():
    rng = np.random.default_rng(3)
    x = random_hexa(rng)
    M = O.unpack300(O.h8_consistent_mass(x, 2.5)[0])
    g = O.h8_gauss_matrices(x)
    vol = g["weight"].sum()
    for c in range(3):
        assert abs(M[c::3, c::3].sum() - 2.5 * vol) < 1e-12 * 2.5 * vol
    assert np.allclose(M[0::3, 1::3], 0)


def cantilever():
    xyz, conn = O.block_mesh(10, 4, 4)
    cons = O.clamp_face(xyz, 0, 0.0)
    dof, N = O.enumerate_dofs(cons)
    b = O.load_tip(xyz, dof, N, 0, 2, -1.0)
    Ke, _ = O.h8_stiffness_batch(O.element_xyz(xyz, conn), 1.0, 0.3)
    return xyz, conn, dof, N, b, Ke


def test_cantilever_skyline_ldlt_vs_jacobi_pcg():
    xyz, conn, dof, N, b, Ke = cantilever()
    assert N == 750
    S = O.Skyline(conn, dof, N)
    S.assemble(Ke)
    F, zems = S.factorized(1e-15)
    assert zems == 0
    xs = S.solve(F, b)
    Cs = O.CSR(xyz.shape[0], conn, dof, N)
    Cs.assemble(Ke)
    assert np.abs(S.multiply(b) - Cs.multiply(b)).max() < 1e-15
    assert np.abs(S.multiply(xs) - b).max() < 1e-10 * np.abs(b).max()
    xp, info = Cs.pcg_jacobi(b, tol=1e-10)
    assert info["status"] == 0 and info["matvecs"] == info["iterations"] + 1
    assert np.abs(xs - xp).max() <= 1e-8 * np.abs(xs).max()
    # LDL^T-preconditioned PCG (the Monte Carlo calculator) converges in one product
    xq, info2 = S.pcg(b, F, tol=1e-10)
    assert info2["matvecs"] == 1 and np.abs(xq - xs).max() <= 1e-12 * np.abs(xs).max()


def test_monte_carlo_first_realization_factor_preconditions_the_others():
    """The reference's Monte Carlo solver (MonteCarloSolverPCGDirectMatrixCalculator.cs:38-80):
    the skyline LDL^T of the first realization's K preconditions PCG on every later
    realization (matvec: that realization's skyline product). It reaches the
    Jacobi-PCG solution of each realization in far fewer iterations."""
    n = 6
    P = O.block_problem(n, 20, 8)
    xi = np.random.default_rng(4).standard_normal((3, 20))
    E = O.kl_field(P["centroids"], P["domain"], P["table"], xi, sigma=0.3)
    S = O.Skyline(P["conn"], P["dof"], P["n_dofs"])
    exyz = O.element_xyz(P["xyz"], P["conn"])
    S.assemble(O.h8_stiffness_batch(exyz, E[0], 0.3)[0])
    F, zems = S.factorized(1e-8)
    assert zems == 0
    for r in (1, 2):
        S.assemble(O.h8_stiffness_batch(exyz, E[r], 0.3)[0])
        x, info = S.pcg(P["b"], F, tol=1e-10)
        xj, ij = O.block_solve_pcg(n, n, n, P["constrained"], E[r], 0.3, P["b"], tol=1e-10)
        assert info["status"] == 0 and ij["status"] == 0
        assert info["iterations"] * 4 < ij["iterations"]
        assert np.abs(x - xj).max() <= 1e-8 * np.abs(xj).max()


def test_skyline_row_index_quirk():
    """rowIndex[1] = 1 is hard-coded (GlobalMatrixAssemblerSkyline.cs:40)."""
    xyz, conn, dof, N, b, Ke = cantilever()
    S = O.Skyline(conn, dof, N)
    assert S.ri[0] == 0 and S.ri[1] == 1


def test_kl_1d_modes_solve_the_eigen_equations_and_are_orthonormal():
    A, l = 16.0, 6.4
    w, a, lam = O.kl_1d_modes(A, l, 12)
    c = 1 / l
    for k in range(12):
        if (k + 1) % 2:
            assert abs(c * np.cos(w[k] * A) - w[k] * np.sin(w[k] * A)) < 1e-10
        else:
            assert abs(w[k] * np.cos(w[k] * A) + c * np.sin(w[k] * A)) < 1e-10
    assert (np.diff(lam) < 0).all()
    x = np.linspace(-A, A, 200001)
    phi = np.array([a[k] * (np.sin(w[k] * x) if (k + 1) % 2 == 0 else np.cos(w[k] * x)) for k in range(6)])
    G = np.trapezoid(phi[:, None, :] * phi[None, :, :], x, axis=2)
    assert np.abs(G - np.eye(6)).max() < 1e-6
    # eigen-equation of the integral operator at a sample point
    K = np.exp(-np.abs(x[:, None][::4000] - x[None, :]) / l)
    lhs = np.trapezoid(K * phi[2][None, :], x, axis=1)
    assert np.abs(lhs - lam[2] * phi[2][::4000]).max() < 1e-4


def test_kl_field_mean_and_reference_form():
    xyz, conn = O.block_mesh(8, 8, 8)
    cen = O.centroids(xyz, conn)
    tab = O.kl_table([8, 8, 8], 1.6, 20, 8)
    assert (np.diff(tab["eig"]) <= 1e-12 * tab["eig"][0]).all()
    xi = np.zeros((1, 20))
    E = O.kl_field(cen, [8, 8, 8], tab, xi, mean=2.0, sigma=0.3, mean_correction=True)
    assert np.allclose(E, 2.0 * np.exp(-0.045))
    E = O.kl_field(cen, [8, 8, 8], tab, xi, mean=1.0, sigma=0.3)
    assert np.allclose(E, 1.0)
    rng = np.random.default_rng(0)
    xi = rng.standard_normal((400, 20))
    g = np.log(O.kl_field(cen, [8, 8, 8], tab, xi, sigma=0.3)) / 0.3
    # variance captured by 20 terms of a unit-variance field stays below 1
    v = g.var(axis=0).mean()
    assert 0.2 < v < 1.0


def test_block_solve_matches_dense_solution():
    xyz, conn = O.block_mesh(3, 3, 3)
    cons = O.clamp_face(xyz, 2, 0.0)
    dof, N = O.enumerate_dofs(cons)
    b = O.load_top_pressure(xyz, dof, N)
    rng = np.random.default_rng(5)
    E = np.exp(0.3 * rng.standard_normal(conn.shape[0]))
    x, info = O.block_solve_pcg(3, 3, 3, cons, E, 0.3, b, tol=1e-12)
    Ke, _ = O.h8_stiffness_batch(O.element_xyz(xyz, conn), E, 0.3)
    C = O.CSR(xyz.shape[0], conn, dof, N)
    C.assemble(Ke)
    rows = np.repeat(np.arange(N), np.diff(C.rp))
    Kd = np.zeros((N, N))
    Kd[rows, C.ci] = C.val
    xd = np.linalg.solve(Kd, b)
    assert info["status"] == 0
    assert np.abs(x - xd).max() <= 1e-10 * np.abs(xd).max()
    assert abs(b.sum() + 9.0) < 1e-12  # total pressure load = area
