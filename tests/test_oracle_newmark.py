"""CPU checks of the oracle's Newmark restatement (NewmarkDynamicAnalyzer.cs):
the direct (skyline LDL^T) and iterative (Jacobi PCG) step solves agree, the
response is linear in the ground-acceleration amplitude, zero load stays at
rest, and the coefficient guards of InitializeCoefficients hold."""
import numpy as np

import msolve_b200 as M
import oracle as O


def _block(n=3):
    xyz, conn = O.block_mesh(n, n, n, 1.0)
    cons = O.clamp_face(xyz, 2, 0.0)
    dof, N = O.enumerate_dofs(cons)
    E = np.exp(0.3 * np.random.default_rng(0).standard_normal(conn.shape[0]))
    tip = dof[np.argmax(xyz.sum(1)), 0]
    return xyz, conn, cons, dof, N, E, tip


def _run(n, cons, E, N, tip, amp=0.1, solver=0, steps=40, f=None):
    return O.block_newmark(n, n, n, cons, E, 0.3, 1.0, 0.01, 0.001, 0.25, 0.5, 0.01, steps, amp, 1.0, 0, N,
                           f_static=f, solver=solver, tol=1e-12, tip_dof=tip)


def test_direct_and_pcg_steps_agree():
    _, _, cons, _, N, E, tip = _block()
    t0, u0, i0 = _run(3, cons, E, N, tip)
    t1, u1, i1 = _run(3, cons, E, N, tip, solver=1)
    assert i0["status"] == 0 and i1["status"] == 0 and i1["iterations"] > 0
    assert np.abs(t0 - t1).max() <= 1e-8 * np.abs(t0).max()
    assert np.abs(u0 - u1).max() <= 1e-8 * np.abs(u0).max()


def test_linear_in_amplitude_and_rest_without_load():
    _, _, cons, _, N, E, tip = _block()
    t1, _, _ = _run(3, cons, E, N, tip, amp=0.1)
    t2, _, _ = _run(3, cons, E, N, tip, amp=0.2)
    assert np.abs(t2 - 2 * t1).max() <= 1e-12 * np.abs(t2).max()
    t0, u0, _ = _run(3, cons, E, N, tip, amp=0.0)
    assert np.abs(t0).max() == 0.0 and np.abs(u0).max() == 0.0
    # the first step has a_g(0) = sin(0) = 0 and starts at rest
    assert t1[0] == 0.0 and t1[1] != 0.0


def test_coefficient_guards():
    _, _, cons, _, N, E, tip = _block()
    st = O.block_newmark(3, 3, 3, cons, E, 0.3, 1.0, 0, 0, 0.25, 0.4, 0.01, 2, 0.1, 1.0, 0, N)[2]["status"]
    assert st != 0  # delta < 0.5
    st = O.block_newmark(3, 3, 3, cons, E, 0.3, 1.0, 0, 0, 0.2, 0.5, 0.01, 2, 0.1, 1.0, 0, N)[2]["status"]
    assert st != 0  # alpha below (0.5 + delta)^2 / 4


def test_sinusoidal_load_history():
    ld = M.MassAccelerationSinusoidalLoad(1.0, 0.01, 2.0, 0.1, dof=0)
    assert ld.time_steps == 200
    assert ld[0] == 0.0 and abs(ld[25] - 0.1) < 1e-15 and ld[200] == 0.0
