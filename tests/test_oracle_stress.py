"""Oracle stress recovery (CalcH8Strains / CalcH8Forces with the elastic
material update), pinned by properties that hold exactly in exact arithmetic:
internal forces equal K_e du, rigid-body motions carry no strain, a uniform
strain field is reproduced at every Gauss point (patch test), and the
stresses are D times the strain increment."""
import numpy as np

import oracle as O


def _elements(n, seed=0, jitter=0.08):
    rng = np.random.default_rng(seed)
    xyz, conn = O.block_mesh(1, 1, 1, 1.0)
    base = xyz[conn].reshape(1, 24)
    return base + jitter * rng.standard_normal((n, 24)), rng


def test_forces_equal_element_stiffness_times_increment():
    X, rng = _elements(20)
    E = np.exp(0.3 * rng.standard_normal(20))
    u = rng.standard_normal((20, 24))
    du = rng.standard_normal((20, 24))
    eps, sig, f, st = O.h8_stress_batch(X, E, 0.3, u, du)
    assert st == 0
    for e in range(20):
        K = O.unpack300(O.h8_stiffness(X[e], E[e], 0.3)[0])
        ref = K @ du[e]
        assert np.abs(f[e] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_rigid_motion_has_no_strain_and_uniform_strain_is_exact():
    X, rng = _elements(10, seed=1)
    for e in range(10):
        x8 = X[e].reshape(8, 3)
        W = rng.standard_normal((3, 3))
        W = W - W.T  # infinitesimal rotation
        t = rng.standard_normal(3)
        rigid = (x8 @ W.T + t).reshape(24)
        eps, _, _, _ = O.h8_stress_batch(X[e], 1.0, 0.3, rigid)
        assert np.abs(eps).max() <= 1e-13 * np.abs(rigid).max()
        G = rng.standard_normal((3, 3))
        uu = (x8 @ G.T).reshape(24)
        eps, _, _, _ = O.h8_stress_batch(X[e], 1.0, 0.3, uu)
        expect = np.array([G[0, 0], G[1, 1], G[2, 2], G[0, 1] + G[1, 0], G[1, 2] + G[2, 1], G[2, 0] + G[0, 2]])
        assert np.abs(eps[0] - expect).max() <= 1e-13 * np.abs(G).max()


def test_stresses_are_D_times_increment_strains():
    X, rng = _elements(5, seed=2)
    u = rng.standard_normal((5, 24))
    du = rng.standard_normal((5, 24))
    _, sig, _, _ = O.h8_stress_batch(X, 2.5, 0.25, u, du)
    deps, _, _, _ = O.h8_stress_batch(X, 2.5, 0.25, du)
    D = O.elastic_D(2.5, 0.25).reshape(6, 6)
    assert np.abs(sig - deps @ D.T).max() <= 1e-13 * np.abs(sig).max()
    _, sig_u, _, _ = O.h8_stress_batch(X, 2.5, 0.25, u)
    eps_u, _, _, _ = O.h8_stress_batch(X, 2.5, 0.25, u)
    assert np.abs(sig_u - eps_u @ D.T).max() <= 1e-13 * np.abs(sig_u).max()
