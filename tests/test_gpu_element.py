"""GPU parity of the batched Hexa8 element kernels against the oracle and the
exact closed form (FP64, 1e-12 relative)."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu

CUBE = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], float)


def test_stiffness_matches_exact_closed_form(ctx, golden):
    for key in ("unit_cube", "parallelepiped"):
        d = golden[key]
        K = M.h8_stiffness_batch(ctx, np.array(d["xyz"])[None], d["E"], d["nu"])[0]
        Kx = np.array(d["K300"])
        assert np.abs(K - Kx).max() <= 1e-12 * np.abs(Kx).max(), key


def test_stiffness_batch_matches_oracle_on_distorted_elements(ctx):
    rng = np.random.default_rng(11)
    n = 1000
    xyz = np.stack([CUBE * rng.uniform(0.5, 2.0, 3) + rng.uniform(-0.15, 0.15, (8, 3)) for _ in range(n)])
    E = rng.uniform(0.5, 3.0, n)
    K = M.h8_stiffness_batch(ctx, xyz, E, 0.27)
    Ko, st = O.h8_stiffness_batch(xyz.reshape(n, 24), E, 0.27)
    assert st == 0
    err = np.abs(K - Ko).max(axis=1) / np.abs(Ko).max(axis=1)
    assert err.max() <= 1e-12


def test_stiffness_of_a_mesh_matches_oracle(ctx):
    m = M.clamped_block_model(5)
    rng = np.random.default_rng(3)
    E = np.exp(0.3 * rng.standard_normal(m.n_elems))
    K = M.h8_stiffness_batch(ctx, m.element_xyz(), E, 0.3)
    Ko, _ = O.h8_stiffness_batch(m.element_xyz(), E, 0.3)
    assert np.abs(K - Ko).max() <= 1e-12 * np.abs(Ko).max()


def test_negative_determinant_raises(ctx):
    bad = CUBE[[1, 0, 3, 2, 5, 4, 7, 6]]
    with pytest.raises(M.InvalidOperationError) as e:
        M.h8_stiffness_batch(ctx, np.stack([CUBE, bad]), 1.0, 0.3)
    assert e.value.code == -1001


def test_invalid_poisson_ratio_raises(ctx):
    with pytest.raises(M.ArgumentError):
        M.h8_stiffness_batch(ctx, CUBE[None], 1.0, 0.5)


def test_empty_batch_is_a_no_op(ctx):
    assert M.h8_stiffness_batch(ctx, np.zeros((0, 24)), np.zeros(0), 0.3).shape == (0, 300)


def test_consistent_mass_matches_oracle(ctx):
    rng = np.random.default_rng(4)
    xyz = np.stack([CUBE * rng.uniform(0.5, 2.0, 3) + rng.uniform(-0.1, 0.1, (8, 3)) for _ in range(64)])
    Mm = M.h8_mass_batch(ctx, xyz, 1.7)
    for e in range(64):
        Mo, st = O.h8_consistent_mass(xyz[e], 1.7)
        assert st == 0
        assert np.abs(Mm[e] - Mo).max() <= 1e-12 * np.abs(Mo).max()
