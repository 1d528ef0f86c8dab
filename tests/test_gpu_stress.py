"""GPU parity of stress recovery (MSG_H8_STRESS_BATCH, MSG_STRESS_BATCH_DEVICE)
against the oracle's CalcH8Strains / CalcH8Forces restatement.

Tolerances: 1e-12 relative (max norm per output) on the same inputs (the
device contracts products into FMAs, the oracle does not); equilibrium of the
assembled internal forces of a converged batch with the load within 1e-8 of
||b|| (the solve stops at a true relative residual of 1e-10)."""
import numpy as np
import pytest

import msolve_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_element_batch_matches_oracle(ctx):
    rng = np.random.default_rng(3)
    xyz, conn = O.block_mesh(1, 1, 1, 1.0)
    n = 333
    X = xyz[conn].reshape(1, 24) + 0.08 * rng.standard_normal((n, 24))
    E = np.exp(0.3 * rng.standard_normal(n))
    u = rng.standard_normal((n, 24))
    du = rng.standard_normal((n, 24))
    for d in (None, du):
        eps, sig, f = M.h8_stress_batch(ctx, X, E, 0.3, u, d)
        eo, so, fo, st = O.h8_stress_batch(X, E, 0.3, u, d)
        assert st == 0
        assert _rel(eps, eo) <= 1e-12 and _rel(sig, so) <= 1e-12 and _rel(f, fo) <= 1e-12


def test_element_batch_rejects_bad_elements(ctx):
    xyz, conn = O.block_mesh(1, 1, 1, 1.0)
    X = xyz[conn].reshape(1, 24).copy()
    X[0, 3 * 6:3 * 7] = X[0, 0:3]  # collapse node 7 onto node 1
    with pytest.raises(M.InvalidOperationError):
        M.h8_stress_batch(ctx, X, 1.0, 0.3, np.zeros((1, 24)))


def test_realization_stresses_match_oracle_and_equilibrium(ctx):
    import torch
    n, R = 6, 12
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 12, 6)
    xi = np.random.default_rng(7).standard_normal((R, 12))
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=12, simulations=R, mode="mixed",
                                                    tolerance=1e-10)
    mc.RandomNumbers = xi
    mc.Solve()
    mesh = M.GpuMesh(ctx, model)
    E = kl.field(mesh, xi)
    dev = torch.device("cuda", 0)
    eps, sig, f = M.realization_stresses(mesh, torch.from_numpy(E).to(dev), model.poisson,
                                         torch.from_numpy(np.asarray(mc.Solutions)).to(dev))
    eps, sig, f = eps.cpu().numpy(), sig.cpu().numpy(), f.cpu().numpy()
    xyz_e = model.xyz[model.conn].reshape(-1, 24)
    for r in (0, R - 1):
        x = np.asarray(mc.Solutions[r])
        u = np.where(model.dof >= 0, x[np.maximum(model.dof, 0)], 0.0)[model.conn].reshape(-1, 24)
        eo, so, fo, st = O.h8_stress_batch(xyz_e, E[r], model.poisson, u)
        assert st == 0
        assert _rel(eps[r], eo) <= 1e-12 and _rel(sig[r], so) <= 1e-12 and _rel(f[r], fo) <= 1e-12
        # assembled internal forces balance the load at the free DOFs
        fint = np.zeros(model.n_dofs)
        d = model.dof[model.conn].reshape(-1, 24)
        ok = d >= 0
        np.add.at(fint, d[ok], f[r][ok])
        b = model.subdomains[0].RHS
        assert np.abs(fint - b).max() <= 1e-8 * np.abs(b).max()
