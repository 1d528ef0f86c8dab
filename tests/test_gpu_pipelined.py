"""MSG_MC_SOLVE_BATCH_PIPELINED: the displacement copy of a batch overlaps the
next batch. Its results equal MSG_MC_SOLVE_BATCH's bit for bit; the X of a
call is complete when the next pipelined call returns (or after
MSG_MC_FLUSH); a plain call after pipelined ones flushes them first."""
import ctypes as C

import numpy as np
import pytest
import torch

import msolve_b200 as M
from msolve_b200 import _native as N

pytestmark = pytest.mark.gpu


def setup(n=6, R=40, K=20):
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, K, 8)
    rng = np.random.default_rng(9)
    return model, kl, [rng.standard_normal((R, K)) for _ in range(3)]


def call(fn, mesh, model, kls, xi, X_ptr, tol=1e-10):
    R = xi.shape[0]
    xi = N.f64(xi)
    b = N.f64(model.subdomains[0].RHS)
    tip, its, res = np.zeros(R), np.zeros(R, dtype=np.int32), np.zeros(R)
    st = fn(mesh.handle, float(model.poisson), C.byref(kls), R, N.ptr(xi), N.ptr(b), N.MSG_MODE_MIXED_BATCHED,
            100000, tol, M.tip_dof(model), X_ptr, N.ptr(tip), N.ptr(its, N._i), N.ptr(res))
    N.check(st, mesh.ctx.handle, "MC batch")
    return tip, its, res


def test_pipelined_batches_equal_plain_calls(ctx):
    model, kl, xis = setup()
    mesh = M.GpuMesh(ctx, model)
    kls = kl.struct()
    L = N.lib()
    R, nd = xis[0].shape[0], model.n_dofs
    ref = []
    for xi in xis:
        X = np.zeros((R, nd))
        ref.append((X,) + call(L.MSG_MC_SOLVE_BATCH, mesh, model, kls, xi, N.ptr(X)))
    bufs = [torch.zeros((R, nd), dtype=torch.float64).pin_memory() for _ in range(2)]
    for k, xi in enumerate(xis):
        X = bufs[k % 2]
        tip, its, res = call(L.MSG_MC_SOLVE_BATCH_PIPELINED, mesh, model, kls, xi,
                             C.cast(C.c_void_p(X.data_ptr()), N._d))
        assert np.array_equal(tip, ref[k][1]) and np.array_equal(its, ref[k][2]) and np.array_equal(res, ref[k][3])
        if k > 0:  # the previous call's displacements are on the host now
            assert np.array_equal(bufs[(k - 1) % 2].numpy(), ref[k - 1][0])
    N.check(L.MSG_MC_FLUSH(ctx.handle), ctx.handle, "MSG_MC_FLUSH")
    assert np.array_equal(bufs[(len(xis) - 1) % 2].numpy(), ref[-1][0])


def test_plain_call_after_pipelined_flushes(ctx):
    model, kl, xis = setup(n=5, R=33)
    mesh = M.GpuMesh(ctx, model)
    kls = kl.struct()
    L = N.lib()
    R, nd = xis[0].shape[0], model.n_dofs
    Xp = torch.zeros((R, nd), dtype=torch.float64).pin_memory()
    call(L.MSG_MC_SOLVE_BATCH_PIPELINED, mesh, model, kls, xis[0], C.cast(C.c_void_p(Xp.data_ptr()), N._d))
    X1 = np.zeros((R, nd))
    call(L.MSG_MC_SOLVE_BATCH, mesh, model, kls, xis[1], N.ptr(X1))
    X0 = np.zeros((R, nd))
    call(L.MSG_MC_SOLVE_BATCH, mesh, model, kls, xis[0], N.ptr(X0))
    assert np.array_equal(Xp.numpy(), X0)  # complete once the plain call returned
    assert not np.array_equal(X0, X1)
