"""GPU test of MSG_PCG_SOLVE_NOALLOC, the PCG solve that allocates no device
memory (for callers that cannot afford cudaMalloc/cudaFree while solving:
those calls synchronise the whole device, and a host that gives the library a
fixed share of device memory may forbid them). Through the C ABI it must give
the same displacements and iteration counts as MSG_PCG_SOLVE, call after call
(the shared scratch array keeps the previous call's contents), leave the
device's free memory unchanged, return MSG_PCG_SOLVE's status and outputs when
the iteration limit is reached, and reject meshes larger than its fixed
scratch.

Collected last (file name) so a stop-at-first-failure run has run every other
test before it; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import msolve_b200 as M
from msolve_b200 import _native as N

pytestmark = pytest.mark.gpu


def _noalloc_call(torch, A, b_dev, x_dev, tol, max_it=20000):
    """One MSG_PCG_SOLVE_NOALLOC call on preallocated device buffers. The
    right-hand side is complete before the call (the entry point runs on the
    context's own stream, which does not wait for torch's stream)."""
    x_dev.fill_(float("nan"))  # must be overwritten
    torch.cuda.synchronize()
    it, rr = C.c_int(0), C.c_double(0)
    st = N.lib().MSG_PCG_SOLVE_NOALLOC(A.handle, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()), max_it,
                                      tol, C.byref(it), C.byref(rr))
    return st, it.value, rr.value


def _noalloc_solve(torch, A, b, tol, max_it=20000):
    b_dev = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_dev = torch.empty_like(b_dev)
    st, its, rr = _noalloc_call(torch, A, b_dev, x_dev, tol, max_it)
    return st, x_dev.cpu().numpy(), its, rr


def _pcg_solve(A, b, tol, max_it):
    """MSG_PCG_SOLVE through the C ABI with host buffers: status, x, iterations,
    relative residual."""
    x = np.zeros_like(b)
    it, rr = C.c_int(0), C.c_double(0)
    st = N.lib().MSG_PCG_SOLVE(A.handle, N.ptr(b), N.ptr(x), max_it, tol, C.byref(it), C.byref(rr))
    return st, x, it.value, rr.value


def test_noalloc_pcg_matches_pcg_solve_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    ctx = M.Context(0)
    rng = np.random.default_rng(17)
    cases = []
    m1 = M.clamped_block_model(10)
    cases.append((m1, np.exp(0.3 * rng.standard_normal(m1.n_elems)), 1e-10))
    m2 = M.cantilever_model()
    cases.append((m2, m2.E_elem, 1e-10))
    for model, E, tol in cases:
        A = M.GpuMesh(ctx, model).assemble(E, model.poisson)
        b0 = model.subdomains[0].RHS.copy()
        for call in range(2):  # two calls in a row, different right-hand sides
            b = b0 * (1.0 + call) + (0.0 if call == 0 else 1e-3 * rng.standard_normal(b0.shape[0]))
            st_ref, x_ref, its_ref, rr_ref = _pcg_solve(A, b, tol, 20000)
            assert st_ref == 0
            st, x, its, rr = _noalloc_solve(torch, A, b, tol)
            assert st == 0, N.lib().MSG_LAST_ERROR(ctx.handle)
            assert its == its_ref
            assert np.isfinite(x).all()
            assert np.abs(x - x_ref).max() <= 1e-12 * np.abs(x_ref).max()
            assert abs(rr - rr_ref) <= 1e-12 * max(rr, 1e-300) + 1e-300


def test_noalloc_pcg_allocates_nothing_on_a_fresh_matrix():
    """On a matrix that MSG_PCG_SOLVE never touched (so none of its workspace
    exists), a warm call leaves the device's free memory unchanged, and the
    result still equals MSG_PCG_SOLVE's."""
    torch = pytest.importorskip("torch")
    ctx = M.Context(0)
    model = M.clamped_block_model(9)
    E = np.exp(0.3 * np.random.default_rng(5).standard_normal(model.n_elems))
    A = M.GpuMesh(ctx, model).assemble(E, model.poisson)
    b = model.subdomains[0].RHS.copy()
    b_dev = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_dev = torch.empty_like(b_dev)
    st, _, _ = _noalloc_call(torch, A, b_dev, x_dev, 1e-10)  # first call: kernels loaded
    assert st == 0, N.lib().MSG_LAST_ERROR(ctx.handle)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st, its, rr = _noalloc_call(torch, A, b_dev, x_dev, 1e-10)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert st == 0
    assert free1 == free0, (free0, free1)
    x = x_dev.cpu().numpy()
    st_ref, x_ref, its_ref, rr_ref = _pcg_solve(A, b, 1e-10, 20000)
    assert st_ref == 0 and its == its_ref
    assert np.abs(x - x_ref).max() <= 1e-12 * np.abs(x_ref).max()


def test_noalloc_pcg_not_converged_matches_pcg_solve():
    """Iteration limit reached: MSG_ERR_NOT_CONVERGED, iterations == max_it, the
    same relative residual, displacements and error message as MSG_PCG_SOLVE."""
    torch = pytest.importorskip("torch")
    ctx = M.Context(0)
    model = M.clamped_block_model(8)
    A = M.GpuMesh(ctx, model).assemble(model.E_elem, model.poisson)
    b = model.subdomains[0].RHS.copy()
    st_ref, x_ref, its_ref, rr_ref = _pcg_solve(A, b, 1e-14, 3)
    msg_ref = N.lib().MSG_LAST_ERROR(ctx.handle)
    assert st_ref == N.MSG_ERR_NOT_CONVERGED and its_ref == 3
    for _ in range(2):
        st, x, its, rr = _noalloc_solve(torch, A, b, 1e-14, max_it=3)
        assert st == N.MSG_ERR_NOT_CONVERGED
        assert N.lib().MSG_LAST_ERROR(ctx.handle) == msg_ref
        assert its == 3
        assert abs(rr - rr_ref) <= 1e-12 * rr_ref
        assert np.isfinite(x).all()
        assert np.abs(x - x_ref).max() <= 1e-12 * np.abs(x_ref).max()


def test_noalloc_pcg_rejects_meshes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    ctx = M.Context(0)
    model = M.clamped_block_model(41)  # 42^3 = 74,088 nodes > 65,536
    A = M.GpuMesh(ctx, model).assemble(model.E_elem, model.poisson)
    st, x, its, rr = _noalloc_solve(torch, A, model.subdomains[0].RHS, 1e-8, max_it=10)
    assert st == N.MSG_ERR_INVALID_ARGUMENT
    assert b"65536" in N.lib().MSG_LAST_ERROR(ctx.handle)
