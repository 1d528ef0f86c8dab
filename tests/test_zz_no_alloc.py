"""GPU test of MSG_PCG_SOLVE_NOALLOC, the PCG solve that allocates no device
memory (for callers that cannot afford cudaMalloc/cudaFree while solving:
those calls synchronise the whole device, and a host that gives the library a
fixed share of device memory may forbid them). Through the C ABI it must give
the same displacements and iteration counts as MSG_PCG_SOLVE, call after call
(the shared scratch array keeps the previous call's contents), and reject
meshes larger than its fixed scratch.

Collected last (file name) so a stop-at-first-failure run has run every other
test before it; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import msolve_b200 as M
from msolve_b200 import _native as N

pytestmark = pytest.mark.gpu


def _noalloc_solve(torch, A, b, tol, max_it=20000):
    b_dev = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_dev = torch.full_like(b_dev, float("nan"))  # must be overwritten
    torch.cuda.synchronize()
    it, rr = C.c_int(0), C.c_double(0)
    st = N.lib().MSG_PCG_SOLVE_NOALLOC(A.handle, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()), max_it,
                                      tol, C.byref(it), C.byref(rr))
    torch.cuda.synchronize()
    return st, x_dev.cpu().numpy(), it.value, rr.value


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
        solver = M.SolverPCG(ctx, model)
        solver.matrix = A
        b0 = model.subdomains[0].RHS.copy()
        for call in range(2):  # two calls in a row, different right-hand sides
            b = b0 * (1.0 + call) + (0.0 if call == 0 else 1e-3 * rng.standard_normal(b0.shape[0]))
            model.subdomains[0].Forces = b
            x_ref = solver.Solve(20000, tol)
            st, x, its, rr = _noalloc_solve(torch, A, b, tol)
            assert st == 0, N.lib().MSG_LAST_ERROR(ctx.handle)
            assert its == solver.iterations
            assert np.isfinite(x).all()
            assert np.abs(x - x_ref).max() <= 1e-12 * np.abs(x_ref).max()
            assert abs(rr - solver.rel_res) <= 1e-12 * max(rr, 1e-300) + 1e-300
        model.subdomains[0].Forces = b0


def test_noalloc_pcg_rejects_meshes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    ctx = M.Context(0)
    model = M.clamped_block_model(41)  # 42^3 = 74,088 nodes > 65,536
    A = M.GpuMesh(ctx, model).assemble(model.E_elem, model.poisson)
    st, x, its, rr = _noalloc_solve(torch, A, model.subdomains[0].RHS, 1e-8, max_it=10)
    assert st == N.MSG_ERR_INVALID_ARGUMENT
    assert b"65536" in N.lib().MSG_LAST_ERROR(ctx.handle)
