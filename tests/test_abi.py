"""CPU tests of the C-ABI library and host logic (no GPU compute): the shared
object loads, exports every entry point include/msolve_gpu.h declares, host-side
helpers agree with the oracle, and argument validation happens before any
device work."""
import ctypes as C
import os
import re

import numpy as np

import msolve_b200 as M
import oracle as O
from msolve_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            syms |= set(re.findall(r"^\s*(?:int|const char\*|void)\s+(MSG_[A-Z0-9_]+)\s*\(", txt, re.M))
    return syms


def test_library_exports_every_header_symbol():
    L = M.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert syms <= set(N.SIGNATURES), syms - set(N.SIGNATURES)
    assert L.MSG_VERSION() == 100


def test_library_is_self_contained_cuda_code():
    """The product .so carries sm_100a device code and does not link the oracle."""
    blob = open(N.LIB_PATH, "rb").read()
    assert b"orc_" not in blob
    assert b"sm_100a" in blob or b"compute_100a" in blob


def test_mesh_generator_matches_oracle_mesh():
    for n in (1, 3, (10, 4, 4)):
        nx, ny, nz = (n, n, n) if isinstance(n, int) else n
        m = M.Hexa8MeshGenerator.block(nx, ny, nz)
        xyz, conn = O.block_mesh(nx, ny, nz)
        assert np.array_equal(m.xyz, xyz) and np.array_equal(m.conn, conn)


def test_loads_and_dofs_match_oracle():
    m = M.clamped_block_model(6)
    xyz, conn = O.block_mesh(6, 6, 6)
    dof, N_ = O.enumerate_dofs(O.clamp_face(xyz, 2, 0.0))
    assert np.array_equal(m.dof, dof) and m.n_dofs == N_
    assert np.array_equal(m.subdomains[0].RHS, O.load_top_pressure(xyz, dof, N_))
    c = M.cantilever_model()
    xyz, conn = O.block_mesh(10, 4, 4)
    dof, N_ = O.enumerate_dofs(O.clamp_face(xyz, 0, 0.0))
    assert c.n_dofs == 750 and np.array_equal(c.subdomains[0].RHS, O.load_tip(xyz, dof, N_, 0, 2, -1.0))


def test_kl_table_matches_oracle():
    for L, l, K in (([32, 32, 32], 6.4, 50), ([8, 16, 24], 3.0, 30)):
        kl = M.LognormalStochasticCoefficientsProvider(L, l, K, 16)
        t = O.kl_table(L, l, K, 16)
        assert np.array_equal(kl.idx, t["idx"])
        assert np.abs(kl.w - t["w"]).max() < 1e-14 * np.abs(t["w"]).max()
        assert np.abs(kl.amp - t["amp"]).max() < 1e-14 * np.abs(t["amp"]).max()
        assert np.abs(kl.eig - t["eig"]).max() < 1e-14 * t["eig"].max()


def test_kl_table_rejects_bad_arguments():
    w = np.zeros((10, 3)); a = np.zeros((10, 3)); i = np.zeros((10, 3), dtype=np.int32); e = np.zeros(10)
    L = np.array([1.0, 1.0, -1.0])
    st = M.lib().MSG_KL_TABLE(N.ptr(L), 1.0, 10, 4, N.ptr(w), N.ptr(a), N.ptr(i, N._i), N.ptr(e))
    assert st == N.MSG_ERR_INVALID_ARGUMENT
    L = np.array([1.0, 1.0, 1.0])
    st = M.lib().MSG_KL_TABLE(N.ptr(L), 1.0, 100, 4, N.ptr(w), N.ptr(a), N.ptr(i, N._i), N.ptr(e))
    assert st == N.MSG_ERR_INVALID_ARGUMENT  # 4^3 < 100 terms


def test_null_handles_are_rejected():
    L = M.lib()
    assert L.MSG_DESTROY(None) == N.MSG_ERR_INVALID_ARGUMENT
    assert L.MSG_MESH_DESTROY(None) == N.MSG_ERR_INVALID_ARGUMENT
    assert L.MSG_MAT_DESTROY(None) == N.MSG_ERR_INVALID_ARGUMENT
    x = np.zeros(3)
    assert L.MSG_MAT_MULTIPLY(None, N.ptr(x), N.ptr(x)) == N.MSG_ERR_INVALID_ARGUMENT
    assert L.MSG_PCG_SOLVE(None, N.ptr(x), N.ptr(x), 10, 1e-6, None, None) == N.MSG_ERR_INVALID_ARGUMENT
    h = N._vp()
    assert L.MSG_CREATE(0, 0, None) == N.MSG_ERR_INVALID_ARGUMENT
    assert L.MSG_CREATE(-1, 0, C.byref(h)) in (N.MSG_ERR_INVALID_ARGUMENT, N.MSG_ERR_NO_DEVICE)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(N, "_lib", None)
    monkeypatch.setattr(N, "LIB_PATH", str(tmp_path / "absent.so"))
    try:
        N.lib()
        raise AssertionError("expected ImportError")
    except ImportError as e:
        assert "no CPU fallback" in str(e)


def header_arities():
    """Parameter count of every entry point the headers declare."""
    out = {}
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            for name, params in re.findall(r"^\s*(?:int|const char\*|void)\s+(MSG_[A-Z0-9_]+)\s*\(([^)]*)\)",
                                           txt, re.M | re.S):
                p = params.strip()
                out[name] = 0 if p in ("", "void") else p.count(",") + 1
    return out


def test_bindings_match_header_declarations():
    """Every entry point the ctypes binding declares (the Python analogue of the
    P/Invoke shim) is declared by the header with the same number of
    parameters, so the binding cannot drift from the ABI."""
    ar = header_arities()
    assert len(ar) >= 20
    assert set(N.SIGNATURES) <= set(ar), set(N.SIGNATURES) - set(ar)
    for name, (_, argtypes) in N.SIGNATURES.items():
        assert len(argtypes) == ar[name], (name, len(argtypes), ar[name])
