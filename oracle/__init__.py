"""CPU oracle for the MSolve Hexa8 solve path -- TEST INFRASTRUCTURE ONLY.

ctypes front end of ``oracle/liboracle.so`` (``oracle/oracle.cpp``), a plain
FP64 C++ restatement of the reference's element, assembly, skyline LDL^T, PCG
and Karhunen-Loeve field algorithms. Only the test suite, the smoke check and
the CPU-baseline legs of ``bench.py`` import this module; the product package
never does.

Parity status: unpinned against reference execution (the reference is C#/.NET
4 plus Intel Fortran and cannot be built here; it ships no golden vectors).
The restatement is pinned by closed-form known answers (exact rational unit
cube stiffness in ``tests/golden``), by agreement of its two independent
element paths (Fortran ``CalcH8K`` and C# ``Hexa8.StiffnessMatrix``), by the
rigid-body null space and by direct-vs-iterative agreement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)


def build() -> None:
    """Compile liboracle.so from oracle.cpp (make, in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_elastic_D": (None, [C.c_double, C.c_double, _d]),
            "orc_h8_gauss_matrices": (C.c_int, [_d, _d, _d, _d, _d, _d, _d]),
            "orc_h8_k": (None, [_d, _d, _d, _d]),
            "orc_h8_stiffness_fortran": (C.c_int, [_d, C.c_double, C.c_double, _d]),
            "orc_h8_stiffness_csharp": (C.c_int, [_d, C.c_double, C.c_double, _d]),
            "orc_h8_consistent_mass": (C.c_int, [_d, C.c_double, _d]),
            "orc_h8_stiffness_batch": (None, [C.c_int, _d, _d, C.c_double, _d, _i]),
            "orc_h8_stress_batch": (None, [C.c_int, _d, _d, C.c_double, _d, _d, _d, _d, _d, _i]),
            "orc_block_nodes": (None, [C.c_int, C.c_int, C.c_int, C.c_double, _d]),
            "orc_block_conn": (None, [C.c_int, C.c_int, C.c_int, _i]),
            "orc_enumerate_dofs": (C.c_int, [C.c_int, _u8, _i]),
            "orc_skyline_rowindex": (C.c_int64, [C.c_int, _i, _i, C.c_int, _i64]),
            "orc_skyline_assemble": (None, [C.c_int, _i, _i, _d, _i64, _d]),
            "orc_skyline_factorize": (C.c_int, [C.c_int, _i64, _d, C.c_double, _i]),
            "orc_skyline_solve": (None, [C.c_int, _i64, _d, _d, _d]),
            "orc_skyline_multiply": (None, [C.c_int, _i64, _d, _d, _d]),
            "orc_csr_pattern": (C.c_int64, [C.c_int, C.c_int, _i, _i, C.c_int, _i64, _i]),
            "orc_csr_assemble": (None, [C.c_int, _i, _i, _d, _i64, _i, _d]),
            "orc_csr_multiply": (None, [C.c_int, _i64, _i, _d, _d, _d]),
            "orc_pcg_csr_jacobi": (C.c_int, [C.c_int, _i64, _i, _d, _d, _d, C.c_int, C.c_double, _i, _i, _d]),
            "orc_pcg_skyline": (C.c_int, [C.c_int, _i64, _d, _d, _d, _d, C.c_int, C.c_double, _i, _i, _d]),
            "orc_kl_1d_modes": (C.c_int, [C.c_double, C.c_double, C.c_int, _d, _d, _d]),
            "orc_kl_table": (C.c_int, [_d, C.c_double, C.c_int, C.c_int, _d, _d, _i, _d]),
            "orc_kl_field": (None, [C.c_int, _d, _d, C.c_int, _d, _d, _i, _d, C.c_int, _d,
                                    C.c_double, C.c_double, C.c_int, _d]),
            "orc_block_solve_pcg": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, _u8, _d, C.c_double,
                                              _d, _d, C.c_int, C.c_double, _i, _d]),
            "orc_block_newmark": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, _u8, _d, C.c_double, C.c_double,
                                            C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                            C.c_double, C.c_double, C.c_int, _d, C.c_int, C.c_double, C.c_int,
                                            _d, _d, _i]),
            "orc_block_solve_pcg_batch": (None, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _u8, _d,
                                                  C.c_double, _d, _d, C.c_int, C.c_int, C.c_double, _i, _i, _d]),
            "orc_block_newmark_batch": (None, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _u8, _d, C.c_double,
                                                C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                                C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, _d, C.c_int,
                                                C.c_double, C.c_int, C.c_int, _d, _d, _i, _i]),
            "orc_kl_field_gaussian": (None, [C.c_int, _d, _d, C.c_int, _d, _d, _i, _d, C.c_int, _d,
                                             C.c_double, C.c_double, _d]),
            "orc_pcg_reorth_csr": (C.c_int, [C.c_int, _i64, _i, _d, _d, _d, _d, _d, _d, C.c_int, _i, C.c_int,
                                             C.c_int, C.c_double, _i, _d]),
            "orc_pc_size": (C.c_int, [C.c_int, C.c_int]),
            "orc_pc_basis": (C.c_int, [C.c_int, C.c_int, _i, _i]),
            "orc_pc_gaussian_matvec": (None, [C.c_int, _i64, _i, _d, C.c_int64, C.c_int, C.c_int, _d, _d]),
            "orc_num_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------- elements
def unpack300(k300):
    """Packed row-wise upper 24x24 (SymmetricMatrix2D.cs:22-49) -> full matrix."""
    k300 = np.asarray(k300)
    K = np.zeros(k300.shape[:-1] + (24, 24))
    iu = np.triu_indices(24)
    K[..., iu[0], iu[1]] = k300
    K[..., iu[1], iu[0]] = k300
    return K


def elastic_D(E, nu):
    D = np.zeros(36)
    lib().orc_elastic_D(E, nu, _p(D))
    return D.reshape(6, 6)


def h8_stiffness(xyz, E, nu, path="fortran"):
    xyz = _f64(xyz).reshape(24)
    K = np.zeros(300)
    fn = lib().orc_h8_stiffness_fortran if path == "fortran" else lib().orc_h8_stiffness_csharp
    st = fn(_p(xyz), float(E), float(nu), _p(K))
    return K, st


def h8_stiffness_batch(xyz, E, nu):
    xyz = _f64(xyz)
    n = xyz.shape[0]
    E = _f64(np.broadcast_to(np.asarray(E, dtype=np.float64), (n,)))
    K = np.zeros((n, 300))
    st = C.c_int(0)
    lib().orc_h8_stiffness_batch(n, _p(xyz), _p(E), float(nu), _p(K), C.byref(st))
    return K, st.value


def h8_stress_batch(xyz, E, nu, u, du=None):
    """Strains, stresses [n][8][6] and internal forces [n][24] per element
    (Hexa8.CalculateStresses + CalculateForces over CalcH8Strains/CalcH8Forces)."""
    xyz = _f64(xyz).reshape(-1, 24)
    n = xyz.shape[0]
    E = _f64(np.broadcast_to(np.asarray(E, dtype=np.float64), (n,)))
    u = _f64(u).reshape(n, 24)
    du = None if du is None else _f64(du).reshape(n, 24)
    eps, sig, f = np.zeros((n, 8, 6)), np.zeros((n, 8, 6)), np.zeros((n, 24))
    st = C.c_int(0)
    lib().orc_h8_stress_batch(n, _p(xyz), _p(E), float(nu), _p(u), None if du is None else _p(du), _p(eps), _p(sig),
                              _p(f), C.byref(st))
    return eps, sig, f, st.value


def h8_gauss_matrices(xyz):
    xyz = _f64(xyz).reshape(24)
    w, S, DS, J, det, B = (np.zeros(8), np.zeros(64), np.zeros(192), np.zeros(72), np.zeros(8), np.zeros(1152))
    st = lib().orc_h8_gauss_matrices(_p(xyz), _p(w), _p(S), _p(DS), _p(J), _p(det), _p(B))
    return dict(weight=w, S=S.reshape(8, 8), DS=DS.reshape(8, 24), J=J.reshape(8, 3, 3), detJ=det,
                B=B.reshape(8, 6, 24), status=st)


def h8_consistent_mass(xyz, rho):
    xyz = _f64(xyz).reshape(24)
    M = np.zeros(300)
    st = lib().orc_h8_consistent_mass(_p(xyz), float(rho), _p(M))
    return M, st


# ---------------------------------------------------------------- mesh
def block_mesh(nx, ny, nz, h=1.0):
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    xyz = np.zeros((nn, 3))
    conn = np.zeros((nx * ny * nz, 8), dtype=np.int32)
    lib().orc_block_nodes(nx, ny, nz, float(h), _p(xyz))
    lib().orc_block_conn(nx, ny, nz, _p(conn, _i))
    return xyz, conn


def enumerate_dofs(constrained):
    cons = np.ascontiguousarray(constrained, dtype=np.uint8)
    dof = np.zeros(cons.shape, dtype=np.int32)
    n = lib().orc_enumerate_dofs(cons.shape[0], _p(cons, _u8), _p(dof, _i))
    return dof, n


def clamp_face(xyz, axis, value=0.0):
    """Constrain every DOF of the nodes on the plane xyz[:, axis] == value."""
    cons = np.zeros((xyz.shape[0], 3), dtype=np.uint8)
    cons[np.isclose(xyz[:, axis], value)] = 1
    return cons


def load_tip(xyz, dof, n_dofs, axis_face=0, comp=2, total=-1.0):
    """Total load split equally over the nodes of the face xyz[:, axis] == max
    (assigned per DOF, Model.AssignNodalLoads Model.cs:227-238)."""
    face = np.isclose(xyz[:, axis_face], xyz[:, axis_face].max())
    b = np.zeros(n_dofs)
    ids = np.nonzero(face)[0]
    for n in ids:
        d = dof[n, comp]
        if d >= 0:
            b[d] = total / len(ids)
    return b


def load_top_pressure(xyz, dof, n_dofs, h=1.0, p=1.0):
    """Uniform pressure p in -z on the top face by consistent bilinear weights:
    each node gets p * h^2 * (number of top-face elements touching it) / 4."""
    zt = xyz[:, 2].max()
    xm, ym = xyz[:, 0].max(), xyz[:, 1].max()
    b = np.zeros(n_dofs)
    for n in np.nonzero(np.isclose(xyz[:, 2], zt))[0]:
        x, y = xyz[n, 0], xyz[n, 1]
        cx = 1 if (np.isclose(x, 0) or np.isclose(x, xm)) else 2
        cy = 1 if (np.isclose(y, 0) or np.isclose(y, ym)) else 2
        d = dof[n, 2]
        if d >= 0:
            b[d] = -p * h * h * cx * cy / 4.0
    return b


def element_xyz(xyz, conn):
    return xyz[conn].reshape(conn.shape[0], 24)


def centroids(xyz, conn):
    """Hexa8WithStochasticMaterial.GetStochasticPoints (:112-140): bounding-box centre."""
    ex = xyz[conn]
    return ex.min(axis=1) + (ex.max(axis=1) - ex.min(axis=1)) / 2


# ---------------------------------------------------------------- skyline / CSR
class Skyline:
    def __init__(self, conn, dof, n_dofs):
        self.conn, self.dof, self.n = _i32(conn), _i32(dof), n_dofs
        self.ri = np.zeros(n_dofs + 1, dtype=np.int64)
        size = lib().orc_skyline_rowindex(conn.shape[0], _p(self.conn, _i), _p(self.dof, _i), n_dofs,
                                          _p(self.ri, _i64))
        self.data = np.zeros(size)

    def assemble(self, Ke):
        Ke = _f64(Ke)
        self.data[:] = 0
        lib().orc_skyline_assemble(self.conn.shape[0], _p(self.conn, _i), _p(self.dof, _i), _p(Ke),
                                   _p(self.ri, _i64), _p(self.data))

    def multiply(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        lib().orc_skyline_multiply(self.n, _p(self.ri, _i64), _p(self.data), _p(x), _p(y))
        return y

    def factorized(self, tol=1e-15):
        f = self.data.copy()
        z = C.c_int(0)
        st = lib().orc_skyline_factorize(self.n, _p(self.ri, _i64), _p(f), tol, C.byref(z))
        if st != 0:
            raise ValueError("near-zero pivot")
        return f, z.value

    def solve(self, factor, b):
        b = _f64(b)
        x = np.zeros(self.n)
        lib().orc_skyline_solve(self.n, _p(self.ri, _i64), _p(factor), _p(b), _p(x))
        return x

    def pcg(self, b, precond_factor, max_it=20000, tol=1e-7):
        b = _f64(b)
        x = np.zeros(self.n)
        it, mv, rr = C.c_int(0), C.c_int(0), C.c_double(0)
        st = lib().orc_pcg_skyline(self.n, _p(self.ri, _i64), _p(self.data), _p(precond_factor), _p(b), _p(x),
                                   max_it, tol, C.byref(it), C.byref(mv), C.byref(rr))
        return x, dict(status=st, iterations=it.value, matvecs=mv.value, rel_res=rr.value)


class CSR:
    def __init__(self, n_nodes, conn, dof, n_dofs):
        self.conn, self.dof, self.n = _i32(conn), _i32(dof), n_dofs
        self.rp = np.zeros(n_dofs + 1, dtype=np.int64)
        nnz = lib().orc_csr_pattern(n_nodes, conn.shape[0], _p(self.conn, _i), _p(self.dof, _i), n_dofs,
                                    _p(self.rp, _i64), None)
        self.ci = np.zeros(nnz, dtype=np.int32)
        lib().orc_csr_pattern(n_nodes, conn.shape[0], _p(self.conn, _i), _p(self.dof, _i), n_dofs,
                              _p(self.rp, _i64), _p(self.ci, _i))
        self.val = np.zeros(nnz)

    def assemble(self, Ke):
        Ke = _f64(Ke)
        self.val[:] = 0
        lib().orc_csr_assemble(self.conn.shape[0], _p(self.conn, _i), _p(self.dof, _i), _p(Ke),
                               _p(self.rp, _i64), _p(self.ci, _i), _p(self.val))

    def multiply(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        lib().orc_csr_multiply(self.n, _p(self.rp, _i64), _p(self.ci, _i), _p(self.val), _p(x), _p(y))
        return y

    def diagonal(self):
        d = np.zeros(self.n)
        for i in range(self.n):
            cols = self.ci[self.rp[i]:self.rp[i + 1]]
            d[i] = self.val[self.rp[i] + np.searchsorted(cols, i)]
        return d

    def pcg_jacobi(self, b, max_it=20000, tol=1e-7):
        b = _f64(b)
        x = np.zeros(self.n)
        it, mv, rr = C.c_int(0), C.c_int(0), C.c_double(0)
        st = lib().orc_pcg_csr_jacobi(self.n, _p(self.rp, _i64), _p(self.ci, _i), _p(self.val), _p(b), _p(x),
                                      max_it, tol, C.byref(it), C.byref(mv), C.byref(rr))
        return x, dict(status=st, iterations=it.value, matvecs=mv.value, rel_res=rr.value)


class SearchVectorStore:
    """Host store of (p, K p) pairs for CSR.pcg_reorth (capacity pairs of length n)."""

    def __init__(self, n, capacity):
        self.P = np.zeros((capacity, n))
        self.Q = np.zeros((capacity, n))
        self.pq = np.zeros(capacity)
        self.capacity, self.count = capacity, 0

    def clear(self, keep_from_top=0):
        self.count = 0 if keep_from_top < 1 else min(self.count, keep_from_top)


def pcg_reorth(csr, store, b, start=False, max_it=20000, tol=1e-7):
    """Re-orthogonalised PCG over the store (SolverPCG + SearchVectors)."""
    b = _f64(b)
    x = np.zeros(csr.n)
    it, rr, cnt = C.c_int(0), C.c_double(0), C.c_int(store.count)
    st = lib().orc_pcg_reorth_csr(csr.n, _p(csr.rp, _i64), _p(csr.ci, _i), _p(csr.val), _p(b), _p(x), _p(store.P),
                                  _p(store.Q), _p(store.pq), store.capacity, C.byref(cnt), int(start), max_it,
                                  tol, C.byref(it), C.byref(rr))
    store.count = cnt.value
    return x, dict(status=st, iterations=it.value, rel_res=rr.value)


def pc_basis(m, p):
    P = lib().orc_pc_size(m, p)
    basis = np.zeros((P, m), dtype=np.int32)
    norms = np.zeros(P, dtype=np.int32)
    lib().orc_pc_basis(m, p, _p(basis, _i), _p(norms, _i))
    return basis, norms


def pc_gaussian_matvec(csr, vals, m, p, u):
    """Galerkin product over the m + 1 matrices vals [m+1][nnz] of csr's pattern."""
    vals = _f64(vals)
    u = _f64(u)
    y = np.zeros_like(u)
    lib().orc_pc_gaussian_matvec(csr.n, _p(csr.rp, _i64), _p(csr.ci, _i), _p(vals), vals.shape[1], m, p, _p(u), _p(y))
    return y


# ---------------------------------------------------------------- KL field
def kl_1d_modes(half_length, corr_len, n):
    w, a, lam = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().orc_kl_1d_modes(float(half_length), float(corr_len), n, _p(w), _p(a), _p(lam))
    return w, a, lam


def kl_table(domain, corr_len, n_terms=50, n1d=16):
    L = _f64(domain)
    w3, a3 = np.zeros((n_terms, 3)), np.zeros((n_terms, 3))
    idx = np.zeros((n_terms, 3), dtype=np.int32)
    eig = np.zeros(n_terms)
    st = lib().orc_kl_table(_p(L), float(corr_len), n_terms, n1d, _p(w3), _p(a3), _p(idx, _i), _p(eig))
    if st:
        raise ValueError("not enough 1-D modes for the requested terms")
    return dict(w=w3, amp=a3, idx=idx, eig=eig)


def kl_field(cen, domain, table, xi, mean=1.0, sigma=0.3, mean_correction=False):
    cen, L, xi = _f64(cen), _f64(domain), _f64(xi)
    R, K = xi.shape
    E = np.zeros((R, cen.shape[0]))
    lib().orc_kl_field(cen.shape[0], _p(cen), _p(L), K, _p(_f64(table["w"])), _p(_f64(table["amp"])),
                       _p(_i32(table["idx"]), _i), _p(_f64(table["eig"])), R, _p(xi), float(mean), float(sigma),
                       int(bool(mean_correction)), _p(E))
    return E


def kl_field_gaussian(cen, domain, table, xi, mean=1.0, cov=0.15):
    """E = mean (1 + sum_k xi_k cov sqrt(eig_k) phi_k(x)) per element centroid
    (GaussianFileStochasticCoefficientsProvider.GetCoefficient)."""
    cen, L, xi = _f64(cen), _f64(domain), _f64(xi)
    R, K = xi.shape
    E = np.zeros((R, cen.shape[0]))
    lib().orc_kl_field_gaussian(cen.shape[0], _p(cen), _p(L), K, _p(_f64(table["w"])), _p(_f64(table["amp"])),
                                _p(_i32(table["idx"]), _i), _p(_f64(table["eig"])), R, _p(xi), float(mean),
                                float(cov), _p(E))
    return E


# ---------------------------------------------------------------- block solve
def block_solve_pcg(nx, ny, nz, constrained, E_elem, nu, b, h=1.0, max_it=50000, tol=1e-10):
    cons = np.ascontiguousarray(constrained, dtype=np.uint8)
    E_elem, b = _f64(E_elem), _f64(b)
    x = np.zeros(b.shape[0])
    it, rr = C.c_int(0), C.c_double(0)
    st = lib().orc_block_solve_pcg(nx, ny, nz, float(h), _p(cons, _u8), _p(E_elem), float(nu), _p(b), _p(x),
                                   max_it, tol, C.byref(it), C.byref(rr))
    return x, dict(status=st, iterations=it.value, rel_res=rr.value)


def block_newmark(nx, ny, nz, constrained, E_elem, nu, rho, ray_alpha, ray_beta, nm_alpha, nm_delta, dt, n_steps,
                  acc_amp, acc_period, acc_dir, n_dofs, f_static=None, solver=0, tol=1e-10, tip_dof=-1, h=1.0):
    """Newmark integration of one realization (NewmarkDynamicAnalyzer.cs:53-315); returns
    (tip history [n_steps], final displacement [n_dofs], info)."""
    cons = np.ascontiguousarray(constrained, dtype=np.uint8)
    E_elem = _f64(E_elem)
    tip = np.zeros(n_steps)
    u = np.zeros(n_dofs)
    its = C.c_int(0)
    fs = _p(_f64(f_static)) if f_static is not None else None
    st = lib().orc_block_newmark(nx, ny, nz, float(h), _p(cons, _u8), _p(E_elem), float(nu), float(rho),
                                 float(ray_alpha), float(ray_beta), float(nm_alpha), float(nm_delta), float(dt),
                                 int(n_steps), float(acc_amp), float(acc_period), int(acc_dir), fs, int(solver),
                                 float(tol), int(tip_dof), _p(tip), _p(u), C.byref(its))
    return tip, u, dict(status=st, iterations=its.value)


def block_solve_pcg_batch(nx, ny, nz, constrained, E, nu, b, h=1.0, max_it=50000, tol=1e-10):
    """block_solve_pcg for every row of E [R][ne], realizations in parallel (one
    per OpenMP thread); returns x [R][n_dofs], status, iterations, rel_res."""
    cons = np.ascontiguousarray(constrained, dtype=np.uint8)
    E, b = _f64(np.atleast_2d(E)), _f64(b)
    R, N = E.shape[0], b.shape[0]
    x = np.zeros((R, N))
    st, it, rr = np.zeros(R, dtype=np.int32), np.zeros(R, dtype=np.int32), np.zeros(R)
    lib().orc_block_solve_pcg_batch(R, nx, ny, nz, float(h), _p(cons, _u8), _p(E), float(nu), _p(b), _p(x), N,
                                    max_it, tol, _p(st, _i), _p(it, _i), _p(rr))
    return x, dict(status=st, iterations=it, rel_res=rr)


def block_newmark_batch(nx, ny, nz, constrained, E, nu, rho, ray_alpha, ray_beta, nm_alpha, nm_delta, dt, n_steps,
                        acc_amp, acc_period, acc_dir, n_dofs, f_static=None, solver=2, tol=1e-12, tip_dof=-1, h=1.0):
    """block_newmark for every row of E [R][ne], realizations in parallel; returns
    (tip histories [R][n_steps], final displacements [R][n_dofs], info)."""
    cons = np.ascontiguousarray(constrained, dtype=np.uint8)
    E = _f64(np.atleast_2d(E))
    R = E.shape[0]
    tip = np.zeros((R, n_steps))
    u = np.zeros((R, n_dofs))
    its, st = np.zeros(R, dtype=np.int32), np.zeros(R, dtype=np.int32)
    fs = _p(_f64(f_static)) if f_static is not None else None
    lib().orc_block_newmark_batch(R, nx, ny, nz, float(h), _p(cons, _u8), _p(E), float(nu), float(rho),
                                  float(ray_alpha), float(ray_beta), float(nm_alpha), float(nm_delta), float(dt),
                                  int(n_steps), float(acc_amp), float(acc_period), int(acc_dir), fs, int(solver),
                                  float(tol), int(tip_dof), int(n_dofs), _p(tip), _p(u), _p(its, _i), _p(st, _i))
    return tip, u, dict(status=st, iterations=its)


def block_problem(n, n_terms=50, n1d=16, corr_frac=0.2):
    """The clamped cube of the Monte Carlo workloads from the oracle alone: an
    n^3 block of unit cubes, z = 0 face clamped, unit pressure on the top face
    (consistent weights), the KL table of the separable exponential kernel with
    correlation length corr_frac * n. Returns a dict with xyz, conn,
    constrained [n_nodes][3] (uint8), dof, n_dofs, b, table, centroids, domain."""
    xyz, conn = block_mesh(n, n, n)
    cons = clamp_face(xyz, 2, 0.0)
    dof, nd = enumerate_dofs(cons)
    b = load_top_pressure(xyz, dof, nd)
    table = kl_table([n, n, n], corr_frac * n, n_terms, n1d)
    return dict(n=n, xyz=xyz, conn=conn, constrained=cons, dof=dof, n_dofs=nd, b=b, table=table,
                centroids=centroids(xyz, conn), domain=[float(n)] * 3)


def num_threads():
    return lib().orc_num_threads()
