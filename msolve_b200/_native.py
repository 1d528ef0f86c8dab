"""ctypes binding of libmsolve_gpu.so (the C ABI declared in include/msolve_gpu.h).

ctypes plays the role P/Invoke plays for the reference's C# code: every call
goes through the same extern "C" entry points a C# shim would bind. The
library is required: there is no CPU fallback, and importing a function that
needs it raises if the shared object is missing or fails to load.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmsolve_gpu.so")

MSG_OK = 0
MSG_ERR_UNKNOWN = -1
MSG_ERR_OUT_OF_MEMORY = -100
MSG_ERR_NEG_DET = -1001
MSG_ERR_NOT_CONVERGED = -2001
MSG_ERR_BREAKDOWN = -2002
MSG_ERR_TIMEOUT = -2003
MSG_ERR_CANCELLED = -2004
MSG_PENDING = 1
MSG_ERR_INVALID_ARGUMENT = -2005
MSG_ERR_CUDA = -2006
MSG_ERR_NOT_STRUCTURED = -2007
MSG_ERR_NO_DEVICE = -2008

MSG_MODE_FP64_BSR = 0
MSG_MODE_MIXED_BATCHED = 1

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)
_i64 = C.POINTER(C.c_int64)
_vp = C.c_void_p


class MSG_KL(C.Structure):
    _fields_ = [
        ("n_terms", C.c_int),
        ("w3", _d),
        ("amp3", _d),
        ("idx3", _i),
        ("eig", _d),
        ("domain", C.c_double * 3),
        ("mean", C.c_double),
        ("sigma", C.c_double),
        ("mean_correction", C.c_int),
        ("gaussian", C.c_int),
    ]


# name -> (restype, argtypes); the exported symbol set of include/msolve_gpu.h
class MSG_NEWMARK(C.Structure):
    _fields_ = [
        ("rho", C.c_double),
        ("rayleigh_alpha", C.c_double),
        ("rayleigh_beta", C.c_double),
        ("alpha", C.c_double),
        ("delta", C.c_double),
        ("dt", C.c_double),
        ("n_steps", C.c_int),
        ("acc_amp", C.c_double),
        ("acc_period", C.c_double),
        ("acc_dof", C.c_int),
    ]


class MSG_RAGGED_SYSTEM(C.Structure):
    _fields_ = [
        ("mesh", _vp),
        ("nu", C.c_double),
        ("kl", C.POINTER(MSG_KL)),
        ("R", C.c_int),
        ("xi", _d),
        ("b", _d),
        ("tip_dof", C.c_int),
        ("X", _d),
        ("tip", _d),
        ("iterations", _i),
        ("rel_res", _d),
    ]


SIGNATURES = {
    "MSG_CREATE": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "MSG_DESTROY": (C.c_int, [_vp]),
    "MSG_LAST_ERROR": (C.c_char_p, [_vp]),
    "MSG_VERSION": (C.c_int, []),
    "MSG_H8_KE_BATCH": (C.c_int, [_vp, C.c_int, _d, _d, C.c_double, _d]),
    "MSG_H8_ME_BATCH": (C.c_int, [_vp, C.c_int, _d, C.c_double, _d]),
    "MSG_PC_SIZE": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "MSG_PC_BASIS": (C.c_int, [C.c_int, C.c_int, _i, _i]),
    "MSG_PC_GALERKIN_MATVEC": (C.c_int, [_vp, C.c_double, C.POINTER(MSG_KL), C.c_int, C.c_int, _d, _d]),
    "MSG_SVS_CREATE": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "MSG_SVS_CLEAR": (C.c_int, [_vp, C.c_int]),
    "MSG_SVS_COUNT": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "MSG_SVS_DESTROY": (C.c_int, [_vp]),
    "MSG_PCG_SOLVE_REORTH": (C.c_int, [_vp, _vp, _d, _d, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_int),
                                       C.POINTER(C.c_double)]),
    "MSG_H8_STRESS_BATCH": (C.c_int, [_vp, C.c_int, _d, _d, C.c_double, _d, _d, _d, _d, _d]),
    "MSG_STRESS_BATCH_DEVICE": (C.c_int, [_vp, C.c_int, _vp, C.c_double, _vp, _vp, _vp, _vp]),
    "MSG_MESH_CREATE": (C.c_int, [_vp, C.c_int, _d, C.c_int, _i, _i, C.c_int, C.POINTER(_vp)]),
    "MSG_MESH_INFO": (C.c_int, [_vp, _i64]),
    "MSG_MESH_DESTROY": (C.c_int, [_vp]),
    "MSG_ASSEMBLE_BSR": (C.c_int, [_vp, _d, C.c_double, C.POINTER(_vp)]),
    "MSG_ASSEMBLE_BSR_KE": (C.c_int, [_vp, _d, C.POINTER(_vp)]),
    "MSG_MAT_MULTIPLY": (C.c_int, [_vp, _d, _d]),
    "MSG_MAT_DIAGONAL": (C.c_int, [_vp, _d]),
    "MSG_MAT_DESTROY": (C.c_int, [_vp]),
    "MSG_PCG_SOLVE": (C.c_int, [_vp, _d, _d, C.c_int, C.c_double, _i, _d]),
    "MSG_PCG_SOLVE_MIXED": (C.c_int, [_vp, _d, _d, C.c_int, C.c_double, _i, _d]),
    "MSG_PCG_SOLVE_NOALLOC": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_double, _i, _d]),
    "MSG_KL_TABLE": (C.c_int, [_d, C.c_double, C.c_int, C.c_int, _d, _d, _i, _d]),
    "MSG_KL_FIELD": (C.c_int, [_vp, C.POINTER(MSG_KL), C.c_int, _d, _d]),
    "MSG_MC_SOLVE_BATCH": (C.c_int, [_vp, C.c_double, C.POINTER(MSG_KL), C.c_int, _d, _d, C.c_int, C.c_int,
                                     C.c_double, C.c_int, _d, _d, _i, _d]),
    "MSG_MC_SOLVE_BATCH_DEVICE": (C.c_int, [_vp, C.c_double, C.POINTER(MSG_KL), C.c_int, _vp, _vp, C.c_int,
                                            C.c_int, C.c_double, C.c_int, _vp, _d, _i, _d]),
    "MSG_MC_SOLVE_BATCH_PIPELINED": (C.c_int, [_vp, C.c_double, C.POINTER(MSG_KL), C.c_int, _d, _d, C.c_int,
                                               C.c_int, C.c_double, C.c_int, _d, _d, _i, _d]),
    "MSG_MC_FLUSH": (C.c_int, [_vp]),
    "MSG_MC_SOLVE_RAGGED": (C.c_int, [_vp, C.c_int, C.POINTER(MSG_RAGGED_SYSTEM), C.c_int, C.c_double]),
    "MSG_NEWMARK_BATCH": (C.c_int, [_vp, C.c_double, C.POINTER(MSG_KL), C.c_int, _d, C.POINTER(MSG_NEWMARK), _d,
                                    C.c_int, C.c_double, C.c_int, _d, _d, _i]),
    "MSG_SERVE_START": (C.c_int, [_vp, C.c_int]),
    "MSG_SERVE_ADD_MODEL": (C.c_int, [_vp, _vp, C.c_double, C.POINTER(MSG_KL), _d, C.c_double, C.c_int, _i]),
    "MSG_SERVE_SUBMIT": (C.c_int, [_vp, C.c_int, _d, C.POINTER(C.c_uint64)]),
    "MSG_SERVE_POLL": (C.c_int, [_vp, C.c_uint64, C.c_int, _d, _i, _d, _d]),
    "MSG_SERVE_CANCEL": (C.c_int, [_vp, C.c_uint64]),
    "MSG_SERVE_STATS": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "MSG_SERVE_LANES": (C.c_int, [_vp, C.c_int, _i, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "MSG_SERVE_STOP": (C.c_int, [_vp]),
    "MSG_SET_OPTION": (C.c_int, [_vp, C.c_char_p, C.c_double]),
    "MSG_STATS": (C.c_int, [_vp, _i64, _d]),
    "MSG_STATS_RESET": (C.c_int, [_vp]),
    "MSG_WAIT_SELFTEST": (C.c_int, [_vp, C.c_int64]),
    "MSG_GET_OPTION": (C.c_int, [_vp, C.c_char_p, C.POINTER(C.c_double)]),
}

_lib = None


class MSolveError(RuntimeError):
    """A non-zero status from the C ABI. `code` is the MSG_ERR_* value."""

    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code


class InvalidOperationError(MSolveError):
    """Maps the codes the reference raises InvalidOperationException for
    (non-convergence, breakdown, singular/negative-determinant elements)."""


class ArgumentError(MSolveError):
    """Maps MSG_ERR_INVALID_ARGUMENT (the reference's ArgumentException)."""


def lib():
    """The loaded product library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C msolve_b200/csrc` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, ctx=None, what=""):
    if status == MSG_OK:
        return
    msg = ""
    if ctx is not None:
        raw = lib().MSG_LAST_ERROR(ctx)
        msg = raw.decode() if raw else ""
    msg = f"{what}: {msg}" if what else msg
    if status == MSG_ERR_INVALID_ARGUMENT:
        raise ArgumentError(status, msg)
    if status in (MSG_ERR_NOT_CONVERGED, MSG_ERR_BREAKDOWN, MSG_ERR_NEG_DET, MSG_ERR_NOT_STRUCTURED):
        raise InvalidOperationError(status, msg)
    raise MSolveError(status, msg)


def ptr(a, t=_d):
    return a.ctypes.data_as(t)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One CUDA device + stream (MSG_CREATE). Closed on garbage collection."""

    def __init__(self, device=0, mem_budget_bytes=0):
        h = _vp()
        st = lib().MSG_CREATE(int(device), int(mem_budget_bytes), C.byref(h))
        if st != MSG_OK:
            raise MSolveError(st, f"MSG_CREATE(device={device}) failed")
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            lib().MSG_DESTROY(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, key, value):
        check(lib().MSG_SET_OPTION(self.handle, key.encode(), float(value)), self.handle, "MSG_SET_OPTION")

    def get_option(self, key):
        v = C.c_double(0.0)
        check(lib().MSG_GET_OPTION(self.handle, key.encode(), C.byref(v)), self.handle, "MSG_GET_OPTION")
        return v.value

    def stats(self):
        n = C.c_int64(0)
        t = np.zeros(8)
        lib().MSG_STATS(self.handle, C.byref(n), ptr(t))
        return dict(launches=n.value, t_field_ms=t[0], t_inner_ms=t[1], reliable_updates=int(t[2]),
                    t_resid_ms=t[3], t_total_ms=t[4], op_launch_ms=t[5], update_launch_ms=t[6],
                    launch_samples=int(t[7]))

    def reset_stats(self):
        lib().MSG_STATS_RESET(self.handle)
