"""Stochastic Galerkin (polynomial chaos, Gaussian germs) on the device:
the basis of PolynomialChaosCoefficientsCalculator and the Galerkin product of
PolynomialChaosSolverPCGMatrixCalculator.MultiplyWithMatrix, over the C ABI
(MSG_PC_SIZE, MSG_PC_BASIS, MSG_PC_GALERKIN_MATVEC)."""
import ctypes as C

import numpy as np

from . import _native as N


def pc_basis(m, p):
    """Multi-indices [P][m] (the reference's order) and squared norms [P]."""
    P = C.c_int(0)
    N.check(N.lib().MSG_PC_SIZE(int(m), int(p), C.byref(P)), None, "MSG_PC_SIZE")
    basis = np.zeros((P.value, m), dtype=np.int32)
    norms = np.zeros(P.value, dtype=np.int32)
    N.check(N.lib().MSG_PC_BASIS(int(m), int(p), N.ptr(basis, N._i), N.ptr(norms, N._i)), None, "MSG_PC_BASIS")
    return basis, norms


class PolynomialChaosSolverPCGMatrixCalculator:
    """The Gaussian Galerkin operator of m KL variables up to degree p on a
    structured mesh (PolynomialChaosSolverPCGMatrixCalculator.cs:21-1089):
    MultiplyWithMatrix(u) returns y = sum_pos sum <xi psi psi> K_pos u for the
    block vector u [P][n_dofs]."""

    def __init__(self, mesh, coefficients_provider, m, p):
        if not getattr(coefficients_provider, "gaussian", False):
            raise TypeError("the Galerkin operator needs a GaussianStochasticCoefficientsProvider")
        self.mesh, self.kl, self.m, self.p = mesh, coefficients_provider, m, p
        self.PsiBasis, self.PsiSquareNorm = pc_basis(m, p)

    @property
    def PsiSize(self):
        return self.PsiBasis.shape[0]

    @property
    def VectorSize(self):
        return self.PsiSize * self.mesh.model.n_dofs

    def MultiplyWithMatrix(self, u):
        u = N.f64(u).reshape(self.PsiSize, self.mesh.model.n_dofs)
        y = np.zeros_like(u)
        s = self.kl.struct()
        N.check(N.lib().MSG_PC_GALERKIN_MATVEC(self.mesh.handle, float(self.mesh.model.poisson), C.byref(s), self.m,
                                               self.p, N.ptr(u), N.ptr(y)), self.mesh.ctx.handle,
                "MSG_PC_GALERKIN_MATVEC")
        return y
