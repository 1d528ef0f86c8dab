"""msolve_b200: B200-native (sm_100a) Hexa8 linear-elastic solve path of MSolve.

The product is ``libmsolve_gpu.so`` (C ABI in ``include/msolve_gpu.h``); this
package is its host-side mirror of the reference's preprocessor, provider,
solver and analyzer interfaces, bound through ctypes.
"""
from ._native import (ArgumentError, Context, InvalidOperationError, MSolveError, MSG_MODE_FP64_BSR,
                      MSG_MODE_MIXED_BATCHED, lib)
from .analyzers import (GaussianStochasticCoefficientsProvider, GpuMatrix, GpuMesh, LinearAnalyzer,
                        LognormalStochasticCoefficientsProvider,
                        MonteCarloAnalyzer, MonteCarloAnalyzerWithStochasticMaterial, NewmarkDynamicAnalyzer,
                        RaggedMonteCarloBatch,
                        SolverPCGReorthogonalizationSearchVectorCalculator, SolverPCGReorthogonalized, ProblemStructural, SolverPCG,
                        StaticAnalyzer, h8_mass_batch, h8_stiffness_batch, h8_stress_batch, realization_stresses)
from .polynomial_chaos import PolynomialChaosSolverPCGMatrixCalculator, pc_basis
from .tuning import Autotuner
from .model import (Hexa8MeshGenerator, MassAccelerationSinusoidalLoad, Model, cantilever_model, clamped_block_model,
                    tip_dof)

__all__ = [
    "ArgumentError", "Autotuner", "Context", "InvalidOperationError", "MSolveError", "MSG_MODE_FP64_BSR", "MSG_MODE_MIXED_BATCHED",
    "lib", "GaussianStochasticCoefficientsProvider", "GpuMatrix", "GpuMesh", "LinearAnalyzer", "LognormalStochasticCoefficientsProvider",
    "MonteCarloAnalyzer", "MonteCarloAnalyzerWithStochasticMaterial", "RaggedMonteCarloBatch",
    "SolverPCGReorthogonalizationSearchVectorCalculator",
    "SolverPCGReorthogonalized", "NewmarkDynamicAnalyzer", "ProblemStructural", "SolverPCG",
    "StaticAnalyzer", "h8_mass_batch", "h8_stiffness_batch", "h8_stress_batch", "realization_stresses",
    "Hexa8MeshGenerator", "MassAccelerationSinusoidalLoad",
    "Model", "PolynomialChaosSolverPCGMatrixCalculator", "pc_basis", "cantilever_model", "clamped_block_model", "tip_dof",
]
