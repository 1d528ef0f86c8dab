"""Host mirror of the reference's solver / provider / analyzer interfaces on
top of the C ABI, so code written against MSolve's StaticAnalyzer ->
LinearAnalyzer -> ISolver chain and its Monte Carlo analyzer can drive the
GPU path with the same call sequence:

    model = clamped_block_model(32)
    ctx = Context(0)
    solver = SolverPCG(ctx, model)                  # ISolver (SolverPCG<T>)
    provider = ProblemStructural(ctx, model)        # IStaticProvider
    static = StaticAnalyzer(provider, LinearAnalyzer(solver))
    static.BuildMatrices(); static.Initialize(); static.Solve()
    model.subdomains[0].Solution

References: IAnalyzer (ISAAR.MSolve.Analyzers/Interfaces/IAnalyzer.cs:9-17),
StaticAnalyzer.cs:10-75, LinearAnalyzer.cs:12-69, ProblemStructural.cs:16-221,
ISolver (ISAAR.MSolve.Solvers/Interfaces/ISolver.cs:8-12),
SolverPCGSkyline.cs:75-108 (Initialize / Solve(20000, 1e-7)),
MonteCarloAnalyzerWithStochasticMaterial.cs:55-296.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import time

import numpy as np

from . import _native as N
from .model import tip_dof as _tip_dof


class GpuMatrix:
    """Assembled FP64 global stiffness on the device (IMatrix2D analogue)."""

    def __init__(self, mesh, handle):
        self.mesh, self.handle = mesh, handle  # keeps the mesh (and its context) alive

    def Multiply(self, x):
        x = N.f64(x)
        y = np.zeros(self.mesh.model.n_dofs)
        N.check(N.lib().MSG_MAT_MULTIPLY(self.handle, N.ptr(x), N.ptr(y)), self.mesh.ctx.handle, "Multiply")
        return y

    def Diagonal(self):
        d = np.zeros(self.mesh.model.n_dofs)
        N.check(N.lib().MSG_MAT_DIAGONAL(self.handle, N.ptr(d)), self.mesh.ctx.handle, "Diagonal")
        return d

    def close(self):
        if self.handle:
            N.lib().MSG_MAT_DESTROY(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuMesh:
    """Device copy of a model's mesh and DOF map (MSG_MESH_CREATE)."""

    def __init__(self, ctx, model):
        if model.dof is None:
            model.ConnectDataStructures()
        self.ctx, self.model = ctx, model
        h = N._vp()
        N.check(N.lib().MSG_MESH_CREATE(ctx.handle, model.n_nodes, N.ptr(model.xyz), model.n_elems,
                                        N.ptr(model.conn, N._i), N.ptr(N.i32(model.dof), N._i), model.n_dofs,
                                        C.byref(h)), ctx.handle, "MSG_MESH_CREATE")
        self.handle = h

    def info(self):
        a = np.zeros(8, dtype=np.int64)
        N.check(N.lib().MSG_MESH_INFO(self.handle, N.ptr(a, N._i64)))
        return dict(structured=bool(a[0]), nx=int(a[1]), ny=int(a[2]), nz=int(a[3]), n_dofs=int(a[4]),
                    n_block_rows=int(a[5]), nnzb=int(a[6]), n_elems=int(a[7]))

    def assemble(self, E_elem, nu):
        h = N._vp()
        E_elem = N.f64(E_elem)
        N.check(N.lib().MSG_ASSEMBLE_BSR(self.handle, N.ptr(E_elem), float(nu), C.byref(h)), self.ctx.handle,
                "MSG_ASSEMBLE_BSR")
        return GpuMatrix(self, h)

    def assemble_from_element_matrices(self, Ke):
        h = N._vp()
        Ke = N.f64(Ke)
        N.check(N.lib().MSG_ASSEMBLE_BSR_KE(self.handle, N.ptr(Ke), C.byref(h)), self.ctx.handle,
                "MSG_ASSEMBLE_BSR_KE")
        return GpuMatrix(self, h)

    def close(self):
        if self.handle:
            N.lib().MSG_MESH_DESTROY(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def h8_stiffness_batch(ctx, xyz, E, nu):
    """MSG_H8_KE_BATCH: packed K_e [n][300] (CalcH8GaussMatrices + CalcH8K)."""
    xyz = N.f64(xyz).reshape(-1, 24)
    n = xyz.shape[0]
    E = N.f64(np.broadcast_to(np.asarray(E, dtype=np.float64), (n,)))
    K = np.zeros((n, 300))
    N.check(N.lib().MSG_H8_KE_BATCH(ctx.handle, n, N.ptr(xyz), N.ptr(E), float(nu), N.ptr(K)), ctx.handle,
            "MSG_H8_KE_BATCH")
    return K


def h8_mass_batch(ctx, xyz, rho):
    """MSG_H8_ME_BATCH: packed consistent mass [n][300] (Hexa8.CalculateConsistentMass)."""
    xyz = N.f64(xyz).reshape(-1, 24)
    M = np.zeros((xyz.shape[0], 300))
    N.check(N.lib().MSG_H8_ME_BATCH(ctx.handle, xyz.shape[0], N.ptr(xyz), float(rho), N.ptr(M)), ctx.handle,
            "MSG_H8_ME_BATCH")
    return M


def h8_stress_batch(ctx, xyz, E, nu, u, du=None):
    """MSG_H8_STRESS_BATCH: Hexa8.CalculateStresses + CalculateForces for n
    elements: strains and stresses [n][8][6] at the Gauss points, internal forces
    [n][24] (stresses from the increment du; du = u when omitted)."""
    xyz = N.f64(xyz).reshape(-1, 24)
    n = xyz.shape[0]
    E = N.f64(np.broadcast_to(np.asarray(E, dtype=np.float64), (n,)))
    u = N.f64(u).reshape(n, 24)
    du = None if du is None else N.f64(du).reshape(n, 24)
    eps, sig, f = np.zeros((n, 8, 6)), np.zeros((n, 8, 6)), np.zeros((n, 24))
    N.check(N.lib().MSG_H8_STRESS_BATCH(ctx.handle, n, N.ptr(xyz), N.ptr(E), float(nu), N.ptr(u),
                                        None if du is None else N.ptr(du), N.ptr(eps), N.ptr(sig), N.ptr(f)),
            ctx.handle, "MSG_H8_STRESS_BATCH")
    return eps, sig, f


def realization_stresses(mesh, E, nu, X, strains=True, stresses=True, forces=True):
    """MSG_STRESS_BATCH_DEVICE: stress recovery of every element of every
    realization on the device. E [R][n_elems] and X [R][n_dofs] are CUDA
    float64 tensors (the KL field and the batch solutions); returns CUDA
    tensors strains, stresses [R][n_elems][8][6] and forces [R][n_elems][24]
    (None where not requested)."""
    import torch
    R = int(X.shape[0])
    ne = mesh.model.n_elems
    assert E.is_cuda and X.is_cuda and E.dtype == torch.float64 and X.dtype == torch.float64
    E = E.contiguous()
    X = X.contiguous()
    out = [torch.empty((R, ne, 8, 6), dtype=torch.float64, device=X.device) if strains else None,
           torch.empty((R, ne, 8, 6), dtype=torch.float64, device=X.device) if stresses else None,
           torch.empty((R, ne, 24), dtype=torch.float64, device=X.device) if forces else None]
    ptrs = [C.c_void_p(t.data_ptr()) if t is not None else None for t in out]
    N.check(N.lib().MSG_STRESS_BATCH_DEVICE(mesh.handle, R, C.c_void_p(E.data_ptr()), float(nu),
                                            C.c_void_p(X.data_ptr()), *ptrs), mesh.ctx.handle,
            "MSG_STRESS_BATCH_DEVICE")
    return tuple(out)


class ProblemStructural:
    """IStaticProvider: builds the global stiffness on the device
    (ProblemStructural.BuildKs / CalculateMatrix, ProblemStructural.cs:63-89, 217-221)."""

    def __init__(self, ctx, model):
        self.ctx, self.model = ctx, model
        self.mesh = GpuMesh(ctx, model)
        self.K = None

    def Reset(self):
        if self.K is not None:
            self.K.close()
        self.K = None

    def CalculateMatrix(self, subdomain=None):
        if self.K is None:
            self.K = self.mesh.assemble(self.model.E_elem, self.model.poisson)
        return self.K


class SolverPCG:
    """ISolver over the device Jacobi-PCG (SolverPCG.Solve, PCG/SolverPCG.cs:105-149).
    Solve() uses (20000, 1e-7) as SolverPCG<T>.Solve() does (SolverPCGSkyline.cs:102-108).
    precision="mixed": FP32 matrix values in the loop, FP64 refinement to the FP64
    true residual (MSG_PCG_SOLVE_MIXED)."""

    def __init__(self, ctx, model, max_iterations=20000, tolerance=1e-7, precision="fp64"):
        self.ctx, self.model = ctx, model
        self.max_iterations, self.tolerance = max_iterations, tolerance
        self.precision = precision
        self.matrix = None
        self.iterations = 0
        self.rel_res = None

    def Initialize(self):
        if self.matrix is None:
            raise N.InvalidOperationError(N.MSG_ERR_INVALID_ARGUMENT, "no matrix: call BuildMatrices first")

    def Solve(self, max_iterations=None, tolerance=None):
        s = self.model.subdomains[0]
        b = N.f64(s.RHS)
        x = np.zeros(self.model.n_dofs)
        it, rr = C.c_int(0), C.c_double(0)
        fn = N.lib().MSG_PCG_SOLVE_MIXED if self.precision == "mixed" else N.lib().MSG_PCG_SOLVE
        st = fn(self.matrix.handle, N.ptr(b), N.ptr(x), int(max_iterations or self.max_iterations),
                float(tolerance or self.tolerance), C.byref(it), C.byref(rr))
        self.iterations, self.rel_res = it.value, rr.value
        s.Solution = x
        N.check(st, self.ctx.handle, "MSG_PCG_SOLVE")
        return x


class SolverPCGReorthogonalizationSearchVectorCalculator:
    """The re-orthogonalising search-vector calculator
    (SolverPCGReorthogonalizationSearchVectorCalculator.cs:11-65) as a device store of
    (p, K p) pairs for one mesh (MSG_SVS_*), at most `capacity` pairs."""

    def __init__(self, mesh, capacity):
        h = C.c_void_p()
        N.check(N.lib().MSG_SVS_CREATE(mesh.handle, int(capacity), C.byref(h)), mesh.ctx.handle, "MSG_SVS_CREATE")
        self.mesh, self.handle, self.capacity = mesh, h, capacity

    @property
    def count(self):
        c = C.c_int(0)
        N.check(N.lib().MSG_SVS_COUNT(self.handle, C.byref(c)))
        return c.value

    def ClearSearchVectors(self, vectors_to_keep_from_top=0):
        N.check(N.lib().MSG_SVS_CLEAR(self.handle, int(vectors_to_keep_from_top)), self.mesh.ctx.handle,
                "MSG_SVS_CLEAR")

    def close(self):
        if self.handle:
            N.lib().MSG_SVS_DESTROY(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolverPCGReorthogonalized(SolverPCG):
    """SolverPCG with the re-orthogonalising search-vector calculator
    (MSG_PCG_SOLVE_REORTH). start_from_store: 0 x0 = 0; 1 the starting vector
    from the stored directions (InitializeStartingVectorFromSearchVectors), the
    store kept; 2 the same starting vector, then a fresh store (for a changed matrix)."""

    def __init__(self, ctx, model, search, max_iterations=20000, tolerance=1e-7, start_from_store=0):
        super().__init__(ctx, model, max_iterations, tolerance)
        self.search, self.start_from_store = search, start_from_store

    def Solve(self, max_iterations=None, tolerance=None, start_from_store=None):
        s = self.model.subdomains[0]
        b = N.f64(s.RHS)
        x = np.zeros(self.model.n_dofs)
        it, rr = C.c_int(0), C.c_double(0)
        start = self.start_from_store if start_from_store is None else start_from_store
        st = N.lib().MSG_PCG_SOLVE_REORTH(self.matrix.handle, self.search.handle, N.ptr(b), N.ptr(x), int(start),
                                          int(max_iterations or self.max_iterations),
                                          float(tolerance or self.tolerance), C.byref(it), C.byref(rr))
        self.iterations, self.rel_res = it.value, rr.value
        s.Solution = x
        N.check(st, self.ctx.handle, "MSG_PCG_SOLVE_REORTH")
        return x


class LinearAnalyzer:
    """IAnalyzer child: Initialize -> solver.Initialize, Solve -> solver.Solve (LinearAnalyzer.cs:57-69)."""

    def __init__(self, solver):
        self.solver = solver
        self.ParentAnalyzer = None

    def BuildMatrices(self):
        if self.ParentAnalyzer is None:
            raise N.InvalidOperationError(N.MSG_ERR_INVALID_ARGUMENT, "linear analyzer needs a parent")
        self.ParentAnalyzer.BuildMatrices()

    def Initialize(self):
        self.solver.Initialize()

    def Solve(self):
        self.solver.Solve()


class StaticAnalyzer:
    """IAnalyzer parent (StaticAnalyzer.cs:18-75)."""

    def __init__(self, provider, child):
        self.provider, self.ChildAnalyzer = provider, child
        child.ParentAnalyzer = self

    def BuildMatrices(self):
        self.ChildAnalyzer.solver.matrix = self.provider.CalculateMatrix(self.provider.model.subdomains[0])

    def Initialize(self):
        self.ChildAnalyzer.Initialize()

    def Solve(self):
        self.ChildAnalyzer.Solve()


class LognormalStochasticCoefficientsProvider:
    """KL lognormal Young's modulus (LognormalFileStochasticCoefficientsProvider.cs:43-193).
    The eigen-data table the reference reads from a file is built analytically
    for the separable exponential kernel (MSG_KL_TABLE)."""

    def __init__(self, domain, corr_len, n_terms=50, n1d=16, mean=1.0, sigma=0.3, mean_correction=False):
        self.domain = np.asarray(domain, dtype=np.float64)
        self.n_terms, self.mean, self.sigma, self.mean_correction = n_terms, mean, sigma, mean_correction
        self.w = np.zeros((n_terms, 3))
        self.amp = np.zeros((n_terms, 3))
        self.idx = np.zeros((n_terms, 3), dtype=np.int32)
        self.eig = np.zeros(n_terms)
        N.check(N.lib().MSG_KL_TABLE(N.ptr(N.f64(self.domain)), float(corr_len), n_terms, n1d, N.ptr(self.w),
                                     N.ptr(self.amp), N.ptr(self.idx, N._i), N.ptr(self.eig)), None, "MSG_KL_TABLE")
        self.RandomVariables = None

    def struct(self):
        s = N.MSG_KL()
        s.n_terms = self.n_terms
        s.w3, s.amp3, s.eig = N.ptr(self.w), N.ptr(self.amp), N.ptr(self.eig)
        s.idx3 = N.ptr(self.idx, N._i)
        for a in range(3):
            s.domain[a] = float(self.domain[a])
        s.mean, s.sigma, s.mean_correction = float(self.mean), float(self.sigma), int(bool(self.mean_correction))
        s.gaussian = 1 if getattr(self, "gaussian", False) else 0
        return s

    def table(self):
        return dict(w=self.w, amp=self.amp, idx=self.idx, eig=self.eig)

    def field(self, mesh, xi):
        xi = N.f64(np.atleast_2d(xi))
        E = np.zeros((xi.shape[0], mesh.model.n_elems))
        s = self.struct()
        N.check(N.lib().MSG_KL_FIELD(mesh.handle, C.byref(s), xi.shape[0], N.ptr(xi), N.ptr(E)), mesh.ctx.handle,
                "MSG_KL_FIELD")
        return E


class GaussianStochasticCoefficientsProvider(LognormalStochasticCoefficientsProvider):
    """KL Gaussian Young's modulus (GaussianFileStochasticCoefficientsProvider.cs:24-108):
    E = mean (1 + sum_k xi_k covariance sqrt(eig_k) phi_k(x)), the reference's
    covariance 0.15 by default, on the same analytic table."""
    gaussian = True

    def __init__(self, domain, corr_len, n_terms=50, n1d=16, mean=1.0, covariance=0.15):
        super().__init__(domain, corr_len, n_terms, n1d, mean=mean, sigma=covariance)
        self.covariance = covariance


def _timespan(seconds):
    """C# TimeSpan.ToString() layout (hh:mm:ss.fffffff), as the reference's -Times.txt lines."""
    ticks = int(round(seconds * 1e7))
    h, rem = divmod(ticks, 36000000000)
    m, rem = divmod(rem, 600000000)
    sec, frac = divmod(rem, 10000000)
    return f"{h:02d}:{m:02d}:{sec:02d}" + (f".{frac:07d}" if frac else "")


def write_randoms(path, table):
    """The reference's random-number file (MonteCarloAnalyzerWithStochasticMaterial.cs:197-203):
    one value per line, expansion term outermost: for j in terms, for i in simulations."""
    table = np.asarray(table, dtype=np.float64)
    with open(path, "w") as f:
        for j in range(table.shape[1]):
            for i in range(table.shape[0]):
                f.write(repr(float(table[i, j])) + "\n")


def read_randoms(path, simulations, expansion_order):
    """Read `simulations` x `expansion_order` values in the layout of write_randoms
    (MonteCarloAnalyzerWithStochasticMaterial.cs:207-215, randomFileSimulations rows)."""
    vals = np.loadtxt(path, dtype=np.float64, ndmin=1)
    need = simulations * expansion_order
    if vals.size < need:
        raise ValueError(f"{path}: {vals.size} values, {need} needed ({simulations} x {expansion_order})")
    return vals[:need].reshape(expansion_order, simulations).T.copy()


class MonteCarloAnalyzerWithStochasticMaterial:
    """The realization loop (MonteCarloAnalyzerWithStochasticMaterial.cs:55-296).
    Initialize() draws xi[simulations][expansion_order] ~ N(0,1) from a seeded
    generator (the reference draws with Troschuetz.Random; the stream is not part
    of parity, the same table feeds every implementation), or reads the
    reference's random-number file (`randoms_read_file_name`, its first
    `random_file_simulations` rows). Solve() runs realizations
    simulation_start_from ... simulation_start_from + simulations - 1 of that
    table through MSG_MC_SOLVE_BATCH in `mode` ("mixed": batched mixed-precision
    launches; "fp64": the plain FP64 drop-in, one realization after another), in
    batches of `batch_size` (all at once by default). Results: Solutions
    [R][n_dofs] (if keep_solutions), TipValues [R], Iterations [R], Residuals [R].

    With `file_name_for_logging` the reference's text files are written:
    randoms{order}.txt next to it when the table is drawn, and per solved
    realization {name}-{order}-{start}.txt (tip value), -Iters.txt (operator
    products; the reference writes a counter it never fills) and -Times.txt
    (rewritten after every batch). With `checkpoint` (a path) the analyzer
    resumes by realization index: after every batch it saves the finished mask
    with the tip values, iterations and residuals next to a fingerprint of the
    realization table; a later Solve() with the same table solves only the
    realizations not yet finished (their Solutions rows stay NaN). With
    `autotune` (True or a tuning.Autotuner, which may carry a JSON cache) the
    mixed mode first picks the loop configuration on the first batch and uses
    it for this Solve() (TunedOptions; the context's options are restored
    afterwards)."""

    def __init__(self, ctx, model, coefficients_provider, expansion_order=50, simulations=1, seed=12345,
                 mode="mixed", max_iterations=20000, tolerance=1e-8, keep_solutions=True, tip_dof=None,
                 randoms_read_file_name="", simulation_start_from=0, random_file_simulations=50000,
                 file_name_for_logging=None, batch_size=None, checkpoint=None, autotune=None):
        self.ctx, self.model, self.kl = ctx, model, coefficients_provider
        self.expansion_order, self.simulations, self.seed = expansion_order, simulations, seed
        self.mode = N.MSG_MODE_MIXED_BATCHED if mode == "mixed" else N.MSG_MODE_FP64_BSR
        self.max_iterations, self.tolerance = max_iterations, tolerance
        self.keep_solutions = keep_solutions
        self.tip_dof = _tip_dof(model) if tip_dof is None else tip_dof
        if simulation_start_from < 0 or simulations < 1:
            raise N.ArgumentError(N.MSG_ERR_INVALID_ARGUMENT, "simulations must be >= 1 and simulation_start_from >= 0")
        self.randoms_read_file_name = randoms_read_file_name
        self.simulation_start_from = simulation_start_from
        self.random_file_simulations = random_file_simulations
        self.file_name_for_logging = file_name_for_logging
        self.batch_size = batch_size
        self.checkpoint = checkpoint
        self.autotune = autotune
        self.TunedOptions = None
        self._mesh = None
        self.RandomNumbers = None

    @property
    def mesh(self):
        if self._mesh is None:
            self._mesh = GpuMesh(self.ctx, self.model)
        return self._mesh

    def Initialize(self):
        order = self.expansion_order
        if self.randoms_read_file_name:
            self.RandomNumbers = read_randoms(self.randoms_read_file_name, self.random_file_simulations, order)
        else:
            rng = np.random.default_rng(self.seed)
            self.RandomNumbers = rng.standard_normal((self.simulations, order))
            if self.file_name_for_logging is not None:
                folder = os.path.dirname(self.file_name_for_logging)
                write_randoms(os.path.join(folder, f"randoms{order}.txt"), self.RandomNumbers)

    def _rows(self):
        s0, R = self.simulation_start_from, self.simulations
        table = np.asarray(self.RandomNumbers, dtype=np.float64)
        if table.ndim != 2 or table.shape[1] < self.expansion_order or table.shape[0] < s0 + R:
            raise N.ArgumentError(N.MSG_ERR_INVALID_ARGUMENT,
                                  f"random-number table {table.shape} does not hold realizations {s0}..{s0 + R - 1} "
                                  f"of {self.expansion_order} terms")
        return np.ascontiguousarray(table[s0:s0 + R, :self.expansion_order])

    def _solve_batch(self, xi):
        """One MSG_MC_SOLVE_BATCH call: (tip, iterations, residuals, solutions or None)."""
        R = xi.shape[0]
        xi = N.f64(xi)
        b = N.f64(self.model.subdomains[0].RHS)
        X = np.zeros((R, self.model.n_dofs)) if self.keep_solutions else None
        tip = np.zeros(R)
        its = np.zeros(R, dtype=np.int32)
        res = np.zeros(R)
        s = self.kl.struct()
        st = N.lib().MSG_MC_SOLVE_BATCH(self.mesh.handle, float(self.model.poisson), C.byref(s), R, N.ptr(xi), N.ptr(b),
                                        self.mode, int(self.max_iterations), float(self.tolerance), int(self.tip_dof),
                                        N.ptr(X) if X is not None else None, N.ptr(tip), N.ptr(its, N._i), N.ptr(res))
        if st not in (N.MSG_OK, N.MSG_ERR_NOT_CONVERGED, N.MSG_ERR_BREAKDOWN):  # per-realization outcomes
            N.check(st, self.ctx.handle, "MSG_MC_SOLVE_BATCH")
        return tip, its, res, X, st

    def _log_names(self):
        base = f"{self.file_name_for_logging}-{self.expansion_order}-{self.simulation_start_from}"
        return base + ".txt", base + "-Iters.txt", base + "-Times.txt"

    def _load_checkpoint(self, xi):
        fp = np.frombuffer(hashlib.sha256(xi.tobytes()).digest(), dtype=np.uint8)
        R = xi.shape[0]
        state = dict(done=np.zeros(R, dtype=bool), tip=np.zeros(R), its=np.zeros(R, dtype=np.int32), res=np.zeros(R),
                     fingerprint=fp)
        if self.checkpoint and os.path.exists(self.checkpoint):
            with np.load(self.checkpoint) as z:
                if not np.array_equal(z["fingerprint"], fp) or int(z["start"]) != self.simulation_start_from:
                    raise ValueError(f"{self.checkpoint}: checkpoint of another realization table or start index")
                for k in ("done", "tip", "its", "res"):
                    state[k] = z[k].copy()
        return state

    def _save_checkpoint(self, state):
        tmp = self.checkpoint + ".tmp.npz"
        np.savez(tmp, start=np.int64(self.simulation_start_from), **state)
        os.replace(tmp, self.checkpoint)

    def Solve(self):
        if self.RandomNumbers is None:
            self.Initialize()
        xi = self._rows()
        R = xi.shape[0]
        state = self._load_checkpoint(xi)
        X = np.full((R, self.model.n_dofs), np.nan) if self.keep_solutions else None
        logging = self.file_name_for_logging is not None
        if logging and not state["done"].any():
            for name in self._log_names()[:2]:
                open(name, "w").close()
        todo = np.flatnonzero(~state["done"])
        batch = int(self.batch_size or R)
        restore = None
        if self.autotune and self.mode == N.MSG_MODE_MIXED_BATCHED and len(todo):
            from .tuning import Autotuner
            tuner = self.autotune if isinstance(self.autotune, Autotuner) else Autotuner(self.ctx)
            self.TunedOptions = tuner.tune_mc(self.mesh, self.kl, xi[todo[:batch]], tol=self.tolerance,
                                              max_iterations=self.max_iterations)
            restore = {k: self.ctx.get_option(k) for k in self.TunedOptions}
            tuner.apply(self.TunedOptions)
        try:
            status = self._solve_todo(xi, todo, batch, state, X)
        finally:
            if restore:
                for k, v in restore.items():
                    self.ctx.set_option(k, v)
        self.Solutions, self.TipValues = X, state["tip"]
        self.Iterations, self.Residuals = state["its"], state["res"]
        if status != N.MSG_OK:
            N.check(status, self.ctx.handle if self.ctx is not None else None, "MSG_MC_SOLVE_BATCH")
        return self.TipValues

    def _solve_todo(self, xi, todo, batch, state, X):
        logging = self.file_name_for_logging is not None
        status = N.MSG_OK
        t_all = time.perf_counter()
        t_solve = 0.0
        for k in range(0, len(todo), batch):
            idx = todo[k:k + batch]
            t0 = time.perf_counter()
            tip, its, res, Xb, st = self._solve_batch(xi[idx])
            t_solve += time.perf_counter() - t0
            if st != N.MSG_OK:
                status = st
            state["tip"][idx], state["its"][idx], state["res"][idx] = tip, its, res
            state["done"][idx] = True
            if X is not None and Xb is not None:
                X[idx] = Xb
            if logging:
                values, iters, times = self._log_names()
                with open(values, "a") as f:
                    f.writelines(repr(float(v)) + "\n" for v in tip)
                with open(iters, "a") as f:
                    f.writelines(f"{int(v)}\n" for v in its)
                with open(times, "w") as f:
                    f.write(f"Elements: {_timespan(0.0)}\nFactorize: {_timespan(0.0)}\n"
                            f"Solution: {_timespan(t_solve)}\nAll: {_timespan(time.perf_counter() - t_all)}\n"
                            f"Total iterations: {int(state['its'][state['done']].sum())}\n")
            if self.checkpoint:
                self._save_checkpoint(state)
        return status

    def statistics(self):
        t = self.TipValues
        return dict(mean=float(np.mean(t)), variance=float(np.var(t, ddof=1)) if len(t) > 1 else 0.0)


class MonteCarloAnalyzer(MonteCarloAnalyzerWithStochasticMaterial):
    """Gaussian-field Monte Carlo (ISAAR.MSolve.Analyzers/MonteCarloAnalyzer.cs:35-198).
    The reference builds K_0 and one matrix K_k per expansion term and solves
    K_0 + sum_k xi_k K_k for every realization. The element stiffness is linear
    in E, so that sum is the stiffness of the field E = mean (1 + sum_k xi_k
    psi_k); the batch evaluates that field and runs the same batched solve as the
    lognormal analyzer (no per-term matrices are stored)."""

    def __init__(self, ctx, model, coefficients_provider, expansion_order=50, simulations=1, **kw):
        if not getattr(coefficients_provider, "gaussian", False):
            raise TypeError("MonteCarloAnalyzer needs a GaussianStochasticCoefficientsProvider")
        super().__init__(ctx, model, coefficients_provider, expansion_order, simulations, **kw)


class RaggedMonteCarloBatch:
    """Monte Carlo realizations of several models of uneven size in one batch
    (MSG_MC_SOLVE_RAGGED): each added system is a model (any Hexa8 mesh), its
    coefficient provider and its random-number rows; Solve() runs the
    realization loop of MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
    (MonteCarloAnalyzerWithStochasticMaterial.cs:232-296) for all of them in the
    same launches (mixed-precision PCG, FP64 true residual below `tolerance`;
    with the context's multigrid option on, each system whose mesh has lattice
    numbering is preconditioned by the V-cycle of its cube lattice, the others
    by the diagonal). Results per system, in the order added: Solutions
    [R][n_dofs] (if keep_solutions), TipValues [R], Iterations [R], Residuals
    [R]. A system's results do not depend on the other systems in the batch.
    The meshes are uploaded once, in add(); Solve() may be called again."""

    def __init__(self, ctx, max_iterations=20000, tolerance=1e-8):
        self.ctx, self.max_iterations, self.tolerance = ctx, max_iterations, tolerance
        self.systems = []
        self.Results = []

    def add(self, model, coefficients_provider, random_numbers, tip_dof=None, keep_solutions=True):
        xi = np.ascontiguousarray(np.atleast_2d(random_numbers)[:, :coefficients_provider.n_terms], dtype=np.float64)
        if xi.shape[1] != coefficients_provider.n_terms or xi.shape[0] < 1:
            raise N.ArgumentError(N.MSG_ERR_INVALID_ARGUMENT,
                                  f"random numbers {xi.shape} for {coefficients_provider.n_terms} KL terms")
        self.systems.append(dict(model=model, kl=coefficients_provider, xi=xi,
                                 tip_dof=_tip_dof(model) if tip_dof is None else tip_dof,
                                 keep=keep_solutions, mesh=GpuMesh(self.ctx, model)))
        return len(self.systems) - 1

    def Solve(self):
        n = len(self.systems)
        arr = (N.MSG_RAGGED_SYSTEM * max(1, n))()
        keep = []  # ctypes structs and arrays alive for the call
        self.Results = []
        for i, y in enumerate(self.systems):
            m, R = y["model"], y["xi"].shape[0]
            res = dict(Solutions=np.zeros((R, m.n_dofs)) if y["keep"] else None, TipValues=np.zeros(R),
                       Iterations=np.zeros(R, dtype=np.int32), Residuals=np.zeros(R))
            kl = y["kl"].struct()
            b = N.f64(m.subdomains[0].RHS)
            keep += [kl, b]
            a = arr[i]
            a.mesh, a.nu, a.kl, a.R = y["mesh"].handle, float(m.poisson), C.pointer(kl), R
            a.xi, a.b, a.tip_dof = N.ptr(y["xi"]), N.ptr(b), int(y["tip_dof"])
            a.X = N.ptr(res["Solutions"]) if y["keep"] else None
            a.tip, a.iterations, a.rel_res = N.ptr(res["TipValues"]), N.ptr(res["Iterations"], N._i), N.ptr(res["Residuals"])
            self.Results.append(res)
        st = N.lib().MSG_MC_SOLVE_RAGGED(self.ctx.handle, n, arr, int(self.max_iterations), float(self.tolerance))
        N.check(st, self.ctx.handle, "MSG_MC_SOLVE_RAGGED")
        return self.Results


class NewmarkDynamicAnalyzer:
    """Implicit Newmark integration (NewmarkDynamicAnalyzer.cs:16-315) of every
    realization of a stochastic-material batch at once. Same parameters as the
    reference (alpha, delta, timeStep, totalTime; the loop runs
    int(totalTime / timeStep) steps), with the structural provider's effective
    matrix K + a0 M + a1 C, Rayleigh damping C = rayleigh_alpha M + rayleigh_beta K
    (Hexa8.DampingMatrix) and a MassAccelerationSinusoidalLoad as ground
    acceleration. BuildMatrices() checks the coefficients (InitializeCoefficients),
    Initialize() draws xi, Solve() runs MSG_NEWMARK_BATCH. Results: TipHistory
    [R][n_steps], Solutions [R][n_dofs] (final displacements), Iterations [R]."""

    def __init__(self, ctx, model, coefficients_provider, alpha, delta, time_step, total_time, load,
                 expansion_order=50, simulations=1, seed=12345, density=1.0, rayleigh_alpha=0.0, rayleigh_beta=0.0,
                 max_iterations=20000, tolerance=1e-8, tip_dof=None, static_loads=False):
        self.ctx, self.model, self.kl = ctx, model, coefficients_provider
        self.alpha, self.delta, self.time_step, self.total_time = alpha, delta, time_step, total_time
        self.load = load
        self.expansion_order, self.simulations, self.seed = expansion_order, simulations, seed
        self.density, self.rayleigh_alpha, self.rayleigh_beta = density, rayleigh_alpha, rayleigh_beta
        self.max_iterations, self.tolerance = max_iterations, tolerance
        self.tip_dof = _tip_dof(model) if tip_dof is None else tip_dof
        self.static_loads = static_loads
        self.mesh = GpuMesh(ctx, model)
        self.RandomNumbers = None

    @property
    def steps(self):
        return int(self.total_time / self.time_step)

    def BuildMatrices(self):
        if self.delta < 0.5:
            raise N.InvalidOperationError(N.MSG_ERR_INVALID_ARGUMENT, "Newmark delta has to be bigger than 0.5.")
        a_limit = 0.25 * (0.5 + self.delta) ** 2
        if self.alpha < a_limit:
            raise N.InvalidOperationError(N.MSG_ERR_INVALID_ARGUMENT,
                                          "Newmark alpha has to be bigger than %s." % a_limit)

    def Initialize(self):
        rng = np.random.default_rng(self.seed)
        self.RandomNumbers = rng.standard_normal((self.simulations, self.expansion_order))

    def params(self):
        nm = N.MSG_NEWMARK()
        nm.rho, nm.rayleigh_alpha, nm.rayleigh_beta = self.density, self.rayleigh_alpha, self.rayleigh_beta
        nm.alpha, nm.delta, nm.dt, nm.n_steps = self.alpha, self.delta, self.time_step, self.steps
        nm.acc_amp, nm.acc_period, nm.acc_dof = self.load.magnitude, self.load.period, self.load.dof
        return nm

    def Solve(self, keep_solutions=True):
        self.BuildMatrices()
        if self.RandomNumbers is None:
            self.Initialize()
        R, S = self.simulations, self.steps
        xi = N.f64(self.RandomNumbers)
        f = N.f64(self.model.subdomains[0].RHS) if self.static_loads else None
        hist = np.zeros((R, S))
        U = np.zeros((R, self.model.n_dofs)) if keep_solutions else None
        its = np.zeros(R, dtype=np.int32)
        s = self.kl.struct()
        nm = self.params()
        st = N.lib().MSG_NEWMARK_BATCH(self.mesh.handle, float(self.model.poisson), C.byref(s), R, N.ptr(xi),
                                       C.byref(nm), N.ptr(f) if f is not None else None, int(self.max_iterations),
                                       float(self.tolerance), int(self.tip_dof), N.ptr(hist),
                                       N.ptr(U) if U is not None else None, N.ptr(its, N._i))
        self.TipHistory, self.Solutions, self.Iterations = hist, U, its
        N.check(st, self.ctx.handle, "MSG_NEWMARK_BATCH")
        return hist
