"""Benchmark: batched mixed-precision Monte Carlo Hexa8 solves on B200.

Workload (one step): a batch of R realizations (default 1024) of a 32^3 Hexa8
block of unit cubes (35,937 nodes, 104,544 free DOFs), z=0 face clamped,
unit pressure on the top face (consistent weights), E_e = exp(sigma g(x_e))
with a 50-term separable-exponential KL field (l = 0.2 * 32, sigma = 0.3),
nu = 0.3, every realization solved to an FP64 true relative residual < tol
(default 1e-9, a decade inside the metric's 1e-8; the displacement error
against FP64 oracle solves of a sample of the batch is measured every run and
reported as rel_err_vs_oracle: about 3e-11) with the matrix-free FP32 PCG +
FP64 refinement path. Each step
draws a fresh xi table (seeded); state is ~4.6 GB per GPU, larger than L2.

value  = realizations solved per second with xi / b / X resident in HBM
         (MSG_MC_SOLVE_BATCH_DEVICE), all ranks summed (weak scaling).
e2e    = the same through the host-buffer entry point with pinned buffers: xi and
         b copied in, every realization's full displacement field copied out;
         MSG_MC_SOLVE_BATCH_PIPELINED, so that each step's copy out overlaps
         the next step's solve (e2e.blocking: MSG_MC_SOLVE_BATCH, which
         returns with the copy done).
fp64_dropin = the plain FP64 drop-in (assembled BSR + Jacobi PCG, one
         realization after another, MSG_MODE_FP64_BSR) on a sample of the batch.
roofline = the dominant kernel (k_op_modal: fused PCG direction update and
         matrix-free FP32 operator), live per-launch CUDA event durations
         inside the timed region.
cpu_baseline = the oracle (C++ FP64 restatement of the reference: assembled
         CSR Jacobi-PCG per realization) on the host cores, a bounded sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: torchrun --nproc-per-node N bench.py --gpus N (one rank per GPU,
realization batches sharded across ranks, one all-reduce of the tip statistics).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Hexa8 PCG solves/s at 1e-8 rel err, batched mixed vs plain FP64; p50/p99 latency"
# DRAM traffic of one k_op_modal launch per realization on the 32^3 lattice: ncu capture
# at R = 512 (dram__bytes_read.sum 1,165.9 MB + dram__bytes_write.sum 845.5 MB) / 512
OP_DRAM_BYTES_PER_REALIZATION = (1165.921e6 + 845.472e6) / 512
# the same for the multigrid loop's direction + operator launch (packed k_lvl_op2<PcgZ>, 3 x 3
# node tiles), 32^3 lattice, ncu capture at R = 512: dram__bytes_read.sum 823.2 MB +
# dram__bytes_write.sum 626.8 MB
MG_OP_DRAM_BYTES_PER_REALIZATION = (823.197e6 + 626.791e6) / 512


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=32)
    p.add_argument("--R", type=int, default=1024)
    p.add_argument("--terms", type=int, default=50)
    p.add_argument("--tol", type=float, default=1e-9)
    p.add_argument("--fp64-sample", type=int, default=8)
    p.add_argument("--cpu-sample", type=int, default=16,
                   help="realizations the in-arm CPU baseline (the oracle) solves")
    p.add_argument("--ref-sample", type=int, default=2,
                   help="--impl reference: realizations of the batch the oracle solves per step")
    p.add_argument("--parity-sample", type=int, default=8,
                   help="realizations of the headline batch checked against FP64 oracle solves")
    p.add_argument("--no-parity", action="store_true", help="skip the oracle comparisons")
    p.add_argument("--newmark-tol", type=float, default=1e-13,
                   help="FP64 true relative residual each Newmark step is solved to (the integration carries step "
                        "errors forward: 1e-13 keeps the displacement history within 1e-8 of an FP64 run)")
    p.add_argument("--newmark-parity", type=int, default=4,
                   help="realizations of the Newmark batch checked against the oracle's FP64 integration")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--reliable-delta", type=float, default=None, help="MSG_SET_OPTION reliable_delta")
    p.add_argument("--chunk", type=int, default=None, help="MSG_SET_OPTION chunk")
    p.add_argument("--no-newmark", action="store_true", help="skip the batched Newmark measurement")
    p.add_argument("--serve-persistent", type=int, default=None, choices=[0, 1],
                   help="MSG_SET_OPTION serve_persistent (serving lanes on persistent grids)")
    p.add_argument("--serve-priority", type=int, default=None, choices=[0, 1],
                   help="MSG_SET_OPTION serve_priority (stream priority by model size)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the library's default loop configuration instead of timing the candidates first")
    p.add_argument("--autotune-cache", default=None, help="JSON cache of tuned configurations (read and written)")
    p.add_argument("--newmark-R", type=int, default=256)
    p.add_argument("--newmark-n", type=int, default=24)
    p.add_argument("--newmark-steps", type=int, default=200)
    p.add_argument("--no-serving", action="store_true", help="skip the serving (continuous batching) measurement")
    p.add_argument("--no-single", action="store_true", help="skip the 64^3 single-solve measurement")
    p.add_argument("--single-n", type=int, default=64)
    p.add_argument("--no-ragged", action="store_true", help="skip the ragged (uneven mesh sizes) batch measurement")
    p.add_argument("--distorted-only", action="store_true",
                   help="only the batched solve of --R realizations on an --n cube with its interior nodes moved "
                        "(the element-by-element path), one JSON line")
    p.add_argument("--ragged-R", type=int, default=64, help="realizations per system of the ragged batch")
    p.add_argument("--ragged-only", action="store_true",
                   help="only the ragged batch of uneven mesh sizes (MSG_MC_SOLVE_RAGGED), one JSON line")
    p.add_argument("--single-only", action="store_true",
                   help="run only the single-solve measurement (FP64 and mixed) and print its JSON object")
    p.add_argument("--serve-rates", default="100,400,1000,2000,5000", help="Poisson arrival rates (requests/s) to run")
    p.add_argument("--serve-requests", type=int, default=300, help="requests per rate")
    p.add_argument("--multigrid", type=int, default=None, choices=[0, 1, 2],
                   help="MSG_SET_OPTION multigrid (1: V-cycle for systems without a mass term, 2: for all)")
    p.add_argument("--mg-levels", type=int, default=None, help="MSG_SET_OPTION multigrid_levels")
    p.add_argument("--mg-sweeps", type=int, default=None, help="MSG_SET_OPTION multigrid_sweeps (coarsest level)")
    p.add_argument("--mg-delta", type=float, default=None, help="MSG_SET_OPTION multigrid_delta")
    p.add_argument("--mg-omega", type=float, default=None, help="MSG_SET_OPTION multigrid_omega")
    p.add_argument("--mg-packed", type=int, default=None, choices=[0, 1],
                   help="MSG_SET_OPTION multigrid_packed (0: level operators on 32-realization tiles)")
    p.add_argument("--option", action="append", default=[], metavar="KEY=VALUE",
                   help="MSG_SET_OPTION before anything runs (repeatable)")
    p.add_argument("--tensor-op", type=int, default=None, choices=[0, 1],
                   help="MSG_SET_OPTION tensor_operator (1: level-0 search-direction launch on the tensor cores)")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu):
        self.gpu, self.proc, self.path = gpu, None, None

    def start(self):
        self.path = f"/tmp/msg_clocks_{os.getpid()}.csv"
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 8:
                try:
                    rows.append((float(f[0]), float(f[1]), f[4], f[5], f[6], f[7]))
                except ValueError:
                    pass
        if not rows:
            return None
        sm = [r[0] for r in rows]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": float(rows[0][1]), "reasons": sorted(reasons),
                "samples": len(rows)}


def make_problem(args):
    import msolve_b200 as M
    model = M.clamped_block_model(args.n)
    kl = M.LognormalStochasticCoefficientsProvider([args.n] * 3, 0.2 * args.n, args.terms, 16)
    return model, kl


def tensor_roofline(args, model, R, op_ms):
    """Tensor-pipe figures of the tensor-core level-0 launch: useful FLOP (the
    24 x 24 element product, 1152 per element and realization) and issued MMA
    FLOP (per x-slab of a 3 x 3 tile of node pencils and 32 realizations: 4 M
    tiles x 4 corner pairs x (N 64 + N 32) x M 128 x K 8), per second."""
    n = args.n
    tiles = ((n + 1 + 2) // 3) ** 2
    issued = 2.0 * 4 * 4 * (128 * 64 * 8 + 128 * 32 * 8) * tiles * ((R + 31) // 32) * n
    sec = op_ms / 1e3
    return {"useful_tflops": 1152.0 * model.n_elems * R / sec / 1e12, "issued_tflops": issued / sec / 1e12,
            "unit": "TFLOP/s (TF32)"}


def workload_config(args, ws):
    """The headline workload, named the same by both arms."""
    n = args.n
    return {"workload": f"batched Monte Carlo, {args.R} realizations x {n}^3 Hexa8 per GPU per step (z=0 clamped, "
                        f"unit top pressure, {args.terms}-term KL lognormal E, sigma 0.3, l 0.2*side, nu 0.3), every "
                        f"realization solved to an FP64 relative residual < {args.tol:g}",
            "realizations_per_gpu": args.R, "mesh": f"{n}x{n}x{n}", "free_dofs": 3 * (n + 1) ** 2 * n,
            "kl_terms": args.terms, "tol_true_residual": args.tol,
            "l2": "inputs larger than L2 (per-GPU batch state ~4.6 GB)", "parallelism": f"realizations x{ws}"}


def oracle_fields(P, xi):
    import oracle as O
    return O.kl_field(P["centroids"], P["domain"], P["table"], np.atleast_2d(xi), sigma=0.3)


def cpu_baseline(args, P, xi_host):
    """Oracle (the restated reference) on the host cores: per realization the KL
    field, FP64 element matrices, CSR assembly and Jacobi-PCG to the same
    tolerance (SolverPCG stopping rule), realizations one after another with
    OpenMP inside each solve; a bounded sample of the batch."""
    import oracle as O
    n, k = args.n, args.cpu_sample
    t0 = time.perf_counter()
    E = oracle_fields(P, xi_host[:k])
    its = []
    for r in range(k):
        x, info = O.block_solve_pcg(n, n, n, P["constrained"], E[r], 0.3, P["b"], tol=args.tol, max_it=100000)
        its.append(info["iterations"])
    dt = time.perf_counter() - t0
    return {"value": k / dt, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{k} realizations of the {n}^3 batch, FP64 KL field + CSR assembly + Jacobi-PCG to tol "
                      f"{args.tol:g} (mean {np.mean(its):.0f} iterations), {dt:.1f} s"}


def mc_parity(args, P, xi_rows, X_rows, tol=1e-12):
    """Max-norm relative displacement error of GPU realizations against FP64
    oracle solves of the same fields converged to `tol`."""
    import oracle as O
    n = args.n
    E = oracle_fields(P, xi_rows)
    errs, its = [], []
    for i in range(E.shape[0]):
        xo, info = O.block_solve_pcg(n, n, n, P["constrained"], E[i], 0.3, P["b"], tol=tol, max_it=100000)
        errs.append(float(np.abs(X_rows[i] - xo).max() / np.abs(xo).max()))
        its.append(info["iterations"])
    return errs, its


def newmark_leg(args, ctx):
    """Batched Newmark dynamics (R realizations x n^3 Hexa8, 200 steps of dt 0.01,
    average acceleration beta 0.25 / gamma 0.5, Rayleigh 0.01 M + 0.001 K,
    ground acceleration 0.1 sin(2 pi t) in x, rho 1), timed end to end through
    MSG_NEWMARK_BATCH after one warm-up call; then a sample of its realizations
    against the oracle's FP64 integration (every step converged to 1e-14)."""
    import msolve_b200 as M
    n, R, S = args.newmark_n, args.newmark_R, args.newmark_steps
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, args.terms, 12)
    dt = 0.01
    load = M.MassAccelerationSinusoidalLoad(1.0, dt, dt * S, 0.1, dof=0)
    corner = int(np.argmax(model.xyz.sum(1)))
    nm = M.NewmarkDynamicAnalyzer(ctx, model, kl, 0.25, 0.5, dt, dt * S, load, expansion_order=args.terms,
                                  simulations=R, density=1.0, rayleigh_alpha=0.01, rayleigh_beta=0.001,
                                  tolerance=args.newmark_tol, tip_dof=int(model.dof[corner, 0]), seed=7)
    nm.Initialize()
    import torch
    nm.Solve(keep_solutions=False)  # warm-up (graph capture, workspace)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    hist = nm.Solve(keep_solutions=False)
    b.record()
    b.synchronize()
    sec = a.elapsed_time(b) / 1e3
    out = {"workload": f"batched Newmark, {R} realizations x {n}^3 Hexa8, {nm.steps} steps (dt 0.01, beta 0.25, "
                       f"gamma 0.5, Rayleigh 0.01 M + 0.001 K, ground acceleration 0.1 sin(2 pi t) in x), "
                       f"FP64 true residual < {args.newmark_tol:g} per step, warm start",
           "seconds": sec, "realization_steps_per_s": R * nm.steps / sec,
           "mean_iterations_per_step": float(np.mean(nm.Iterations)) / nm.steps,
           "tip_ux_final_mean": float(np.mean(hist[:, -1]))}
    k = min(args.newmark_parity, R)
    if not args.no_parity and k > 0:
        import oracle as O
        nm.Solve(keep_solutions=True)  # same realizations again, final fields kept
        P = O.block_problem(n, args.terms, 12)
        rows = np.linspace(0, R - 1, k).astype(int)
        E = oracle_fields(P, nm.RandomNumbers[rows])
        t0 = time.perf_counter()
        tip_err, u_err = [], []
        for i, r in enumerate(rows):
            t, u, info = O.block_newmark(n, n, n, P["constrained"], E[i], model.poisson, 1.0, 0.01, 0.001, 0.25, 0.5,
                                         dt, nm.steps, 0.1, 1.0, 0, model.n_dofs, solver=2, tol=1e-14,
                                         tip_dof=nm.tip_dof)
            tip_err.append(float(np.abs(hist[r] - t).max() / np.abs(t).max()))
            u_err.append(float(np.abs(nm.Solutions[r] - u).max() / np.abs(u).max()))
        out["oracle"] = {"realizations": [int(r) for r in rows], "tip_history_rel_err_max": max(tip_err),
                         "final_field_rel_err_max": max(u_err), "tip_history_rel_err": tip_err,
                         "final_field_rel_err": u_err, "oracle_seconds": time.perf_counter() - t0,
                         "oracle": "FP64 CSR Newmark restatement, each step Jacobi-PCG (warm start) to 1e-14; "
                                   "errors in the max norm relative to the oracle's maximum"}
    return out


def single_leg(args, ctx):
    """One large static solve (64^3 Hexa8, E = 1, nu 0.3, z=0 clamped, unit top
    pressure): (a) the FP64 assembled drop-in (MSG_PCG_SOLVE) and (b) FP32 matrix
    values + FP64 refinement (MSG_PCG_SOLVE_MIXED), both to the relative
    residual 1e-8, timed after one warm-up solve each. Algorithmic bytes per
    iteration: the SpMV (72 B FP64 / 36 B FP32 values + 4 B column per 3x3
    block, each vector read or written once) and the update pass (FP64: r, q, x,
    p, D^-1 read, r, x written; mixed: p, q, r, d, D^-1 read, p, r, d written, in
    FP32); hbm_frac = those bytes per iteration / time per iteration / the
    measured copy bandwidth."""
    import torch
    import msolve_b200 as M
    n = args.single_n
    model = M.clamped_block_model(n)
    mesh = M.GpuMesh(ctx, model)
    A = mesh.assemble(np.ones(model.n_elems), model.poisson)
    info = mesh.info()
    out = {"workload": f"{n}^3 Hexa8 static solve, {model.n_dofs} free DOFs, {info['nnzb']} 3x3 blocks, "
                       f"Jacobi PCG to ||r||/||b|| < 1e-8", "n_dofs": model.n_dofs, "nnzb": info["nnzb"]}
    sols = {}
    # the mixed variant stops on the FP64 true residual; run to 1e-8 (the
    # configuration) it ends 1.1e-8 from the oracle on this block, so it is also
    # run to 5e-9 (mixed_tol_5e-9), which ends inside 1e-8
    for name, prec, tol in (("fp64", "fp64", 1e-8), ("mixed", "mixed", 1e-8), ("mixed_tol_5e-9", "mixed", 5e-9)):
        s = M.SolverPCG(ctx, model, max_iterations=100000, tolerance=tol, precision=prec)
        s.matrix = A
        sols[name] = s.Solve().copy()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        s.Solve()
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        per_it = ms / max(1, s.iterations)
        # vectors of the SpMV pass: FP64 D^-1, r, p_old read and p_new, q written (the direction is formed in
        # that pass); mixed p (gathered), r, D^-1 read and q written in FP32
        spmv_bytes = ((72 if prec == "fp64" else 36) * info["nnzb"] + 4 * info["nnzb"]
                      + (5 * 8 if prec == "fp64" else 4 * 4) * 3 * model.n_nodes)
        update_bytes = (7 * 8 if prec == "fp64" else 8 * 4) * 3 * model.n_nodes
        peak, peak_src = load_peaks()
        out[name] = {"ms": ms, "iterations": s.iterations, "rel_res": s.rel_res, "ms_per_iteration": per_it,
                     "dof_iterations_per_s": model.n_dofs * s.iterations / (ms / 1e3),
                     "spmv_bytes_per_iteration": spmv_bytes, "update_bytes_per_iteration": update_bytes,
                     "hbm_frac": (spmv_bytes + update_bytes) / (per_it * 1e-3) / (peak * 1e9),
                     "hbm_peak": f"{peak:g} GB/s ({peak_src})"}
    out["mixed_over_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    out["mixed_tol_5e-9_over_fp64"] = out["fp64"]["ms"] / out["mixed_tol_5e-9"]["ms"]
    A.close()
    if not args.no_parity:
        import oracle as O
        P = O.block_problem(n, 1, 4)
        t0 = time.perf_counter()
        xo, info = O.block_solve_pcg(n, n, n, P["constrained"], np.ones(n ** 3), 0.3, P["b"], tol=1e-11,
                                     max_it=100000)
        out["oracle"] = {"oracle": "FP64 CSR Jacobi-PCG restatement of SolverPCG to 1e-11",
                         "iterations": info["iterations"], "seconds": time.perf_counter() - t0}
        for name in sols:
            out[name]["rel_err_vs_oracle"] = float(np.abs(sols[name] - xo).max() / np.abs(xo).max())
    return out


def cantilever_leg(args, ctx):
    """The plain small case: the linear-static cantilever of 10 x 4 x 4 unit
    cubes (275 nodes, 750 free DOFs), E = 1, nu 0.3, x = 0 face clamped, total
    load -1 in z split over the 25 nodes of the x = 10 face, FP64. The GPU FP64
    drop-in (MSG_PCG_SOLVE, Jacobi-PCG to the recursive 1e-10, timed after one
    warm-up solve) against the oracle on the host: skyline LDL^T (factorisation
    and substitution) and CSR Jacobi-PCG to 1e-10, both built from the oracle's
    own mesh, DOF and load functions."""
    import torch
    import msolve_b200 as M
    import oracle as O
    nx, ny, nz = 10, 4, 4
    model = M.cantilever_model(nx, ny, nz)
    xyz, conn = O.block_mesh(nx, ny, nz)
    cons = O.clamp_face(xyz, 0)
    dof, nd = O.enumerate_dofs(cons)
    b = O.load_tip(xyz, dof, nd, axis_face=0, comp=2, total=-1.0)
    assert nd == model.n_dofs and np.array_equal(b, model.subdomains[0].RHS)
    mesh = M.GpuMesh(ctx, model)
    A = mesh.assemble(np.ones(model.n_elems), model.poisson)
    s = M.SolverPCG(ctx, model, max_iterations=20000, tolerance=1e-10, precision="fp64")
    s.matrix = A
    s.Solve()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    xg = s.Solve().copy()
    ev1.record()
    ev1.synchronize()
    gpu_ms = ev0.elapsed_time(ev1)
    A.close()
    Ke = O.h8_stiffness_batch(O.element_xyz(xyz, conn), np.ones(conn.shape[0]), 0.3)[0]
    t0 = time.perf_counter()
    sk = O.Skyline(conn, dof, nd)
    sk.assemble(Ke)
    f, _ = sk.factorized()
    xs = sk.solve(f, b)
    sky_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    cs = O.CSR(xyz.shape[0], conn, dof, nd)
    cs.assemble(Ke)
    xp, info = cs.pcg_jacobi(b, tol=1e-10)
    pcg_ms = (time.perf_counter() - t0) * 1e3
    scale = np.abs(xs).max()
    return {"workload": "linear-static cantilever, 10 x 4 x 4 unit cubes, 750 free DOFs, E 1, nu 0.3, total load -1 "
                        "in z over the x = 10 face, FP64",
            "gpu_fp64_pcg_ms": gpu_ms, "gpu_iterations": s.iterations,
            "cpu_skyline_ldlt_ms": sky_ms, "cpu_csr_pcg_ms": pcg_ms, "cpu_pcg_iterations": info["iterations"],
            "cpu_threads": O.num_threads(),
            "rel_err_gpu_pcg_vs_skyline": float(np.abs(xg - xs).max() / scale),
            "rel_err_cpu_pcg_vs_skyline": float(np.abs(xp - xs).max() / scale)}


def cpu_serving_baseline(args, sides):
    """The oracle on the host cores, one request at a time, for the serving
    sides it solves within seconds (8 to 32; the 48^3 solve takes about half a
    minute and is left out): KL field, element matrices, CSR assembly and
    Jacobi-PCG to 1e-8, one realization of a fresh field per side."""
    import oracle as O
    per = {}
    for n in sides:
        if n > 32:
            continue
        P = O.block_problem(n, args.terms, 12)
        xi = np.random.default_rng(500 + n).standard_normal((1, args.terms))
        t0 = time.perf_counter()
        E = oracle_fields(P, xi)
        _, info = O.block_solve_pcg(n, n, n, P["constrained"], E[0], 0.3, P["b"], tol=1e-8, max_it=100000)
        per[str(n)] = {"service_ms": (time.perf_counter() - t0) * 1e3, "iterations": info["iterations"]}
    mean = float(np.mean([v["service_ms"] for v in per.values()])) if per else None
    return {"sides": per, "mean_service_ms_sides_8_to_32": mean, "cores": O.num_threads(),
            "max_throughput_per_s_sides_8_to_32": 1e3 / mean if mean else None}


def ragged_leg(args, ctx):
    """Monte Carlo systems of uneven size in one batch (MSG_MC_SOLVE_RAGGED): the
    serving sides {8, 16, 24, 32, 48} (cube lattices) and blocks of side 16, 24
    and 32 with their interior nodes moved by up to 0.2 (not lattices),
    args.ragged_R realizations each with its own 50-term KL field (sigma 0.3,
    l 0.2 * side), to the FP64 true residual < 1e-8; the cube lattices run the
    lattice loop, the moved-node blocks share the element-by-element batch, each
    system preconditioned by the V-cycle of its cube lattice (the diagonal with
    the multigrid option 0). Timed as one ragged batch, as the same systems one
    ragged call each, and as one MSG_MC_SOLVE_BATCH call (the analyzer) per
    system; each batch is built and solved once first (its meshes, their
    lattices and the workspace then exist), the time of a call is the median of
    three calls on the host clock (xi and b in, X of the 48^3 lattice and the
    distorted 24^3 and every tip value out); the oracle solves one realization
    of the 48^3 lattice and of the distorted 24^3 (FP64 CSR Jacobi-PCG to 1e-12)."""
    import msolve_b200 as M
    R, tol = args.ragged_R, 1e-8
    specs = [(8, False), (16, False), (24, False), (32, False), (48, False), (16, True), (24, True), (32, True)]
    systems = []
    for i, (n, dist) in enumerate(specs):
        model = M.clamped_block_model(n)
        if dist:
            rng = np.random.default_rng(100 + n)
            inner = (model.xyz > 0.5).all(axis=1) & (model.xyz < n - 0.5).all(axis=1)
            model.xyz[inner] += 0.2 * rng.uniform(-1, 1, (int(inner.sum()), 3))
        kl = M.LognormalStochasticCoefficientsProvider([n] * 3, 0.2 * n, args.terms, 16)
        xi = np.random.default_rng(1000 + i).standard_normal((R, args.terms))
        systems.append((n, dist, model, kl, xi))
    keep = {4, 6}  # the 48^3 lattice and the distorted 24^3

    def batch(sel):
        b = M.RaggedMonteCarloBatch(ctx, tolerance=tol)
        for j in sel:
            _, _, model, kl, xi = systems[j]
            b.add(model, kl, xi, keep_solutions=j in keep)
        b.Solve()  # warm-up: meshes, their lattices and the workspace exist from here on
        return b

    def timed(b, reps=3):
        ms = []
        for _ in range(reps):
            t0 = time.perf_counter()
            res = b.Solve()
            ms.append((time.perf_counter() - t0) * 1e3)
        return res, float(np.median(ms))

    idx = list(range(len(systems)))
    mixed_batch = batch(idx)
    singles = [batch([j]) for j in idx]
    res, ms = timed(mixed_batch)
    seq_ms = sum(timed(b)[1] for b in singles)
    # each system through MSG_MC_SOLVE_BATCH on its own (the lattice loop for the
    # cube lattices, the element-by-element loop for the distorted block)
    own_ms = 0.0
    for j in idx:
        _, _, model, kl, xi = systems[j]
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=kl.n_terms,
                                                        simulations=xi.shape[0], mode="mixed", tolerance=tol,
                                                        keep_solutions=j in keep)
        mc.RandomNumbers = xi
        own_ms += timed(mc)[1]
    dof_its = sum(systems[j][2].n_dofs * float(res[j]["Iterations"].sum()) for j in idx)
    prec = "Jacobi-PCG" if ctx.get_option("multigrid") == 0 else "PCG preconditioned by each system's V-cycle"
    out = {"workload": f"{len(specs)} Monte Carlo systems in one batch: cube lattices of side 8, 16, 24, 32, 48 and "
                       f"16^3, 24^3, 32^3 blocks with interior nodes moved by up to 0.2, {R} realizations each, "
                       f"{args.terms}-term KL lognormal E, {prec} (FP32 element-by-element operator, FP64 "
                       f"iterate) to the FP64 true relative residual < {tol:g}",
           "systems": [{"mesh": f"{n}^3" + (" distorted" if dist else ""), "free_dofs": model.n_dofs,
                        "mean_iterations": float(res[j]["Iterations"].mean())}
                       for j, (n, dist, model, _, _) in enumerate(systems)],
           "ragged_ms": ms, "one_call_per_system_ms": seq_ms, "ragged_over_one_call_per_system": seq_ms / ms,
           "mc_batch_per_system_ms": own_ms, "ragged_over_mc_batch_per_system": own_ms / ms,
           "solves_per_s": len(idx) * R / (ms / 1e3), "dof_iterations_per_s": dof_its / (ms / 1e3),
           "max_true_rel_residual": float(max(r["Residuals"].max() for r in res))}
    if not args.no_parity:
        import oracle as O
        errs = {}
        for j in sorted(keep):
            n, dist, model, kl, xi = systems[j]
            P = O.block_problem(n, args.terms, 16)
            E = O.kl_field(O.centroids(model.xyz, model.conn), P["domain"], P["table"], xi[:1], sigma=0.3)[0]
            if dist:
                C = O.CSR(model.n_nodes, model.conn, model.dof, model.n_dofs)
                C.assemble(O.h8_stiffness_batch(model.element_xyz(), E, model.poisson)[0])
                xo, _ = C.pcg_jacobi(model.subdomains[0].RHS, tol=1e-12)
            else:
                xo, _ = O.block_solve_pcg(n, n, n, P["constrained"], E, 0.3, P["b"], tol=1e-12, max_it=100000)
            x = res[j]["Solutions"][0]
            errs[out["systems"][j]["mesh"]] = float(np.abs(x - xo).max() / np.abs(xo).max())
        out["rel_err_vs_oracle"] = errs
    return out


def distorted_leg(args, ctx):
    """The Monte Carlo batch of args.R realizations on the args.n cube with its
    interior nodes moved by up to 0.2 in each axis (not a cube lattice: the
    element-by-element loop of MSG_MC_SOLVE_BATCH in mixed mode, preconditioned
    by the V-cycle of the cube lattice of the same numbering, or by the
    diagonal with the multigrid option 0), 50-term KL field, FP64 true
    residual < args.tol; one warm-up call, then args.steps timed calls (device
    time of the call and of its loop)."""
    import msolve_b200 as M
    n, R = args.n, args.R
    model = M.clamped_block_model(n)
    rng = np.random.default_rng(5)
    inner = (model.xyz > 0.5).all(axis=1) & (model.xyz < n - 0.5).all(axis=1)
    model.xyz[inner] += 0.2 * rng.uniform(-1, 1, (int(inner.sum()), 3))
    kl = M.LognormalStochasticCoefficientsProvider([n] * 3, 0.2 * n, args.terms, 16)
    xi = np.random.default_rng(1).standard_normal((R, args.terms))
    mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=args.terms, simulations=R,
                                                    mode="mixed", tolerance=args.tol, keep_solutions=False)
    mc.RandomNumbers = xi
    mc.Solve()
    calls, loops = [], []
    for _ in range(max(1, args.steps)):
        mc.Solve()
        st = ctx.stats()
        calls.append(st["t_total_ms"])
        loops.append(st["t_inner_ms"])
    best = min(calls)
    prec = "diagonal" if ctx.get_option("multigrid") == 0 else "V-cycle of the cube lattice of the same numbering"
    return {"workload": f"{R} realizations x {n}^3 Hexa8 with interior nodes moved by up to 0.2 (not a cube "
                        f"lattice), {args.terms}-term KL lognormal E, PCG with the FP32 element-by-element "
                        f"operator ({prec} preconditioner) and FP64 true residual < {args.tol:g}",
            "solves_per_s": R / (best / 1e3), "call_ms": calls, "loop_ms": loops,
            "true_residual_steps": st["reliable_updates"], "mean_iterations": float(np.mean(mc.Iterations)),
            "max_true_rel_residual": float(mc.Residuals.max())}


def serving_leg(args, ctx):
    """Serving: Poisson arrivals (seeded) of single-realization requests on cube
    meshes of side {8, 16, 24, 32, 48} (uniform), fresh xi per request, tol 1e-8,
    through MSG_SERVE_* (continuous batching, 64 slots per model). Latency =
    submit to finish, measured by the server."""
    import msolve_b200 as M
    from msolve_b200.serving import Server
    sides = (8, 16, 24, 32, 48)
    srv = Server(ctx, max_batch=64)
    models = {}
    try:
        for n in sides:
            model = M.clamped_block_model(n)
            kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, args.terms, 12)
            models[n] = srv.add_model(model, kl, tol=1e-8)
        out = {"workload": f"Poisson arrivals, cube side uniform in {list(sides)}, one realization per request "
                           f"({args.terms}-term KL lognormal E, sigma 0.3), FP64 true residual < 1e-8, 64 slots per "
                           f"model, continuous batching", "rates": []}
        largest = None
        # warm-up: one request per model
        for n in sides:
            srv.poll(srv.submit(models[n], np.zeros(args.terms)), timeout_ms=-1)
        for rate in [float(v) for v in args.serve_rates.split(",") if v]:
            rng = np.random.default_rng(int(rate))
            k = args.serve_requests
            gaps = rng.exponential(1.0 / rate, k)
            which = rng.choice(sides, k)
            xis = rng.standard_normal((k, args.terms))
            reqs = []
            t0 = time.perf_counter()
            t_next = t0
            for i in range(k):
                t_next += gaps[i]
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                reqs.append((int(which[i]), srv.submit(models[int(which[i])], xis[i])))
            lat = {n: [] for n in sides}
            its = []
            for i, (n, rq) in enumerate(reqs):
                o = srv.poll(rq, timeout_ms=-1)
                lat[n].append(o["latency_ms"])
                its.append(o["iterations"])
                if n == max(sides):
                    largest = (xis[i], o["X"])
            wall = time.perf_counter() - t0
            allv = np.concatenate([np.array(v) for v in lat.values() if v])
            out["rates"].append({
                "rate_per_s": rate, "requests": k, "throughput_per_s": k / wall,
                "p50_ms": float(np.percentile(allv, 50)), "p99_ms": float(np.percentile(allv, 99)),
                "per_side": {str(n): {"count": len(v), "p50_ms": float(np.percentile(v, 50)),
                                      "p99_ms": float(np.percentile(v, 99))} for n, v in lat.items() if v},
                "mean_iterations": float(np.mean(its))})
        out["fp64_one_at_a_time"] = fp64_serving_baseline(args, ctx, sides,
                                                           [float(v) for v in args.serve_rates.split(",") if v])
        if not args.no_cpu:
            out["cpu_oracle_one_at_a_time"] = cpu_serving_baseline(args, sides)
        if not args.no_parity and largest is not None:
            import oracle as O
            n = max(sides)
            P = O.block_problem(n, args.terms, 12)
            E = oracle_fields(P, largest[0])
            xo, info = O.block_solve_pcg(n, n, n, P["constrained"], E[0], 0.3, P["b"], tol=1e-12, max_it=100000)
            out["oracle"] = {"side": n, "rel_err": float(np.abs(largest[1] - xo).max() / np.abs(xo).max()),
                             "oracle": "FP64 CSR Jacobi-PCG restatement of SolverPCG to 1e-12, one served request"}
        return out
    finally:
        srv.stop()


def fp64_serving_baseline(args, ctx, sides, rates):
    """The plain FP64 path serving the same kind of stream one request at a
    time: per request its KL field, the assembled FP64 BSR matrix and the FP64
    Jacobi-PCG drop-in (MSG_PCG_SOLVE, the reference's stopping rule at 1e-8),
    each request's service time measured on the GPU box. A single FIFO server
    gives each arrival process's latencies exactly: finish_i =
    max(arrival_i, finish_{i-1}) + service_i."""
    import msolve_b200 as M
    rng = np.random.default_rng(7)
    k = args.serve_requests
    which = rng.choice(sides, k)
    xis = rng.standard_normal((k, args.terms))
    meshes = {}
    for n in sides:
        model = M.clamped_block_model(n)
        kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, args.terms, 12)
        solver = M.SolverPCG(ctx, model, max_iterations=100000, tolerance=1e-8, precision="fp64")
        meshes[n] = (model, M.GpuMesh(ctx, model), kl, solver)

    def serve(n, xi):
        model, mesh, kl, solver = meshes[n]
        A = mesh.assemble(kl.field(mesh, xi)[0], model.poisson)
        solver.matrix = A
        solver.Solve()
        A.close()
        return solver.iterations

    for n in sides:  # warm-up
        serve(n, np.zeros(args.terms))
    service, its = np.zeros(k), np.zeros(k)
    for i in range(k):
        t0 = time.perf_counter()
        its[i] = serve(int(which[i]), xis[i])
        service[i] = time.perf_counter() - t0
    out = {"workload": f"the same kind of stream ({k} requests, sides uniform in {list(sides)}), one request at a "
                       f"time: KL field + FP64 BSR assembly + FP64 Jacobi-PCG (MSG_PCG_SOLVE, tol 1e-8)",
           "service_ms_mean": 1e3 * float(service.mean()), "mean_iterations": float(its.mean()),
           "max_throughput_per_s": k / float(service.sum()), "rates": []}
    for rate in rates:
        arrive = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, k))
        finish = np.zeros(k)
        prev = 0.0
        for i in range(k):
            prev = max(arrive[i], prev) + service[i]
            finish[i] = prev
        lat = 1e3 * (finish - arrive)
        out["rates"].append({"rate_per_s": rate, "throughput_per_s": k / float(finish[-1] - arrive[0]),
                             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))})
    return out


def run_reference(args):
    """The reference's CPU implementation of the path (the oracle port: the
    reference is C#/.NET + Intel Fortran, which cannot be built here) on the
    host cores, on the headline workload: each step solves a bounded sample of
    the batch's realizations (KL field, FP64 element matrices, assembly and
    SolverPCG-rule Jacobi-PCG per realization, one after another, OpenMP inside
    each solve). Realizations are independent, so solves/s of the sample is
    the batch's rate. Rank 0 alone runs; the other ranks exit."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    import oracle as O
    P = O.block_problem(args.n, args.terms, 16)
    rng = np.random.default_rng(99)
    n, k = args.n, args.ref_sample
    times, its = [], []
    for s in range(args.warmup + args.steps):
        xi = rng.standard_normal((k, args.terms))
        t0 = time.perf_counter()
        E = oracle_fields(P, xi)
        for r in range(k):
            _, info = O.block_solve_pcg(n, n, n, P["constrained"], E[r], 0.3, P["b"], tol=args.tol, max_it=100000)
            its.append(info["iterations"])
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    T = float(np.sum(times))
    v = args.steps * k / T
    sample = (f"each step {k} realizations of the {args.R}-realization batch (FP64 KL field, element matrices, CSR "
              f"assembly, Jacobi-PCG to tol {args.tol:g}, mean {np.mean(its):.0f} iterations), one after another "
              f"with OpenMP inside each solve")
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(args, ws),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "latency_ms": {"p50": 1e3 * float(np.percentile(times, 50)) / k,
                           "p99": 1e3 * float(np.percentile(times, 99)) / k}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import msolve_b200 as M
    from msolve_b200 import _native as N

    ctx = M.Context(local)
    for kv in args.option:
        k, v = kv.split("=", 1)
        ctx.set_option(k, float(v))
    if args.reliable_delta is not None:
        ctx.set_option("reliable_delta", args.reliable_delta)
    if args.single_only:
        print(json.dumps(single_leg(args, ctx)))
        return
    if args.distorted_only or args.ragged_only:
        if args.multigrid is not None:
            ctx.set_option("multigrid", args.multigrid)
        print(json.dumps(distorted_leg(args, ctx) if args.distorted_only else ragged_leg(args, ctx)))
        return
    if args.chunk is not None:
        ctx.set_option("chunk", args.chunk)
    if args.tensor_op is not None:
        ctx.set_option("tensor_operator", args.tensor_op)
    if args.multigrid is not None:
        ctx.set_option("multigrid", args.multigrid)
    for key, val in (("multigrid_levels", args.mg_levels), ("multigrid_sweeps", args.mg_sweeps),
                     ("multigrid_delta", args.mg_delta), ("multigrid_omega", args.mg_omega),
                     ("serve_persistent", args.serve_persistent), ("serve_priority", args.serve_priority),
                     ("multigrid_packed", args.mg_packed)):
        if val is not None:
            ctx.set_option(key, val)
    model, kl = make_problem(args)
    mesh = M.GpuMesh(ctx, model)
    R, K_terms = args.R, args.terms
    Nd = model.n_dofs
    tip = M.tip_dof(model)
    dev = torch.device("cuda", local)
    steps_total = args.warmup + args.steps
    # every step draws a global table of ws * R realizations; this rank solves its shard
    from msolve_b200 import distributed as D
    lo, hi = D.shard(ws * R, ws, rank)
    xi_all = torch.from_numpy(np.stack([D.global_xi(1000 + s, ws * R, K_terms)[lo:hi]
                                        for s in range(steps_total + 1)]))
    xi_dev = xi_all.to(dev)
    b_dev = torch.from_numpy(model.subdomains[0].RHS).to(dev)
    X_dev = torch.empty(R, Nd, dtype=torch.float64, device=dev)
    kls = kl.struct()
    tip_h = np.zeros(R)
    its_h = np.zeros(R, dtype=np.int32)
    res_h = np.zeros(R)
    L = N.lib()

    def solve_device(step, mode=N.MSG_MODE_MIXED_BATCHED, count=R):
        st = L.MSG_MC_SOLVE_BATCH_DEVICE(mesh.handle, model.poisson, C.byref(kls), count,
                                         C.c_void_p(xi_dev[step].data_ptr()), C.c_void_p(b_dev.data_ptr()), mode,
                                         200000, args.tol, tip, C.c_void_p(X_dev.data_ptr()), N.ptr(tip_h),
                                         N.ptr(its_h, N._i), N.ptr(res_h))
        N.check(st, ctx.handle, "MSG_MC_SOLVE_BATCH_DEVICE")

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    # loop configuration (tile shapes, preconditioner) picked by the project's autotuner
    # on this rank's own batch, unless an option was forced on the command line
    tuned = None
    forced = any(v is not None for v in (args.multigrid, args.mg_levels, args.chunk, args.mg_packed,
                                         args.tensor_op))
    if not args.no_autotune and not forced:
        from msolve_b200.tuning import Autotuner
        tuner = Autotuner(ctx, args.autotune_cache)
        opts = tuner.tune_mc(mesh, kl, xi_all[0].numpy(), tol=args.tol)
        tuner.apply(opts)
        rec = tuner.cache[tuner.last_key]
        tuned = {"options": opts, "candidates": [{"options": c["options"], "seconds": round(c["seconds"], 4)}
                                                 for c in rec["candidates"]]}

    for s in range(args.warmup):
        solve_device(s)
    barrier()
    ctx.reset_stats()
    launches0 = ctx.stats()["launches"]
    clocks = Clocks(local)
    clocks.start()
    lat, iters, resmax, phases = [], [], [], []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    for s in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        solve_device(args.warmup + s)
        b.record()
        b.synchronize()
        lat.append(a.elapsed_time(b))
        stp = ctx.stats()
        phases.append({k: round(stp[k], 1) for k in ("t_field_ms", "t_inner_ms", "t_resid_ms", "t_total_ms")}
                      | {"reliable_updates": stp["reliable_updates"]})
        iters.append(its_h[:R].copy())
        resmax.append(float(res_h[:R].max()))
    e1.record()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    st = ctx.stats()
    launches = st["launches"] - launches0
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if ws > 1:
        import torch.distributed as dist
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = ws * R * args.steps / (ms_max / 1e3)

    # Monte Carlo statistics of the last step: one all-reduce of (count, sum u, sum u^2)
    mom = D.combine_moments(tip_h[:R], device=dev)
    tip_mean, tip_var, cnt = mom["mean"], mom["variance"], mom["count"]

    # roofline of the dominant kernel, the fused direction + matrix-free FP32 operator
    # (live per-launch samples from the timed region): k_lvl_op<PcgZ> in the multigrid
    # loop, k_op_modal in the Jacobi loop
    mg = ctx.get_option("multigrid") != 0
    op_ms = st["op_launch_ms"]
    nn = model.n_nodes
    ne = model.n_elems
    Rp = (R + 31) // 32 * 32
    # algorithmic bytes of one launch, FP32, realization-innermost, each value once.
    # multigrid: read z, p_{k-1}, d (3 per node), E (1 per element); write p_k, d, q (3 per node).
    # Jacobi: read r, p_{k-1}, d (3 per node), dinv (1 per node), E; write p_k, d, q (3 per node)
    tensor = mg and ctx.get_option("tensor_operator") != 0
    if mg:
        op_kernel = ("k_lvl_op2<PcgZ> (multigrid loop, level 0: fused search direction p = z + beta p + "
                     "matrix-free FP32 operator, two realizations per lane in packed FP32)")
        if tensor:
            op_kernel = ("k_lvl_tc<PcgZ> (multigrid loop, level 0: fused search direction p = z + beta p + element "
                         "product E Khat u on the tensor cores, tcgen05.mma kind::tf32 with a three-term split)")
        op_bytes = 4.0 * Rp * ((3 + 3 + 3 + 3 + 3 + 3) * nn + ne)
        per_r = None if tensor else MG_OP_DRAM_BYTES_PER_REALIZATION
    else:
        op_kernel = "k_op_modal (fused PCG direction update + matrix-free FP32 Hexa8 operator)"
        op_bytes = 4.0 * Rp * ((3 + 3 + 3 + 1 + 3 + 3 + 3) * nn + ne)
        per_r = OP_DRAM_BYTES_PER_REALIZATION
    hbm, peak_kind = load_peaks()
    achieved = op_bytes / (op_ms / 1e3) / 1e9 if op_ms > 0 else 0.0
    # DRAM bytes per launch from one ncu capture of the same kernel at 512 realizations
    # (dram__bytes_read.sum + dram__bytes_write.sum), scaled by the realizations processed
    traffic = per_r * Rp if (per_r and args.n == 32) else None

    line = None
    # e2e through the host-buffer entry points (pinned buffers), on every rank at
    # once (each rank its own batch and host buffers; the slowest rank's time):
    # every step copies its xi in and every realization's displacements out.
    # Blocking: MSG_MC_SOLVE_BATCH returns with X on the host. Pipelined (the e2e
    # value): MSG_MC_SOLVE_BATCH_PIPELINED leaves each step's X copy in flight
    # while the next step solves (two host buffers, flushed inside the timed region).
    xi_h = torch.empty(R, K_terms, dtype=torch.float64).pin_memory()
    b_h = torch.from_numpy(model.subdomains[0].RHS.copy()).pin_memory()
    X_hs = [torch.empty(R, Nd, dtype=torch.float64).pin_memory() for _ in range(2)]
    n_e2e = max(3, args.steps)

    def host_call(fn, X_h):
        stt = fn(mesh.handle, model.poisson, C.byref(kls), R, C.cast(C.c_void_p(xi_h.data_ptr()), N._d),
                 C.cast(C.c_void_p(b_h.data_ptr()), N._d), N.MSG_MODE_MIXED_BATCHED, 200000, args.tol, tip,
                 C.cast(C.c_void_p(X_h.data_ptr()), N._d), N.ptr(tip_h), N.ptr(its_h, N._i), N.ptr(res_h))
        N.check(stt, ctx.handle, "MC batch (host buffers)")

    def slowest(ms):  # the slowest rank's time (every rank calls it, in the same order)
        if ws == 1:
            return ms
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def start_together():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    e2e_lat = []
    for s in range(1 + n_e2e):  # one untimed call, then at least 3 timed
        xi_h.copy_(xi_all[steps_total])
        start_together()
        t0 = time.perf_counter()
        host_call(L.MSG_MC_SOLVE_BATCH, X_hs[0])
        if s > 0:
            e2e_lat.append(slowest(1e3 * (time.perf_counter() - t0)))
    e2e_blocking = ws * R / (np.mean(e2e_lat) / 1e3)
    host_call(L.MSG_MC_SOLVE_BATCH_PIPELINED, X_hs[1])  # untimed
    N.check(L.MSG_MC_FLUSH(ctx.handle), ctx.handle, "MSG_MC_FLUSH")
    start_together()
    t0 = time.perf_counter()
    for s in range(n_e2e):
        xi_h.copy_(xi_all[steps_total])
        host_call(L.MSG_MC_SOLVE_BATCH_PIPELINED, X_hs[s % 2])
    N.check(L.MSG_MC_FLUSH(ctx.handle), ctx.handle, "MSG_MC_FLUSH")
    e2e_ms = slowest(1e3 * (time.perf_counter() - t0) / n_e2e)
    e2e_value = ws * R / (e2e_ms / 1e3)
    if rank == 0:
        X_h = X_hs[(n_e2e - 1) % 2]
        # parity: realizations of the e2e batch (host outputs of the public entry
        # point) against FP64 oracle solves of the same fields converged to 1e-12
        parity = None
        if not args.no_parity:
            import oracle as O
            P = O.block_problem(args.n, K_terms, 16)
            rows = np.linspace(0, R - 1, min(args.parity_sample, R)).astype(int)
            t0 = time.perf_counter()
            errs, oits = mc_parity(args, P, xi_all[steps_total].numpy()[rows], X_h.numpy()[rows])
            parity = {"realizations": [int(r) for r in rows], "rel_err_max": max(errs), "rel_err": errs,
                      "oracle_iterations_mean": float(np.mean(oits)), "oracle_seconds": time.perf_counter() - t0,
                      "oracle": "FP64 CSR Jacobi-PCG restatement of SolverPCG to 1e-12 per realization; max-norm "
                                "displacement error relative to the oracle's maximum"}
        # plain FP64 drop-in throughput on a sample of the batch (same tolerance, reference stopping rule)
        k = args.fp64_sample
        solve_device(0, N.MSG_MODE_FP64_BSR, 1)  # warm
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        solve_device(0, N.MSG_MODE_FP64_BSR, k)
        b.record()
        b.synchronize()
        fp64_rate = k / (a.elapsed_time(b) / 1e3)
        fp64_its = float(np.mean(its_h[:k]))
        # the batched mixed loop with the diagonal (Jacobi) preconditioner on the same
        # batch: precision + batching alone against the FP64 drop-in, without multigrid
        mg_opt = ctx.get_option("multigrid")
        ctx.set_option("multigrid", 0)
        solve_device(steps_total - 1)  # warm (graph capture)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        solve_device(steps_total - 1)
        b.record()
        b.synchronize()
        jac_ms = a.elapsed_time(b)
        jac_its = float(np.mean(its_h[:R]))
        ctx.set_option("multigrid", mg_opt)
        cpu = None
        if not args.no_cpu and ws == 1:
            import oracle as O
            cpu = cpu_baseline(args, O.block_problem(args.n, K_terms, 16), xi_all[0].numpy())
        its_all = np.concatenate(iters)
        # the other configurations are single-GPU measurements: the 1-GPU run reports
        # them, a multi-GPU run (the other ranks waiting) only the scaled batch
        solo = ws == 1
        newmark = newmark_leg(args, ctx) if solo and not args.no_newmark else None
        serving = serving_leg(args, ctx) if solo and not args.no_serving else None
        single = single_leg(args, ctx) if solo and not args.no_single else None
        ragged = ragged_leg(args, ctx) if solo and not args.no_ragged else None
        cantilever = cantilever_leg(args, ctx) if solo and not args.no_cpu else None
        distorted = None
        if solo and not args.no_ragged:  # the same element-by-element loop on one mesh that is not a lattice
            dargs = argparse.Namespace(**vars(args))
            dargs.R, dargs.steps = 512, 2
            distorted = distorted_leg(dargs, ctx)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": workload_config(args, ws),
            "method": f"mixed FP32 matrix-free PCG ({'geometric multigrid V(1,1)' if mg else 'Jacobi'} "
                      f"preconditioner) + FP64 refinement to the FP64 true residual",
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(R * K_terms * 8 + Nd * 8),
                    "d2h_bytes_per_step": int(R * Nd * 8 + R * (8 + 4 + 8)), "ms_per_step": e2e_ms,
                    "api": "MSG_MC_SOLVE_BATCH_PIPELINED (each step's displacement copy to pinned host memory "
                           "overlaps the next step's solve; MSG_MC_FLUSH inside the timed region)",
                    "blocking": {"value": e2e_blocking, "api": "MSG_MC_SOLVE_BATCH (returns with X on the host)"}},
            "gpu_launches": int(launches),
            "tuned": tuned,
            "roofline": {"kernel": op_kernel,
                         "bound": "hbm", "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm if hbm else None, "traffic": traffic,
                         "peak_kind": peak_kind, "launch_ms": op_ms, "bytes_per_launch": op_bytes,
                         ("iteration_ms" if mg else "update_launch_ms"): st["update_launch_ms"],
                         "samples": st["launch_samples"],
                         "tensor": tensor_roofline(args, model, R, op_ms) if tensor else None},
            "cpu_baseline": cpu,
            "clocks": clk,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "steps": [round(v, 1) for v in lat]},
            "phases_ms": phases,
            "iterations": {"mean": float(its_all.mean()), "max": int(its_all.max()),
                           "reliable_updates_last_step": st["reliable_updates"]},
            "max_true_rel_residual": max(resmax),
            "rel_err_vs_oracle": parity["rel_err_max"] if parity else None,
            "parity": parity,
            "fp64_dropin": {"solves_per_s": fp64_rate, "sample": k, "mean_iterations": fp64_its,
                            "note": "assembled BSR FP64 Jacobi-PCG, one realization after another, tol on the "
                                    "recursive residual as the reference"},
            "mixed_over_fp64": value / ws / fp64_rate,
            "mixed_jacobi": {"solves_per_s": R / (jac_ms / 1e3), "ms": jac_ms, "mean_iterations": jac_its,
                             "note": "the same batched mixed loop with the diagonal preconditioner (multigrid 0)"},
            "mixed_jacobi_over_fp64": R / (jac_ms / 1e3) / fp64_rate,
            "tip_uz": {"mean": tip_mean, "variance": tip_var, "realizations": int(cnt)},
            "newmark": newmark,
            "serving": serving,
            "single_solve": single,
            "ragged": ragged,
            "distorted_mesh": distorted,
            "cantilever": cantilever,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
