"""Autotuner of the batched loop's launch configuration.

The batched mixed-precision solve has run-time choices that change its tile
and block shapes and its per-iteration work, but never its results beyond the
FP64 stopping rule. The choices are:

  multigrid           V-cycle preconditioned loop (1; 2 also for systems with
                      a mass term) or the Jacobi loop (0);
  multigrid_packed    level operators on 3 x 3 node tiles of 64 realizations
                      (two per lane, packed FP32: 1) or of 32 realizations (0);
  multigrid_levels    depth of the V-cycle.

Which one is fastest depends on the lattice, the batch (the number of work
items against the SM count) and the device. The Autotuner times each candidate on the
caller's own problem, keeps the fastest, and caches the choice in a JSON file
keyed by device, lattice, padded batch and system kind, so later runs with
the same key apply it without timing.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time

import numpy as np

from . import _native as N

TUNABLE = ("multigrid", "multigrid_packed", "multigrid_levels")


def static_candidates():
    """Candidates for systems without a mass term (static solves, serving)."""
    return [
        {"multigrid": 1, "multigrid_packed": 1, "multigrid_levels": 6},
        {"multigrid": 1, "multigrid_packed": 0, "multigrid_levels": 6},
        {"multigrid": 1, "multigrid_packed": 1, "multigrid_levels": 3},
        {"multigrid": 0, "multigrid_packed": 1, "multigrid_levels": 6},
    ]


def mass_candidates():
    """Candidates for systems with a mass term (Newmark steps)."""
    return [
        {"multigrid": 1, "multigrid_packed": 1, "multigrid_levels": 6},  # the Jacobi loop for these systems
        {"multigrid": 2, "multigrid_packed": 1, "multigrid_levels": 6},
        {"multigrid": 2, "multigrid_packed": 0, "multigrid_levels": 6},
    ]


def tuning_key(device, nx, ny, nz, R, mass):
    """Cache key: device name, lattice, batch padded to 64 realizations, system kind."""
    Rp = (int(R) + 63) // 64 * 64
    return f"{device}|{nx}x{ny}x{nz}|R{Rp}|{'mass' if mass else 'static'}"


def device_name(index=0):
    try:
        import torch
        if torch.cuda.is_available():
            p = torch.cuda.get_device_properties(index)
            return f"{p.name} sm_{p.major}{p.minor} x{p.multi_processor_count}"
    except Exception:
        pass
    return f"device{index}"


class Autotuner:
    """Times candidate configurations on a context and keeps the fastest per key.

    `measure(options)` returns seconds for one solve with the options applied.
    The context's options are saved before and restored after every candidate,
    and tune() leaves them unchanged; apply() sets a tuned choice."""

    def __init__(self, ctx, cache_path=None):
        self.ctx = ctx
        self.cache_path = cache_path
        self.last_key = None
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def _save(self):
        if not self.cache_path:
            return
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def tune(self, key, measure, candidates, repeats=1):
        self.last_key = key
        if key in self.cache:
            return dict(self.cache[key]["options"])
        saved = {k: self.ctx.get_option(k) for k in TUNABLE}
        results = []
        try:
            for cand in candidates:
                for k, v in cand.items():
                    self.ctx.set_option(k, v)
                t = min(float(measure(cand)) for _ in range(max(1, repeats)))
                results.append((t, dict(cand)))
                for k, v in saved.items():
                    self.ctx.set_option(k, v)
        finally:
            for k, v in saved.items():
                self.ctx.set_option(k, v)
        best_t, best = min(results, key=lambda r: r[0])
        self.cache[key] = {"options": best, "seconds": best_t,
                           "candidates": [{"options": c, "seconds": t} for t, c in results]}
        self._save()
        return dict(best)

    def apply(self, options):
        for k, v in options.items():
            self.ctx.set_option(k, v)

    def tune_mc(self, mesh, kl, xi, tol=1e-8, max_iterations=20000, device=None, candidates=None):
        """Tune the batched Monte Carlo solve of `mesh` for the realizations xi
        [R][terms] (timed through MSG_MC_SOLVE_BATCH with tip outputs only:
        one warm-up call and one timed call per candidate). Returns the options."""
        model = mesh.model
        xi = N.f64(xi)
        R = xi.shape[0]
        b = N.f64(model.subdomains[0].RHS)
        tip, its, res = np.zeros(R), np.zeros(R, dtype=np.int32), np.zeros(R)
        s = kl.struct()

        def measure(_opts):
            dt = 0.0
            for rep in range(2):
                t0 = time.perf_counter()
                st = N.lib().MSG_MC_SOLVE_BATCH(mesh.handle, float(model.poisson), C.byref(s), R, N.ptr(xi), N.ptr(b),
                                                N.MSG_MODE_MIXED_BATCHED, int(max_iterations), float(tol), 0, None,
                                                N.ptr(tip), N.ptr(its, N._i), N.ptr(res))
                dt = time.perf_counter() - t0
                N.check(st, self.ctx.handle, "MSG_MC_SOLVE_BATCH (tuning)")
            return dt

        if model.structured is None:
            raise N.ArgumentError(N.MSG_ERR_INVALID_ARGUMENT, "the batched solve needs a structured lattice model")
        nx, ny, nz = model.structured[:3]
        key = tuning_key(device or device_name(self.ctx.device), nx, ny, nz, R, False)
        return self.tune(key, measure, candidates or static_candidates())
