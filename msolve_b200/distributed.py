"""Realization sharding of the Monte Carlo and Newmark batches over ranks.

The reference's realization loop (MonteCarloAnalyzerWithStochasticMaterial.cs:258-276)
solves independent systems one after another. Here ranks (one process per
GPU) take contiguous shards of one global xi table, solve their shard as one
batch with no collective on the data path, and combine the statistics of the
quantity of interest with a single all-reduce of (n, sum u, sum u^2) at the
end. Every rank derives the same global table from the seed, so the union of
the shards is the single-process run and the statistics match it to rounding.
"""
from __future__ import annotations

import numpy as np


def shard(R, world, rank):
    """[start, stop) of rank's realizations: contiguous, the first R % world ranks one more."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    base, extra = divmod(int(R), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def global_xi(seed, R, n_terms):
    """The global N(0,1) table [R][n_terms] (identical on every rank)."""
    return np.random.default_rng(seed).standard_normal((int(R), int(n_terms)))


def combine_moments(values, group=None, device=None):
    """Mean and sample variance of `values` over all ranks of `group` (one
    all-reduce of three FP64 sums; without torch.distributed, the local values)."""
    v = np.asarray(values, dtype=np.float64)
    sums = np.array([v.size, v.sum(), (v * v).sum()], dtype=np.float64)
    try:
        import torch
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            t = torch.from_numpy(sums)
            if device is not None:
                t = t.to(device)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            sums = t.cpu().numpy()
    except ImportError:
        pass
    n, s1, s2 = sums
    mean = s1 / n if n > 0 else 0.0
    var = (s2 - n * mean * mean) / (n - 1) if n > 1 else 0.0
    return {"count": int(round(n)), "mean": float(mean), "variance": float(var)}


def sharded_batch(xi_global, solve, world, rank, group=None, device=None):
    """Solve this rank's shard with `solve(xi_shard) -> per-realization values`
    and combine the moments over the ranks. Returns (local values, shard, moments)."""
    lo, hi = shard(xi_global.shape[0], world, rank)
    local = np.asarray(solve(xi_global[lo:hi]), dtype=np.float64) if hi > lo else np.zeros(0)
    return local, (lo, hi), combine_moments(local, group=group, device=device)
