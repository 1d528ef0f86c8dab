"""Realization sharding over ranks (CPU, gloo, world size 2): shards cover the
global table exactly once, and the combined tip statistics of a sharded Monte
Carlo run equal the single-process ones. The per-realization solve is the
oracle's FP64 PCG here (the GPU batch is the same call per shard)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

import msolve_b200 as M
from msolve_b200 import distributed as D
import oracle as O


def test_shards_partition_the_batch():
    for R in (0, 1, 7, 32, 1000):
        for world in (1, 2, 3, 8):
            spans = [D.shard(R, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == R
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and b - a >= d - c
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1
    with pytest.raises(ValueError):
        D.shard(4, 2, 2)


def _tip_solver(n):
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, 6, 4)
    cen = O.centroids(model.xyz, model.conn)
    cons = (model.dof < 0).astype(np.uint8)
    tip = M.tip_dof(model)

    def solve(xi):
        E = O.kl_field(cen, [n, n, n], kl.table(), xi, mean=kl.mean, sigma=kl.sigma,
                       mean_correction=kl.mean_correction)
        out = []
        for r in range(xi.shape[0]):
            x, info = O.block_solve_pcg(n, n, n, cons, E[r], model.poisson, model.subdomains[0].RHS, tol=1e-12)
            assert info["status"] == 0
            out.append(x[tip])
        return out
    return solve


def _worker(rank, world, port, path):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    xi = D.global_xi(11, 7, 6)
    local, span, mom = D.sharded_batch(xi, _tip_solver(3), world, rank)
    np.save(os.path.join(path, f"r{rank}.npy"), np.array([span[0], span[1], mom["count"], mom["mean"],
                                                         mom["variance"], *local]))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_statistics_match_single_process():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        rows = [np.load(os.path.join(d, f"r{r}.npy")) for r in range(world)]
    xi = D.global_xi(11, 7, 6)
    ref = np.array(_tip_solver(3)(xi))
    single = D.combine_moments(ref)
    tips = np.concatenate([r[5:] for r in rows])
    # the oracle's OpenMP reductions depend on the thread count of each process
    assert np.abs(tips - ref).max() <= 1e-10 * np.abs(ref).max()
    for r in rows:
        assert int(r[2]) == 7
        assert abs(r[3] - single["mean"]) <= 1e-12 * abs(single["mean"])
        assert abs(r[4] - single["variance"]) <= 1e-10 * abs(single["variance"])
