"""Host logic of the Monte Carlo analyzer (no GPU): the reference's
random-number file layout and start index
(MonteCarloAnalyzerWithStochasticMaterial.cs:182-216, 232-296), its per-
realization log files, and resume by realization index from a checkpoint. The
batch solve is replaced by a deterministic stand-in, so these tests exercise
only the bookkeeping around MSG_MC_SOLVE_BATCH."""
import os

import numpy as np
import pytest

import msolve_b200 as M
from msolve_b200 import _native as N
from msolve_b200.analyzers import read_randoms, write_randoms


class FakeBatch(M.MonteCarloAnalyzerWithStochasticMaterial):
    """Tip value = a fixed function of the realization's xi row; fails on call `fail_at`."""

    def __init__(self, *a, fail_at=None, **kw):
        super().__init__(None, M.clamped_block_model(2), None, *a, keep_solutions=False, tip_dof=0, **kw)
        self.calls, self.fail_at = [], fail_at

    def _solve_batch(self, xi):
        if self.fail_at is not None and len(self.calls) == self.fail_at:
            raise RuntimeError("simulated failure")
        self.calls.append(xi.shape[0])
        tip = np.tanh(xi) @ np.arange(1.0, xi.shape[1] + 1)
        its = (np.abs(xi[:, 0]) * 10).astype(np.int32) + 1
        return tip, its, np.full(xi.shape[0], 1e-11), None, N.MSG_OK


def test_randoms_file_layout(tmp_path):
    t = np.random.default_rng(1).standard_normal((7, 3))
    p = tmp_path / "randoms3.txt"
    write_randoms(p, t)
    lines = p.read_text().split()
    assert len(lines) == 21
    assert float(lines[1]) == t[1, 0] and float(lines[7]) == t[0, 1]  # term outermost, simulations inner
    assert np.array_equal(read_randoms(p, 7, 3), t)
    assert np.array_equal(read_randoms(p, 5, 3)[:, 0], t[:5, 0])  # first rows of the first term's block
    with pytest.raises(ValueError):
        read_randoms(p, 8, 3)


def test_drawn_table_is_written_and_read_back(tmp_path):
    prefix = str(tmp_path / "monteCarlo")
    a = FakeBatch(expansion_order=4, simulations=6, seed=5, file_name_for_logging=prefix)
    a.Solve()
    path = tmp_path / "randoms4.txt"
    assert path.exists()
    b = FakeBatch(expansion_order=4, simulations=6, randoms_read_file_name=str(path), random_file_simulations=6)
    b.Solve()
    assert np.array_equal(b.TipValues, a.TipValues)


def test_start_index_selects_rows(tmp_path):
    t = np.random.default_rng(2).standard_normal((10, 3))
    path = tmp_path / "r.txt"
    write_randoms(path, t)
    a = FakeBatch(expansion_order=3, simulations=4, randoms_read_file_name=str(path), random_file_simulations=10,
                  simulation_start_from=5)
    tip = a.Solve()
    assert np.array_equal(tip, np.tanh(t[5:9]) @ np.arange(1.0, 4.0))
    bad = FakeBatch(expansion_order=3, simulations=6, randoms_read_file_name=str(path), random_file_simulations=10,
                    simulation_start_from=5)
    with pytest.raises(N.ArgumentError):
        bad.Solve()


def test_log_files(tmp_path):
    prefix = str(tmp_path / "mc")
    a = FakeBatch(expansion_order=3, simulations=5, file_name_for_logging=prefix, batch_size=2)
    a.Solve()
    values = (tmp_path / "mc-3-0.txt").read_text().split()
    iters = (tmp_path / "mc-3-0-Iters.txt").read_text().split()
    times = (tmp_path / "mc-3-0-Times.txt").read_text().splitlines()
    assert [float(v) for v in values] == list(a.TipValues)
    assert [int(v) for v in iters] == list(a.Iterations)
    assert times[0].startswith("Elements: ") and times[-1] == f"Total iterations: {int(a.Iterations.sum())}"


def test_resume_after_failure(tmp_path):
    ck = str(tmp_path / "mc.npz")
    full = FakeBatch(expansion_order=5, simulations=11, seed=3)
    full.Solve()
    first = FakeBatch(expansion_order=5, simulations=11, seed=3, batch_size=3, checkpoint=ck, fail_at=2)
    with pytest.raises(RuntimeError):
        first.Solve()
    assert first.calls == [3, 3] and os.path.exists(ck)
    again = FakeBatch(expansion_order=5, simulations=11, seed=3, batch_size=3, checkpoint=ck)
    again.Solve()
    assert again.calls == [3, 2]  # only the 5 realizations not finished before the failure
    assert np.array_equal(again.TipValues, full.TipValues)
    assert np.array_equal(again.Iterations, full.Iterations)
    done = FakeBatch(expansion_order=5, simulations=11, seed=3, batch_size=3, checkpoint=ck)
    done.Solve()
    assert done.calls == [] and np.array_equal(done.TipValues, full.TipValues)


def test_checkpoint_of_another_table_is_refused(tmp_path):
    ck = str(tmp_path / "mc.npz")
    FakeBatch(expansion_order=3, simulations=4, seed=1, checkpoint=ck).Solve()
    with pytest.raises(ValueError):
        FakeBatch(expansion_order=3, simulations=4, seed=2, checkpoint=ck).Solve()
