"""Serving (MSG_SERVE_*): continuous batching of independent realizations.
Results against FP64 oracle solves (1e-8 max-norm), bitwise identity of a
request alone and inside a changing mix, bitwise identity with the batched
Monte Carlo solve under per-chunk true-residual steps, cancellation, and two
models served side by side."""
import numpy as np
import pytest

import msolve_b200 as M
from msolve_b200 import _native as N
from msolve_b200.serving import Server
import oracle as O

pytestmark = pytest.mark.gpu


def _problem(n, n_terms=12):
    model = M.clamped_block_model(n)
    kl = M.LognormalStochasticCoefficientsProvider([n, n, n], 0.2 * n, n_terms, 6)
    return model, kl


def _oracle(model, kl, xi, n):
    cen = O.centroids(model.xyz, model.conn)
    E = O.kl_field(cen, [n, n, n], kl.table(), xi[None, :], mean=kl.mean, sigma=kl.sigma,
                   mean_correction=kl.mean_correction)[0]
    cons = (model.dof < 0).astype(np.uint8)
    x, info = O.block_solve_pcg(n, n, n, cons, E, model.poisson, model.subdomains[0].RHS, tol=1e-13, max_it=100000)
    return x


@pytest.fixture
def server(ctx):
    srv = Server(ctx, max_batch=32)
    yield srv
    srv.stop()


def test_requests_match_oracle(server):
    n = 6
    model, kl = _problem(n)
    m = server.add_model(model, kl, tol=1e-10)
    xis = np.random.default_rng(5).standard_normal((10, 12))
    reqs = [server.submit(m, xi) for xi in xis]
    for xi, rq in zip(xis, reqs):
        out = server.poll(rq, timeout_ms=-1)
        assert out["rel_res"] < 1e-10 and out["iterations"] > 0 and out["latency_ms"] > 0
        xo = _oracle(model, kl, xi, n)
        assert np.abs(out["X"] - xo).max() <= 1e-8 * np.abs(xo).max()


def test_alone_and_mixed_are_bitwise_equal(server):
    n = 6
    model, kl = _problem(n)
    m = server.add_model(model, kl, tol=1e-10)
    rng = np.random.default_rng(9)
    xa = rng.standard_normal(12)
    alone = server.poll(server.submit(m, xa), timeout_ms=-1)
    others = rng.standard_normal((45, 12))
    first = [server.submit(m, xi) for xi in others[:20]]
    server.poll(first[0], timeout_ms=-1)  # the batch is running when the request joins
    ra = server.submit(m, xa)
    rest = [server.submit(m, xi) for xi in others[20:]]
    mixed = server.poll(ra, timeout_ms=-1)
    for rq in first[1:] + rest:
        server.poll(rq, timeout_ms=-1)
    assert np.array_equal(alone["X"], mixed["X"])
    assert alone["iterations"] == mixed["iterations"] and alone["rel_res"] == mixed["rel_res"]


def test_matches_batched_solve_with_fixed_updates(ctx, server):
    n, R = 6, 8
    model, kl = _problem(n)
    xis = np.random.default_rng(2).standard_normal((R, 12))
    ctx.set_option("fixed_updates", 1)
    try:
        mc = M.MonteCarloAnalyzerWithStochasticMaterial(ctx, model, kl, expansion_order=12, simulations=R,
                                                        mode="mixed", tolerance=1e-10)
        mc.RandomNumbers = xis
        mc.Solve()
    finally:
        ctx.set_option("fixed_updates", 0)
    m = server.add_model(model, kl, tol=1e-10)
    outs = [server.poll(server.submit(m, xi), timeout_ms=-1) for xi in xis]
    for r in range(R):
        assert np.array_equal(outs[r]["X"], mc.Solutions[r]), r
        assert outs[r]["iterations"] == mc.Iterations[r]


def test_cancel(server):
    n = 8
    model, kl = _problem(n)
    m = server.add_model(model, kl, tol=1e-12)
    xis = np.random.default_rng(4).standard_normal((70, 12))
    reqs = [server.submit(m, xi) for xi in xis]  # 70 > 32 slots: the tail waits in the queue
    server.cancel(reqs[-1])
    server.cancel(reqs[0])
    with pytest.raises(N.MSolveError) as e:
        server.poll(reqs[-1], timeout_ms=-1)
    assert e.value.code == N.MSG_ERR_CANCELLED
    with pytest.raises(N.MSolveError):
        server.poll(reqs[0], timeout_ms=-1)
    for rq in reqs[1:-1]:
        assert server.poll(rq, timeout_ms=-1)["rel_res"] < 1e-12
    assert server.stats() == {"queued": 0, "running": 0}


def test_two_models_side_by_side(server):
    probs = [(4,) + _problem(4), (8,) + _problem(8)]
    ids = [server.add_model(model, kl, tol=1e-10) for _, model, kl in probs]
    rng = np.random.default_rng(6)
    jobs = []
    for k in range(12):
        which = k % 2
        xi = rng.standard_normal(12)
        jobs.append((which, xi, server.submit(ids[which], xi)))
    for which, xi, rq in jobs:
        n, model, kl = probs[which]
        out = server.poll(rq, timeout_ms=-1)
        xo = _oracle(model, kl, xi, n)
        assert np.abs(out["X"] - xo).max() <= 1e-8 * np.abs(xo).max()


def test_poll_without_wait_and_unknown_request(server):
    model, kl = _problem(4)
    m = server.add_model(model, kl, tol=1e-10)
    rq = server.submit(m, np.zeros(12))
    out = server.poll(rq, timeout_ms=0)
    while out is None:
        out = server.poll(rq, timeout_ms=50)
    with pytest.raises(N.ArgumentError):
        server.poll(rq, timeout_ms=0)  # forgotten after the successful poll


def test_scheduling_options_do_not_change_results(ctx):
    """One CTA per work item and shortest-first stream priorities change only
    when work runs, not what it computes: two models served side by side give
    the same bits under every scheduling option."""
    models = [_problem(n) for n in (6, 10)]
    rng = np.random.default_rng(21)
    xis = rng.standard_normal((2, 6, 12))
    results = []
    for persistent, priority in ((1, 0), (0, 0), (0, 1)):
        ctx.set_option("serve_persistent", persistent)
        ctx.set_option("serve_priority", priority)
        srv = Server(ctx, max_batch=32)
        try:
            ms = [srv.add_model(model, kl, tol=1e-10) for model, kl in models]
            reqs = [[srv.submit(m, xi) for xi in xis[i]] for i, m in enumerate(ms)]
            results.append([[srv.poll(rq, timeout_ms=-1)["X"] for rq in rs] for rs in reqs])
        finally:
            srv.stop()
            ctx.set_option("serve_persistent", 1)
            ctx.set_option("serve_priority", 0)
    for other in results[1:]:
        for a_model, b_model in zip(results[0], other):
            for a, b in zip(a_model, b_model):
                assert np.array_equal(a, b)


def test_lanes_grow_with_the_backlog_and_retire_when_idle(ctx):
    """A burst larger than one lane's slots makes the manager add lanes of the
    same model; the results do not depend on the lane a request landed in
    (bitwise equal to the same requests served one at a time), and the extra
    lanes are retired once idle."""
    import time
    n = 6
    model, kl = _problem(n)
    rng = np.random.default_rng(31)
    xis = rng.standard_normal((200, 12))
    srv = Server(ctx, max_batch=32)
    try:
        m = srv.add_model(model, kl, tol=1e-10)
        assert srv.lanes(m)["lanes"] == 1
        alone = [srv.poll(srv.submit(m, xi), timeout_ms=-1)["X"] for xi in xis[:4]]
        reqs = [srv.submit(m, xi) for xi in xis]
        outs = [srv.poll(rq, timeout_ms=-1) for rq in reqs]
        assert srv.lanes()["added"] >= 2
        for a, o in zip(alone, outs[:4]):
            assert np.array_equal(a, o["X"])
        assert all(o["rel_res"] < 1e-10 for o in outs)
        t0 = time.time()
        while srv.lanes(m)["lanes"] > 1 and time.time() - t0 < 10:
            time.sleep(0.2)
        assert srv.lanes(m)["lanes"] == 1
        assert srv.lanes()["retired"] >= 1
    finally:
        srv.stop()


def test_admission_waits_for_device_memory(ctx):
    """A context whose memory budget holds the two models' first lanes and
    room for one more: bursts on both models queue until a lane frees memory,
    and every request completes with the bits of an unconstrained server."""
    models = [_problem(n) for n in (6, 8)]
    rng = np.random.default_rng(41)
    xis = rng.standard_normal((2, 150, 12))
    ref = []
    srv = Server(ctx, max_batch=32)
    try:
        ms = [srv.add_model(model, kl, tol=1e-10) for model, kl in models]
        for i, m in enumerate(ms):
            ref.append([srv.poll(rq, timeout_ms=-1)["X"] for rq in [srv.submit(m, xi) for xi in xis[i][:20]]])
    finally:
        srv.stop()
    probe = M.Context(0)
    s0 = Server(probe, max_batch=32)
    meshes = []
    try:
        used0 = probe.get_option("memory_used")
        s0.add_model(*models[0], tol=1e-10)
        lane6 = probe.get_option("memory_used") - used0
        s0.add_model(*models[1], tol=1e-10)
        base = probe.get_option("memory_used")
        lane8 = base - used0 - lane6
    finally:
        s0.stop()
        probe.close()
    tight = M.Context(0, int(base + 1.2 * max(lane6, lane8)))
    srv = Server(tight, max_batch=32)
    try:
        ms = [srv.add_model(model, kl, tol=1e-10) for model, kl in models]
        reqs = [[srv.submit(m, xi) for xi in xis[i]] for i, m in enumerate(ms)]
        outs = [[srv.poll(rq, timeout_ms=-1) for rq in rs] for rs in reqs]
        assert tight.get_option("memory_used") <= tight.get_option("memory_budget")
        for i in range(2):
            assert all(o["rel_res"] < 1e-10 for o in outs[i])
            for a, o in zip(ref[i], outs[i][:20]):
                assert np.array_equal(a, o["X"])
        assert srv.lanes()["lanes"] <= 3
    finally:
        srv.stop()
        tight.close()


def test_router_over_two_budgeted_contexts():
    """Two contexts of one GPU with different memory budgets behind a router:
    requests land where the most budget is free, and every result equals, bit
    for bit, the same request on a single unconstrained server."""
    from msolve_b200.serving import Router
    model, kl = _problem(6)
    xis = np.random.default_rng(51).standard_normal((24, 12))
    single = Server(M.Context(0), max_batch=32)
    try:
        m = single.add_model(model, kl, tol=1e-10)
        ref = [single.poll(single.submit(m, xi), timeout_ms=-1)["X"] for xi in xis]
    finally:
        single.stop()
    ctxs = [M.Context(0, 6 << 30), M.Context(0, 2 << 30)]
    r = Router([Server(c, max_batch=32) for c in ctxs])
    try:
        mm = r.add_model(model, kl, tol=1e-10)
        assert r.choose() == 0  # 6 GB budget, the larger free share
        reqs = [r.submit(mm, xi) for xi in xis]
        assert {i for i, _ in reqs} == {0}
        outs = [r.poll(rq) for rq in reqs]
        for a, o in zip(ref, outs):
            assert np.array_equal(a, o["X"])
    finally:
        r.stop()
        for c in ctxs:
            c.close()
