"""Host logic of the serving router (msolve_b200.serving.Router), with stand-in
servers (no GPU): a request goes to the server with the most free device
memory for new lanes (budget - used with a budget, else the device's free
memory), ties to the fewest requests queued and running, then the lowest
index; models are registered on every server and requests come back from the
server that took them."""
from msolve_b200.serving import Router


class _Ctx:
    def __init__(self, budget, used, device_free):
        self.v = {"memory_budget": budget, "memory_used": used, "device_free_memory": device_free}

    def get_option(self, key):
        return self.v[key]


class _Server:
    def __init__(self, budget, used, device_free, queued=0, running=0):
        self.ctx = _Ctx(budget, used, device_free)
        self.queued, self.running = queued, running
        self.models, self.submitted, self.stopped = [], [], False

    def stats(self):
        return {"queued": self.queued, "running": self.running}

    def add_model(self, model, kl, tol=1e-8, max_iterations=20000):
        self.models.append((model, kl, tol))
        return len(self.models) - 1

    def submit(self, model_id, xi):
        self.submitted.append((model_id, xi))
        self.queued += 1
        return ("rq", len(self.submitted))

    def poll(self, rq, timeout_ms=-1):
        return {"from": self, "rq": rq}

    def stop(self):
        self.stopped = True


def test_router_prefers_free_memory_then_load():
    a = _Server(budget=10e9, used=8e9, device_free=100e9)      # 2 GB free in its budget
    b = _Server(budget=0, used=5e9, device_free=30e9)          # no budget: the device's 30 GB
    c = _Server(budget=40e9, used=10e9, device_free=100e9)     # 30 GB free in its budget
    r = Router([a, b, c])
    m = r.add_model("model", "kl", tol=1e-9)
    assert all(s.models == [("model", "kl", 1e-9)] for s in (a, b, c))
    assert m == [0, 0, 0]
    # b and c tie on free memory; both idle: the lower index
    req = r.submit(m, [0.0])
    assert req[0] == 1 and b.submitted == [(0, [0.0])]
    # b now has one queued request: c is preferred
    req = r.submit(m, [1.0])
    assert req[0] == 2
    assert r.poll(req)["from"] is c
    # memory dominates load: a heavily loaded server with more free memory still wins
    c.ctx.v["memory_used"] = 5e9
    c.running = 100
    assert r.choose() == 2
    r.stop()
    assert a.stopped and b.stopped and c.stopped


def test_router_needs_a_server():
    try:
        Router([])
    except ValueError:
        return
    raise AssertionError("expected ValueError")
