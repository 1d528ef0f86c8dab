"""Host mirror of the serving entry points (MSG_SERVE_*): continuous batching of
independent realizations of registered models on one context, lanes of
max_batch slots added and retired by device memory (the context's budget).

    srv = Server(ctx, max_batch=64)
    m = srv.add_model(model, kl, tol=1e-8)        # one structured mesh + material + KL table + load
    rid = srv.submit(m, xi)                        # one realization
    out = srv.poll(rid, timeout_ms=-1)             # dict(X, iterations, rel_res, latency_ms)

A request's result does not depend on what else is in flight (bitwise)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .analyzers import GpuMesh


class Router:
    """Requests over several servers (one per GPU, or several budgeted contexts
    of one GPU): each submit goes to the server with the most free device
    memory for new lanes (budget - used when its context has a budget, else
    its device's free memory), ties to the one with the fewest requests
    queued and running. Models are registered on every server; requests are
    independent, so there is no collective.

        r = Router([Server(Context(d), 64) for d in range(n_gpus)])
        m = r.add_model(model, kl, tol=1e-8)
        req = r.submit(m, xi)
        out = r.poll(req)"""

    def __init__(self, servers):
        if not servers:
            raise ValueError("a router needs at least one server")
        self.servers = list(servers)

    def add_model(self, model, coefficients_provider, tol=1e-8, max_iterations=20000):
        return [s.add_model(model, coefficients_provider, tol=tol, max_iterations=max_iterations)
                for s in self.servers]

    def free_memory(self, i):
        ctx = self.servers[i].ctx
        budget = ctx.get_option("memory_budget")
        if budget > 0:
            return budget - ctx.get_option("memory_used")
        return ctx.get_option("device_free_memory")

    def choose(self):
        """Index of the server the next request goes to."""
        def key(i):
            st = self.servers[i].stats()
            return (-self.free_memory(i), st["queued"] + st["running"], i)
        return min(range(len(self.servers)), key=key)

    def submit(self, model, xi):
        i = self.choose()
        return i, self.servers[i].submit(model[i], xi)

    def poll(self, request, timeout_ms=-1):
        i, rq = request
        return self.servers[i].poll(rq, timeout_ms=timeout_ms)

    def stop(self):
        for s in self.servers:
            s.stop()


class Server:
    def __init__(self, ctx, max_batch=64):
        self.ctx = ctx
        self._models = []
        N.check(N.lib().MSG_SERVE_START(ctx.handle, int(max_batch)), ctx.handle, "MSG_SERVE_START")

    def add_model(self, model, coefficients_provider, tol=1e-8, max_iterations=20000):
        mesh = GpuMesh(self.ctx, model)
        s = coefficients_provider.struct()
        b = N.f64(model.subdomains[0].RHS)
        mid = C.c_int(0)
        st = N.lib().MSG_SERVE_ADD_MODEL(self.ctx.handle, mesh.handle, float(model.poisson), C.byref(s), N.ptr(b),
                                         float(tol), int(max_iterations), C.byref(mid))
        N.check(st, self.ctx.handle, "MSG_SERVE_ADD_MODEL")
        self._models.append((mesh, model, coefficients_provider, s))
        return mid.value

    def submit(self, model_id, xi):
        xi = N.f64(xi)
        rid = C.c_uint64(0)
        N.check(N.lib().MSG_SERVE_SUBMIT(self.ctx.handle, int(model_id), N.ptr(xi), C.byref(rid)), self.ctx.handle,
                "MSG_SERVE_SUBMIT")
        return rid.value, int(model_id)

    def poll(self, request, timeout_ms=-1):
        """None while pending; else dict(X, iterations, rel_res, latency_ms). Raises on failure."""
        rid, model_id = request
        n_dofs = self._models[model_id][1].n_dofs
        X = np.zeros(n_dofs)
        its = C.c_int(0)
        res = C.c_double(0)
        lat = C.c_double(0)
        st = N.lib().MSG_SERVE_POLL(self.ctx.handle, C.c_uint64(rid), int(timeout_ms), N.ptr(X), C.byref(its),
                                    C.byref(res), C.byref(lat))
        if st == N.MSG_PENDING:
            return None
        N.check(st, self.ctx.handle, "MSG_SERVE_POLL")
        return {"X": X, "iterations": its.value, "rel_res": res.value, "latency_ms": lat.value}

    def cancel(self, request):
        N.check(N.lib().MSG_SERVE_CANCEL(self.ctx.handle, C.c_uint64(request[0])), self.ctx.handle, "MSG_SERVE_CANCEL")

    def stats(self):
        q, r = C.c_int64(0), C.c_int64(0)
        N.check(N.lib().MSG_SERVE_STATS(self.ctx.handle, C.byref(q), C.byref(r)), self.ctx.handle, "MSG_SERVE_STATS")
        return {"queued": q.value, "running": r.value}

    def lanes(self, model_id=-1):
        """Lanes admitting requests (of one model, or all), lanes added and retired so far."""
        n, a, r = C.c_int(0), C.c_int64(0), C.c_int64(0)
        N.check(N.lib().MSG_SERVE_LANES(self.ctx.handle, int(model_id), C.byref(n), C.byref(a), C.byref(r)),
                self.ctx.handle, "MSG_SERVE_LANES")
        return {"lanes": n.value, "added": a.value, "retired": r.value}

    def stop(self):
        N.lib().MSG_SERVE_STOP(self.ctx.handle)
        self._models = []
