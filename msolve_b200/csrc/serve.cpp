// Serving: requests (one realization of a registered model each) are queued,
// admitted into free slots of their model's lane at chunk boundaries, and
// returned as soon as their own FP64 true residual is below the model's
// tolerance (continuous batching). One worker thread per model drives its
// lane on the lane's own stream, so models of different sizes overlap on the
// GPU; the C entry points only touch the queues under the server mutex.
// No counterpart in the reference (its Monte Carlo loop is sequential,
// ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:258-276).
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>

#include "msg_internal.h"

namespace msg {

struct ServeRequest {
  int model = 0;
  std::vector<double> xi;
  std::chrono::steady_clock::time_point t0;
  int slot = -1;
  bool finished = false, cancelled = false;
  int status = MSG_OK;
  std::vector<double> X;
  int its = 0;
  double res = 0.0, latency_ms = 0.0;
};

struct ServeModel {
  Lane* lane = nullptr;
  std::deque<uint64_t> queue;
  std::vector<uint64_t> slot_req;  // 0 = free
  std::vector<int> state, its;
  std::vector<double> res;
  int running = 0;
  std::thread worker;
};

struct Server {
  Context* ctx = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  int capacity = 32;
  uint64_t next_id = 1;
  int error = MSG_OK;
  std::deque<ServeModel> models;  // deque: references stay valid while models are added
  std::unordered_map<uint64_t, ServeRequest> reqs;

  void run(ServeModel& m);
  ~Server() {
    {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
    }
    cv_work.notify_all();
    for (auto& m : models)
      if (m.worker.joinable()) m.worker.join();
    for (auto& m : models) lane_destroy(m.lane);
  }
};

void Server::run(ServeModel& m) {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_work.wait(lk, [&] { return stop || m.running > 0 || !m.queue.empty(); });
    if (stop) return;
    // admit queued requests into free slots (host staging only)
    const int cap = lane_capacity(m.lane);
    for (int s = 0; s < cap && !m.queue.empty(); ++s) {
      if (m.slot_req[s]) continue;
      const uint64_t id = m.queue.front();
      m.queue.pop_front();
      auto it = reqs.find(id);
      if (it == reqs.end() || it->second.cancelled) continue;
      it->second.slot = s;
      m.slot_req[s] = id;
      lane_stage(m.lane, s, it->second.xi.data());
      ++m.running;
    }
    if (m.running == 0) continue;
    // one cycle without the lock (GPU work and a stream sync)
    lk.unlock();
    int n_active = 0;
    const int st = lane_cycle(m.lane, m.state.data(), m.its.data(), m.res.data(), &n_active);
    lk.lock();
    if (st != MSG_OK) {
      // a failed cycle fails every request of the lane
      error = st;
      for (size_t s = 0; s < m.slot_req.size(); ++s) {
        if (!m.slot_req[s]) continue;
        auto it = reqs.find(m.slot_req[s]);
        if (it != reqs.end()) {
          it->second.finished = true;
          it->second.status = st;
        }
        m.slot_req[s] = 0;
      }
      m.running = 0;
      cv_done.notify_all();
      continue;
    }
    for (size_t s = 0; s < m.slot_req.size(); ++s) {
      const uint64_t id = m.slot_req[s];
      if (!id || m.state[s] == 0) continue;
      m.slot_req[s] = 0;
      --m.running;
      auto it = reqs.find(id);
      if (it == reqs.end()) continue;
      std::vector<double> X;
      int fs = MSG_OK;
      if (!it->second.cancelled) {
        // fetch without the lock (the request map may change meanwhile)
        X.resize(lane_n_dofs(m.lane));
        lk.unlock();
        fs = lane_fetch(m.lane, (int)s, X.data());
        lk.lock();
        it = reqs.find(id);
        if (it == reqs.end()) continue;
      }
      ServeRequest& r = it->second;
      if (!r.cancelled) {
        r.X.swap(X);
        r.its = m.its[s];
        r.res = m.res[s];
        r.status = fs != MSG_OK ? fs
                   : m.state[s] == 1 ? MSG_OK
                   : m.state[s] == 2 ? MSG_ERR_BREAKDOWN
                                     : MSG_ERR_NOT_CONVERGED;
      }
      r.finished = true;
      r.latency_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r.t0).count();
    }
    // cancelled requests still occupying slots are stopped at the next cycle
    for (size_t s = 0; s < m.slot_req.size(); ++s) {
      if (!m.slot_req[s]) continue;
      auto it = reqs.find(m.slot_req[s]);
      if (it != reqs.end() && it->second.cancelled) lane_abort(m.lane, (int)s);
    }
    cv_done.notify_all();
  }
}

static Server* server_of(Context* ctx) { return static_cast<Server*>(ctx->server); }

void server_destroy(Context* ctx) {
  delete server_of(ctx);
  ctx->server = nullptr;
}

}  // namespace msg

using namespace msg;

#define SERVE_GUARD(ctx)                                            \
  if (!(ctx)) return MSG_ERR_INVALID_ARGUMENT;                      \
  std::lock_guard<std::recursive_mutex> _g((ctx)->mu);              \
  Server* srv = server_of(ctx);                                     \
  if (!srv) return set_error((ctx), MSG_ERR_INVALID_ARGUMENT, "serving is not started on this context")

extern "C" {

int MSG_SERVE_START(MSG_CTX ctx, int max_batch) {
  if (!ctx) return MSG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> g(ctx->mu);
  if (ctx->server) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "serving already started");
  if (max_batch <= 0 || max_batch > 65536) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "max_batch out of range");
  Server* s = new Server();
  s->ctx = ctx;
  s->capacity = max_batch;
  ctx->server = s;
  return MSG_OK;
}

int MSG_SERVE_ADD_MODEL(MSG_CTX ctx, MSG_MESH mesh, double nu, const MSG_KL* kl, const double* b, double tol,
                        int max_it, int* model_id) {
  SERVE_GUARD(ctx);
  if (!mesh || !kl || !b || !model_id) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "null argument");
  if (mesh->ctx != ctx) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "mesh belongs to another context");
  Lane* lane = nullptr;
  MSG_TRY(lane_create(ctx, mesh, nu, kl, b, srv->capacity, tol, max_it, &lane));
  std::lock_guard<std::mutex> g2(srv->mu);
  ServeModel m;
  m.lane = lane;
  const int cap = lane_capacity(lane);
  m.slot_req.assign(cap, 0);
  m.state.assign(cap, 0);
  m.its.assign(cap, 0);
  m.res.assign(cap, 0.0);
  srv->models.push_back(std::move(m));
  ServeModel& added = srv->models.back();
  added.worker = std::thread([srv, &added] { srv->run(added); });
  *model_id = (int)srv->models.size() - 1;
  return MSG_OK;
}

int MSG_SERVE_SUBMIT(MSG_CTX ctx, int model_id, const double* xi, uint64_t* id) {
  SERVE_GUARD(ctx);
  if (!xi || !id) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> g2(srv->mu);
  if (model_id < 0 || model_id >= (int)srv->models.size())
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown model %d", model_id);
  ServeModel& m = srv->models[model_id];
  ServeRequest r;
  r.model = model_id;
  r.xi.assign(xi, xi + lane_n_terms(m.lane));
  r.t0 = std::chrono::steady_clock::now();
  const uint64_t rid = srv->next_id++;
  srv->reqs.emplace(rid, std::move(r));
  m.queue.push_back(rid);
  *id = rid;
  srv->cv_work.notify_all();
  return MSG_OK;
}

int MSG_SERVE_POLL(MSG_CTX ctx, uint64_t id, int timeout_ms, double* X, int* iterations, double* rel_res,
                   double* latency_ms) {
  if (!ctx) return MSG_ERR_INVALID_ARGUMENT;
  Server* srv = nullptr;
  {
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    srv = server_of(ctx);
    if (!srv) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "serving is not started on this context");
  }
  // wait without the context lock (the worker never takes it)
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return MSG_ERR_INVALID_ARGUMENT;
  if (!it->second.finished && timeout_ms != 0) {
    auto done = [&] {
      auto jt = srv->reqs.find(id);
      return jt == srv->reqs.end() || jt->second.finished;
    };
    if (timeout_ms < 0)
      srv->cv_done.wait(lk, done);
    else
      srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done);
    it = srv->reqs.find(id);
    if (it == srv->reqs.end()) return MSG_ERR_INVALID_ARGUMENT;
  }
  ServeRequest& r = it->second;
  if (!r.finished) return MSG_PENDING;
  const int st = r.cancelled ? MSG_ERR_CANCELLED : r.status;
  if (X && !r.cancelled && !r.X.empty()) std::memcpy(X, r.X.data(), sizeof(double) * r.X.size());
  if (iterations) *iterations = r.its;
  if (rel_res) *rel_res = r.res;
  if (latency_ms) *latency_ms = r.latency_ms;
  srv->reqs.erase(it);
  return st;
}

int MSG_SERVE_CANCEL(MSG_CTX ctx, uint64_t id) {
  SERVE_GUARD(ctx);
  std::lock_guard<std::mutex> g2(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown request");
  ServeRequest& r = it->second;
  if (r.finished) return MSG_OK;
  r.cancelled = true;
  if (r.slot < 0) {
    // still queued: it never reaches the GPU
    auto& q = srv->models[r.model].queue;
    for (auto qi = q.begin(); qi != q.end(); ++qi)
      if (*qi == id) {
        q.erase(qi);
        break;
      }
    r.finished = true;
    srv->cv_done.notify_all();
  }
  return MSG_OK;
}

int MSG_SERVE_STATS(MSG_CTX ctx, int64_t* queued, int64_t* running) {
  SERVE_GUARD(ctx);
  std::lock_guard<std::mutex> g2(srv->mu);
  int64_t nq = 0, nr = 0;
  for (auto& m : srv->models) {
    nq += (int64_t)m.queue.size();
    nr += m.running;
  }
  if (queued) *queued = nq;
  if (running) *running = nr;
  return MSG_OK;
}

int MSG_SERVE_STOP(MSG_CTX ctx) {
  if (!ctx) return MSG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> g(ctx->mu);
  if (!ctx->server) return MSG_OK;
  server_destroy(ctx);
  return MSG_OK;
}

}  // extern "C"
