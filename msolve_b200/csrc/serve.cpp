// Serving: requests (one realization of a registered model each) are queued,
// admitted into free slots of one of their model's lanes at chunk boundaries,
// and returned as soon as their own FP64 true residual is below the model's
// tolerance (continuous batching). A lane is a batch of `capacity` slots of
// one model with its device state; admission is by device memory: a model
// gets its first lane when it is registered, and a manager thread adds lanes
// while the model's queue outgrows its free slots and the context's memory
// budget (MSG_CREATE) has room, and retires idle extra lanes when another
// model's requests need the memory (or after a second of idleness). One
// worker thread per lane drives it on the lane's own stream, so lanes of
// different sizes overlap on the GPU; the C entry points only touch the
// queues under the server mutex.
// No counterpart in the reference (its Monte Carlo loop is sequential,
// ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:258-276).
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <thread>
#include <unordered_map>

#include "msg_internal.h"

namespace msg {

using Clock = std::chrono::steady_clock;
constexpr int kMaxLanesPerModel = 8;

struct ServeRequest {
  int model = 0;
  std::vector<double> xi;
  Clock::time_point t0;
  int slot = -1;
  bool finished = false, cancelled = false;
  int status = MSG_OK;
  std::vector<double> X;
  int its = 0;
  double res = 0.0, latency_ms = 0.0;
};

struct ServeLane {
  Lane* lane = nullptr;
  std::vector<uint64_t> slot_req;  // 0 = free
  std::vector<int> state, its;
  std::vector<double> res;
  int running = 0;
  bool first = false;   // the model's first lane: kept while the server runs
  bool retire = false;  // stop admitting; the worker exits once its slots are empty
  bool exited = false;
  Clock::time_point idle_since = Clock::now();
  std::thread worker;
};

// A registered model: what a new lane needs (mesh, material, a copy of the KL
// table and of the load), its queue and its lanes.
struct ServeModel {
  Mesh* mesh = nullptr;
  double nu = 0.3, tol = 1e-8;
  int max_it = 0;
  MSG_KL kl{};
  std::vector<double> w3, amp3, eig, b;
  std::vector<int> idx3;
  std::deque<uint64_t> queue;
  std::list<ServeLane> lanes;  // list: references stay valid while lanes come and go
  int free_slots() const {
    int f = 0;
    for (const ServeLane& l : lanes)
      if (!l.retire) f += (int)l.slot_req.size() - l.running;
    return f;
  }
};

struct Server {
  Context* ctx = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_manage;
  std::atomic<bool> stop{false};
  int capacity = 32;
  uint64_t next_id = 1;
  int error = MSG_OK;
  std::deque<ServeModel> models;  // deque: references stay valid while models are added
  std::unordered_map<uint64_t, ServeRequest> reqs;
  std::thread manager;
  int64_t lanes_added = 0, lanes_retired = 0;

  void run(ServeModel& m, ServeLane& l);
  void manage();
  int add_lane(ServeModel& m, bool first);
  ~Server() {
    {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
    }
    cv_work.notify_all();
    cv_manage.notify_all();
    if (manager.joinable()) manager.join();
    for (auto& m : models)
      for (auto& l : m.lanes)
        if (l.worker.joinable()) l.worker.join();
    for (auto& m : models) {
      for (auto& l : m.lanes) lane_destroy(l.lane);
      if (m.mesh) release(m.mesh);
    }
  }
};

// Create a lane for model m (the context lock must be held) and start its worker.
int Server::add_lane(ServeModel& m, bool first) {
  Lane* lane = nullptr;
  MSG_TRY(lane_create(ctx, m.mesh, m.nu, &m.kl, m.b.data(), capacity, m.tol, m.max_it, &lane));
  std::lock_guard<std::mutex> g(mu);
  m.lanes.emplace_back();
  ServeLane& l = m.lanes.back();
  l.lane = lane;
  l.first = first;
  const int cap = lane_capacity(lane);
  l.slot_req.assign(cap, 0);
  l.state.assign(cap, 0);
  l.its.assign(cap, 0);
  l.res.assign(cap, 0.0);
  l.worker = std::thread([this, &m, &l] { run(m, l); });
  ++lanes_added;
  cv_work.notify_all();
  return MSG_OK;
}

void Server::run(ServeModel& m, ServeLane& l) {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_work.wait(lk, [&] { return stop || l.retire || l.running > 0 || !m.queue.empty(); });
    if (stop || (l.retire && l.running == 0)) {
      l.exited = true;
      cv_manage.notify_all();
      return;
    }
    // admit queued requests into free slots (host staging only)
    const int cap = (int)l.slot_req.size();
    for (int s = 0; s < cap && !m.queue.empty() && !l.retire; ++s) {
      if (l.slot_req[s]) continue;
      const uint64_t id = m.queue.front();
      m.queue.pop_front();
      auto it = reqs.find(id);
      if (it == reqs.end() || it->second.cancelled) continue;
      it->second.slot = s;
      l.slot_req[s] = id;
      lane_stage(l.lane, s, it->second.xi.data());
      ++l.running;
    }
    if (l.running == 0) continue;
    if (!m.queue.empty()) cv_manage.notify_all();  // a backlog beyond this lane: maybe another lane
    // one cycle without the lock (GPU work and a stream sync)
    lk.unlock();
    int n_active = 0;
    const int st = lane_cycle(l.lane, l.state.data(), l.its.data(), l.res.data(), &n_active);
    lk.lock();
    if (st != MSG_OK) {
      // a failed cycle fails every request of the lane
      error = st;
      for (size_t s = 0; s < l.slot_req.size(); ++s) {
        if (!l.slot_req[s]) continue;
        auto it = reqs.find(l.slot_req[s]);
        if (it != reqs.end()) {
          it->second.finished = true;
          it->second.status = st;
        }
        l.slot_req[s] = 0;
      }
      l.running = 0;
      l.idle_since = Clock::now();
      cv_done.notify_all();
      continue;
    }
    for (size_t s = 0; s < l.slot_req.size(); ++s) {
      const uint64_t id = l.slot_req[s];
      if (!id || l.state[s] == 0) continue;
      l.slot_req[s] = 0;
      --l.running;
      auto it = reqs.find(id);
      if (it == reqs.end()) continue;
      std::vector<double> X;
      int fs = MSG_OK;
      if (!it->second.cancelled) {
        // fetch without the lock (the request map may change meanwhile)
        X.resize(lane_n_dofs(l.lane));
        lk.unlock();
        fs = lane_fetch(l.lane, (int)s, X.data());
        lk.lock();
        it = reqs.find(id);
        if (it == reqs.end()) continue;
      }
      ServeRequest& r = it->second;
      if (!r.cancelled) {
        r.X.swap(X);
        r.its = l.its[s];
        r.res = l.res[s];
        r.status = fs != MSG_OK ? fs
                   : l.state[s] == 1 ? MSG_OK
                   : l.state[s] == 2 ? MSG_ERR_BREAKDOWN
                                     : MSG_ERR_NOT_CONVERGED;
      }
      r.finished = true;
      r.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - r.t0).count();
    }
    if (l.running == 0) {
      l.idle_since = Clock::now();
      cv_manage.notify_all();
    }
    // cancelled requests still occupying slots are stopped at the next cycle
    for (size_t s = 0; s < l.slot_req.size(); ++s) {
      if (!l.slot_req[s]) continue;
      auto it = reqs.find(l.slot_req[s]);
      if (it != reqs.end() && it->second.cancelled) lane_abort(l.lane, (int)s);
    }
    cv_done.notify_all();
  }
}

// Lanes by memory: add a lane to a model whose queue outgrows its free slots
// while the context's budget allows; when it does not, retire idle extra lanes
// of the other models (their memory returns to the budget) and try again.
// Extra lanes idle for a second are retired as well.
void Server::manage() {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    cv_manage.wait_for(lk, std::chrono::milliseconds(200));
    if (stop) return;
    // join and free the lanes whose workers have exited (models by index: a model
    // added while the lock is released appends to the deque, which moves no
    // element but invalidates iterators)
    for (size_t mi = 0; mi < models.size(); ++mi) {
      ServeModel& m = models[mi];
      for (auto it = m.lanes.begin(); it != m.lanes.end();) {
        if (!it->exited) {
          ++it;
          continue;
        }
        std::thread w = std::move(it->worker);
        Lane* lane = it->lane;
        it = m.lanes.erase(it);
        lk.unlock();
        if (w.joinable()) w.join();
        // the context lock before the server lock, as the entry points take them; a
        // server being destroyed holds the context lock and waits for this thread
        bool locked = false;
        while (!(locked = ctx->mu.try_lock()) && !stop) std::this_thread::sleep_for(std::chrono::microseconds(200));
        lane_destroy(lane);
        if (locked) ctx->mu.unlock();
        if (stop) return;
        lk.lock();
        ++lanes_retired;
      }
    }
    const auto now = Clock::now();
    for (size_t mi = 0; mi < models.size(); ++mi) {
      ServeModel& m = models[mi];
      for (auto& l : m.lanes)
        if (!l.first && !l.retire && l.running == 0 && m.queue.empty() && now - l.idle_since > std::chrono::seconds(1)) {
          l.retire = true;
          cv_work.notify_all();
        }
    }
    // models with more queued requests than free slots
    for (size_t mi = 0; mi < models.size(); ++mi) {
      ServeModel& m = models[mi];
      if ((int)m.queue.size() <= m.free_slots() || (int)m.lanes.size() >= kMaxLanesPerModel) continue;
      lk.unlock();
      while (!ctx->mu.try_lock()) {
        if (stop) return;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
      }
      const int st = add_lane(m, false);
      ctx->mu.unlock();
      lk.lock();
      if (st == MSG_ERR_OUT_OF_MEMORY) {
        // no room: retire idle extra lanes of other models; the next round retries
        bool any = false;
        for (size_t mj = 0; mj < models.size(); ++mj)
          for (auto& l : models[mj].lanes)
            if (mj != mi && !l.first && !l.retire && l.running == 0) {
              l.retire = true;
              any = true;
            }
        if (any) cv_work.notify_all();
      } else if (st != MSG_OK) {
        error = st;
      }
    }
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
  s->manager = std::thread([s] { s->manage(); });
  return MSG_OK;
}

int MSG_SERVE_ADD_MODEL(MSG_CTX ctx, MSG_MESH mesh, double nu, const MSG_KL* kl, const double* b, double tol,
                        int max_it, int* model_id) {
  SERVE_GUARD(ctx);
  if (!mesh || !kl || !b || !model_id) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "null argument");
  if (mesh->ctx != ctx) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "mesh belongs to another context");
  if (kl->n_terms <= 0 || kl->n_terms > 64 || !kl->w3 || !kl->amp3 || !kl->idx3 || !kl->eig)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "KL table: 1..64 terms with all four arrays");
  ServeModel* m = nullptr;
  {
    std::lock_guard<std::mutex> g2(srv->mu);
    srv->models.emplace_back();
    m = &srv->models.back();
  }
  // the model keeps what later lanes need: its own copies of the KL table and the load
  const int K = kl->n_terms;
  m->mesh = mesh;
  retain(mesh);
  m->nu = nu;
  m->tol = tol;
  m->max_it = max_it;
  m->w3.assign(kl->w3, kl->w3 + 3 * K);
  m->amp3.assign(kl->amp3, kl->amp3 + 3 * K);
  m->idx3.assign(kl->idx3, kl->idx3 + 3 * K);
  m->eig.assign(kl->eig, kl->eig + K);
  m->b.assign(b, b + mesh->n_dofs);
  m->kl = *kl;
  m->kl.w3 = m->w3.data();
  m->kl.amp3 = m->amp3.data();
  m->kl.idx3 = m->idx3.data();
  m->kl.eig = m->eig.data();
  const int st = srv->add_lane(*m, true);
  if (st != MSG_OK) {
    // leave a model without lanes behind: its requests are refused
    std::lock_guard<std::mutex> g2(srv->mu);
    m->max_it = -1;
    return st;
  }
  *model_id = (int)srv->models.size() - 1;
  return MSG_OK;
}

int MSG_SERVE_SUBMIT(MSG_CTX ctx, int model_id, const double* xi, uint64_t* id) {
  SERVE_GUARD(ctx);
  if (!xi || !id) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> g2(srv->mu);
  if (model_id < 0 || model_id >= (int)srv->models.size() || srv->models[model_id].max_it < 0)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown model %d", model_id);
  ServeModel& m = srv->models[model_id];
  ServeRequest r;
  r.model = model_id;
  r.xi.assign(xi, xi + m.kl.n_terms);
  r.t0 = Clock::now();
  const uint64_t rid = srv->next_id++;
  srv->reqs.emplace(rid, std::move(r));
  m.queue.push_back(rid);
  *id = rid;
  srv->cv_work.notify_all();
  if ((int)m.queue.size() > m.free_slots()) srv->cv_manage.notify_all();
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
  // wait without the context lock (the workers never take it)
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
    for (auto& l : m.lanes) nr += l.running;
  }
  if (queued) *queued = nq;
  if (running) *running = nr;
  return MSG_OK;
}

int MSG_SERVE_LANES(MSG_CTX ctx, int model_id, int* lanes, int64_t* added, int64_t* retired) {
  SERVE_GUARD(ctx);
  std::lock_guard<std::mutex> g2(srv->mu);
  if (model_id < -1 || model_id >= (int)srv->models.size())
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown model %d", model_id);
  int n = 0;
  for (size_t mi = 0; mi < srv->models.size(); ++mi)
    if (model_id < 0 || (int)mi == model_id)
      for (auto& l : srv->models[mi].lanes) n += l.retire ? 0 : 1;
  if (lanes) *lanes = n;
  if (added) *added = srv->lanes_added;
  if (retired) *retired = srv->lanes_retired;
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
