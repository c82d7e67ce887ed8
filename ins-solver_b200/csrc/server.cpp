// Serving loop: concurrent solves of independent requests on one GPU.
//
// No counterpart in the reference, which solves one system at a time inside
// its time step. Requests arrive through sipg_server_submit at any time; `slots`
// worker threads each take the first queued request that can run now (a slot is
// free, its operator is not busy with another request, and its solver state is
// resident or fits the HBM budget) and solve it on the solver's own CUDA stream,
// so the kernels of different requests overlap on the device. Solver states stay
// resident between requests with the same operator, kind and options; idle ones
// are released least recently used first when a new state needs room.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "runtime.hpp"

namespace sipg {
void solver_set_cancel(sipg_solver* s, const std::atomic<int>* flag);
}

using Clock = std::chrono::steady_clock;
using namespace sipg;

namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Device bytes of a solver's state (work vectors, multigrid levels, assembled
// blocks, algebraic coarse levels), estimated from the operator's sizes.
size_t estimate_bytes(const sipg_op* op, int kind, const sipg_solver_opts& o) {
  const size_t K = op->mesh->K, nc = op->ncomp, NF = op->mesh->dim + 1;
  const size_t n = nc * K * op->Np;
  size_t b = 10 * n * sizeof(double);  // Krylov vectors, host-transfer buffers
  if (kind == SIPG_SOLVER_BLOCK_JACOBI) b += n * op->Np * sizeof(double);
  if (kind == SIPG_SOLVER_PMULTIGRID) {
    const size_t ts = o.precision == SIPG_FP32 ? 4 : 8;
    for (int l = 0; l < o.n_levels && l < 4; ++l) {
      const int p = l == 0 ? op->order : o.orders[l];
      const size_t np = (size_t)(op->mesh->dim == 3 ? (p + 1) * (p + 2) * (p + 3) / 6 : (p + 1) * (p + 2) / 2);
      const size_t nl = nc * K * np;
      b += nl * (12 + 7 * ts);                              // inverse diagonals, level vectors
      if (l > 0) b += K * np * 24 + K * NF * 2 * (np + 2) * 12;  // level operator, traces
      if (l > 0 && p == 1) b += (NF + 1) * np * np * K * 12;  // assembled blocks
    }
    b += op->mesh->Nv * 400;  // algebraic coarse levels
  }
  return b + (1u << 20);
}

struct Request {
  long long id = 0;
  sipg_op* op = nullptr;
  int kind = 0;
  sipg_solver_opts opts{};
  std::vector<double> b;
  double* x = nullptr;
  Clock::time_point t_submit, t_start, t_done;
  std::atomic<int> cancel{0};
  int state = 0;  // 0 queued, 1 running, 2 done
  sipg_request_result res{};
};

struct Resident {
  sipg_op* op = nullptr;
  int kind = 0;
  sipg_solver_opts opts{};
  sipg_solver* solver = nullptr;
  size_t bytes = 0;
  bool busy = false;
  unsigned long long last_use = 0;
  bool matches(const Request& r) const {
    return op == r.op && kind == r.kind && std::memcmp(&opts, &r.opts, sizeof(opts)) == 0;
  }
};

}  // namespace

struct sipg_server {
  sipg_server_opts o{};
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<long long, std::shared_ptr<Request>> all;
  std::vector<std::unique_ptr<Resident>> resident;
  size_t resident_bytes = 0;
  std::set<sipg_op*> busy_ops;
  std::vector<std::thread> workers;
  bool stop = false;
  long long next_id = 1;
  int running = 0;
  unsigned long long tick = 0;

  // Resident state for r (existing, or newly reserved within the budget); null: wait.
  Resident* reserve(const Request& r) {
    for (auto& s : resident)
      if (s->matches(r)) return s->busy ? nullptr : s.get();
    const size_t need = estimate_bytes(r.op, r.kind, r.opts);
    while (resident_bytes + need > o.hbm_budget_bytes) {
      Resident* lru = nullptr;
      for (auto& s : resident)
        if (!s->busy && (!lru || s->last_use < lru->last_use)) lru = s.get();
      if (!lru) return nullptr;  // everything resident is in use: wait
      evict(lru);
    }
    auto s = std::make_unique<Resident>();
    s->op = r.op;
    s->kind = r.kind;
    s->opts = r.opts;
    s->bytes = need;
    resident_bytes += need;
    resident.push_back(std::move(s));
    return resident.back().get();
  }
  void evict(Resident* s) {
    if (s->solver) sipg_solver_destroy(s->solver);
    resident_bytes -= s->bytes;
    resident.erase(std::find_if(resident.begin(), resident.end(), [&](auto& p) { return p.get() == s; }));
  }
  void finish(Request& r, int status) {
    r.t_done = Clock::now();
    r.res.status = status;
    r.res.queue_ms = r.state == 0 ? ms_between(r.t_submit, r.t_done) : ms_between(r.t_submit, r.t_start);
    r.res.run_ms = r.state == 0 ? 0.0 : ms_between(r.t_start, r.t_done);
    r.res.total_ms = ms_between(r.t_submit, r.t_done);
    r.state = 2;
  }

  void worker() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      std::shared_ptr<Request> req;
      Resident* slot = nullptr;
      for (auto it = queue.begin(); it != queue.end(); ++it) {
        if (busy_ops.count((*it)->op)) continue;
        slot = reserve(**it);
        if (!slot) continue;
        req = *it;
        queue.erase(it);
        break;
      }
      if (!req) {
        if (stop) return;
        cv_work.wait(lk);
        continue;
      }
      slot->busy = true;
      busy_ops.insert(req->op);
      req->state = 1;
      req->t_start = Clock::now();
      ++running;
      lk.unlock();
      int st = SIPG_OK;
      sipg_solve_info info{};
      if (!slot->solver) {
        st = sipg_solver_create(req->op, req->kind, &req->opts, &slot->solver);
        if (st != SIPG_OK) slot->solver = nullptr;
      }
      if (st == SIPG_OK) {
        solver_set_cancel(slot->solver, &req->cancel);
        st = sipg_solver_solve_host(slot->solver, req->b.data(), req->x, &info);
        solver_set_cancel(slot->solver, nullptr);
      }
      const bool hard = st != SIPG_OK && st != SIPG_NOT_CONVERGED && st != SIPG_BREAKDOWN && st != SIPG_CANCELLED;
      if (hard) std::snprintf(req->res.error, sizeof(req->res.error), "%s", sipg_last_error());
      lk.lock();
      --running;
      req->res.info = info;
      finish(*req, st);
      slot->busy = false;
      slot->last_use = ++tick;
      // a solver that failed with an error may hold inconsistent state: the next
      // request of its kind gets a new one
      if (!slot->solver || hard) evict(slot);
      busy_ops.erase(req->op);
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

extern "C" {

int sipg_server_create(const sipg_server_opts* o, sipg_server** out) {
  return guarded([&] {
    if (!o || !out || o->slots < 1 || o->slots > 64) throw Error(SIPG_INVALID_ARG, "server options");
    auto s = std::make_unique<sipg_server>();
    s->o = *o;
    SIPG_CUDA(cudaGetDevice(&s->device));
    if (s->o.hbm_budget_bytes == 0) {
      size_t free_b = 0, total = 0;
      SIPG_CUDA(cudaMemGetInfo(&free_b, &total));
      s->o.hbm_budget_bytes = (size_t)(0.9 * (double)free_b);
    }
    for (int i = 0; i < o->slots; ++i) s->workers.emplace_back([p = s.get()] { p->worker(); });
    *out = s.release();
  });
}

int sipg_server_submit(sipg_server* s, sipg_op* op, int kind, const sipg_solver_opts* o, const double* b, double* x,
                       long long* id) {
  return guarded([&] {
    if (!s || !op || !b || !x || !id || kind < 0 || kind > SIPG_SOLVER_PMULTIGRID)
      throw Error(SIPG_INVALID_ARG, "submit arguments");
    auto r = std::make_shared<Request>();
    r->op = op;
    r->kind = kind;
    if (o) r->opts = *o;
    else sipg_solver_default_opts(kind, &r->opts);
    const size_t n = (size_t)op->ncomp * op->mesh->K * op->Np;
    r->b.assign(b, b + n);
    r->x = x;
    if (estimate_bytes(op, kind, r->opts) > s->o.hbm_budget_bytes)
      throw Error(SIPG_OUT_OF_MEMORY, "request rejected: its solver state exceeds the HBM budget");
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) throw Error(SIPG_CANCELLED, "server stopping");
    r->id = s->next_id++;
    *id = r->id;
    s->all[r->id] = r;
    s->queue.push_back(r);
    s->cv_work.notify_one();
  });
}

int sipg_server_poll(sipg_server* s, long long id, int* done, sipg_request_result* res) {
  return guarded([&] {
    if (!s || !done) throw Error(SIPG_INVALID_ARG, "poll arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) throw Error(SIPG_INVALID_ARG, "unknown request");
    *done = it->second->state == 2;
    if (*done) {
      if (res) *res = it->second->res;
      s->all.erase(it);
    }
  });
}

int sipg_server_wait(sipg_server* s, long long id, sipg_request_result* res) {
  return guarded([&] {
    if (!s) throw Error(SIPG_INVALID_ARG, "wait arguments");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) throw Error(SIPG_INVALID_ARG, "unknown request");
    auto r = it->second;
    s->cv_done.wait(lk, [&] { return r->state == 2; });
    if (res) *res = r->res;
    s->all.erase(id);
  });
}

int sipg_server_cancel(sipg_server* s, long long id) {
  return guarded([&] {
    if (!s) throw Error(SIPG_INVALID_ARG, "cancel arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) throw Error(SIPG_INVALID_ARG, "unknown request");
    auto& r = it->second;
    if (r->state == 0) {
      s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
      s->finish(*r, SIPG_CANCELLED);
      s->cv_done.notify_all();
    } else if (r->state == 1) {
      r->cancel.store(1);
    }
  });
}

int sipg_server_stats(sipg_server* s, int* resident_solvers, size_t* resident_bytes, int* queued, int* running) {
  return guarded([&] {
    if (!s) throw Error(SIPG_INVALID_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (resident_solvers) *resident_solvers = (int)s->resident.size();
    if (resident_bytes) *resident_bytes = s->resident_bytes;
    if (queued) *queued = (int)s->queue.size();
    if (running) *running = s->running;
  });
}

void sipg_server_destroy(sipg_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto& r : s->queue) s->finish(*r, SIPG_CANCELLED);
    s->queue.clear();
    for (auto& kv : s->all)
      if (kv.second->state == 1) kv.second->cancel.store(1);
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  for (auto& t : s->workers) t.join();
  for (auto& r : s->resident)
    if (r->solver) sipg_solver_destroy(r->solver);
  delete s;
}

}  // extern "C"
