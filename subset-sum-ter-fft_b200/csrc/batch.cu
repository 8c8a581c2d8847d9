// tergpu_attempt_batch: many independent attempt ranges on one device at once
// (include/tergpu.h).
//
// Continuous batching over `slots` concurrent attempt pipelines, each a host
// thread with its own stream and private workspace.  The unit of work is one
// attempt of one request: a request's attempts are independent (each draws its
// own targets from seed + attempt), so they spread over free slots.  A request
// is decided by its lowest attempt whose status is not NoWitnessThisAttempt --
// exactly the attempt the sequential loop of tergpu_attempt_run would stop at --
// and attempts above a known decisive one are never started; every attempt runs
// exactly tergpu_attempt_run's code, so a request's result is the same alone
// and in the mix.
//
// Admission: requests in arrival order; a request's next attempt starts when a
// slot is free and the predicted device bytes of the running attempts (one
// preflight figure per attempt) stay within the memory budget; a request that
// does not fit waits and later requests that fit go ahead.  Requests the
// preflight refuses (InvalidConfiguration, or ResourceLimit against their own
// ceiling or the whole budget) complete at once with that status.

#include "tergpu.h"
#include "tergpu_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <system_error>
#include <thread>
#include <vector>

namespace tergpu {
std::mutex g_slots_mu;
std::vector<std::unique_ptr<Workspace>> g_slots;  // idle slot workspaces, any device

std::unique_ptr<Workspace> take_slot(int device) {
  {
    std::lock_guard<std::mutex> lock(g_slots_mu);
    for (auto it = g_slots.begin(); it != g_slots.end(); ++it) {
      if ((*it)->device == device) {
        std::unique_ptr<Workspace> w = std::move(*it);
        g_slots.erase(it);
        return w;
      }
    }
  }
  return make_workspace(device, /*blocking=*/true);
}

void give_slot(std::unique_ptr<Workspace> w) {
  release_buffers(*w);
  if (cudaStreamSynchronize(w->stream) != cudaSuccess) {  // a broken slot is not kept
    destroy_workspace(*w);
    return;
  }
  std::lock_guard<std::mutex> lock(g_slots_mu);
  g_slots.push_back(std::move(w));
}

void release_slots() {
  std::lock_guard<std::mutex> lock(g_slots_mu);
  for (auto& w : g_slots) destroy_workspace(*w);
  g_slots.clear();
}

namespace {

using Clock = std::chrono::steady_clock;

constexpr int8_t kPending = -1;  // attempt not finished (or never started)

struct Request {
  uint32_t count = 0;        // attempts in the range
  uint32_t next = 0;         // next attempt index to start
  std::vector<int8_t> unit;  // per attempt: kPending, or its status
  bool admitted = false, done = false;
  uint64_t held = 0;         // largest bytes an attempt's workspace held
  std::vector<std::pair<uint32_t, std::array<uint8_t, 128>>> witnesses;  // of Found attempts
};

struct Unit {
  uint64_t req;
  uint32_t k;
};

struct Engine {
  const tergpu_batch_in* in = nullptr;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Unit> ready;
  std::vector<Request> req;
  std::vector<uint64_t> predicted;  // admission bytes of one attempt (stage buffers)
  std::vector<uint64_t> reported;   // device_bytes as the request alone reports it
  uint64_t running = 0, finished = 0, inflight_bytes = 0;
  bool graphs = true;  // slots keep their per-shape graph plans (reserved in the budget)
  bool stop = false;
  int worker_error = TERGPU_COMPLETED;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
};

// The sequential loop's stopping point: the lowest attempt whose status is not
// NoWitness decides once every attempt below it has finished.  Returns its
// index (count when every attempt is NoWitness), or -1 while undecided.
int64_t decisive(const Request& r) {
  for (uint32_t k = 0; k < r.count; ++k) {
    if (r.unit[k] == kPending) return -1;
    if (r.unit[k] != TERGPU_NO_WITNESS_THIS_ATTEMPT) return k;
  }
  return r.count;
}

// The lowest finished attempt already known to decide; attempts at or above
// it need not start.
uint32_t stop_bound(const Request& r) {
  for (uint32_t k = 0; k < r.count; ++k) {
    if (r.unit[k] != kPending && r.unit[k] != TERGPU_NO_WITNESS_THIS_ATTEMPT) return k;
  }
  return r.count;
}

// With e->mu held, once a request is decided at attempt j: its result.
void finish_request(Engine* e, uint64_t r, int64_t j) {
  Request& q = e->req[r];
  tergpu_attempt_out* o = &e->in->outs[r];
  const uint32_t first = e->in->jobs[r].attempt_first;
  if (static_cast<uint32_t>(j) == q.count) {
    o->status = TERGPU_ATTEMPT_LIMIT_REACHED;
    o->attempts_run = q.count;
  } else if (q.unit[j] == TERGPU_FOUND) {
    o->status = TERGPU_FOUND;
    o->attempts_run = static_cast<uint32_t>(j) + 1;
    o->found_attempt = first + static_cast<uint32_t>(j);
    for (const auto& w : q.witnesses) {
      if (w.first == static_cast<uint32_t>(j)) std::memcpy(o->witness, w.second.data(), w.second.size());
    }
  } else {
    o->status = q.unit[j];  // an error stops the sequential loop before that attempt counts
    o->attempts_run = static_cast<uint32_t>(j);
  }
  o->device_bytes = e->reported[r];
  o->device_bytes_held = q.held;
  q.done = true;
  ++e->finished;
  if (e->in->finish_ms != nullptr) e->in->finish_ms[r] = e->now_ms();
}

void worker_main(Engine* e) {
  std::unique_ptr<Workspace> ws;
  try {
    ws = take_slot(e->in->device);
  } catch (const Failure& f) {
    std::lock_guard<std::mutex> lock(e->mu);
    e->worker_error = f.status;
  }
  for (;;) {
    Unit u{};
    {
      std::unique_lock<std::mutex> lock(e->mu);
      e->cv_work.wait(lock, [e] { return e->stop || !e->ready.empty(); });
      if (e->ready.empty()) break;
      u = e->ready.front();
      e->ready.pop_front();
    }
    tergpu_attempt_in one = e->in->jobs[u.req];
    one.device = e->in->device;
    if (!e->graphs) one.flags |= TERGPU_ATTEMPT_NO_GRAPH;
    // the largest attempts (n = 108: seconds of sweep) yield SMs to the others
    if (one.n >= 108) one.flags |= TERGPU_ATTEMPT_BACKGROUND;
    one.attempt_first += u.k;
    one.attempt_count = 1;
    tergpu_attempt_out* dst = &e->in->outs[u.req];
    tergpu_attempt_stats stat{};
    tergpu_attempt_out out{};
    out.stats = &stat;
    int st = TERGPU_DEVICE_ERROR;
    if (ws) {
      try {
        st = attempt_body(&one, &out, ws.get());
      } catch (const Failure& f) {
        st = f.status;
      } catch (const std::bad_alloc&) {
        st = TERGPU_RESOURCE_LIMIT;
      } catch (...) {
        st = TERGPU_DEVICE_ERROR;
      }
    }
    // one attempt's "limit reached" is the sequential loop's NoWitness for it
    const int8_t unit = static_cast<int8_t>(
        st == TERGPU_ATTEMPT_LIMIT_REACHED ? TERGPU_NO_WITNESS_THIS_ATTEMPT : st);
    // the slot's buffers go back to the device pool: each running attempt holds
    // only its own bytes, so the running attempts stay within the budget
    if (ws) release_buffers(*ws);
    {
      std::lock_guard<std::mutex> lock(e->mu);
      Request& q = e->req[u.req];
      q.unit[u.k] = unit;
      q.held = std::max(q.held, out.device_bytes_held);
      if (dst->stats != nullptr && out.attempts_run == 1) dst->stats[u.k] = stat;
      if (out.r1 != 0) {
        dst->r1 = out.r1;
        dst->r2 = out.r2;
        dst->level3_size = out.level3_size;
      }
      if (unit == TERGPU_FOUND) {
        std::array<uint8_t, 128> w{};
        std::memcpy(w.data(), out.witness, w.size());
        q.witnesses.emplace_back(u.k, w);
      }
      e->inflight_bytes -= e->predicted[u.req];
      --e->running;
      if (!q.done) {
        const int64_t j = decisive(q);
        if (j >= 0) finish_request(e, u.req, j);
      }
    }
    e->cv_done.notify_all();
  }
  if (ws) give_slot(std::move(ws));
}

int batch_body(const tergpu_batch_in* in, tergpu_batch_out* out) {
  if (in->count != 0 && (in->jobs == nullptr || in->outs == nullptr)) {
    t_error = "jobs or outs missing";
    return TERGPU_INVALID_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || in->device < 0 || in->device >= ndev) {
    t_error = "no CUDA device " + std::to_string(in->device);
    return TERGPU_DEVICE_ERROR;
  }
  check(cudaSetDevice(in->device), "cudaSetDevice");
  uint64_t budget = in->memory_budget_bytes;
  if (budget == 0) {
    size_t free_b = 0, total_b = 0;
    check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    budget = static_cast<uint64_t>(static_cast<double>(free_b) * 0.9);
  }
  const uint32_t slots = in->slots == 0 ? 8u : std::min<uint32_t>(in->slots, 256u);
  Engine e;
  e.in = in;
  e.predicted.assign(in->count, 0);
  e.reported.assign(in->count, 0);
  e.req.resize(in->count);
  std::memset(out, 0, sizeof *out);

  // arrival order (stable by index for equal arrivals)
  std::vector<uint64_t> order(in->count);
  std::iota(order.begin(), order.end(), 0ull);
  if (in->arrival_ms != nullptr) {
    std::stable_sort(order.begin(), order.end(), [in](uint64_t a, uint64_t b) {
      return in->arrival_ms[a] < in->arrival_ms[b];
    });
  }
  // preflight every request (host arithmetic only) and clear its result
  // (keeping the caller's stats buffer); the batch runs no L1 export.  A
  // request's own preflight decides its refusals, as alone; admission counts
  // its stage-by-stage bytes, and each slot's graph plans (kept between
  // requests, one per shape n = 36 / 72) are reserved up front.  When slots x
  // plans leave no room for the largest request, every attempt runs stage by
  // stage instead (same results) and nothing is reserved.
  std::vector<int> refused(in->count, -1);
  std::map<uint32_t, uint64_t> plan_of;  // shape n -> graph plan bytes
  uint64_t largest = 0;
  for (uint64_t i = 0; i < in->count; ++i) {
    tergpu_attempt_out* o = &in->outs[i];
    tergpu_attempt_stats* keep_stats = o->stats;
    std::memset(o, 0, sizeof *o);
    o->stats = keep_stats;
    tergpu_attempt_in pre = in->jobs[i];
    pre.flags |= TERGPU_ATTEMPT_PREFLIGHT;
    tergpu_attempt_out pout{};
    const int st = attempt_body(&pre, &pout, nullptr);
    e.predicted[i] = e.reported[i] = pout.device_bytes;
    if (st == TERGPU_COMPLETED) {
      tergpu_attempt_out sout{};
      pre.flags |= TERGPU_ATTEMPT_NO_GRAPH;
      if (attempt_body(&pre, &sout, nullptr) == TERGPU_COMPLETED) {
        e.predicted[i] = sout.device_bytes;
        if (pout.device_bytes > sout.device_bytes) {
          uint64_t& p = plan_of[pre.n];
          p = std::max(p, pout.device_bytes - sout.device_bytes);
        }
      }
    }
    if (st != TERGPU_COMPLETED) {
      refused[i] = st;
    } else if (e.predicted[i] > budget) {
      refused[i] = TERGPU_RESOURCE_LIMIT;
    } else if (in->jobs[i].values_le == nullptr || in->jobs[i].target_le == nullptr ||
               in->jobs[i].attempt_count == 0) {
      refused[i] = TERGPU_INVALID_INPUT;
    } else {
      o->r1 = pout.r1;
      o->r2 = pout.r2;
      o->level3_size = pout.level3_size;
    }
    e.req[i].count = refused[i] >= 0 ? 0 : in->jobs[i].attempt_count;
    e.req[i].unit.assign(e.req[i].count, kPending);
    if (refused[i] < 0) largest = std::max(largest, e.predicted[i]);
  }
  uint64_t reserve = 0;
  for (const auto& kv : plan_of) reserve += kv.second * slots;
  if (reserve != 0 && reserve + largest <= budget) {
    budget -= reserve;
    out->peak_predicted_bytes = reserve;
  } else {
    e.graphs = false;
    reserve = 0;
    for (uint64_t i = 0; i < in->count; ++i) e.reported[i] = e.predicted[i];
  }

  e.t0 = Clock::now();
  std::vector<std::thread> workers;
  workers.reserve(slots);
  for (uint32_t s = 0; s < slots; ++s) workers.emplace_back(worker_main, &e);

  std::vector<uint64_t> open;  // arrived requests with attempts left to start, in arrival order
  size_t next = 0;
  {
    std::unique_lock<std::mutex> lock(e.mu);
    while (e.finished < in->count) {
      const double now = e.now_ms();
      while (next < order.size() &&
             (in->arrival_ms == nullptr || in->arrival_ms[order[next]] <= now)) {
        const uint64_t r = order[next++];
        if (refused[r] >= 0) {
          in->outs[r].status = refused[r];
          in->outs[r].device_bytes = e.reported[r];
          if (in->admit_ms != nullptr) in->admit_ms[r] = now;
          if (in->finish_ms != nullptr) in->finish_ms[r] = now;
          e.req[r].done = true;
          ++e.finished;
          ++out->refused;
        } else {
          open.push_back(r);
        }
      }
      // start attempts: the earliest request first, each request's attempts in order
      for (auto it = open.begin(); it != open.end() && e.running < slots;) {
        Request& q = e.req[*it];
        const uint32_t bound = q.done ? 0u : stop_bound(q);
        while (q.next < bound && e.running < slots &&
               e.inflight_bytes + e.predicted[*it] <= budget) {
          if (!q.admitted) {
            q.admitted = true;
            if (in->admit_ms != nullptr) in->admit_ms[*it] = e.now_ms();
          }
          e.inflight_bytes += e.predicted[*it];
          ++e.running;
          e.ready.push_back(Unit{*it, q.next++});
          out->peak_running = std::max<uint32_t>(out->peak_running, static_cast<uint32_t>(e.running));
          out->peak_predicted_bytes = std::max(out->peak_predicted_bytes, reserve + e.inflight_bytes);
          e.cv_work.notify_one();
        }
        if (q.done || q.next >= stop_bound(q)) {
          it = open.erase(it);  // nothing more to start for this request
        } else {
          ++it;
        }
      }
      if (e.finished >= in->count) break;
      if (next < order.size() && in->arrival_ms != nullptr) {
        const double wait = in->arrival_ms[order[next]] - e.now_ms();
        if (wait > 0) e.cv_done.wait_for(lock, std::chrono::duration<double, std::milli>(wait));
      } else {
        e.cv_done.wait(lock);
      }
    }
    e.stop = true;
  }
  e.cv_work.notify_all();
  for (auto& t : workers) t.join();
  out->total_ms = e.now_ms();
  if (e.worker_error != TERGPU_COMPLETED) {
    t_error = "a batch slot could not create its stream or workspace";
    return e.worker_error;
  }
  return TERGPU_COMPLETED;
}

}  // namespace
}  // namespace tergpu

extern "C" int tergpu_attempt_batch(const tergpu_batch_in* in, tergpu_batch_out* out) {
  using namespace tergpu;
  t_error.clear();
  if (in == nullptr || out == nullptr) {
    t_error = "null argument";
    return TERGPU_INVALID_INPUT;
  }
  try {
    return batch_body(in, out);
  } catch (const Failure& f) {
    return f.status;
  } catch (const std::bad_alloc&) {
    t_error = "host allocation failed";
    return TERGPU_RESOURCE_LIMIT;
  } catch (const std::system_error&) {
    t_error = "could not start the slot threads";
    return TERGPU_DEVICE_ERROR;
  }
}
