// tergpu_attempt_batch: many independent attempt ranges on one device at once
// (include/tergpu.h).
//
// Continuous batching over `slots` concurrent attempt pipelines, each a host
// thread with its own stream and private workspace.  A scheduler admits
// requests in arrival order as a slot frees up and as long as the predicted
// device bytes of the running requests (the preflight of each request) stay
// within the memory budget; a request that has arrived but does not fit waits
// while later, smaller requests that fit go ahead.  Requests whose preflight
// refuses them (InvalidConfiguration, or ResourceLimit against their own
// ceiling or the whole budget) complete at once with that status.  Every
// request runs exactly the code of tergpu_attempt_run, so its result is the
// same alone and in the mix; only the timing differs.

#include "tergpu.h"
#include "tergpu_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <system_error>
#include <thread>
#include <vector>

namespace tergpu {
namespace {

using Clock = std::chrono::steady_clock;

struct Engine {
  const tergpu_batch_in* in = nullptr;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> ready;  // admitted, waiting for a slot thread
  uint64_t running = 0, finished = 0;
  uint64_t inflight_bytes = 0;
  bool stop = false;
  std::vector<uint64_t> predicted;
  int worker_error = TERGPU_COMPLETED;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
};

void worker_main(Engine* e, int slot) {
  (void)slot;
  std::unique_ptr<Workspace> ws;
  try {
    ws = make_workspace(e->in->device, /*blocking=*/true);
  } catch (const Failure& f) {
    std::lock_guard<std::mutex> lock(e->mu);
    e->worker_error = f.status;
  }
  for (;;) {
    uint64_t job = 0;
    {
      std::unique_lock<std::mutex> lock(e->mu);
      e->cv_work.wait(lock, [e] { return e->stop || !e->ready.empty(); });
      if (e->ready.empty()) break;
      job = e->ready.front();
      e->ready.pop_front();
    }
    tergpu_attempt_in req = e->in->jobs[job];
    req.device = e->in->device;
    tergpu_attempt_out* out = &e->in->outs[job];
    int st = TERGPU_DEVICE_ERROR;
    if (ws) {
      try {
        st = attempt_body(&req, out, ws.get());
      } catch (const Failure& f) {
        st = f.status;
      } catch (const std::bad_alloc&) {
        st = TERGPU_RESOURCE_LIMIT;
      }
    }
    out->status = st;
    // the slot's buffers go back to the device pool: each request holds only its
    // own bytes while it runs, so the running requests stay within the budget
    if (ws) release_buffers(*ws);
    {
      std::lock_guard<std::mutex> lock(e->mu);
      if (e->in->finish_ms != nullptr) e->in->finish_ms[job] = e->now_ms();
      e->inflight_bytes -= e->predicted[job];
      --e->running;
      ++e->finished;
    }
    e->cv_done.notify_all();
  }
  if (ws) destroy_workspace(*ws);
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
  std::memset(out, 0, sizeof *out);

  // arrival order (stable by index for equal arrivals)
  std::vector<uint64_t> order(in->count);
  std::iota(order.begin(), order.end(), 0ull);
  if (in->arrival_ms != nullptr) {
    std::stable_sort(order.begin(), order.end(), [in](uint64_t a, uint64_t b) {
      return in->arrival_ms[a] < in->arrival_ms[b];
    });
  }
  // preflight every request (host arithmetic only)
  std::vector<int> refused(in->count, -1);
  for (uint64_t i = 0; i < in->count; ++i) {
    tergpu_attempt_in pre = in->jobs[i];
    pre.flags |= TERGPU_ATTEMPT_PREFLIGHT;
    tergpu_attempt_out pout{};
    const int st = attempt_body(&pre, &pout, nullptr);
    e.predicted[i] = pout.device_bytes;
    if (st != TERGPU_COMPLETED) {
      refused[i] = st;
    } else if (pout.device_bytes > budget) {
      refused[i] = TERGPU_RESOURCE_LIMIT;
    } else if (in->jobs[i].values_le == nullptr || in->jobs[i].target_le == nullptr ||
               in->jobs[i].attempt_count == 0) {
      refused[i] = TERGPU_INVALID_INPUT;
    }
  }

  e.t0 = Clock::now();
  std::vector<std::thread> workers;
  workers.reserve(slots);
  for (uint32_t s = 0; s < slots; ++s) workers.emplace_back(worker_main, &e, static_cast<int>(s));

  std::vector<uint64_t> waiting;  // arrived, not admitted, in arrival order
  size_t next = 0;
  {
    std::unique_lock<std::mutex> lock(e.mu);
    while (e.finished < in->count) {
      const double now = e.now_ms();
      while (next < order.size() &&
             (in->arrival_ms == nullptr || in->arrival_ms[order[next]] <= now)) {
        const uint64_t job = order[next++];
        if (refused[job] >= 0) {
          tergpu_attempt_out* o = &in->outs[job];
          tergpu_attempt_stats* keep = o->stats;
          std::memset(o, 0, sizeof *o);
          o->stats = keep;
          o->status = refused[job];
          o->device_bytes = e.predicted[job];
          if (in->admit_ms != nullptr) in->admit_ms[job] = now;
          if (in->finish_ms != nullptr) in->finish_ms[job] = now;
          ++e.finished;
          ++out->refused;
        } else {
          waiting.push_back(job);
        }
      }
      // admit whatever fits, in arrival order
      for (auto it = waiting.begin(); it != waiting.end();) {
        if (e.running >= slots) break;
        if (e.inflight_bytes + e.predicted[*it] > budget) {
          ++it;
          continue;
        }
        e.inflight_bytes += e.predicted[*it];
        ++e.running;
        if (in->admit_ms != nullptr) in->admit_ms[*it] = e.now_ms();
        e.ready.push_back(*it);
        it = waiting.erase(it);
        out->peak_running = std::max<uint32_t>(out->peak_running, static_cast<uint32_t>(e.running));
        out->peak_predicted_bytes = std::max(out->peak_predicted_bytes, e.inflight_bytes);
        e.cv_work.notify_one();
      }
      if (e.finished >= in->count) break;
      if (next < order.size() && in->arrival_ms != nullptr) {
        const double wait = in->arrival_ms[order[next]] - e.now_ms();
        if (wait > 0) {
          e.cv_done.wait_for(lock, std::chrono::duration<double, std::milli>(wait));
        }
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
