// C ABI of the B200 root backend (include/tergpu.h).
//
// One workspace per device, grown on demand and reused across calls; calls on
// the same device are serialized by that workspace's mutex.  Every call checks
// its predicted device bytes against the caller's ceiling before it allocates
// anything, so a refused call returns TERGPU_RESOURCE_LIMIT with no partial
// result (the reference's ResourceLimit contract, src/full_ter.cpp:3174-3185).

#include "tergpu.h"
#include "root_kernels.cuh"
#include "tergpu_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

namespace tergpu {

thread_local std::string t_error;

enum Slot {
  kSlotKeyLo = 0, kSlotKeyHi = 3, kSlotInId = 6, kSlotRes = 9, kSlotHi = 12, kSlotId = 15,
  kSlotCnt = 18, kSlotOff = 21, kSlotCur = 24, kSlotCells = 27, kSlotTriples = 28,
  kSlotCounters = 29, kSlotRecords = 30, kSlotFlags = 33, kSlotQWin = 34, kSlotRes4 = 35,
  kSlotHi4 = 36, kSlotId4 = 37, kSlotWin4 = 38, kSlotCnt4 = 39, kSlotOff4 = 40, kSlotCur4 = 41,
  kSlotStageKey = 42, kSlotStageHi = 43, kSlotStageId = 44, kSlotStageTab = 45, kSlots = 46
};

std::mutex g_mu;
std::vector<std::unique_ptr<Workspace>> g_ws;

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    t_error = std::string(what) + ": " + cudaGetErrorString(e);
    throw Failure{e == cudaErrorMemoryAllocation ? TERGPU_RESOURCE_LIMIT : TERGPU_DEVICE_ERROR};
  }
}

Workspace& workspace(int device) {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto& w : g_ws) {
    if (w->device == device) return *w;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    t_error = "no CUDA device " + std::to_string(device);
    throw Failure{TERGPU_DEVICE_ERROR};
  }
  g_ws.push_back(make_workspace(device));
  return *g_ws.back();
}

// Loading the library asks the CUDA context this process will create for 32
// hardware work queues (CUDA_DEVICE_MAX_CONNECTIONS; CUDA's default is 8 and it
// maps streams onto them in order): the batch engine runs two streams per slot,
// and with fewer queues than streams a short request's kernel waits behind an
// n = 108 sweep queued earlier on another slot's stream.  A value the caller set
// is kept; a context created before the library is loaded keeps its own count.
__attribute__((constructor)) void ask_for_work_queues() {
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
}

std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

// The library's stream-ordered memory pool of `device`, created on first use.
// It keeps freed memory instead of returning it at every synchronization
// (workspaces grow and shrink across calls), and it never reuses a block whose
// free is still pending on another stream by making the allocating stream wait
// for that stream: with the default pool's internal dependencies, a short
// request's allocation could wait for a whole n = 108 sweep launched on another
// slot's stream.  Such a block stays unused until its free has completed.
cudaMemPool_t library_pool(int device) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  auto it = g_pools.find(device);
  if (it != g_pools.end()) return it->second;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
  uint64_t keep = ~0ull;
  check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
  int off = 0;
  check(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &off),
        "cudaMemPoolSetAttribute");
  g_pools[device] = pool;
  return pool;
}

void trim_library_pools() {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  for (auto& kv : g_pools) cudaMemPoolTrimTo(kv.second, 0);
}

std::unique_ptr<Workspace> make_workspace(int device, bool blocking) {
  auto w = std::make_unique<Workspace>();
  w->device = device;
  check(cudaSetDevice(device), "cudaSetDevice");
  w->pool = library_pool(device);
  if (blocking) {
    // batch slots: small requests' work ahead of background (n >= 108) attempts
    int least = 0, greatest = 0;
    check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
    check(cudaStreamCreateWithPriority(&w->stream, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
    check(cudaStreamCreateWithPriority(&w->stream_low, cudaStreamNonBlocking, least), "cudaStreamCreate");
  } else {
    check(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  }
  check(cudaEventCreate(&w->start), "cudaEventCreate");
  check(cudaEventCreate(&w->mid), "cudaEventCreate");
  check(cudaEventCreate(&w->stop), "cudaEventCreate");
  if (blocking) {
    check(cudaEventCreateWithFlags(&w->sync_event, cudaEventBlockingSync | cudaEventDisableTiming),
          "cudaEventCreate");
  }
  return w;
}

void cancel_word(Workspace& w) {
  if (w.cancel_host == nullptr) {
    void* h = nullptr;
    check(cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable), "cudaHostAlloc");
    void* d = nullptr;
    check(cudaHostGetDevicePointer(&d, h, 0), "cudaHostGetDevicePointer");
    w.cancel_host = static_cast<volatile int*>(h);
    w.cancel_dev = static_cast<const volatile int*>(d);
  }
  *w.cancel_host = 0;
}

void sync_stream(Workspace& w, cudaStream_t st, const char* what) {
  if (w.sync_event != nullptr) {
    check(cudaEventRecord(w.sync_event, st), what);
    check(cudaEventSynchronize(w.sync_event), what);
  } else {
    check(cudaStreamSynchronize(st), what);
  }
}

void release_buffers(Workspace& w) {
  cudaSetDevice(w.device);
  for (auto& kv : w.buf) {
    if (kv.second.ptr != nullptr) cudaFreeAsync(kv.second.ptr, w.stream);
  }
  w.buf.clear();
}

void destroy_workspace(Workspace& w) {
  release_buffers(w);
  if (w.stream) cudaStreamSynchronize(w.stream);
  w.plans.clear();
  if (w.start) cudaEventDestroy(w.start);
  if (w.mid) cudaEventDestroy(w.mid);
  if (w.stop) cudaEventDestroy(w.stop);
  if (w.sync_event) cudaEventDestroy(w.sync_event);
  if (w.stream) cudaStreamDestroy(w.stream);
  if (w.stream_low) {
    cudaStreamSynchronize(w.stream_low);
    cudaStreamDestroy(w.stream_low);
  }
  w.stream_low = nullptr;
  if (w.cancel_host) cudaFreeHost(const_cast<int*>(w.cancel_host));
  w.cancel_host = nullptr;
  w.cancel_dev = nullptr;
  w.start = w.mid = w.stop = w.sync_event = nullptr;
  w.stream = nullptr;
}

void* ensure_bytes(Workspace& w, int slot, size_t bytes) {
  bytes = std::max<size_t>(bytes, 256);
  Buffer& b = w.buf[slot];
  if (b.bytes < bytes) {
    cudaStream_t s = w.alloc_stream != nullptr ? w.alloc_stream : w.stream;
    if (b.ptr != nullptr) check(cudaFreeAsync(b.ptr, s), "cudaFreeAsync");
    b.ptr = nullptr;
    b.bytes = 0;
    check(cudaMallocFromPoolAsync(&b.ptr, bytes, w.pool, s), "cudaMallocFromPoolAsync");
    b.bytes = bytes;
  }
  return b.ptr;
}

uint32_t ceil_log2(uint64_t v) {
  uint32_t b = 0;
  while ((1ull << b) < v) ++b;
  return b;
}

// v1: about 1024 D entries per family and about 256 filter bits per D entry.
// v2: about 2048 D entries per family; the filter has about 8x as many words as
// a B family has entries (measured best at n=108: 19 filter bits, false-pass
// rate |D_u| / 2^(wb+5) ~ 0.3 %); narrower filters make the probes of 32
// consecutive sorted B entries nearly conflict-free but pass too many pairs.
// v3 (bank-free probes, one CTA per SM): 16x as many words (20 filter bits at
// n=108, false-pass rate ~ 0.16 %).
Tuning choose_tuning(uint64_t n_x, uint64_t n_d, uint32_t fast_bits, uint32_t projected,
                     uint32_t fb_req, uint32_t filter_req, uint32_t variant, uint32_t shards,
                     uint64_t n_q, uint32_t block_log2) {
  Tuning t;
  t.variant = variant == 0 ? 3u : variant;
  const bool v2 = t.variant != 1;
  uint32_t fb_max = std::min<uint32_t>(14, fast_bits - 2);
  if (projected != 0) fb_max = std::min<uint32_t>(fb_max, projected - 6);
  if (fb_req != 0) {
    t.fb = fb_req;
  } else if (t.variant == 4) {
    // v4: about 256 D entries per family (a table survivor rate of about
    // 2 |D_u| / 2^14, B families of a few rows of 32)
    const double ideal = std::log2(std::max<double>(1.0, static_cast<double>(n_d) / 256.0));
    t.fb = static_cast<uint32_t>(std::max(6.0, std::floor(ideal + 0.5)));
    t.fb = std::min<uint32_t>(t.fb, std::min<uint32_t>(16, fast_bits > 34 ? fast_bits - 32 : 6));
    if (projected != 0) t.fb = std::min(t.fb, fb_max);
    t.fb = std::max<uint32_t>(t.fb, 6);
  } else {
    const double per = v2 ? 2048.0 : 1024.0;
    const double ideal = std::log2(std::max<double>(1.0, static_cast<double>(n_d) / per));
    t.fb = static_cast<uint32_t>(std::max(6.0, std::floor(ideal + 0.5)));
    if (t.variant == 3 && n_d >= (128u << 7)) {
      // small roots (the n = 72 root, 3.6e4 targets): 128 families of ~280
      // entries keep 24 warps per CTA busy (measured 0.33 ms against 0.44 ms
      // with 64 families)
      t.fb = std::max<uint32_t>(t.fb, 7);
    }
    t.fb = std::min(t.fb, fb_max);
    t.fb = std::max<uint32_t>(t.fb, 6);
  }
  const uint64_t avg_d = std::max<uint64_t>(1, n_d >> t.fb);
  const uint64_t avg_x = std::max<uint64_t>(1, n_x >> t.fb);
  if (filter_req != 0) {
    t.wb = filter_req - 5;
  } else if (t.variant == 3 || t.variant == 4) {
    t.wb = 15;  // v3: the widest filter the 24-warp CTA holds (best measured at n = 72 and 108)
  } else if (v2) {
    t.wb = std::clamp<uint32_t>(ceil_log2(avg_x) + 3, 6, 14);
  } else {
    t.wb = std::clamp<uint32_t>(ceil_log2(avg_d * 256) - 5, 10, 14);
  }
  t.sort_bits = std::min<uint32_t>(t.wb, 12);
  const uint32_t nfam = 1u << t.fb;
  const uint32_t nloc = std::max<uint32_t>(1, nfam / shards);  // target families per shard
  const bool one_cta = t.variant == 3 || t.variant == 4;     // one CTA of 24 warps per SM
  uint64_t target_ctas = 148 * (one_cta ? 1 : 2) * 8;          // about 8 waves of resident CTAs
  if (n_q != 0) {
    const double pairs = static_cast<double>(n_q) * static_cast<double>(n_x) / shards;
    target_ctas = std::min<uint64_t>(target_ctas, static_cast<uint64_t>(pairs / (1u << 20)) + 1);
    // very large joins: blocks of about 2^block_log2 pairs, so SMs come free
    // often for work of higher priority on the device (a block's filter build
    // is microseconds)
    target_ctas = std::max<uint64_t>(target_ctas, static_cast<uint64_t>(pairs / std::ldexp(1.0, block_log2)));
  }
  t.s_split = static_cast<uint32_t>(std::clamp<uint64_t>((target_ctas + nloc - 1) / nloc, 1, nfam));
  // every CTA gets at least about 8 work items (A family x chunk of 256 B entries)
  // per warp: with fewer, warps idle at the end of the CTA (the n = 72 root with
  // 128 families of ~144 B entries had 26 items for 24 warps: half the SM time
  // idle; 8 per warp measured 5 % more batched n = 72 attempts per second than 4)
  const uint64_t chunks = (avg_x + 255) / 256;
  const uint64_t warps = one_cta ? kSweep3Warps : kSweepWarps;
  const uint64_t most = std::max<uint64_t>(1, nfam * chunks / (8 * warps));
  t.s_split = static_cast<uint32_t>(std::min<uint64_t>(t.s_split, most));
  return t;
}

// Slots of the staged scatter's temp copy: the longest list that takes it (0: none).
uint64_t staged_slots(const uint64_t count[3], uint32_t fb) {
  uint64_t m = 0;
  for (int l = 0; l < 3; ++l) {
    if (staged_partition(Count(count[l]), fb)) m = std::max<uint64_t>(m, count[l] + (1ull << fb) + 16);
  }
  return m;
}

uint64_t partition_bytes(const uint64_t count[3], uint32_t fb, uint32_t variant, bool one_pass) {
  uint64_t b = 0;
  for (int l = 0; l < 3; ++l) {
    const uint64_t slots = count[l] + (1ull << fb) + 16;
    b += slots * (8 + 1 + 4);
    b += 3ull * ((1ull << fb) + 1) * 4;
  }
  if (variant == 4) {  // A windows, the B lane-slot layout with its windows and tables
    b += (count[0] + (1ull << fb) + 16) * 4;
    b += v4_slots(count[1], fb) * (8 + 1 + 4 + 4);
    b += 3ull * ((1ull << fb) + 1) * 4;
  }
  const uint64_t staged = one_pass ? 0 : staged_slots(count, fb);
  if (staged != 0) b += staged * (8 + 1 + 4) + staged_table_words(fb) * 4ull;
  return b;
}

bool autotune_requested(uint32_t flags) { return (flags & TERGPU_ROOT_AUTOTUNE) != 0; }

// 0: the default (variant 3, or the autotuner's pick), 1 or 2 when a flag forces one.
uint32_t sweep_variant(uint32_t flags) {
  if ((flags & TERGPU_ROOT_SWEEP_V1) != 0) return 1;
  if ((flags & TERGPU_ROOT_SWEEP_V2) != 0) return 2;
  if ((flags & TERGPU_ROOT_SWEEP_V4) != 0) return 4;
  return 0;
}

uint32_t checked_shards(uint32_t index, uint32_t count) {
  const uint32_t n = count == 0 ? 1u : count;
  if (n > 64 || (n & (n - 1)) != 0 || index >= n) {
    t_error = "shard_count must be 0 or a power of two <= 64, and shard_index below it";
    throw Failure{TERGPU_INVALID_INPUT};
  }
  return n;
}

uint32_t enqueue_join(const JoinBuffers& b, const JoinWork& j, const Tuning& tu, cudaEvent_t mid,
                      cudaStream_t st, uint32_t* launches) {
  const uint32_t Q = j.quotient_bits;
  const uint32_t F = std::min<uint32_t>(Q, 64);
  const uint32_t hi_bits = Q - F;
  const uint32_t nfam = 1u << tu.fb;
  const uint64_t fast_mask = F >= 64 ? ~0ull : ((1ull << F) - 1ull);
  ListView views[3];
  check(cudaMemsetAsync(b.counters, 0, kCounters * 8, st), "memset");
  for (int l = 0; l < 3; ++l) {
    check(cudaMemsetAsync(b.cnt[l], 0, nfam * 4ull, st), "memset");
    launch_hist(j.key_lo[l], j.count[l], nfam - 1, b.cnt[l], st);
    const uint32_t hi_mask = hi_bits ? ((1u << hi_bits) - 1u) : 0u;
    if (b.stage.key != nullptr && staged_partition(j.count[l], tu.fb)) {
      launch_scan_staged(b.cnt[l], nfam, b.off[l], b.cur[l], tu.fb, b.stage.table, st);
      *launches += launch_scatter_staged(j.key_lo[l], j.key_hi[l], j.id[l], j.count[l], tu.fb, fast_mask,
                                         hi_mask, b.cur[l], b.stage, b.res[l], b.hi[l], b.id[l], st);
    } else {
      launch_scan(b.cnt[l], nfam, b.off[l], b.cur[l], st);
      launch_scatter(j.key_lo[l], j.key_hi[l], j.id[l], j.count[l], tu.fb, fast_mask, hi_mask, b.cur[l],
                     b.res[l], b.hi[l], b.id[l], st);
      *launches += j.count[l].cap != 0 ? 1 : 0;
    }
    views[l] = ListView{b.res[l], b.hi[l], b.id[l], b.off[l], b.cnt[l]};
    *launches += (j.count[l].cap != 0 ? 1 : 0) + 1;
  }
  launch_max_family(b.cnt[0], nfam, b.counters, kMaxQ, st);
  launch_max_family(b.cnt[1], nfam, b.counters, kMaxX, st);
  *launches += 2;
  // v3 and v4 need full 32-bit windows (mrb >= 32); below that the
  // B-in-registers sweep (v2) runs, exact for any family order.
  uint32_t main_variant = (tu.variant == 3 || tu.variant == 4) && F - tu.fb < 32 ? 2u : tu.variant;
  if (main_variant == 4 && b.res4 == nullptr) main_variant = 3;
  ListView x4view{};
  if (main_variant == 4) {
    // A probe windows; the B list in lane slots, one bank per lane
    launch_window4(b.res[0], Count(j.count[0].cap + nfam + 16), b.qwin, st);
    launch_rows4(b.res[1], b.off[1], b.cnt[1], nfam, b.cnt4, st);
    launch_scan(b.cnt4, nfam, b.off4, b.cur4, st);
    launch_arrange4(b.res[1], b.hi[1], b.id[1], b.off[1], b.cnt[1], b.off4, b.cnt4, nfam, b.res4, b.hi4,
                    b.id4, b.win4, st);
    launch_max_family(b.cnt4, nfam, b.counters, kMaxX, st);
    *launches += 5;
    x4view = ListView{b.res4, b.hi4, b.id4, b.off4, b.cnt4, b.win4};
  } else if (main_variant == 3 && j.count[1].cap != 0) {
    // B families in lane slots of distinct residual classes mod 32 (bank-free probes)
    launch_family_arrange(b.res[1], b.hi[1], b.id[1], b.off[1], b.cnt[1], nfam, j.count[1].cap >> tu.fb, st);
    *launches += 1;
  } else if (main_variant == 2 && j.count[1].cap != 0) {
    // B families sorted by the top filter-word bits of the full-width window
    launch_family_sort(b.res[1], b.hi[1], b.id[1], b.off[1], b.cnt[1], nfam, F - tu.fb, tu.sort_bits, st);
    *launches += 1;
  }
  auto sweep = [&](const SweepArgs& sa) {
    if (main_variant == 4 && sa.mrb >= 32 && sa.project == 0) {
      SweepArgs a4 = sa;
      a4.q.win = b.qwin;
      a4.x = x4view;
      launch_sweep4(a4, st);
    } else if (main_variant == 3 && sa.mrb >= 32) {
      launch_sweep3(sa, st);
    } else if (main_variant == 1) {
      launch_sweep(sa, sa.mrb < 32, st);
    } else {
      launch_sweep2(sa, sa.mrb < 32, st);
    }
  };
  check(cudaGetLastError(), "partition launch");
  if (mid != nullptr) check(cudaEventRecord(mid, st), "event");
  SweepArgs a{};
  a.q = views[0];
  a.x = views[1];
  a.y = views[2];
  a.cells = j.cells;
  a.fb = tu.fb;
  a.s_split = tu.s_split;
  a.shard = j.shard;
  a.shards = j.shards;
  a.wb = tu.wb;
  a.rb = F - tu.fb;
  a.hi_bits = hi_bits;
  a.triples = b.triples;
  a.cap = j.cap;
  a.counters = b.counters;
  a.cancel = j.cancel;
  if (j.main_sweep) {
    a.project = 0;
    a.mrb = F - tu.fb;
    sweep(a);
    *launches += 1;
  }
  if (j.projected_bits != 0) {
    a.project = 1;
    a.visit = j.visit;
    a.mrb = j.projected_bits - tu.fb;
    sweep(a);
    *launches += 1;
  }
  return main_variant;
}

// ---- autotuner: per root shape, the fastest (family bits, filter bits, sweep
// variant) among the neighbours of the size-based choice, timed as device time
// (partition + sweep) on one 64th of the root's target families (shard 0 of
// 64: all of A and B against 1/64 of D); cached for the life of the process.
// Replaces the reference's CPU probe dispatcher (ter2_root/frozen/ter_arwlf.cpp:612-747)
// on the device side.  The choice changes only the time, never a result.
struct ShapeKey {
  uint32_t q, la, lb, ld, proj;
  bool operator<(const ShapeKey& o) const {
    return std::tie(q, la, lb, ld, proj) < std::tie(o.q, o.la, o.lb, o.ld, o.proj);
  }
};
struct Tuned {
  uint32_t fb = 0, filter_bits = 0, variant = 0;
};
std::mutex g_tune_mu;
std::map<ShapeKey, Tuned> g_tuned;

uint32_t size_bucket(uint64_t n) {
  return n == 0 ? 0u : static_cast<uint32_t>(std::lround(4.0 * std::log2(static_cast<double>(n))));
}

Tuned autotune(Workspace& w, const JoinInput& in, uint64_t input_bytes, float* spent_ms) {
  const uint32_t F = std::min<uint32_t>(in.quotient_bits, 64);
  // neighbours of each variant's own size-based choice
  (void)0;
  Tuned best;
  float best_ms = 0;
  *spent_ms = 0;
  for (uint32_t variant : {3u, 2u}) {
    for (int dfb = -1; dfb <= 1; ++dfb) {
      for (int dfl = -1; dfl <= 1; ++dfl) {
        JoinInput j = in;
        j.autotune = false;
        j.count_only = true;
        j.capacity = 0;
        j.projected_bits = 0;
        j.shard = 0;
        j.shards = 64;
        const Tuning base = choose_tuning(in.count[1], in.count[2], F, 0, 0, 0, variant, 1, in.count[0]);
        if (variant == 4 && dfl != 0) continue;  // v4's table has no width to tune
        j.family_bits = static_cast<uint32_t>(static_cast<int>(base.fb) + dfb);
        j.filter_bits = static_cast<uint32_t>(static_cast<int>(base.wb) + 5 + dfl);
        j.sweep_variant = variant;
        if (j.family_bits < 6 || j.family_bits + 2 > F || j.filter_bits < 10 || j.filter_bits > 20) continue;
        try {
          const JoinResult r = run_join(w, j, input_bytes);
          const float ms = r.partition_ms + r.sweep_ms;
          *spent_ms += r.join_ms;
          if (best.fb == 0 || ms < best_ms) {
            best_ms = ms;
            best = Tuned{j.family_bits, j.filter_bits, variant};
          }
        } catch (const Failure&) {
          t_error.clear();  // a candidate outside the supported range: skip it
        }
      }
    }
  }
  return best;
}

// Partition + sweep(s) on keys already on the device.  The only host
// synchronization is the final download of counters and family sizes.
JoinResult run_join(Workspace& w, const JoinInput& in, uint64_t input_bytes) {
  if (in.autotune && in.family_bits == 0 && in.filter_bits == 0 && in.sweep_variant == 0 &&
      in.count[0] != 0 && in.count[1] != 0 && in.count[2] != 0) {
    const ShapeKey key{in.quotient_bits, size_bucket(in.count[0]), size_bucket(in.count[1]),
                       size_bucket(in.count[2]), in.projected_bits};
    Tuned t;
    float spent = 0;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) t = it->second;
    }
    if (t.fb == 0) {
      t = autotune(w, in, input_bytes, &spent);
      std::lock_guard<std::mutex> lock(g_tune_mu);
      if (t.fb != 0) g_tuned[key] = t;
    }
    JoinInput j = in;
    j.autotune = false;
    if (t.fb != 0) {
      j.family_bits = t.fb;
      j.filter_bits = t.filter_bits;
      j.sweep_variant = t.variant;
    }
    JoinResult r = run_join(w, j, input_bytes);
    r.tune_ms = spent;
    return r;
  }
  JoinResult r;
  const uint32_t Q = in.quotient_bits;
  const uint32_t F = std::min<uint32_t>(Q, 64);
  r.tuning = choose_tuning(in.count[1], in.count[2], F, in.projected_bits, in.family_bits,
                           in.filter_bits, in.sweep_variant, in.shards, in.count[0],
                           in.background ? kBackgroundBlockLog2 : kJoinBlockLog2);
  const Tuning& tu = r.tuning;
  checked_shards(in.shard, in.shards);
  if (tu.fb < 6 || tu.fb > 16 || tu.fb + 2 > F || tu.wb < 5 || tu.wb > 15 ||
      (in.projected_bits != 0 && (in.projected_bits > F || in.projected_bits < tu.fb + 1))) {
    t_error = "family/filter bits outside the supported range for this quotient width";
    throw Failure{TERGPU_INVALID_INPUT};
  }
  const uint32_t nfam = 1u << tu.fb;
  const uint64_t need = input_bytes + partition_bytes(in.count, tu.fb, tu.variant, in.one_pass) +
                        (in.count_only ? 0 : in.capacity * 12) + 4096 + 64;
  r.device_bytes = need;
  if (in.memory_limit_bytes != 0 && need > in.memory_limit_bytes) {
    t_error = "predicted device bytes " + std::to_string(need) + " exceed the ceiling " +
              std::to_string(in.memory_limit_bytes);
    throw Failure{TERGPU_RESOURCE_LIMIT};
  }
  cudaStream_t st = in.stream;
  uint64_t* res[3];
  uint8_t* hi[3];
  uint32_t* ids[3];
  uint32_t *cnt[3], *off[3], *cur[3];
  for (int l = 0; l < 3; ++l) {
    const uint64_t slots = in.count[l] + nfam + 16;
    res[l] = ensure<uint64_t>(w, kSlotRes + l, slots * 8);
    hi[l] = ensure<uint8_t>(w, kSlotHi + l, slots);
    ids[l] = ensure<uint32_t>(w, kSlotId + l, slots * 4);
    cnt[l] = ensure<uint32_t>(w, kSlotCnt + l, (nfam + 1) * 4ull);
    off[l] = ensure<uint32_t>(w, kSlotOff + l, (nfam + 1) * 4ull);
    cur[l] = ensure<uint32_t>(w, kSlotCur + l, (nfam + 1) * 4ull);
  }
  unsigned long long* counters = ensure<unsigned long long>(w, kSlotCounters, kCounters * 8);
  uint32_t* d_triples = ensure<uint32_t>(w, kSlotTriples, std::max<uint64_t>(in.capacity, 1) * 12);
  JoinBuffers jb{};
  if (tu.variant == 4 && F - tu.fb >= 32 && (!in.count_only || in.projected_bits == 0)) {
    const uint64_t s4 = v4_slots(in.count[1], tu.fb);
    jb.qwin = ensure<uint32_t>(w, kSlotQWin, (in.count[0] + nfam + 16) * 4);
    jb.res4 = ensure<uint64_t>(w, kSlotRes4, s4 * 8);
    jb.hi4 = ensure<uint8_t>(w, kSlotHi4, s4);
    jb.id4 = ensure<uint32_t>(w, kSlotId4, s4 * 4);
    jb.win4 = ensure<uint32_t>(w, kSlotWin4, s4 * 4);
    jb.cnt4 = ensure<uint32_t>(w, kSlotCnt4, (nfam + 1) * 4ull);
    jb.off4 = ensure<uint32_t>(w, kSlotOff4, (nfam + 1) * 4ull);
    jb.cur4 = ensure<uint32_t>(w, kSlotCur4, (nfam + 1) * 4ull);
  }
  const uint64_t staged = in.one_pass ? 0 : staged_slots(in.count, tu.fb);
  if (staged != 0) {
    jb.stage.key = ensure<uint64_t>(w, kSlotStageKey, staged * 8);
    jb.stage.hi = ensure<uint8_t>(w, kSlotStageHi, staged);
    jb.stage.id = ensure<uint32_t>(w, kSlotStageId, staged * 4);
    jb.stage.table = ensure<uint32_t>(w, kSlotStageTab, staged_table_words(tu.fb) * 4ull);
  }
  const uint8_t* d_cells = in.cells_device;
  if (d_cells == nullptr && in.cells != nullptr) {
    uint8_t* c = ensure<uint8_t>(w, kSlotCells, 4096);
    check(cudaMemcpyAsync(c, in.cells, 4096, cudaMemcpyHostToDevice, st), "cells upload");
    d_cells = c;
  }
  check(cudaEventRecord(w.start, st), "event");
  for (int l = 0; l < 3; ++l) {
    jb.res[l] = res[l];
    jb.hi[l] = hi[l];
    jb.id[l] = ids[l];
    jb.cnt[l] = cnt[l];
    jb.off[l] = off[l];
    jb.cur[l] = cur[l];
  }
  jb.counters = counters;
  jb.triples = d_triples;
  JoinWork jw{};
  for (int l = 0; l < 3; ++l) {
    jw.key_lo[l] = in.key_lo[l];
    jw.key_hi[l] = in.key_hi[l];
    jw.id[l] = in.id[l];
    jw.count[l] = Count(in.count[l]);
  }
  jw.quotient_bits = Q;
  jw.cells = d_cells;
  jw.shard = in.shard;
  jw.shards = in.shards;
  jw.cap = in.count_only ? 0 : in.capacity;
  jw.main_sweep = !in.count_only || in.projected_bits == 0;
  jw.projected_bits = in.projected_bits;
  jw.visit = in.visit;
  jw.cancel = in.cancel;
  r.tuning.variant = enqueue_join(jb, jw, tu, w.mid, st, &r.launches);
  check(cudaGetLastError(), "sweep launch");
  check(cudaEventRecord(w.stop, st), "event");
  unsigned long long hc[kCounters];
  std::vector<uint32_t> hcnt[2];
  check(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, st), "counters");
  for (int l = 0; l < 2; ++l) {
    hcnt[l].resize(nfam);
    check(cudaMemcpyAsync(hcnt[l].data(), cnt[l], nfam * 4ull, cudaMemcpyDeviceToHost, st),
          "count download");
  }
  sync_stream(w, st, "join");
  check(cudaEventElapsedTime(&r.join_ms, w.start, w.stop), "elapsed");
  check(cudaEventElapsedTime(&r.partition_ms, w.start, w.mid), "elapsed");
  check(cudaEventElapsedTime(&r.sweep_ms, w.mid, w.stop), "elapsed");
  std::vector<uint8_t> hcells;
  if (d_cells != nullptr) {
    hcells.resize(4096);
    if (in.cells != nullptr) {
      std::memcpy(hcells.data(), in.cells, 4096);
    } else {
      check(cudaMemcpyAsync(hcells.data(), d_cells, 4096, cudaMemcpyDeviceToHost, st), "cells download");
      sync_stream(w, st, "cells download");
    }
  }
  // B sizes by t mod 64: the cell mask and the shard (shards | 64) see only that
  const uint32_t cls = std::min<uint32_t>(nfam, 64);
  uint64_t bsum[64] = {};
  for (uint32_t t = 0; t < nfam; ++t) bsum[t & (cls - 1u)] += hcnt[1][t];
  for (uint32_t s = 0; s < nfam; ++s) {
    uint64_t b = 0;
    for (uint32_t c = 0; c < cls; ++c) {
      if (((s + c) & (nfam - 1u) & (in.shards - 1u)) != in.shard) continue;
      if (!hcells.empty() && hcells[((s & 63u) << 6) | c] == 0) continue;
      b += bsum[c];
    }
    r.pairs += static_cast<uint64_t>(hcnt[0][s]) * b;
  }
  r.triples = hc[kTriples];
  r.survivors = hc[kSurvivors];
  r.fast = hc[kFast];
  r.projected = hc[kProjected];
  r.d_triples = d_triples;
  return r;
}

void fill_out(const JoinResult& j, tergpu_root_out* out) {
  out->triples_count = j.triples;
  out->logical_pairs = j.pairs;
  out->filter_survivors = j.survivors;
  out->fast_hits = j.fast;
  out->projected_hits = j.projected;
  out->device_bytes = j.device_bytes;
  out->join_ms = j.join_ms;
  out->partition_ms = j.partition_ms;
  out->sweep_ms = j.sweep_ms;
  out->family_bits = j.tuning.fb;
  out->filter_bits = j.tuning.wb + 5;
  out->kernel_launches = j.launches;
  out->sweep_variant = j.tuning.variant;
  out->tune_ms = j.tune_ms;
}

int guarded(const char* what, int (*body)(const void*, void*), const void* in, void* out) {
  (void)what;
  t_error.clear();
  try {
    return body(in, out);
  } catch (const Failure& f) {
    return f.status;
  } catch (const std::bad_alloc&) {
    t_error = "host allocation failed";
    return TERGPU_RESOURCE_LIMIT;
  } catch (...) {
    t_error = "unexpected exception";
    return TERGPU_DEVICE_ERROR;
  }
}

int root_run_body(const void* vin, void* vout) {
  const auto* in = static_cast<const tergpu_root_in*>(vin);
  auto* out = static_cast<tergpu_root_out*>(vout);
  const auto t0 = std::chrono::steady_clock::now();
  if (in == nullptr || out == nullptr) {
    t_error = "null argument";
    return TERGPU_INVALID_INPUT;
  }
  const uint32_t Q = in->quotient_bits;
  if (Q < 8 || Q > TERGPU_MAX_QUOTIENT_BITS) {
    t_error = "quotient width outside [8, 72]";
    return TERGPU_UNSUPPORTED_WIDTH;
  }
  const bool count_only = (in->flags & TERGPU_ROOT_COUNT_ONLY) != 0;
  const bool resident = (in->flags & TERGPU_ROOT_DEVICE_INPUTS) != 0;
  for (int l = 0; l < 3; ++l) {
    if (in->count[l] >= 0x80000000ull || (in->count[l] != 0 && in->key_lo[l] == nullptr) ||
        (Q > 64 && in->count[l] != 0 && in->key_hi[l] == nullptr)) {
      t_error = "list pointers or sizes invalid";
      return TERGPU_INVALID_INPUT;
    }
  }
  if (!count_only && out->capacity != 0 && out->triples == nullptr) {
    t_error = "triples buffer missing";
    return TERGPU_INVALID_INPUT;
  }
  Workspace& w = workspace(in->device);
  std::lock_guard<std::mutex> lock(w.mu);
  check(cudaSetDevice(w.device), "cudaSetDevice");
  cudaStream_t st = in->stream != nullptr ? static_cast<cudaStream_t>(in->stream) : w.stream;
  w.alloc_stream = st;
  uint64_t input_bytes = 0;
  if (!resident) {
    for (int l = 0; l < 3; ++l) input_bytes += in->count[l] * 13 + 64;
  }
  if (in->memory_limit_bytes != 0 && input_bytes > in->memory_limit_bytes) {
    t_error = "input keys alone exceed the device ceiling";
    return TERGPU_RESOURCE_LIMIT;
  }
  JoinInput j{};
  j.quotient_bits = Q;
  j.stream = st;
  for (int l = 0; l < 3; ++l) {
    j.count[l] = in->count[l];
    if (resident) {
      j.key_lo[l] = in->key_lo[l];
      j.key_hi[l] = Q > 64 ? in->key_hi[l] : nullptr;
      j.id[l] = in->id[l];
      continue;
    }
    uint64_t* dlo = ensure<uint64_t>(w, kSlotKeyLo + l, in->count[l] * 8 + 8);
    if (in->count[l]) {
      check(cudaMemcpyAsync(dlo, in->key_lo[l], in->count[l] * 8, cudaMemcpyHostToDevice, st),
            "key upload");
    }
    j.key_lo[l] = dlo;
    j.key_hi[l] = nullptr;
    if (Q > 64) {
      uint8_t* dhi = ensure<uint8_t>(w, kSlotKeyHi + l, in->count[l] + 8);
      if (in->count[l]) {
        check(cudaMemcpyAsync(dhi, in->key_hi[l], in->count[l], cudaMemcpyHostToDevice, st),
              "key upload");
      }
      j.key_hi[l] = dhi;
    }
    j.id[l] = nullptr;
    if (in->id[l] != nullptr) {
      uint32_t* did = ensure<uint32_t>(w, kSlotInId + l, in->count[l] * 4 + 8);
      if (in->count[l]) {
        check(cudaMemcpyAsync(did, in->id[l], in->count[l] * 4, cudaMemcpyHostToDevice, st),
              "id upload");
      }
      j.id[l] = did;
    }
  }
  j.cells = resident ? nullptr : in->cells;
  j.cells_device = resident ? in->cells : nullptr;
  j.projected_bits = in->projected_bits;
  j.family_bits = in->family_bits;
  j.filter_bits = in->filter_bits;
  j.memory_limit_bytes = in->memory_limit_bytes;
  j.capacity = count_only ? 0 : out->capacity;
  j.count_only = count_only;
  j.sweep_variant = sweep_variant(in->flags);
  j.autotune = autotune_requested(in->flags) && j.sweep_variant == 0;
  j.one_pass = (in->flags & TERGPU_ROOT_PARTITION_ONE_PASS) != 0;
  j.shard = in->shard_index;
  j.shards = checked_shards(in->shard_index, in->shard_count);
  const JoinResult res = run_join(w, j, input_bytes);
  fill_out(res, out);
  int status = TERGPU_COMPLETED;
  if (!count_only) {
    if (res.triples > out->capacity) {
      status = TERGPU_OUTPUT_OVERFLOW;
    } else if (res.triples != 0) {
      check(cudaMemcpyAsync(out->triples, res.d_triples, res.triples * 12, cudaMemcpyDeviceToHost,
                            st), "triples download");
      check(cudaStreamSynchronize(st), "triples download");
    }
  }
  out->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return status;
}

typedef unsigned __int128 u128;

u128 words_to_u128(const uint32_t* w, uint32_t words) {
  u128 v = 0;
  for (uint32_t k = 0; k < words && k < 4; ++k) v |= ((u128)w[k]) << (32 * k);
  return v;
}

int root_records_body(const void* vin, void* vout) {
  const auto* in = static_cast<const tergpu_root_records_in*>(vin);
  auto* out = static_cast<tergpu_root_records_out*>(vout);
  const auto t0 = std::chrono::steady_clock::now();
  if (in == nullptr || out == nullptr) {
    t_error = "null argument";
    return TERGPU_INVALID_INPUT;
  }
  const uint32_t n = in->n;
  if (n == 0 || n % 36 != 0 || n > 128 || in->r1 == 0 || in->r1 >= n) {
    t_error = "records root requires 36 | n <= 128 and 0 < r1 < n";
    return TERGPU_INVALID_CONFIGURATION;
  }
  const uint32_t w64 = (n + 63) / 64, w32 = (n + 31) / 32;
  if (in->record_bytes != 16 * w64 + 4 * w32) {
    t_error = "record_bytes does not match n";
    return TERGPU_INVALID_INPUT;
  }
  const uint32_t Q = n - in->r1;
  if (Q < 8 || Q > TERGPU_MAX_QUOTIENT_BITS) {
    t_error = "root quotient width outside [8, 72]";
    return TERGPU_UNSUPPORTED_WIDTH;
  }
  for (int l = 0; l < 3; ++l) {
    if (in->count[l] >= 0x80000000ull || (in->count[l] && in->records[l] == nullptr) ||
        in->child_target[l] == nullptr) {
      t_error = "record lists invalid";
      return TERGPU_INVALID_INPUT;
    }
  }
  if (in->root_target == nullptr) {
    t_error = "root target missing";
    return TERGPU_INVALID_INPUT;
  }
  const bool count_only = (in->flags & TERGPU_ROOT_COUNT_ONLY) != 0;
  if (!count_only && out->root.capacity != 0 && out->root.triples == nullptr) {
    t_error = "triples buffer missing";
    return TERGPU_INVALID_INPUT;
  }
  const u128 nmask = n >= 128 ? ~(u128)0 : ((((u128)1) << n) - 1);
  const u128 T = words_to_u128(in->root_target, w32) & nmask;
  u128 c[3];
  u128 tau_res = T;
  for (int l = 0; l < 3; ++l) {
    c[l] = words_to_u128(in->child_target[l], w32) & nmask;
    tau_res = (tau_res - c[l]) & nmask;
  }
  const u128 qmask = Q >= 128 ? ~(u128)0 : ((((u128)1) << Q) - 1);
  const u128 tau = (tau_res >> in->r1) & qmask;
  out->tau_lo = static_cast<uint64_t>(tau);
  out->tau_hi = static_cast<uint64_t>(tau >> 64);

  Workspace& w = workspace(in->device);
  std::lock_guard<std::mutex> lock(w.mu);
  check(cudaSetDevice(w.device), "cudaSetDevice");
  w.alloc_stream = w.stream;
  uint64_t input_bytes = 0;
  for (int l = 0; l < 3; ++l) input_bytes += in->count[l] * (in->record_bytes + 9) + 64;
  if (in->memory_limit_bytes != 0 && input_bytes > in->memory_limit_bytes) {
    t_error = "input records alone exceed the device ceiling";
    return TERGPU_RESOURCE_LIMIT;
  }
  JoinInput j{};
  j.quotient_bits = Q;
  j.stream = w.stream;
  uint8_t* drec[3];
  for (int l = 0; l < 3; ++l) {
    j.count[l] = in->count[l];
    drec[l] = ensure<uint8_t>(w, kSlotRecords + l, in->count[l] * in->record_bytes + 16);
    if (in->count[l]) {
      check(cudaMemcpyAsync(drec[l], in->records[l], in->count[l] * in->record_bytes,
                            cudaMemcpyHostToDevice, w.stream), "records upload");
    }
    uint64_t* dlo = ensure<uint64_t>(w, kSlotKeyLo + l, in->count[l] * 8 + 8);
    uint8_t* dhi = ensure<uint8_t>(w, kSlotKeyHi + l, in->count[l] + 8);
    RecordKeyArgs k{};
    k.records = drec[l];
    k.count = in->count[l];
    k.record_bytes = in->record_bytes;
    k.res_offset = 16 * w64;
    k.words32 = w32;
    k.n = n;
    k.r1 = in->r1;
    k.qbits = Q;
    k.child_lo = static_cast<uint64_t>(c[l]);
    k.child_hi = static_cast<uint64_t>(c[l] >> 64);
    k.tau_lo = out->tau_lo;
    k.tau_hi = out->tau_hi;
    k.negate = l == 2;
    k.key_lo = dlo;
    k.key_hi = dhi;
    launch_record_keys(k, w.stream);
    j.key_lo[l] = dlo;
    j.key_hi[l] = dhi;
    j.id[l] = nullptr;
  }
  check(cudaGetLastError(), "key derivation");
  j.cells = in->cells;
  j.projected_bits = in->projected_bits;
  j.family_bits = in->family_bits;
  j.filter_bits = in->filter_bits;
  j.memory_limit_bytes = in->memory_limit_bytes;
  j.capacity = count_only ? 0 : out->root.capacity;
  j.count_only = count_only;
  j.sweep_variant = sweep_variant(in->flags);
  j.autotune = autotune_requested(in->flags) && j.sweep_variant == 0;
  j.one_pass = (in->flags & TERGPU_ROOT_PARTITION_ONE_PASS) != 0;
  j.shard = in->shard_index;
  j.shards = checked_shards(in->shard_index, in->shard_count);
  const JoinResult res = run_join(w, j, input_bytes);
  fill_out(res, &out->root);
  out->residue_exact = out->structural = out->valid_roots = 0;
  int status = TERGPU_COMPLETED;
  if (!count_only) {
    if (res.triples > out->root.capacity) {
      status = TERGPU_OUTPUT_OVERFLOW;
    } else if (res.triples != 0) {
      uint8_t* dflags = ensure<uint8_t>(w, kSlotFlags, res.triples + 16);
      unsigned long long* counters = ensure<unsigned long long>(w, kSlotCounters, kCounters * 8);
      check(cudaMemsetAsync(counters, 0, kCounters * 8, w.stream), "memset");
      AuthorityArgs au{};
      for (int l = 0; l < 3; ++l) au.records[l] = drec[l];
      au.record_bytes = in->record_bytes;
      au.res_offset = 16 * w64;
      au.words32 = w32;
      au.words64 = w64;
      au.n = n;
      au.root_lo = static_cast<uint64_t>(T);
      au.root_hi = static_cast<uint64_t>(T >> 64);
      au.triples = res.d_triples;
      au.count = res.triples;
      au.flags = dflags;
      au.counters = counters;
      launch_authority(au, w.stream);
      check(cudaGetLastError(), "authority launch");
      unsigned long long hc[3];
      check(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, w.stream), "counters");
      check(cudaMemcpyAsync(out->root.triples, res.d_triples, res.triples * 12,
                            cudaMemcpyDeviceToHost, w.stream), "triples download");
      if (out->triple_flags != nullptr) {
        check(cudaMemcpyAsync(out->triple_flags, dflags, res.triples, cudaMemcpyDeviceToHost,
                              w.stream), "flags download");
      }
      check(cudaStreamSynchronize(w.stream), "authority");
      out->residue_exact = hc[0];
      out->structural = hc[1];
      out->valid_roots = hc[2];
    }
  }
  out->root.total_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return status;
}

}  // namespace tergpu

extern "C" {

int tergpu_root_run(const tergpu_root_in* in, tergpu_root_out* out) {
  return tergpu::guarded("tergpu_root_run", tergpu::root_run_body, in, out);
}

int tergpu_root_run_records(const tergpu_root_records_in* in, tergpu_root_records_out* out) {
  return tergpu::guarded("tergpu_root_run_records", tergpu::root_records_body, in, out);
}

int tergpu_device_count(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) return 0;
  return count;
}

int tergpu_abi_version(void) { return TERGPU_ABI_VERSION; }

uint64_t tergpu_fnv1a(const void* bytes, uint64_t size, uint64_t state) {
  const auto* p = static_cast<const uint8_t*>(bytes);
  for (uint64_t i = 0; i < size; ++i) {
    state ^= p[i];
    state *= 0x100000001b3ULL;
  }
  return state;
}

void tergpu_release(void) {
  tergpu::release_slots();
  std::lock_guard<std::mutex> lock(tergpu::g_mu);
  for (auto& w : tergpu::g_ws) {
    std::lock_guard<std::mutex> inner(w->mu);
    tergpu::destroy_workspace(*w);
  }
  tergpu::g_ws.clear();
  tergpu::trim_library_pools();
}

const char* tergpu_last_error(void) { return tergpu::t_error.c_str(); }

}  // extern "C"
