// Host-side machinery shared by the C ABI entry points of libtergpu.so:
// per-device workspaces (grow-only device buffers reused across calls), error
// reporting, and the partition + sweep join driver.
#pragma once

#include <cuda_runtime.h>

#include "count.cuh"
#include "root_kernels.cuh"
#include "tergpu.h"

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>

namespace tergpu {

extern thread_local std::string t_error;

struct Failure {
  int status;
};

// Throws Failure (ResourceLimit for an allocation failure, DeviceError else).
void check(cudaError_t e, const char* what);

struct Buffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

// Device buffers, a stream and timing events for one call at a time.  Buffers
// are stream-ordered allocations from the library's own pool of the device
// (library_pool: no reuse that would make one stream wait for another's work),
// on alloc_stream, or on `stream` when that is null, so growing one workspace
// never waits for work that other workspaces have in flight on the device.
struct Workspace {
  int device = 0;
  cudaStream_t stream = nullptr;
  // batch slots: `stream` has the device's highest priority and stream_low its
  // lowest (TERGPU_ATTEMPT_BACKGROUND); null elsewhere
  cudaStream_t stream_low = nullptr;
  cudaStream_t alloc_stream = nullptr;  // the stream the current call launches on
  cudaEvent_t start = nullptr, mid = nullptr, stop = nullptr;
  // batch slots wait on a blocking-sync event (the host thread sleeps instead of
  // spinning: many slots share the host cores); the shared workspace spins
  cudaEvent_t sync_event = nullptr;
  std::map<int, Buffer> buf;
  // captured attempt graphs by shape (n), with buffers of their own: kept across
  // calls and across release_buffers, freed by destroy_workspace
  std::map<uint32_t, std::shared_ptr<void>> plans;
  std::mutex mu;
  // cancel word of this workspace's calls: pinned host memory the sweep reads
  // through its device mapping (cancel_word() allocates it on first use)
  volatile int* cancel_host = nullptr;
  cudaMemPool_t pool = nullptr;  // library_pool(device)
  const volatile int* cancel_dev = nullptr;
};

// The workspace's cancel word (host and device views), cleared.
void cancel_word(Workspace& w);

// Waits until the work queued so far on `st` is done (see Workspace::sync_event).
void sync_stream(Workspace& w, cudaStream_t st, const char* what);

// The shared workspace of a device (created on first use; calls through it are
// serialized by its mutex).
Workspace& workspace(int device);

// A workspace with its own stream and events; `blocking` makes its waits yield the
// host thread (the batch engine's slots).
std::unique_ptr<Workspace> make_workspace(int device, bool blocking = false);
// Frees a workspace's buffers, stream and events (waits for its stream).
void destroy_workspace(Workspace& w);
// Returns a workspace's buffers to the device pool (stream-ordered, no wait).
void release_buffers(Workspace& w);

// The batch engine's slot workspaces: kept between calls with their graph
// plans (a server's slots stay warm), freed by release_slots (tergpu_release).
std::unique_ptr<Workspace> take_slot(int device);
void give_slot(std::unique_ptr<Workspace> w);
void release_slots();

// Grow-only device buffer in slot `slot` of the workspace.
void* ensure_bytes(Workspace& w, int slot, size_t bytes);
template <typename T>
T* ensure(Workspace& w, int slot, size_t bytes) {
  return static_cast<T*>(ensure_bytes(w, slot, bytes));
}

struct Tuning {
  uint32_t fb = 6, wb = 12, s_split = 1, sort_bits = 0;
  // sweep: 1 (A in registers), 2 (B in registers), 3 (v2 + bank-free probes),
  // 4 (0/1 probe table over 14-bit windows, B laid out one bank per lane)
  uint32_t variant = 3;
};

// Device-resident inputs of one join: keys per list.
struct JoinInput {
  uint32_t quotient_bits;
  uint64_t count[3];
  const uint64_t* key_lo[3];  // device
  const uint8_t* key_hi[3];   // device or null
  const uint32_t* id[3];      // device or null
  const uint8_t* cells;       // host or null
  const uint8_t* cells_device;  // device or null (takes precedence)
  uint32_t projected_bits;
  uint32_t family_bits, filter_bits;
  uint64_t memory_limit_bytes;
  uint64_t capacity;
  bool count_only;
  uint32_t sweep_variant;  // 0: default (3), else 1, 2 or 3
  bool autotune = false;   // pick fb / filter bits / variant by timing a sample first
  bool one_pass = false;   // no staged two-pass scatter for long lists
  bool background = false; // CTAs of about 2^kBackgroundBlockLog2 pairs (work of higher
                           // priority on the device gets SMs sooner)
  uint32_t shard = 0, shards = 1;  // join only target families u == shard (mod shards)
  cudaStream_t stream;
  VisitBound visit{};      // projected counts only before this bound (root_kernels.cuh)
  const volatile int* cancel = nullptr;  // device view of a cancel word, or null
};

struct JoinResult {
  uint64_t triples = 0, pairs = 0, survivors = 0, fast = 0, projected = 0;
  uint64_t device_bytes = 0;
  float join_ms = 0, partition_ms = 0, sweep_ms = 0;
  uint32_t launches = 0;
  float tune_ms = 0;       // device time the autotuner spent on this shape (0: cached)
  Tuning tuning;
  uint32_t* d_triples = nullptr;  // device, capacity triples (valid until the next join)
};

// Checks a (shard_index, shard_count) pair of the C ABI and returns the shard
// count (count 0 means 1).  Throws Failure(InvalidInput) unless the count is a
// power of two in [1, 64] and the index is below it.
uint32_t checked_shards(uint32_t index, uint32_t count);

// Pairs per sweep CTA of a very large join, as a power of two: about 25 ms of
// one SM in the foreground, about 2 ms for background work (an n = 108 attempt
// beside short requests: an SM comes free every ~10 us on average).
constexpr uint32_t kJoinBlockLog2 = 29;
constexpr uint32_t kBackgroundBlockLog2 = 25;

// Family bits, filter bits, CTAs per family and variant of one join from its
// list sizes (requested values win when not zero).  With the A list size n_q,
// small joins get fewer CTAs (about 2^20 pairs each at least), so a join of a
// few million pairs does not occupy every SM with CTAs that mostly build filters,
// and very large joins get CTAs of at most about 2^block_log2 pairs.
Tuning choose_tuning(uint64_t n_x, uint64_t n_d, uint32_t fast_bits, uint32_t projected,
                     uint32_t fb_req, uint32_t filter_req, uint32_t variant, uint32_t shards,
                     uint64_t n_q = 0, uint32_t block_log2 = kJoinBlockLog2);

// Device buffers of one join, sized by the caller for the lists' count bounds:
// per list res / hi / id (bound + 2^fb + 16 entries), cnt / off / cur
// (2^fb + 1 words), the counters (kCounters) and the triples (3 * cap words).
struct JoinBuffers {
  uint64_t* res[3];
  uint8_t* hi[3];
  uint32_t* id[3];
  uint32_t *cnt[3], *off[3], *cur[3];
  unsigned long long* counters;
  uint32_t* triples;
  // v4 (null: v4 is not run): the A list's probe windows (A slots), the B list
  // in the lane-slot layout (v4_slots(count_B, fb) slots) with its windows, and
  // that layout's family sizes and offsets (2^fb + 1 words each)
  uint32_t* qwin = nullptr;
  uint64_t* res4 = nullptr;
  uint8_t* hi4 = nullptr;
  uint32_t* id4 = nullptr;
  uint32_t* win4 = nullptr;
  uint32_t *cnt4 = nullptr, *off4 = nullptr, *cur4 = nullptr;
  // temp copy for the staged two-pass scatter (null: every list takes the
  // one-pass scatter); sized for the longest staged list
  StageBuffers stage{};
};

// Lane slots the v4 layout of a B list of `count` entries in 2^fb families can
// take: every family is padded to whole rows of 32 with at most
// kArrange4ExtraRows rows more than the minimum.
inline uint64_t v4_slots(uint64_t count, uint32_t fb) {
  return count + (static_cast<uint64_t>(32) * (kArrange4ExtraRows + 1)) * (uint64_t{1} << fb) + 64;
}

// The inputs of one join: keys per list with host or device counts.
struct JoinWork {
  const uint64_t* key_lo[3];
  const uint8_t* key_hi[3];
  const uint32_t* id[3];
  Count count[3];
  uint32_t quotient_bits;
  const uint8_t* cells;  // device or null
  uint32_t shard, shards;
  uint64_t cap;          // triples written (0: count only)
  bool main_sweep;       // the full-width sweep (false: projected counts only)
  uint32_t projected_bits;
  VisitBound visit{};
  const volatile int* cancel = nullptr;
};

// The join's device work on `st` -- partition, family layout, sweep(s) -- with
// no host synchronization (a captured graph can hold it): the triples count
// and the other counters stay in b.counters.  Records `mid` after the
// partition when not null.  Returns the sweep variant that ran.
uint32_t enqueue_join(const JoinBuffers& b, const JoinWork& j, const Tuning& tu, cudaEvent_t mid,
                      cudaStream_t st, uint32_t* launches);

// Partition + sweep on keys already on the device (throws Failure).
JoinResult run_join(Workspace& w, const JoinInput& in, uint64_t input_bytes);

// One attempt range (tergpu_attempt_run's body) on `own`, a private workspace,
// or on the device's shared workspace when `own` is null.  Returns the status.
int attempt_body(const tergpu_attempt_in* in, tergpu_attempt_out* out, Workspace* own);

// Slots 0..99 belong to the root entry points; the attempt driver uses 100+.
constexpr int kAttemptSlotBase = 100;

}  // namespace tergpu
