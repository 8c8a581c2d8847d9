// tergpu_root_run_noalloc: the root join for callers that must not allocate.
//
// Some callers cannot call cudaMalloc at all: code running inside another
// framework's memory pool (which owns every device allocation and forbids
// side allocations), a process whose device memory is fully reserved up
// front, or a latency-critical service loop where an allocation could
// synchronize the device or fail under fragmentation.  This entry point serves
// them: it takes device-resident inputs and a device output buffer from the
// caller and keeps every intermediate array (the partitioned key lists, the
// family tables and the counters) in one fixed, file-scope device array.
//
// The array is kNoAllocScratchBytes (32 MiB) on every device that loads the
// library, and it stays there until the process exits.  A root whose
// intermediates do not fit is refused with TERGPU_RESOURCE_LIMIT before any
// work is queued (about 2.4 million key entries over the three lists).
//
// Set-up: the first call on a device looks up the device address of the array
// (cudaGetSymbolAddress, with that device current) and remembers it; it is a
// lookup, not an allocation.  Every call also waits for its stream to finish
// the join (it reads the counters back), so a call on a stream that is being
// captured is refused with TERGPU_INVALID_INPUT and the capture is left intact.
// The call makes `device` current for its work and restores the caller's
// current device before it returns.
//
// Every call uses the same array and leaves the last call's contents in it; the
// call clears what must start at zero.  Two calls whose work overlaps on the
// GPU (different streams, or different host threads) race on the array and
// corrupt each other's results: run them one after the other.

#include "tergpu.h"
#include "root_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

namespace tergpu {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;
constexpr uint32_t kNoAllocMaxFamilyBits = 10;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

thread_local char t_noalloc_error[256] = "";

int fail(int status, const char* msg) {
  std::snprintf(t_noalloc_error, sizeof t_noalloc_error, "%s", msg);
  return status;
}

int fail_cuda(cudaError_t e, const char* what) {
  std::snprintf(t_noalloc_error, sizeof t_noalloc_error, "%s: %s", what, cudaGetErrorString(e));
  return TERGPU_DEVICE_ERROR;
}

// Carves 256-byte aligned pieces out of the static array.
struct Carver {
  unsigned char* base;
  size_t used;
  template <typename T>
  T* take(size_t bytes) {
    used = (used + 255) & ~size_t{255};
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

uint32_t ceil_log2_u64(uint64_t v) {
  uint32_t b = 0;
  while ((uint64_t{1} << b) < v) ++b;
  return b;
}

}  // namespace
}  // namespace tergpu

extern "C" const char* tergpu_noalloc_last_error(void) { return tergpu::t_noalloc_error; }

namespace tergpu {
namespace {
// Restores the calling thread's current device on every return path.
struct DeviceGuard {
  int saved = -1;
  DeviceGuard() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceGuard() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};
}  // namespace
}  // namespace tergpu

extern "C" int tergpu_root_run_noalloc(const tergpu_root_in* in, tergpu_root_out* out) {
  using namespace tergpu;
  t_noalloc_error[0] = '\0';
  const DeviceGuard restore;
  const auto t0 = std::chrono::steady_clock::now();
  if (in == nullptr || out == nullptr) return fail(TERGPU_INVALID_INPUT, "null argument");
  if ((in->flags & TERGPU_ROOT_DEVICE_INPUTS) == 0) {
    return fail(TERGPU_INVALID_INPUT,
                "the no-allocation entry needs device-resident inputs (TERGPU_ROOT_DEVICE_INPUTS)");
  }
  const uint32_t Q = in->quotient_bits;
  if (Q < 8 || Q > TERGPU_MAX_QUOTIENT_BITS) return fail(TERGPU_UNSUPPORTED_WIDTH, "quotient width outside [8, 72]");
  const bool count_only = (in->flags & TERGPU_ROOT_COUNT_ONLY) != 0;
  if (!count_only && out->capacity != 0 && out->triples == nullptr) {
    return fail(TERGPU_INVALID_INPUT, "device triples buffer missing");
  }
  if (in->projected_bits != 0) {
    return fail(TERGPU_INVALID_INPUT, "projected counts are not offered by the no-allocation entry");
  }
  for (int l = 0; l < 3; ++l) {
    if (in->count[l] >= 0x80000000ull || (in->count[l] != 0 && in->key_lo[l] == nullptr) ||
        (Q > 64 && in->count[l] != 0 && in->key_hi[l] == nullptr)) {
      return fail(TERGPU_INVALID_INPUT, "list pointers or sizes invalid");
    }
  }
  const int device = in->device;
  if (device < 0 || device >= kMaxDevices) return fail(TERGPU_DEVICE_ERROR, "device ordinal out of range");

  // Tuning: about 2048 D entries per family, at most 2^10 families (the family
  // tables then stay small enough for the host side to read on its stack).
  const uint32_t F = std::min<uint32_t>(Q, 64);
  const uint32_t hi_bits = Q - F;
  uint32_t fb = in->family_bits;
  if (fb == 0) {
    const double ideal = std::log2(std::max<double>(1.0, static_cast<double>(in->count[2]) / 2048.0));
    fb = static_cast<uint32_t>(std::max(6.0, std::floor(ideal + 0.5)));
    fb = std::min(fb, std::min<uint32_t>(kNoAllocMaxFamilyBits, F - 2));
  }
  if (fb < 6 || fb > kNoAllocMaxFamilyBits || fb + 2 > F) {
    return fail(TERGPU_INVALID_INPUT, "family bits outside [6, 10] for the no-allocation entry");
  }
  const uint32_t nfam = 1u << fb;
  const uint64_t avg_x = std::max<uint64_t>(1, in->count[1] >> fb);
  uint32_t wb = in->filter_bits != 0 ? in->filter_bits - 5
                                     : std::clamp<uint32_t>(ceil_log2_u64(avg_x) + 3, 6, 14);
  if (wb < 5 || wb > 15) return fail(TERGPU_INVALID_INPUT, "filter bits outside [10, 20]");
  const uint32_t s_split = std::clamp<uint32_t>((148u * 16u + nfam - 1) / nfam, 1, nfam);

  // Plan the pieces of the static array before touching the device.
  size_t need = 0;
  {
    Carver plan{nullptr, 0};
    for (int l = 0; l < 3; ++l) {
      const uint64_t slots = in->count[l] + nfam + 16;
      plan.take<uint64_t>(slots * 8);
      plan.take<uint8_t>(slots);
      plan.take<uint32_t>(slots * 4);
      for (int k = 0; k < 3; ++k) plan.take<uint32_t>((nfam + 1) * 4ull);
    }
    plan.take<unsigned long long>(kCounters * 8);
    need = plan.used;
  }
  if (need > kNoAllocScratchBytes) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "root needs %zu bytes of scratch; the no-allocation entry has %zu (32 MiB)", need,
                  kNoAllocScratchBytes);
    return fail(TERGPU_RESOURCE_LIMIT, msg);
  }

  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(in->stream);
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing(st, &capturing)) != cudaSuccess) return fail_cuda(e, "cudaStreamIsCapturing");
  if (capturing != cudaStreamCaptureStatusNone) {
    return fail(TERGPU_INVALID_INPUT,
                "the no-allocation entry waits for its stream and cannot run on a capturing stream");
  }
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (g_scratch_ptr[device] == nullptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress");
      g_scratch_ptr[device] = p;
    }
  }
  Carver carve{static_cast<unsigned char*>(g_scratch_ptr[device]), 0};
  ListView views[3];
  uint64_t* res[3];
  uint8_t* hi[3];
  uint32_t* ids[3];
  uint32_t *cnt[3], *off[3], *cur[3];
  for (int l = 0; l < 3; ++l) {
    const uint64_t slots = in->count[l] + nfam + 16;
    res[l] = carve.take<uint64_t>(slots * 8);
    hi[l] = carve.take<uint8_t>(slots);
    ids[l] = carve.take<uint32_t>(slots * 4);
    cnt[l] = carve.take<uint32_t>((nfam + 1) * 4ull);
    off[l] = carve.take<uint32_t>((nfam + 1) * 4ull);
    cur[l] = carve.take<uint32_t>((nfam + 1) * 4ull);
  }
  unsigned long long* counters = carve.take<unsigned long long>(kCounters * 8);

  const uint64_t fast_mask = F >= 64 ? ~0ull : ((1ull << F) - 1ull);
  if ((e = cudaMemsetAsync(counters, 0, kCounters * 8, st)) != cudaSuccess) return fail_cuda(e, "memset");
  for (int l = 0; l < 3; ++l) {
    if ((e = cudaMemsetAsync(cnt[l], 0, nfam * 4ull, st)) != cudaSuccess) return fail_cuda(e, "memset");
    launch_hist(in->key_lo[l], in->count[l], nfam - 1, cnt[l], st);
    launch_scan(cnt[l], nfam, off[l], cur[l], st);
    launch_scatter(in->key_lo[l], Q > 64 ? in->key_hi[l] : nullptr, in->id[l], in->count[l], fb,
                   fast_mask, hi_bits ? ((1u << hi_bits) - 1u) : 0u, cur[l], res[l], hi[l], ids[l], st);
    views[l] = ListView{res[l], hi[l], ids[l], off[l], cnt[l]};
  }
  launch_max_family(cnt[0], nfam, counters, kMaxQ, st);
  launch_max_family(cnt[1], nfam, counters, kMaxX, st);
  if (in->count[1] != 0) {
    launch_family_sort(res[1], hi[1], ids[1], off[1], cnt[1], nfam, F - fb, std::min<uint32_t>(wb, 12), st);
  }
  SweepArgs a{};
  a.q = views[0];
  a.x = views[1];
  a.y = views[2];
  a.cells = in->cells;  // device pointer or null
  a.fb = fb;
  a.s_split = s_split;
  a.shard = 0;
  a.shards = 1;
  a.wb = wb;
  a.rb = F - fb;
  a.mrb = F - fb;
  a.hi_bits = hi_bits;
  a.project = 0;
  a.triples = count_only ? nullptr : out->triples;
  a.cap = count_only ? 0 : out->capacity;
  a.counters = counters;
  launch_sweep2(a, a.mrb < 32, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail_cuda(e, "launch");

  unsigned long long hc[kCounters];
  uint32_t hcnt[2][1u << kNoAllocMaxFamilyBits];
  uint8_t hcells[4096];
  if ((e = cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(hcnt[0], cnt[0], nfam * 4ull, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(hcnt[1], cnt[1], nfam * 4ull, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (in->cells != nullptr &&
       (e = cudaMemcpyAsync(hcells, in->cells, 4096, cudaMemcpyDeviceToHost, st)) != cudaSuccess)) {
    return fail_cuda(e, "result download");
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, "join");
  uint64_t pairs = 0;
  for (uint32_t s = 0; s < nfam; ++s) {
    for (uint32_t t = 0; t < nfam; ++t) {
      if (in->cells != nullptr && hcells[((s & 63u) << 6) | (t & 63u)] == 0) continue;
      pairs += static_cast<uint64_t>(hcnt[0][s]) * hcnt[1][t];
    }
  }
  out->triples_count = hc[kTriples];
  out->logical_pairs = pairs;
  out->filter_survivors = hc[kSurvivors];
  out->fast_hits = hc[kFast];
  out->projected_hits = 0;
  out->device_bytes = need;
  out->join_ms = 0;
  out->partition_ms = 0;
  out->sweep_ms = 0;
  out->family_bits = fb;
  out->filter_bits = wb + 5;
  uint32_t launches = 2 + (in->count[1] != 0 ? 1 : 0) + 1;  // max-family x2, family sort, sweep
  for (int l = 0; l < 3; ++l) launches += (in->count[l] != 0 ? 2 : 0) + 1;  // hist + scatter, scan
  out->kernel_launches = launches;
  out->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (!count_only && hc[kTriples] > out->capacity) return TERGPU_OUTPUT_OVERFLOW;
  return TERGPU_COMPLETED;
}
