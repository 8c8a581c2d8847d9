// Host-side machinery shared by the C ABI entry points of libtergpu.so:
// per-device workspaces (grow-only device buffers reused across calls), error
// reporting, and the partition + sweep join driver.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
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

struct Workspace {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t start = nullptr, mid = nullptr, stop = nullptr;
  std::map<int, Buffer> buf;
  std::mutex mu;
};

// The workspace of a device (created on first use).
Workspace& workspace(int device);

// Grow-only device buffer in slot `slot` of the workspace.
void* ensure_bytes(Workspace& w, int slot, size_t bytes);
template <typename T>
T* ensure(Workspace& w, int slot, size_t bytes) {
  return static_cast<T*>(ensure_bytes(w, slot, bytes));
}

struct Tuning {
  uint32_t fb = 6, wb = 12, s_split = 1, sort_bits = 0;
  uint32_t variant = 3;  // sweep: 1 (A in registers), 2 (B in registers), 3 (v2 + bank-free probes)
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
  uint32_t shard = 0, shards = 1;  // join only target families u == shard (mod shards)
  cudaStream_t stream;
};

struct JoinResult {
  uint64_t triples = 0, pairs = 0, survivors = 0, fast = 0, projected = 0;
  uint64_t device_bytes = 0;
  float join_ms = 0, partition_ms = 0, sweep_ms = 0;
  uint32_t launches = 0;
  Tuning tuning;
  uint32_t* d_triples = nullptr;  // device, capacity triples (valid until the next join)
};

// Checks a (shard_index, shard_count) pair of the C ABI and returns the shard
// count (count 0 means 1).  Throws Failure(InvalidInput) unless the count is a
// power of two in [1, 64] and the index is below it.
uint32_t checked_shards(uint32_t index, uint32_t count);

// Partition + sweep on keys already on the device (throws Failure).
JoinResult run_join(Workspace& w, const JoinInput& in, uint64_t input_bytes);

// Slots 0..99 belong to the root entry points; the attempt driver uses 100+.
constexpr int kAttemptSlotBase = 100;

}  // namespace tergpu
