#pragma once

// Drop-in GPU root backend for the reference's ter2_root plugin point.
//
// A fifth peer of run_k2 / run_k2_wide / run_arwlf / run_hash_join with exactly
// run_hash_join's signature (reference ter2_root/campaign/ter_hash_join_root.hpp:38-40).
// It is compiled against the reference's headers and links the C ABI in
// include/tergpu.h; nothing here does arithmetic of its own.
//
// Contract, as for run_hash_join:
//   * inputs are borrowed, immutable and host resident;
//   * the sink is not reset: callers time reset + call;
//   * every full-Q triple reaches sink.emit_triple(a, b, c) once, with
//     multiplicity, on the calling thread (order is unspecified, the sink's
//     digest is order-independent);
//   * InvalidInput / ResourceLimit / DeviceError leave the sink unchanged.

#include "ter_a64_chqr.hpp"

#include <cstddef>
#include <cstdint>
#include <limits>

namespace ter::gpu_root {

namespace rg = ter::root_generalization;
namespace mr8 = ter::microreport8;
namespace a64 = ter::a64;

enum class Status : std::uint8_t { Completed, InvalidInput, ResourceLimit, DeviceError };

struct Config {
  // Device bytes the call may hold (workspace plus uploaded keys).
  std::size_t memory_limit_bytes = std::numeric_limits<std::size_t>::max();
  int device = 0;
  std::uint32_t projected_bits = 0;  // > 0: also count triples equal on key bits [0, k)
  std::uint32_t family_bits = 0;     // 0: autotuned
  std::uint32_t filter_bits = 0;     // 0: autotuned
};

struct Telemetry {
  std::uint64_t logical_pairs = 0;
  std::uint64_t filter_survivors = 0;
  std::uint64_t fast_hits = 0;
  std::uint64_t full_hits = 0;
  std::uint64_t projected_hits = 0;
  std::uint64_t device_bytes = 0;
  double join_ms = 0.0;
  double total_ms = 0.0;
  std::uint32_t family_bits = 0;
  std::uint32_t filter_bits = 0;
};

[[nodiscard]] Status run_gpu_root(const mr8::Dataset& data, const rg::RootIndex& index,
                                  const a64::FamilyKeys& keys, const Config& config,
                                  rg::RootSink& sink, Telemetry* telemetry = nullptr);

[[nodiscard]] const char* status_label(Status status) noexcept;

}  // namespace ter::gpu_root
