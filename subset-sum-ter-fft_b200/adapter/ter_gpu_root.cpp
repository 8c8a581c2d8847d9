#include "ter_gpu_root.hpp"

#include "tergpu.h"

#include <dlfcn.h>

#include <array>
#include <cstdlib>
#include <mutex>
#include <new>
#include <vector>

namespace ter::gpu_root {

namespace {

// The C ABI is resolved on first use, so a host without the GPU library still
// runs every other backend.  TERGPU_LIBRARY names the shared object; otherwise
// the dynamic linker's search path finds libtergpu.so.  A library built for
// another ABI version (a different tergpu_root_in layout) is not used.
using RootRunFn = int (*)(const tergpu_root_in*, tergpu_root_out*);
using AbiVersionFn = int (*)(void);

RootRunFn resolve_root_run() noexcept {
  static std::once_flag once;
  static RootRunFn fn = nullptr;
  std::call_once(once, [] {
    const char* path = std::getenv("TERGPU_LIBRARY");
    void* handle = dlopen(path != nullptr ? path : "libtergpu.so", RTLD_NOW | RTLD_LOCAL);
    if (handle != nullptr) {
      const auto version = reinterpret_cast<AbiVersionFn>(dlsym(handle, "tergpu_abi_version"));
      if (version != nullptr && version() == TERGPU_ABI_VERSION) {
        fn = reinterpret_cast<RootRunFn>(dlsym(handle, "tergpu_root_run"));
      }
    }
  });
  return fn;
}

}  // namespace

const char* status_label(const Status status) noexcept {
  switch (status) {
    case Status::Completed: return "Completed";
    case Status::InvalidInput: return "InvalidInput";
    case Status::ResourceLimit: return "ResourceLimit";
    case Status::DeviceError: return "DeviceError";
  }
  return "Unknown";
}

Status run_gpu_root(const mr8::Dataset& data, const rg::RootIndex& index,
                    const a64::FamilyKeys& keys, const Config& config, rg::RootSink& sink,
                    Telemetry* const telemetry) {
  if (telemetry != nullptr) { *telemetry = Telemetry{}; }
  // The same admission rules as run_hash_join (ter_hash_join_root.cpp:76-104).
  if (!data.ok || !keys.ok || keys.full_bits < 25U || keys.full_bits > 69U ||
      keys.fast_bits != std::min(keys.full_bits, 64U) ||
      keys.residual_bits != keys.fast_bits - 6U || keys.hi_bits != keys.full_bits - keys.fast_bits ||
      sink.data != &data || sink.index != &index || sink.depth != rg::SinkDepth::Full) {
    return Status::InvalidInput;
  }
  const std::array<const std::array<std::vector<mr8::Posting>, rg::kFamilies>*, 3> families{
      &data.q_family, &data.x_family, &data.y_family};
  const std::uint64_t residual_mask = (std::uint64_t{1} << keys.residual_bits) - 1U;
  const std::uint32_t hi_mask = (1U << keys.hi_bits) - 1U;

  // Flatten family-major: the full low-F key is (residual << 6) | family.
  std::array<std::vector<std::uint64_t>, 3> key_lo;
  std::array<std::vector<std::uint8_t>, 3> key_hi;
  std::array<std::vector<std::uint32_t>, 3> ids;
  try {
    for (std::size_t l = 0U; l < 3U; ++l) {
      std::size_t total = 0U;
      for (std::uint32_t f = 0U; f < rg::kFamilies; ++f) {
        const auto& postings = (*families[l])[f];
        if (postings.size() != keys.key[l][f].size() || postings.size() != keys.hi[l][f].size()) {
          return Status::InvalidInput;
        }
        total += postings.size();
      }
      key_lo[l].reserve(total);
      key_hi[l].reserve(total);
      ids[l].reserve(total);
      for (std::uint32_t f = 0U; f < rg::kFamilies; ++f) {
        const auto& postings = (*families[l])[f];
        for (std::size_t i = 0U; i < postings.size(); ++i) {
          const std::uint64_t residual = keys.key[l][f][i];
          if (residual > residual_mask || keys.hi[l][f][i] > hi_mask ||
              (residual & mr8::kResidualMask) != postings[i].value) {
            return Status::InvalidInput;
          }
          key_lo[l].push_back((residual << 6U) | f);
          key_hi[l].push_back(keys.hi[l][f][i]);
          ids[l].push_back(postings[i].id);
        }
      }
    }
  } catch (const std::bad_alloc&) {
    return Status::ResourceLimit;
  }

  const RootRunFn root_run = resolve_root_run();
  if (root_run == nullptr) { return Status::DeviceError; }

  tergpu_root_in in{};
  in.quotient_bits = keys.full_bits;
  for (std::size_t l = 0U; l < 3U; ++l) {
    in.count[l] = key_lo[l].size();
    in.key_lo[l] = key_lo[l].data();
    in.key_hi[l] = key_hi[l].data();
    in.id[l] = ids[l].data();
  }
  in.cells = index.selected.data();
  in.projected_bits = config.projected_bits;
  in.device = config.device;
  in.memory_limit_bytes =
      config.memory_limit_bytes == std::numeric_limits<std::size_t>::max() ? 0U
                                                                            : config.memory_limit_bytes;
  in.family_bits = config.family_bits;
  in.filter_bits = config.filter_bits;

  // Full-Q outputs are rare (about |A||B||C| / 2^Q); start small and retry once
  // with the exact count when the first capacity was too small.
  std::vector<std::uint32_t> triples;
  tergpu_root_out out{};
  std::uint64_t capacity = 4096U;
  for (int round = 0; round < 2; ++round) {
    try {
      triples.assign(static_cast<std::size_t>(capacity) * 3U, 0U);
    } catch (const std::bad_alloc&) {
      return Status::ResourceLimit;
    }
    out = tergpu_root_out{};
    out.triples = triples.data();
    out.capacity = capacity;
    const int status = root_run(&in, &out);
    if (status == TERGPU_OUTPUT_OVERFLOW && round == 0) {
      capacity = out.triples_count;
      continue;
    }
    if (status == TERGPU_RESOURCE_LIMIT) { return Status::ResourceLimit; }
    if (status == TERGPU_INVALID_INPUT || status == TERGPU_UNSUPPORTED_WIDTH) {
      return Status::InvalidInput;
    }
    if (status != TERGPU_COMPLETED) { return Status::DeviceError; }
    break;
  }
  for (std::uint64_t i = 0U; i < out.triples_count; ++i) {
    sink.emit_triple(triples[3U * i], triples[3U * i + 1U], triples[3U * i + 2U]);
  }
  if (telemetry != nullptr) {
    telemetry->logical_pairs = out.logical_pairs;
    telemetry->filter_survivors = out.filter_survivors;
    telemetry->fast_hits = out.fast_hits;
    telemetry->full_hits = out.triples_count;
    telemetry->projected_hits = out.projected_hits;
    telemetry->device_bytes = out.device_bytes;
    telemetry->join_ms = out.join_ms;
    telemetry->total_ms = out.total_ms;
    telemetry->family_bits = out.family_bits;
    telemetry->filter_bits = out.filter_bits;
  }
  return Status::Completed;
}

}  // namespace ter::gpu_root
