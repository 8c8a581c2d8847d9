// Element counts for kernels that run either with a count known on the host or
// inside a captured CUDA graph, where the count is produced on the device by an
// earlier kernel of the same graph.
#pragma once

#include <cstdint>

namespace tergpu {

struct Count {
  uint64_t cap = 0;                          // the count, or its bound when `dev` is set
  const unsigned long long* dev = nullptr;   // device count read at kernel start (bounded by cap)

  Count() = default;
  Count(uint64_t n) : cap(n) {}  // NOLINT: a host count converts implicitly
  Count(uint64_t bound, const unsigned long long* d) : cap(bound), dev(d) {}

#ifdef __CUDACC__
  __device__ __forceinline__ uint64_t get() const {
    if (dev == nullptr) return cap;
    const unsigned long long v = *dev;
    return v < cap ? v : cap;
  }
#endif
};

}  // namespace tergpu
