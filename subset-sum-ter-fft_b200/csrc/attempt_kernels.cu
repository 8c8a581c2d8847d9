// Kernels of the attempt pipeline below the root (see attempt_kernels.cuh).
//
// Reference behaviour restated (file:line in the reference project):
//   level-3 enumeration ........ src/full_ter.cpp:540-617 (lexicographic k-subsets)
//   L3 -> L2 binary merge ...... src/full_ter.cpp:827-933
//   L2 -> L1 projected quotient  src/arithmetic.cpp:9-53, src/full_ter.cpp:1170-1279
//   parent construction ........ src/packed.cpp:15-38, src/full_ter.cpp:732-790, 1079-1136
//   canonical order ............ src/full_ter.cpp:320-326 (packed_less), 624-633

#include "attempt_kernels.cuh"
#include "root_kernels.cuh"

#include <cooperative_groups.h>
#include <cuda_runtime.h>

namespace tergpu {
namespace {

namespace cg = cooperative_groups;

typedef unsigned __int128 u128;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 8;
constexpr uint32_t kTile = kRadixThreads * kRadixItems;  // 2048
constexpr uint32_t kScanChunk = 2048;

__device__ __forceinline__ u128 nmask128(uint32_t n) {
  return n >= 128 ? ~(u128)0 : ((((u128)1) << n) - 1);
}

__device__ uint64_t binom(uint32_t m, uint32_t k) {
  if (k > m) return 0;
  uint64_t r = 1;
  for (uint32_t i = 0; i < k; ++i) r = r * (m - i) / (i + 1);
  return r;
}

int blocks_for(uint64_t n, int threads, int cap = 148 * 16) {
  uint64_t b = (n + threads - 1) / threads;
  if (b > (uint64_t)cap) b = cap;
  return b == 0 ? 1 : (int)b;
}

// Blocks for a grid-stride kernel over `c`.  A device count (a captured graph's
// launch, sized by a capacity the real count mostly stays far below) gets about
// two CTAs per SM, so the launch does not spend SM time on empty CTAs.
int blocks_for_count(const Count& c, int threads) {
  return blocks_for(c.cap, threads, c.dev != nullptr ? 148 * 2 : 148 * 16);
}

__device__ __forceinline__ ConstEntryArrays offset_view(ConstEntryArrays e, uint64_t off) {
  return ConstEntryArrays{e.pos0 + off, e.pos1 + off, e.res_lo + off, e.res_hi + off};
}

__global__ void k_enumerate_half(const uint64_t* __restrict__ weights, uint32_t n, uint32_t second,
                                 uint64_t count, EntryArrays out) {
  const uint32_t half = n / 2, k = n / 36;
  const u128 mask = nmask128(n);
  for (uint64_t rank0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; rank0 < count;
       rank0 += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t rank = rank0;
    uint32_t c = 0;
    uint64_t p0 = 0, p1 = 0;
    u128 res = 0;
    for (uint32_t i = 0; i < k; ++i) {
      // the number of combinations whose i-th element is c is C(half - 1 - c, k - 1 - i)
      for (;;) {
        const uint64_t b = binom(half - 1 - c, k - 1 - i);
        if (rank < b) break;
        rank -= b;
        ++c;
      }
      const uint32_t coord = c + (second ? half : 0u);
      if (coord < 64) p0 |= 1ull << coord; else p1 |= 1ull << (coord - 64);
      res = (res + (((u128)weights[2 * coord + 1] << 64) | weights[2 * coord])) & mask;
      ++c;
    }
    out.pos0[rank0] = p0;
    out.pos1[rank0] = p1;
    out.res_lo[rank0] = (uint64_t)res;
    out.res_hi[rank0] = (uint64_t)(res >> 64);
  }
}

__global__ void k_bucket_hist(const uint64_t* __restrict__ res_lo, uint64_t n, uint32_t mask,
                              uint32_t* __restrict__ cnt) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    atomicAdd(&cnt[(uint32_t)res_lo[i] & mask], 1u);
  }
}

__global__ void k_bucket_scatter(const uint64_t* __restrict__ res_lo, uint64_t n, uint32_t mask,
                                 uint32_t* __restrict__ cur, uint32_t* __restrict__ order) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    order[atomicAdd(&cur[(uint32_t)res_lo[i] & mask], 1u)] = (uint32_t)i;
  }
}

__global__ void k_copy_u32(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i];
}

__global__ void k_l2_count(ConstEntryArrays left, uint64_t nl, const uint32_t* __restrict__ off,
                           uint32_t mask, uint64_t t, uint32_t* __restrict__ counts) {
  for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < nl;
       l += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t b = (uint32_t)(t - left.res_lo[l]) & mask;
    counts[l] = off[b + 1] - off[b];
  }
}

__global__ void k_l2_fill(ConstEntryArrays left, uint64_t nl, ConstEntryArrays right,
                          const uint32_t* __restrict__ off, const uint32_t* __restrict__ order,
                          uint32_t mask, uint64_t t, uint32_t n, const uint32_t* __restrict__ starts,
                          EntryArrays out) {
  const u128 nm = nmask128(n);
  for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < nl;
       l += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t b = (uint32_t)(t - left.res_lo[l]) & mask;
    const u128 rl = ((u128)left.res_hi[l] << 64) | left.res_lo[l];
    uint32_t at = starts[l];
    for (uint32_t k = off[b]; k < off[b + 1]; ++k, ++at) {
      const uint32_t r = order[k];
      const u128 rr = ((u128)right.res_hi[r] << 64) | right.res_lo[r];
      const u128 sum = (rl + rr) & nm;
      out.pos0[at] = left.pos0[l] | right.pos0[r];
      out.pos1[at] = left.pos1[l] | right.pos1[r];
      out.res_lo[at] = (uint64_t)sum;
      out.res_hi[at] = (uint64_t)(sum >> 64);
    }
  }
}

__global__ void k_l2_count_all(ConstEntryArrays left, uint64_t nl, const uint32_t* __restrict__ off,
                               uint32_t mask, MergeTargets t, const MergeTargets* __restrict__ dt,
                               uint32_t* __restrict__ counts) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < 9 * nl;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = (uint32_t)(x / nl);
    const uint64_t l = x - (uint64_t)m * nl;
    const uint64_t tm = dt != nullptr ? dt->t[m] : t.t[m];
    const uint32_t b = (uint32_t)(tm - left.res_lo[l]) & mask;
    counts[x] = off[b + 1] - off[b];
  }
}

__global__ void k_l2_bounds(const uint32_t* __restrict__ starts, uint64_t nl, uint32_t* __restrict__ bounds) {
  if (threadIdx.x < 10) bounds[threadIdx.x] = starts[(uint64_t)threadIdx.x * nl];
}

__global__ void k_l2_fill_all(ConstEntryArrays left, uint64_t nl, ConstEntryArrays right,
                              const uint32_t* __restrict__ off, const uint32_t* __restrict__ order,
                              uint32_t mask, MergeTargets t, const MergeTargets* __restrict__ dt,
                              uint32_t n, const uint32_t* __restrict__ starts, uint64_t cap,
                              EntryArrays out) {
  const u128 nm = nmask128(n);
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < 9 * nl;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = (uint32_t)(x / nl);
    const uint64_t l = x - (uint64_t)m * nl;
    const uint64_t tm = dt != nullptr ? dt->t[m] : t.t[m];
    const uint32_t b = (uint32_t)(tm - left.res_lo[l]) & mask;
    const u128 rl = ((u128)left.res_hi[l] << 64) | left.res_lo[l];
    uint32_t at = starts[x];
    for (uint32_t k = off[b]; k < off[b + 1] && at < cap; ++k, ++at) {
      const uint32_t r = order[k];
      const u128 rr = ((u128)right.res_hi[r] << 64) | right.res_lo[r];
      const u128 sum = (rl + rr) & nm;
      out.pos0[at] = left.pos0[l] | right.pos0[r];
      out.pos1[at] = left.pos1[l] | right.pos1[r];
      out.res_lo[at] = (uint64_t)sum;
      out.res_hi[at] = (uint64_t)(sum >> 64);
    }
  }
}

// One CTA of 1024 threads per segment: bitonic sort of (pos0, pos1, index) in
// shared memory (ties are identical digit vectors, so the order among them does
// not matter), then the first of every run of equal keys is kept, compacted in
// order.  Padding keys (all ones) sort last; no entry has all 64 bits of pos0 set.
__global__ void __launch_bounds__(1024) k_canon_small(ConstEntryArrays raw, Segments seg,
                                                      const uint32_t* __restrict__ dbounds, uint64_t cap,
                                                      EntryArrays out, unsigned long long* __restrict__ kept,
                                                      unsigned int* __restrict__ overflow) {
  extern __shared__ __align__(16) uint64_t csm[];
  uint64_t* k0 = csm;
  uint64_t* k1 = k0 + kCanonSmallCap;
  uint16_t* ix = reinterpret_cast<uint16_t*>(k1 + kCanonSmallCap);
  uint32_t* pos = reinterpret_cast<uint32_t*>(ix + kCanonSmallCap);
  __shared__ uint32_t warp_tot[32];
  const uint32_t s = blockIdx.x;
  const uint32_t m = dbounds != nullptr ? dbounds[s + 1] - dbounds[s] : seg.cnt[s];
  const uint32_t base = dbounds != nullptr ? dbounds[s] : seg.off[s];
  if (m > kCanonSmallCap || (uint64_t)base + m > cap) {  // only with device bounds: the caller falls back
    if (threadIdx.x == 0) {
      kept[s] = 0;
      if (overflow != nullptr) atomicOr(overflow, 1u);
    }
    return;
  }
  uint32_t p = 1;
  while (p < m) p <<= 1;
  for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) {
    const bool ok = i < m;
    k0[i] = ok ? raw.pos0[base + i] : ~0ull;
    k1[i] = ok ? raw.pos1[base + i] : ~0ull;
    ix[i] = (uint16_t)i;
  }
  __syncthreads();
  for (uint32_t k = 2; k <= p; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) {
        const uint32_t o = i ^ j;
        if (o > i) {
          const bool up = (i & k) == 0;
          const bool greater = k0[i] > k0[o] || (k0[i] == k0[o] && k1[i] > k1[o]);
          const bool less = k0[i] < k0[o] || (k0[i] == k0[o] && k1[i] < k1[o]);
          if (up ? greater : less) {
            const uint64_t a0 = k0[i], a1 = k1[i];
            const uint16_t ai = ix[i];
            k0[i] = k0[o];
            k1[i] = k1[o];
            ix[i] = ix[o];
            k0[o] = a0;
            k1[o] = a1;
            ix[o] = ai;
          }
        }
      }
      __syncthreads();
    }
  }
  // keep flags and their exclusive scan (four items per thread, in order)
  const uint32_t per = (kCanonSmallCap + blockDim.x - 1) / blockDim.x;
  const uint32_t begin = threadIdx.x * per;
  uint32_t local = 0;
  for (uint32_t i = begin; i < begin + per && i < m; ++i) {
    local += (i == 0 || k0[i] != k0[i - 1] || k1[i] != k1[i - 1]) ? 1u : 0u;
  }
  uint32_t v = local;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(kFull, v, d);
    if (lane >= (uint32_t)d) v += o;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < blockDim.x / 32 ? warp_tot[lane] : 0;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, w, d);
      if (lane >= (uint32_t)d) w += o;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  uint32_t run = v - local + (warp > 0 ? warp_tot[warp - 1] : 0);
  for (uint32_t i = begin; i < begin + per && i < m; ++i) {
    if (i == 0 || k0[i] != k0[i - 1] || k1[i] != k1[i - 1]) pos[run++] = ix[i];
  }
  __syncthreads();
  const uint32_t total = warp_tot[(blockDim.x / 32) - 1];
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
    const uint32_t src = base + pos[i];
    out.pos0[base + i] = raw.pos0[src];
    out.pos1[base + i] = raw.pos1[src];
    out.res_lo[base + i] = raw.res_lo[src];
    out.res_hi[base + i] = raw.res_hi[src];
  }
  if (threadIdx.x == 0) kept[s] = total;
}

// One CTA of 1024 threads: exclusive scan of n <= 65536 values; out[n] = total.
// Tiles of 8192 values pass through shared memory, so global reads and writes
// are coalesced; each thread scans 8 consecutive values of a tile (one pad
// word per 32 keeps those reads free of bank conflicts).
__global__ void __launch_bounds__(1024) k_scan_small(const uint32_t* __restrict__ in, uint32_t n,
                                                     uint32_t* __restrict__ out) {
  constexpr uint32_t kPer = 8, kTileN = 1024 * kPer;
  __shared__ uint32_t tile[kTileN + kTileN / 32];
  __shared__ uint32_t warp_tot[32];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t carry = 0;
  for (uint32_t base = 0; base < n; base += kTileN) {
    const uint32_t m = min(kTileN, n - base);
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      const uint32_t i = threadIdx.x + 1024u * k;
      tile[i + (i >> 5)] = i < m ? in[base + i] : 0u;
    }
    __syncthreads();
    uint32_t v[kPer];
    uint32_t local = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      const uint32_t i = threadIdx.x * kPer + k;
      v[k] = tile[i + (i >> 5)];
      local += v[k];
    }
    uint32_t x = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, x, d);
      if (lane >= (uint32_t)d) x += o;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = warp_tot[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(kFull, w, d);
        if (lane >= (uint32_t)d) w += o;
      }
      warp_tot[lane] = w;
    }
    __syncthreads();
    uint32_t run = carry + x - local + (warp > 0 ? warp_tot[warp - 1] : 0u);
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      const uint32_t i = threadIdx.x * kPer + k;
      tile[i + (i >> 5)] = run;
      run += v[k];
    }
    carry += warp_tot[31];
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      const uint32_t i = threadIdx.x + 1024u * k;
      if (i < m) out[base + i] = tile[i + (i >> 5)];
    }
    __syncthreads();  // the next tile reuses tile[] and warp_tot[]
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// ---- generic exclusive scan of uint32 (three kernels) ----------------------
__global__ void k_chunk_sums(const uint32_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t warp_tot[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t v = 0;
  for (uint32_t i = threadIdx.x; i < kScanChunk; i += blockDim.x) {
    if (base + i < n) v += in[base + i];
  }
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(kFull, v, d);
  if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += warp_tot[w];
    sums[blockIdx.x] = t;
  }
}

// One CTA: exclusive scan of nb chunk sums in place; sums[nb] = total.
__global__ void k_scan_sums(uint32_t* __restrict__ sums, uint32_t nb) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
  const uint32_t begin = threadIdx.x * per, end = min(nb, begin + per);
  uint32_t local = 0;
  for (uint32_t i = begin; i < end; ++i) local += sums[i];
  uint32_t v = local;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(kFull, v, d);
    if (lane >= (uint32_t)d) v += o;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < blockDim.x / 32 ? warp_tot[lane] : 0;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, w, d);
      if (lane >= (uint32_t)d) w += o;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  uint32_t run = v - local + (warp > 0 ? warp_tot[warp - 1] : 0);
  for (uint32_t i = begin; i < end; ++i) {
    const uint32_t c = sums[i];
    sums[i] = run;
    run += c;
  }
  if (threadIdx.x == blockDim.x - 1) sums[nb] = run;
}

// Each CTA (1024 threads, 2 items each) scans its chunk with the chunk's offset.
__global__ void k_chunk_scan(const uint32_t* __restrict__ in, uint64_t n, const uint32_t* __restrict__ sums,
                             uint32_t nb, uint32_t* __restrict__ out) {
  __shared__ uint32_t warp_tot[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk + 2ull * threadIdx.x;
  const uint32_t a0 = base < n ? in[base] : 0u;
  const uint32_t a1 = base + 1 < n ? in[base + 1] : 0u;
  const uint32_t local = a0 + a1;
  uint32_t v = local;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(kFull, v, d);
    if (lane >= (uint32_t)d) v += o;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_tot[lane];
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, w, d);
      if (lane >= (uint32_t)d) w += o;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  const uint32_t run = sums[blockIdx.x] + v - local + (warp > 0 ? warp_tot[warp - 1] : 0);
  if (base < n) out[base] = run;
  if (base + 1 < n) out[base + 1] = run + a0;
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[nb];
}

__global__ void k_l2_quotients(ConstEntryArrays l, Count cnt, const uint32_t* __restrict__ doff,
                               uint32_t b1, uint32_t r2, uint64_t t_lo, uint64_t t_hi, int negate,
                               uint64_t tau, const uint64_t* __restrict__ dvals,
                               uint64_t* __restrict__ key) {
  if (doff != nullptr) l = offset_view(l, *doff);
  if (dvals != nullptr) {
    t_lo = dvals[0];
    t_hi = dvals[1];
    tau = dvals[2];
  }
  const u128 m1 = nmask128(b1);
  const u128 t = (((u128)t_hi << 64) | t_lo) & m1;
  const uint64_t qmask = (b1 - r2) >= 64 ? ~0ull : ((1ull << (b1 - r2)) - 1ull);
  const uint64_t count = cnt.get();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const u128 r = (((u128)l.res_hi[i] << 64) | l.res_lo[i]) & m1;
    uint64_t q = (uint64_t)(((r - t) & m1) >> r2) & qmask;
    if (negate) q = (tau - q) & qmask;
    key[i] = q;
  }
}

__global__ void k_l1_parents(const uint32_t* __restrict__ triples, Count ntc, ConstEntryArrays x,
                             ConstEntryArrays y, ConstEntryArrays z, const uint32_t* __restrict__ doff,
                             uint32_t n, uint32_t ones, EntryArrays out,
                             unsigned long long* __restrict__ count,
                             unsigned long long* __restrict__ rejects) {
  if (doff != nullptr) {
    x = offset_view(x, doff[0]);
    y = offset_view(y, doff[1]);
    z = offset_view(z, doff[2]);
  }
  const u128 nm = nmask128(n);
  const uint64_t nt = ntc.get();
  unsigned long long c_struct = 0, c_dist = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nt;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = triples[3 * i], b = triples[3 * i + 1], c = triples[3 * i + 2];
    const uint64_t a0 = x.pos0[a], a1 = x.pos1[a], b0 = y.pos0[b], b1 = y.pos1[b];
    const uint64_t c0 = z.pos0[c], c1 = z.pos1[c];
    // binary digits: a coordinate set in two children leaves {-1, 0, 1}
    // (add_three's structural reject); then the digit counts (its distribution reject)
    const uint64_t two0 = (a0 & b0) | (a0 & c0) | (b0 & c0);
    const uint64_t two1 = (a1 & b1) | (a1 & c1) | (b1 & c1);
    const uint64_t p0 = a0 | b0 | c0, p1 = a1 | b1 | c1;
    if ((two0 | two1) != 0) {
      ++c_struct;
      continue;
    }
    if ((uint32_t)(__popcll(p0) + __popcll(p1)) != ones) {
      ++c_dist;
      continue;
    }
    const u128 s = ((((u128)x.res_hi[a] << 64) | x.res_lo[a]) + (((u128)y.res_hi[b] << 64) | y.res_lo[b]) +
                    (((u128)z.res_hi[c] << 64) | z.res_lo[c])) & nm;
    // the kept parents of the warp's current step take consecutive slots with one
    // atomic (their order is free: the canonical sort follows)
    const cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long at = 0;
    if (g.thread_rank() == 0) at = atomicAdd(count, static_cast<unsigned long long>(g.size()));
    at = g.shfl(at, 0) + g.thread_rank();
    out.pos0[at] = p0;
    out.pos1[at] = p1;
    out.res_lo[at] = (uint64_t)s;
    out.res_hi[at] = (uint64_t)(s >> 64);
  }
  if (rejects != nullptr) {
    for (int d = 16; d > 0; d >>= 1) {
      c_struct += __shfl_down_sync(0xFFFFFFFFu, c_struct, d);
      c_dist += __shfl_down_sync(0xFFFFFFFFu, c_dist, d);
    }
    if ((threadIdx.x & 31u) == 0u) {
      if (c_struct != 0) atomicAdd(&rejects[0], c_struct);
      if (c_dist != 0) atomicAdd(&rejects[1], c_dist);
    }
  }
}

// ---- stable LSD radix sort on (pos0, pos1) ---------------------------------
__global__ void k_radix_init(ConstEntryArrays in, Count cnt, uint64_t* khi, uint64_t* klo, uint32_t* idx) {
  const uint64_t n = cnt.get();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    khi[i] = in.pos0[i];
    klo[i] = in.pos1[i];
    idx[i] = (uint32_t)i;
  }
}

__device__ __forceinline__ uint32_t digit_of(uint64_t hi, uint64_t lo, uint32_t word, uint32_t shift) {
  return (uint32_t)(((word ? hi : lo) >> shift) & 255u);
}

// counts[d * nb + b]: items of digit d in tile b
__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const uint64_t* __restrict__ khi,
                                                              const uint64_t* __restrict__ klo, Count cnt,
                                                              uint32_t word, uint32_t shift, uint32_t nb,
                                                              uint32_t* __restrict__ counts) {
  __shared__ uint32_t hist[256];
  const uint64_t n = cnt.get();
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  if (base >= n) {  // a tile past the device count (grids are sized by capacity): zero counts
    counts[(uint64_t)threadIdx.x * nb + blockIdx.x] = 0;
    return;
  }
  hist[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < kTile; i += kRadixThreads) {
    if (base + i < n) atomicAdd(&hist[digit_of(khi[base + i], klo[base + i], word, shift)], 1u);
  }
  __syncthreads();
  counts[(uint64_t)threadIdx.x * nb + blockIdx.x] = hist[threadIdx.x];
}

// Stable scatter of one tile: warp w owns items [w*256, w*256+256) of the tile in
// rounds of 32 (item order == index order); equal digits are ranked with
// __match_any_sync, per-warp digit counts give the offsets between warps.
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(
    const uint64_t* __restrict__ khi, const uint64_t* __restrict__ klo, const uint32_t* __restrict__ idx,
    Count cnt, uint32_t word, uint32_t shift, uint32_t nb, const uint32_t* __restrict__ offsets,
    uint64_t* __restrict__ ohi, uint64_t* __restrict__ olo, uint32_t* __restrict__ oidx) {
  const uint64_t n = cnt.get();
  if ((uint64_t)blockIdx.x * kTile >= n) return;  // nothing to scatter (uniform per block)
  __shared__ uint32_t wcnt[kRadixThreads / 32][256];
  __shared__ uint32_t goff[256];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t d = lane; d < 256; d += 32) wcnt[warp][d] = 0;
  goff[threadIdx.x] = offsets[(uint64_t)threadIdx.x * nb + blockIdx.x];
  __syncwarp();
  const uint64_t base = (uint64_t)blockIdx.x * kTile + warp * 256u;
  uint64_t vh[kRadixItems], vl[kRadixItems];
  uint32_t vi[kRadixItems], dg[kRadixItems], rk[kRadixItems];
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    const uint64_t i = base + r * 32u + lane;
    const bool ok = i < n;
    vh[r] = ok ? khi[i] : 0;
    vl[r] = ok ? klo[i] : 0;
    vi[r] = ok ? idx[i] : 0;
    dg[r] = ok ? digit_of(vh[r], vl[r], word, shift) : 256u;
    const uint32_t peers = __match_any_sync(kFull, dg[r]);
    const uint32_t before = wcnt[warp][dg[r] & 255u];
    __syncwarp();
    rk[r] = before + __popc(peers & ((1u << lane) - 1u));
    if (ok && lane == (uint32_t)(__ffs(peers) - 1)) wcnt[warp][dg[r]] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // exclusive prefix over warps for digit d = threadIdx.x
  {
    uint32_t run = 0;
    for (uint32_t w = 0; w < kRadixThreads / 32; ++w) {
      const uint32_t c = wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    if (dg[r] < 256u) {
      const uint32_t pos = goff[dg[r]] + wcnt[warp][dg[r]] + rk[r];
      ohi[pos] = vh[r];
      olo[pos] = vl[r];
      oidx[pos] = vi[r];
    }
  }
}

__global__ void k_unique_flags(ConstEntryArrays in, const uint32_t* __restrict__ perm, Count cnt,
                               uint32_t* __restrict__ flags) {
  const uint64_t n = cnt.get();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt.cap;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (i >= n) {  // beyond a device count: nothing to keep (the scan runs to the bound)
      flags[i] = 0;
      continue;
    }
    const uint32_t p = perm[i];
    uint32_t keep = 1;
    if (i > 0) {
      const uint32_t q = perm[i - 1];
      keep = (in.pos0[p] != in.pos0[q] || in.pos1[p] != in.pos1[q]) ? 1u : 0u;
    }
    flags[i] = keep;
  }
}

__global__ void k_gather_kept(ConstEntryArrays in, const uint32_t* __restrict__ perm, Count cnt,
                              const uint32_t* __restrict__ flags, const uint32_t* __restrict__ starts,
                              EntryArrays out, unsigned long long* kept) {
  const uint64_t n = cnt.get();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (!flags[i]) continue;
    const uint32_t p = perm[i], at = starts[i];
    out.pos0[at] = in.pos0[p];
    out.pos1[at] = in.pos1[p];
    out.res_lo[at] = in.res_lo[p];
    out.res_hi[at] = in.res_hi[p];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *kept = starts[cnt.cap];
}

__global__ void k_or_reduce(ConstEntryArrays in, uint64_t n, unsigned long long* acc) {
  uint64_t a = 0, b = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    a |= in.pos0[i];
    b |= in.pos1[i];
  }
  for (int d = 16; d > 0; d >>= 1) {
    a |= __shfl_down_sync(kFull, a, d);
    b |= __shfl_down_sync(kFull, b, d);
  }
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicOr(&acc[0], (unsigned long long)a);
    if (b) atomicOr(&acc[1], (unsigned long long)b);
  }
}

__global__ void k_copy_count(const unsigned long long* __restrict__ src, unsigned long long* __restrict__ dst) {
  *dst = *src;
}

__global__ void k_pack_records(ConstEntryArrays in, Count cnt, uint32_t nbits, uint8_t* __restrict__ rec) {
  const uint64_t n = cnt.get();
  const uint32_t w64 = (nbits + 63) / 64, w32 = (nbits + 31) / 32;
  const uint32_t rb = 16 * w64 + 4 * w32;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t* w = reinterpret_cast<uint32_t*>(rec + i * rb);
    const uint64_t pos[2] = {in.pos0[i], in.pos1[i]};
    for (uint32_t k = 0; k < w64; ++k) {
      w[2 * k] = (uint32_t)pos[k];
      w[2 * k + 1] = (uint32_t)(pos[k] >> 32);
      w[2 * (w64 + k)] = 0u;
      w[2 * (w64 + k) + 1] = 0u;
    }
    const uint64_t res[2] = {in.res_lo[i], in.res_hi[i]};
    for (uint32_t k = 0; k < w32; ++k) w[4 * w64 + k] = (uint32_t)(res[k / 2] >> (32 * (k % 2)));
  }
}

}  // namespace

void launch_enumerate_half(const uint64_t* weights, uint32_t n, uint32_t second_half, uint64_t count,
                           EntryArrays out, cudaStream_t st) {
  k_enumerate_half<<<blocks_for(count, 256), 256, 0, st>>>(weights, n, second_half, count, out);
}

void launch_bucket_right(ConstEntryArrays right, uint64_t nr, uint32_t r2, uint32_t* bucket_cnt,
                         uint32_t* bucket_off, uint32_t* bucket_cur, uint32_t* order, cudaStream_t st) {
  const uint32_t nbk = 1u << r2;
  cudaMemsetAsync(bucket_cnt, 0, (nbk + 1) * 4ull, st);
  k_bucket_hist<<<blocks_for(nr, 256), 256, 0, st>>>(right.res_lo, nr, nbk - 1, bucket_cnt);
  // bucket_off[0..nbk] = exclusive scan (scratch: bucket_cur, at least nbk/2048 + 2 words)
  launch_scan_u32(bucket_cnt, nbk, bucket_off, bucket_cur + nbk + 1, st);
  k_copy_u32<<<blocks_for(nbk, 256), 256, 0, st>>>(bucket_off, nbk, bucket_cur);
  k_bucket_scatter<<<blocks_for(nr, 256), 256, 0, st>>>(right.res_lo, nr, nbk - 1, bucket_cur, order);
}

void launch_l2_count(ConstEntryArrays left, uint64_t nl, const uint32_t* bucket_off, uint32_t r2,
                     uint64_t t_lo, uint32_t* counts, cudaStream_t st) {
  k_l2_count<<<blocks_for(nl, 256), 256, 0, st>>>(left, nl, bucket_off, (1u << r2) - 1u, t_lo, counts);
}

void launch_l2_fill(ConstEntryArrays left, uint64_t nl, ConstEntryArrays right, const uint32_t* bucket_off,
                    const uint32_t* order, uint32_t r2, uint64_t t_lo, uint32_t n, const uint32_t* starts,
                    EntryArrays out, cudaStream_t st) {
  k_l2_fill<<<blocks_for(nl, 128), 128, 0, st>>>(left, nl, right, bucket_off, order, (1u << r2) - 1u, t_lo,
                                                 n, starts, out);
}

void launch_scan_u32(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* scratch, cudaStream_t st) {
  const uint32_t nb = (uint32_t)((n + kScanChunk - 1) / kScanChunk);
  if (nb == 0) {
    cudaMemsetAsync(out, 0, 4, st);
    return;
  }
  if (n <= 65536) {
    k_scan_small<<<1, 1024, 0, st>>>(in, (uint32_t)n, out);
    return;
  }
  k_chunk_sums<<<nb, 256, 0, st>>>(in, n, scratch);
  k_scan_sums<<<1, 1024, 0, st>>>(scratch, nb);
  k_chunk_scan<<<nb, 1024, 0, st>>>(in, n, scratch, nb, out);
}

void launch_l2_count_all(ConstEntryArrays left, uint64_t nl, const uint32_t* bucket_off, uint32_t r2,
                         const MergeTargets& t, uint32_t* counts, cudaStream_t st,
                         const MergeTargets* dt) {
  k_l2_count_all<<<blocks_for(9 * nl, 256), 256, 0, st>>>(left, nl, bucket_off, (1u << r2) - 1u, t, dt,
                                                          counts);
}

void launch_l2_bounds(const uint32_t* starts, uint64_t nl, uint32_t* bounds, cudaStream_t st) {
  k_l2_bounds<<<1, 32, 0, st>>>(starts, nl, bounds);
}

void launch_l2_fill_all(ConstEntryArrays left, uint64_t nl, ConstEntryArrays right,
                        const uint32_t* bucket_off, const uint32_t* order, uint32_t r2,
                        const MergeTargets& t, uint32_t n, const uint32_t* starts, EntryArrays out,
                        cudaStream_t st, const MergeTargets* dt, uint64_t cap) {
  k_l2_fill_all<<<blocks_for(9 * nl, 128), 128, 0, st>>>(left, nl, right, bucket_off, order,
                                                        (1u << r2) - 1u, t, dt, n, starts, cap, out);
}

void launch_canon_small(ConstEntryArrays raw, const Segments& seg, uint32_t nseg, EntryArrays out,
                        unsigned long long* kept, cudaStream_t st, const uint32_t* dbounds,
                        unsigned int* overflow, uint64_t cap) {
  if (nseg == 0) return;
  const size_t smem = kCanonSmallCap * (8 + 8 + 2 + 4);
  allow_max_smem(reinterpret_cast<const void*>(k_canon_small));
  k_canon_small<<<nseg, 1024, smem, st>>>(raw, seg, dbounds, cap, out, kept, overflow);
}

void prepare_attempt_kernels() {
  allow_max_smem(reinterpret_cast<const void*>(k_canon_small));
}

void launch_l2_quotients(ConstEntryArrays l, Count count, uint32_t b1, uint32_t r2, uint64_t t_lo,
                         uint64_t t_hi, int negate, uint64_t tau, uint64_t* key, cudaStream_t st,
                         const uint32_t* doff, const uint64_t* dvals) {
  if (count.cap == 0) return;
  k_l2_quotients<<<blocks_for_count(count, 256), 256, 0, st>>>(l, count, doff, b1, r2, t_lo, t_hi, negate,
                                                             tau, dvals, key);
}

void launch_l1_parents(const uint32_t* triples, Count ntriples, ConstEntryArrays x, ConstEntryArrays y,
                       ConstEntryArrays z, uint32_t n, uint32_t expected_ones, EntryArrays out,
                       unsigned long long* count, cudaStream_t st, const uint32_t* doff,
                       unsigned long long* rejects) {
  cudaMemsetAsync(count, 0, 8, st);
  if (rejects != nullptr) cudaMemsetAsync(rejects, 0, 16, st);
  if (ntriples.cap == 0) return;
  k_l1_parents<<<blocks_for_count(ntriples, 256), 256, 0, st>>>(triples, ntriples, x, y, z, doff, n,
                                                              expected_ones, out, count, rejects);
}

uint64_t radix_scratch_words(uint64_t count) {
  const uint64_t nb = (count + kTile - 1) / kTile;
  const uint64_t cells = 256 * nb;
  // keys ping-pong (4 x u64 = 8 words per item), idx ping-pong (2 words / item),
  // digit counts and offsets (cells + 1 each), scan scratch
  return count * 10 + 2 * (cells + 1) + cells / kScanChunk + 64;
}

void radix_sort_entries(ConstEntryArrays in, Count cnt, uint64_t vary_pos0, uint64_t vary_pos1,
                        uint32_t* perm_out, uint32_t* scratch, cudaStream_t st) {
  const uint64_t count = cnt.cap;
  if (count == 0) return;
  const uint32_t nb = (uint32_t)((count + kTile - 1) / kTile);
  const uint64_t cells = 256ull * nb;
  uint64_t* khi[2];
  uint64_t* klo[2];
  uint32_t* idx[2];
  uint64_t* w64 = reinterpret_cast<uint64_t*>(scratch);
  khi[0] = w64;
  klo[0] = w64 + count;
  khi[1] = w64 + 2 * count;
  klo[1] = w64 + 3 * count;
  uint32_t* w32 = reinterpret_cast<uint32_t*>(w64 + 4 * count);
  idx[0] = w32;
  idx[1] = w32 + count;
  uint32_t* counts = w32 + 2 * count;
  uint32_t* offsets = counts + cells + 1;
  uint32_t* scan_scratch = offsets + cells + 1;
  k_radix_init<<<blocks_for_count(cnt, 256), 256, 0, st>>>(in, cnt, khi[0], klo[0], idx[0]);
  int cur = 0;
  for (uint32_t word = 0; word < 2; ++word) {  // word 0: pos1 (less significant), word 1: pos0
    const uint64_t vary = word == 0 ? vary_pos1 : vary_pos0;
    for (uint32_t shift = 0; shift < 64; shift += 8) {
      if (((vary >> shift) & 255u) == 0) continue;  // digit constant (zero) in every key
      k_radix_hist<<<nb, kRadixThreads, 0, st>>>(khi[cur], klo[cur], cnt, word, shift, nb, counts);
      launch_scan_u32(counts, cells, offsets, scan_scratch, st);
      k_radix_scatter<<<nb, kRadixThreads, 0, st>>>(khi[cur], klo[cur], idx[cur], cnt, word, shift, nb,
                                                    offsets, khi[1 - cur], klo[1 - cur], idx[1 - cur]);
      cur = 1 - cur;
    }
  }
  cudaMemcpyAsync(perm_out, idx[cur], count * 4, cudaMemcpyDeviceToDevice, st);
}

void launch_gather_unique(ConstEntryArrays in, const uint32_t* perm, Count cnt, EntryArrays out,
                          uint32_t* flags, uint32_t* starts, uint32_t* scratch, unsigned long long* kept,
                          cudaStream_t st) {
  const uint64_t count = cnt.cap;
  if (count == 0) {
    cudaMemsetAsync(kept, 0, 8, st);
    return;
  }
  k_unique_flags<<<blocks_for_count(cnt, 256), 256, 0, st>>>(in, perm, cnt, flags);
  launch_scan_u32(flags, count, starts, scratch, st);
  k_gather_kept<<<blocks_for_count(cnt, 256), 256, 0, st>>>(in, perm, cnt, flags, starts, out, kept);
}

void launch_or_reduce(ConstEntryArrays in, uint64_t count, unsigned long long* acc, cudaStream_t st) {
  cudaMemsetAsync(acc, 0, 16, st);
  if (count == 0) return;
  k_or_reduce<<<blocks_for(count, 256), 256, 0, st>>>(in, count, acc);
}

void launch_copy_count(const unsigned long long* src, unsigned long long* dst, cudaStream_t st) {
  k_copy_count<<<1, 1, 0, st>>>(src, dst);
}

void launch_pack_records(ConstEntryArrays in, Count count, uint32_t n, uint8_t* records, cudaStream_t st) {
  if (count.cap == 0) return;
  k_pack_records<<<blocks_for_count(count, 256), 256, 0, st>>>(in, count, n, records);
}

}  // namespace tergpu
