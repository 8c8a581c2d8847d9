// tergpu_attempt_run: exact depth-3 TER attempts on the device (include/tergpu.h).
//
// Host side of the attempt loop: FiniteSanity parameters, per-attempt targets,
// the stage sequence and its memory preflight, witness selection and
// verification.  Device work: attempt_kernels.cu (levels 3..1) and the root
// join of root_kernels.cu / tergpu_api.cu.

#include "attempt_kernels.cuh"
#include "root_kernels.cuh"
#include "tergpu.h"
#include "tergpu_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <tuple>
#include <atomic>
#include <functional>
#include <thread>
#include <vector>

namespace tergpu {
namespace {

typedef unsigned __int128 u128;

u128 mask128(uint32_t bits) { return bits >= 128 ? ~(u128)0 : ((((u128)1) << bits) - 1); }

// ---- FiniteSanity parameters: r = floor(log2 R) / 2 with
// R1 = (n/2)! / ((n/6)!)^3 and R2 = (n/6)! / ((n/18)!)^3 (every epsilon zero;
// reference src/full_ter.cpp:2699-2759).  Exact small bignum arithmetic.
uint32_t floor_log2_multinomial3(uint32_t total, uint32_t part) {
  std::vector<uint32_t> w{1};
  auto mul = [&w](uint32_t m) {
    uint64_t carry = 0;
    for (auto& x : w) {
      const uint64_t t = (uint64_t)x * m + carry;
      x = (uint32_t)t;
      carry = t >> 32;
    }
    if (carry) w.push_back((uint32_t)carry);
  };
  auto div = [&w](uint32_t d) {
    uint64_t rem = 0;
    for (size_t i = w.size(); i-- > 0;) {
      const uint64_t cur = (rem << 32) | w[i];
      w[i] = (uint32_t)(cur / d);
      rem = cur % d;
    }
    while (w.size() > 1 && w.back() == 0) w.pop_back();
  };
  for (uint32_t i = 2; i <= total; ++i) mul(i);
  for (int copy = 0; copy < 3; ++copy)
    for (uint32_t i = 2; i <= part; ++i) div(i);
  uint32_t top = w.back(), bits = 0;
  while (top >>= 1) ++bits;
  return (uint32_t)(w.size() - 1) * 32 + bits;
}

// ---- targets of one attempt: SplitMix64(seed), one draw per 32-bit word, even
// words take the low half (src/full_ter.cpp:519-532, 2364-2386).
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  u128 residue(uint32_t bits) {
    const uint32_t words = (bits + 31) / 32;
    u128 v = 0;
    for (uint32_t i = 0; i < words; ++i) {
      const uint64_t r = next();
      v |= ((u128)(uint32_t)(i % 2 == 0 ? r : r >> 32)) << (32 * i);
    }
    return v & mask128(bits);
  }
};

struct Targets {
  u128 t1[3];
  u128 t2[9];
};

Targets random_targets(uint64_t seed, uint32_t r1, uint32_t r2, u128 T) {
  SplitMix rng{seed};
  Targets t;
  t.t1[0] = rng.residue(r1);
  t.t1[1] = rng.residue(r1);
  t.t1[2] = (T - t.t1[0] - t.t1[1]) & mask128(r1);
  for (int g = 0; g < 3; ++g) {
    t.t2[3 * g] = rng.residue(r2);
    t.t2[3 * g + 1] = rng.residue(r2);
    t.t2[3 * g + 2] = (t.t1[g] - t.t2[3 * g] - t.t2[3 * g + 1]) & mask128(r2);
  }
  return t;
}

// GuidedPlanted targets (TerTargetMode::GuidedPlanted): the planted root's
// half-balanced decomposition (build_guided_tree, src/full_ter.cpp:2230-2317)
// into three level-1 vectors -- in each half the root's ones, in coordinate
// order, go n/12 to each child -- and nine level-2 vectors -- each level-1
// vector's ones in each half go n/36 to each of its three children (FiniteSanity
// shapes have no -1 digits, so the decomposition's other patterns are empty);
// each target is its vector's residue masked to r1 or r2 bits (guided_targets,
// src/full_ter.cpp:2412-2428).  False when the planted root is not binary with
// n/4 ones in each half.
bool guided_targets(const uint8_t* planted, uint32_t n, uint32_t r1, uint32_t r2, const uint64_t* values_le,
                    Targets* t, std::vector<std::vector<uint8_t>>* level2 = nullptr) {
  if (planted == nullptr) return false;
  const uint32_t w64 = (n + 63) / 64;
  for (uint32_t half = 0; half < 2; ++half) {
    uint32_t ones = 0;
    for (uint32_t c = half * n / 2; c < (half + 1) * n / 2; ++c) {
      if (planted[c] > 1) return false;
      ones += planted[c];
    }
    if (ones != n / 4) return false;
  }
  // deal each half's set coordinates of `parent` out to three children, `per` each
  auto split = [n](const std::vector<uint8_t>& parent, uint32_t per) {
    std::array<std::vector<uint8_t>, 3> kids;
    for (auto& k : kids) k.assign(n, 0);
    for (uint32_t half = 0; half < 2; ++half) {
      uint32_t seen = 0;
      for (uint32_t c = half * n / 2; c < (half + 1) * n / 2; ++c) {
        if (parent[c] == 0) continue;
        kids[std::min<uint32_t>(seen / per, 2)][c] = 1;
        ++seen;
      }
    }
    return kids;
  };
  const u128 nm = mask128(n);
  auto residue = [&](const std::vector<uint8_t>& v) {
    u128 s = 0;
    for (uint32_t c = 0; c < n; ++c) {
      if (v[c] == 0) continue;
      u128 w = values_le[c * w64];
      if (w64 > 1) w |= (u128)values_le[c * w64 + 1] << 64;
      s = (s + w) & nm;
    }
    return s;
  };
  const std::vector<uint8_t> root(planted, planted + n);
  const auto l1 = split(root, n / 12);
  for (int g = 0; g < 3; ++g) {
    t->t1[g] = residue(l1[g]) & mask128(r1);
    const auto l2 = split(l1[g], n / 36);
    for (int k = 0; k < 3; ++k) {
      t->t2[3 * g + k] = residue(l2[k]) & mask128(r2);
      if (level2 != nullptr) level2->push_back(l2[k]);
    }
  }
  return true;
}

uint64_t binom_host(uint32_t m, uint32_t k) {
  if (k > m) return 0;
  uint64_t r = 1;
  for (uint32_t i = 0; i < k; ++i) r = r * (m - i) / (i + 1);
  return r;
}

enum : int {
  S_L3 = kAttemptSlotBase,        // +0..+7: left and right halves
  S_WEIGHTS = S_L3 + 8,
  S_BCNT, S_BOFF, S_BCUR, S_ORDER,
  S_L2RAW,                        // +0..+3
  S_L2CNT = S_L2RAW + 4, S_L2START, S_SCAN,
  S_L2 = S_SCAN + 1,              // 9 lists x 4 arrays
  S_SORT = S_L2 + 36, S_PERM, S_FLAGS, S_STARTS, S_SCAN2, S_ACC,
  S_KEYS,                         // +0..+2
  S_CAND = S_KEYS + 3,            // +0..+3
  S_L1 = S_CAND + 4,              // 3 lists x 4 arrays
  S_REC = S_L1 + 12,              // +0..+2
  S_RKLO = S_REC + 3,             // +0..+2
  S_RKHI = S_RKLO + 3,            // +0..+2
  S_AFLAGS = S_RKHI + 3, S_ACOUNT, S_BOUNDS, S_KEPT9
};

EntryArrays entry_slot(Workspace& w, int slot, uint64_t count) {
  const size_t b = (count + 16) * 8;
  return EntryArrays{ensure<uint64_t>(w, slot, b), ensure<uint64_t>(w, slot + 1, b),
                     ensure<uint64_t>(w, slot + 2, b), ensure<uint64_t>(w, slot + 3, b)};
}

ConstEntryArrays as_const(const EntryArrays& e) {
  return ConstEntryArrays{e.pos0, e.pos1, e.res_lo, e.res_hi};
}

// Entries [off, ...) of a list, as a list of their own.
EntryArrays view(const EntryArrays& e, uint64_t off) {
  return EntryArrays{e.pos0 + off, e.pos1 + off, e.res_lo + off, e.res_hi + off};
}

template <typename T>
void download(Workspace& w, T* dst, const T* src, size_t n, cudaStream_t st) {
  check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, st), "download");
  sync_stream(w, st, "sync");
}

// Canonical order of `count` entries in `raw`: radix sort + unique into `dst`
// (room for `count` entries).
uint64_t canonicalize(Workspace& w, const EntryArrays& raw, uint64_t count, const EntryArrays& dst,
                      cudaStream_t st) {
  unsigned long long* acc = ensure<unsigned long long>(w, S_ACC, 64);
  if (count == 0) return 0;
  launch_or_reduce(as_const(raw), count, acc, st);
  unsigned long long vary[2];
  download(w, vary, acc, 2, st);
  uint32_t* scratch = ensure<uint32_t>(w, S_SORT, radix_scratch_words(count) * 4);
  uint32_t* perm = ensure<uint32_t>(w, S_PERM, (count + 16) * 4);
  radix_sort_entries(as_const(raw), count, vary[0], vary[1], perm, scratch, st);
  uint32_t* flags = ensure<uint32_t>(w, S_FLAGS, (count + 16) * 4);
  uint32_t* starts = ensure<uint32_t>(w, S_STARTS, (count + 16) * 4);
  uint32_t* scan2 = ensure<uint32_t>(w, S_SCAN2, (count / 2048 + 64) * 4);
  launch_gather_unique(as_const(raw), perm, count, dst, flags, starts, scan2, acc + 2, st);
  unsigned long long kept = 0;
  download(w, &kept, acc + 2, 1, st);
  return kept;
}

void cancelled_check(const tergpu_attempt_in* in) {
  if (in->cancel != nullptr && *in->cancel != 0) {
    t_error = "full TER execution was cancelled";
    throw Failure{TERGPU_CANCELLED};
  }
}

// Mirrors the caller's host cancel flag into the workspace's cancel word while
// the call runs, so the sweep kernels (which read only device-visible memory)
// stop within a few work items of a cancel instead of at the next stage.
class CancelMirror {
 public:
  CancelMirror(const volatile int32_t* src, volatile int* dst) : src_(src), dst_(dst) {
    if (src_ == nullptr || dst_ == nullptr) return;
    thread_ = std::thread([this] {
      while (!done_.load(std::memory_order_relaxed)) {
        if (*src_ != 0) *dst_ = 1;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
      }
    });
  }
  ~CancelMirror() {
    done_.store(true);
    if (thread_.joinable()) thread_.join();
  }
  CancelMirror(const CancelMirror&) = delete;
  CancelMirror& operator=(const CancelMirror&) = delete;

 private:
  const volatile int32_t* src_;
  volatile int* dst_;
  std::atomic<bool> done_{false};
  std::thread thread_;
};

double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

// ---- graph mode: one attempt as one captured CUDA graph (n = 36 and 72) ----
//
// Every size-dependent step reads its counts on the device (Count) and works in
// fixed-capacity buffers owned by the plan, so an attempt is a fixed sequence
// of launches: captured once per workspace and shape, replayed per attempt
// after the attempt's values (targets) are copied into a device parameter
// block.  The kernels and their order are those of the stage-by-stage path; a
// capacity that would overflow is flagged on the device and that attempt runs
// again on the stage-by-stage path, so results are identical either way.

struct GraphParams {
  MergeTargets t2;        // L3 -> L2 targets mod 2^r2
  uint64_t q[9][3];       // L2 list 3g + l of the ternary merge: {t_lo, t_hi, tau_g}
  uint64_t rk[3][4];      // L1 list l: {child_lo, child_hi, tau_lo, tau_hi} of the root keys
  uint64_t root[2];       // T
};

struct GraphCounts {      // device counts the host reads after an attempt
  uint32_t bounds[10];    // raw L2 list boundaries (bounds[9]: L3 -> L2 pairs)
  unsigned long long kept9[9];
  unsigned long long l2_triples[3];
  unsigned long long ncand[3];
  unsigned long long l1[3];
  unsigned long long root_counters[kCounters];
  unsigned long long auth[3];
  unsigned long long l1rej[3][2];  // per group: structural, distribution rejects
  unsigned int overflow;  // a segment above the canonical-sort capacity
};

struct GraphPlan {
  uint32_t n = 0, r1 = 0, r2 = 0;
  uint64_t l3 = 0, cap_l2 = 0, cap_t = 0, cap_r = 0;
  Tuning tu_l2{}, tu_root{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // buffers
  EntryArrays left{}, right{}, raw{}, l2all{}, cand{}, l1[3]{};
  uint64_t* d_weights = nullptr;
  uint32_t *bcnt = nullptr, *boff = nullptr, *bcur = nullptr, *order = nullptr;
  uint32_t *counts = nullptr, *starts = nullptr, *scan = nullptr;
  uint64_t* keys[3]{};
  JoinBuffers jb{};
  uint32_t* sort_scratch = nullptr;
  uint32_t *perm = nullptr, *flags = nullptr, *starts2 = nullptr, *scan2 = nullptr;
  uint8_t* recs[3]{};
  uint64_t* rk_lo[3]{};
  uint8_t* rk_hi[3]{};
  uint8_t* aflags = nullptr;
  const volatile int* cancel = nullptr;  // the workspace's cancel word (device view)
  GraphParams* d_params = nullptr;
  GraphParams* h_params = nullptr;  // pinned
  GraphCounts* d_counts = nullptr;
  GraphCounts* h_counts = nullptr;  // pinned
  uint32_t* h_triples = nullptr;    // pinned, cap_r * 3
  uint8_t* h_aflags = nullptr;      // pinned, cap_r
  uint64_t bytes = 0;

  char* base = nullptr;  // one device allocation holds every buffer (null: size only)

  template <typename T>
  T* alloc(uint64_t count) {
    const uint64_t b = (std::max<uint64_t>(count * sizeof(T), 256) + 255) & ~255ull;
    const uint64_t at = bytes;
    bytes += b;
    return base != nullptr ? reinterpret_cast<T*>(base + at) : nullptr;
  }
  EntryArrays entries(uint64_t count) {
    return EntryArrays{alloc<uint64_t>(count + 16), alloc<uint64_t>(count + 16), alloc<uint64_t>(count + 16),
                       alloc<uint64_t>(count + 16)};
  }
  ~GraphPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (base) cudaFree(base);
    if (h_params) cudaFreeHost(h_params);
    if (h_counts) cudaFreeHost(h_counts);
    if (h_triples) cudaFreeHost(h_triples);
    if (h_aflags) cudaFreeHost(h_aflags);
  }
};

// ---- the reference's telemetry hashes (src/full_ter.cpp:2431-2577): a chain
// hash ^= value, hash *= 1099511628211 from 1469598103934665603 over 64-bit values.
struct Fnv64 {
  uint64_t h = 1469598103934665603ULL;
  void mix(uint64_t v) {
    h ^= v;
    h *= 1099511628211ULL;
  }
};

// One BigEntry of stage_fingerprint: digits.n, the packed digit words (W64
// positive then W64 negative, all zero at FiniteSanity), then the residue's
// 32-bit words without the zero words above the top one (BigInt keeps none).
void mix_entry(Fnv64& f, uint32_t n, uint64_t pos0, uint64_t pos1, u128 res) {
  const uint32_t w64 = (n + 63) / 64;
  f.mix(n);
  f.mix(pos0);
  if (w64 > 1) f.mix(pos1);
  for (uint32_t k = 0; k < w64; ++k) f.mix(0);
  uint32_t words = 4;
  while (words > 0 && (uint32_t)(res >> (32 * (words - 1))) == 0) --words;
  for (uint32_t k = 0; k < words; ++k) f.mix((uint32_t)(res >> (32 * k)));
}

// stage_fingerprint of `count` device lists in canonical order: each list's
// size, then its entries (downloaded to the host; the chain is sequential).
uint64_t lists_fingerprint(Workspace& w, uint32_t n, const EntryArrays* lists, const uint64_t* sizes,
                           int count, cudaStream_t st) {
  Fnv64 f;
  std::vector<uint64_t> p0, p1, rl, rh;
  for (int l = 0; l < count; ++l) {
    const uint64_t m = sizes[l];
    f.mix(m);
    if (m == 0) continue;
    p0.resize(m);
    p1.resize(m);
    rl.resize(m);
    rh.resize(m);
    check(cudaMemcpyAsync(p0.data(), lists[l].pos0, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(p1.data(), lists[l].pos1, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(rl.data(), lists[l].res_lo, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(rh.data(), lists[l].res_hi, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    sync_stream(w, st, "fingerprint");
    for (uint64_t i = 0; i < m; ++i) mix_entry(f, n, p0[i], p1[i], ((u128)rh[i] << 64) | rl[i]);
  }
  return f.h;
}

// The root's prefilter width and tile bits: min(24, Q, 32) and min(15, p)
// (src/full_ter.cpp:1681-1686, include/ter/limitations.hpp:563-570).
uint32_t root_prefilter_bits(uint32_t Q) { return std::min<uint32_t>(std::min<uint32_t>(24, Q), 32); }
uint32_t root_tile_bits(uint32_t p) { return std::min<uint32_t>(15, p); }

// Position of a root triple in the reference's tiled visit order (see
// VisitBound): window m, bucket i of A, A's and B's EntryIds, then C's EntryId
// descending.
struct VisitKey {
  uint32_t m, i, a, b, c;
  bool before(const VisitKey& o) const {
    if (m != o.m) return m < o.m;
    if (i != o.i) return i < o.i;
    if (a != o.a) return a < o.a;
    if (b != o.b) return b < o.b;
    return c > o.c;
  }
};

// The root's outcome under the attempt's policy, from its full-Q triples and
// their authority flags (k_authority): the retained parents (canonical order)
// and the reference's root counters (the visitor's, src/full_ter.cpp:1537-1622).
struct RootOutcome {
  uint64_t modular = 0, structural = 0, distribution = 0, valid = 0;
  bool stopped = false;  // FirstWitness stopped at `stop`
  VisitKey stop{};
  std::vector<std::array<uint64_t, 2>> parents;
};

RootOutcome pick_root(Workspace& w, cudaStream_t st, uint32_t n, uint32_t Q, uint32_t policy,
                      const uint32_t* trip, const uint8_t* flags, uint64_t count, const uint64_t* d_key_a,
                      const uint64_t* d_key_b, uint8_t* const recs[3], uint32_t rb) {
  const uint32_t w64 = (n + 63) / 64;
  RootOutcome o;
  std::vector<uint64_t> mod;  // the visitor's modular candidates
  for (uint64_t i = 0; i < count; ++i) {
    if ((flags[i] & 1) != 0) {
      mod.push_back(i);
    } else if (Q <= 64) {
      // a decisive quotient match always has the exact residue
      t_error = "root triple with a full quotient match but another residue";
      throw Failure{TERGPU_INVARIANT_VIOLATION};
    }
  }
  auto parent_of = [&](uint64_t i) {
    std::array<uint64_t, 2> p{0, 0};
    for (int l = 0; l < 3; ++l) {
      uint32_t wds[4] = {0, 0, 0, 0};  // the record's pos words (w64 <= 2)
      // on the attempt's own stream: the legacy default stream is shared by every
      // thread of the process (the batch engine's other slots included)
      check(cudaMemcpyAsync(wds, recs[l] + (uint64_t)trip[3 * i + l] * rb, w64 * 8, cudaMemcpyDeviceToHost,
                            st),
            "record download");
      sync_stream(w, st, "record download");
      p[0] |= (uint64_t)wds[0] | ((uint64_t)wds[1] << 32);
      if (w64 > 1) p[1] |= (uint64_t)wds[2] | ((uint64_t)wds[3] << 32);
    }
    return p;
  };
  bool any_valid = false;
  for (uint64_t i : mod) any_valid = any_valid || (flags[i] & 4) != 0;
  std::vector<uint64_t> counted = mod;
  if (policy == TERGPU_ROOT_POLICY_FIRST_WITNESS && any_valid) {
    const uint32_t p = root_prefilter_bits(Q), tb = root_tile_bits(p);
    const uint64_t pm = (1ull << p) - 1ull;
    std::vector<VisitKey> keys(mod.size());
    int64_t first = -1;
    for (size_t k = 0; k < mod.size(); ++k) {
      const uint64_t i = mod[k];
      uint64_t ka = 0, kb = 0;
      check(cudaMemcpyAsync(&ka, d_key_a + trip[3 * i], 8, cudaMemcpyDeviceToHost, st), "key download");
      check(cudaMemcpyAsync(&kb, d_key_b + trip[3 * i + 1], 8, cudaMemcpyDeviceToHost, st), "key download");
      sync_stream(w, st, "key download");
      const uint32_t bi = (uint32_t)((ka & pm) >> tb);
      keys[k] = VisitKey{bi + (uint32_t)((kb & pm) >> tb), bi, trip[3 * i], trip[3 * i + 1], trip[3 * i + 2]};
      if ((flags[i] & 4) != 0 && (first < 0 || keys[k].before(keys[first]))) first = (int64_t)k;
    }
    o.stopped = true;
    o.stop = keys[first];
    counted.clear();
    for (size_t k = 0; k < mod.size(); ++k)
      if (!o.stop.before(keys[k])) counted.push_back(mod[k]);  // visited up to the stop
    o.parents.push_back(parent_of(mod[first]));
  }
  o.modular = counted.size();
  for (uint64_t i : counted) {
    o.structural += (flags[i] >> 3) & 1;
    o.distribution += (flags[i] >> 4) & 1;
    o.valid += (flags[i] >> 2) & 1;
  }
  if (o.stopped) {
    o.valid = 1;
  } else if (policy == TERGPU_ROOT_POLICY_FULL_CANONICAL) {
    for (uint64_t i : counted)
      if ((flags[i] & 4) != 0) o.parents.push_back(parent_of(i));
    std::sort(o.parents.begin(), o.parents.end());
    o.parents.erase(std::unique(o.parents.begin(), o.parents.end()), o.parents.end());
  }
  return o;
}

// ---- audit (TERGPU_ATTEMPT_AUDIT): the reference's scalar oracles per stage
// (binary_oracle and ternary_oracle, src/full_ter.cpp:2061-2160, compared with
// the optimized stages at :3186-3222, :3318-3334 and :3449-3465).  Where a
// stage's oracle work is at most kAuditCap pairs or triples (the reference's
// kCubicCandidateTripleCap, include/ter/limitations.hpp:89), its device output
// is recomputed on the host by plain enumeration of the stage's inputs and
// compared: the canonical output list and the provenance -- which children
// made each output (the L3 -> L2 merge's raw parents, the ternary merges' and
// the root's index triples with their decisions).  A difference is
// InvariantViolation, as in the reference.
constexpr uint64_t kAuditCap = 1000000;

struct HostEntry {
  uint64_t p0, p1;
  u128 res;
  bool operator<(const HostEntry& o) const {
    if (p0 != o.p0) return p0 < o.p0;
    if (p1 != o.p1) return p1 < o.p1;
    return res < o.res;
  }
  bool operator==(const HostEntry& o) const { return p0 == o.p0 && p1 == o.p1 && res == o.res; }
};

std::vector<HostEntry> host_entries(Workspace& w, const EntryArrays& e, uint64_t m, cudaStream_t st) {
  std::vector<uint64_t> p0(m), p1(m), rl(m), rh(m);
  if (m != 0) {
    check(cudaMemcpyAsync(p0.data(), e.pos0, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(p1.data(), e.pos1, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(rl.data(), e.res_lo, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    check(cudaMemcpyAsync(rh.data(), e.res_hi, m * 8, cudaMemcpyDeviceToHost, st), "d2h");
    sync_stream(w, st, "audit download");
  }
  std::vector<HostEntry> v(m);
  for (uint64_t i = 0; i < m; ++i) v[i] = HostEntry{p0[i], p1[i], ((u128)rh[i] << 64) | rl[i]};
  return v;
}

// Canonical order (digit words ascending, pos0 first) without repeated digits.
std::vector<HostEntry> canonical_entries(std::vector<HostEntry> v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end(),
                      [](const HostEntry& a, const HostEntry& b) { return a.p0 == b.p0 && a.p1 == b.p1; }),
          v.end());
  return v;
}

[[noreturn]] void audit_failed(const char* what) {
  t_error = std::string("audit: ") + what + " disagrees with the scalar oracle";
  throw Failure{TERGPU_INVARIANT_VIOLATION};
}

// L3 -> L2 merge: every pair (a of the left half, b of the right half) with
// res_a + res_b = t (mod 2^r2), binary digits (disjoint supports) and n/18 ones.
// The device's raw parents (one per matching pair) and its canonical list.
void audit_binary(uint32_t n, uint32_t r2, u128 t, const std::vector<HostEntry>& left,
                  const std::vector<HostEntry>& right, std::vector<HostEntry> raw_dev,
                  const std::vector<HostEntry>& canon_dev) {
  const u128 nm = mask128(n), m2 = mask128(r2);
  std::vector<HostEntry> raw;
  for (const HostEntry& a : left) {
    for (const HostEntry& b : right) {
      const u128 s = (a.res + b.res) & nm;
      if (((s - t) & m2) != 0) continue;
      if (((a.p0 & b.p0) | (a.p1 & b.p1)) != 0) continue;
      const uint64_t p0 = a.p0 | b.p0, p1 = a.p1 | b.p1;
      if ((uint32_t)(__builtin_popcountll(p0) + __builtin_popcountll(p1)) != n / 18) continue;
      raw.push_back(HostEntry{p0, p1, s});
    }
  }
  std::sort(raw.begin(), raw.end());
  std::sort(raw_dev.begin(), raw_dev.end());
  if (raw != raw_dev) audit_failed("an L3 -> L2 merge's parents (provenance)");
  if (canonical_entries(std::move(raw)) != canon_dev) audit_failed("an L3 -> L2 list");
}

struct Triple {
  uint32_t a, b, c;
  bool operator<(const Triple& o) const {
    return std::tie(a, b, c) < std::tie(o.a, o.b, o.c);
  }
  bool operator==(const Triple& o) const { return a == o.a && b == o.b && c == o.c; }
};

// A ternary merge: every triple with res_a + res_b + res_c = t (mod 2^bits)
// (the candidates), and among them those with disjoint supports (else a
// structural reject) and `ones` ones (else a distribution reject): the parents.
struct TernaryOracle {
  std::vector<Triple> candidates;
  std::vector<uint8_t> decision;  // 0 parent, 1 structural reject, 2 distribution reject
  std::vector<HostEntry> parents;
};

TernaryOracle ternary_oracle(uint32_t n, uint32_t bits, u128 t, uint32_t ones, const std::vector<HostEntry>& A,
                             const std::vector<HostEntry>& B, const std::vector<HostEntry>& C) {
  const u128 nm = mask128(n), mb = mask128(bits);
  TernaryOracle o;
  for (uint32_t i = 0; i < A.size(); ++i) {
    for (uint32_t j = 0; j < B.size(); ++j) {
      const u128 ab = A[i].res + B[j].res;
      for (uint32_t k = 0; k < C.size(); ++k) {
        const u128 s = (ab + C[k].res) & nm;
        if (((s - t) & mb) != 0) continue;
        o.candidates.push_back(Triple{i, j, k});
        const uint64_t two0 = (A[i].p0 & B[j].p0) | (A[i].p0 & C[k].p0) | (B[j].p0 & C[k].p0);
        const uint64_t two1 = (A[i].p1 & B[j].p1) | (A[i].p1 & C[k].p1) | (B[j].p1 & C[k].p1);
        const uint64_t p0 = A[i].p0 | B[j].p0 | C[k].p0, p1 = A[i].p1 | B[j].p1 | C[k].p1;
        if ((two0 | two1) != 0) {
          o.decision.push_back(1);
        } else if ((uint32_t)(__builtin_popcountll(p0) + __builtin_popcountll(p1)) != ones) {
          o.decision.push_back(2);
        } else {
          o.decision.push_back(0);
          o.parents.push_back(HostEntry{p0, p1, s});
        }
      }
    }
  }
  return o;
}

bool cubic_fits(uint64_t a, uint64_t b, uint64_t c) {
  return a == 0 || b == 0 || c == 0 || (a * b <= kAuditCap && a * b * c <= kAuditCap);
}

// stage_fingerprint of the retained L0 parents: each parent's digits and the
// root target as its residue (every retained parent is residue-exact).
uint64_t l0_fingerprint(uint32_t n, const std::vector<std::array<uint64_t, 2>>& parents, u128 T) {
  Fnv64 f;
  f.mix(parents.size());
  for (const auto& p : parents) mix_entry(f, n, p[0], p[1], T);
  return f.h;
}

// Expected level sizes of the FiniteSanity shape (the preflight's means).
double expected_l1(uint64_t l3, uint32_t r1, uint32_t r2) {
  const double l2 = (double)l3 * l3 / std::ldexp(1.0, r2);
  return l2 * l2 * l2 / std::ldexp(1.0, r1 - r2) * 0.3;
}

// The capture: the stage-by-stage path's launches with device counts.
void capture_attempt(GraphPlan& g, cudaStream_t st) {
  const uint32_t n = g.n, r1 = g.r1, r2 = g.r2;
  const uint64_t l3 = g.l3;
  const uint32_t w64 = (n + 63) / 64, w32 = (n + 31) / 32;
  const uint32_t rb = 16 * w64 + 4 * w32;
  GraphCounts* dc = g.d_counts;
  GraphParams* dp = g.d_params;
  MergeTargets none{};
  uint32_t launches = 0;
  check(cudaMemsetAsync(&dc->overflow, 0, sizeof(unsigned int), st), "memset");
  // L3 -> L2
  launch_l2_count_all(as_const(g.left), l3, g.boff, r2, none, g.counts, st, &dp->t2);
  launch_scan_u32(g.counts, 9 * l3, g.starts, g.scan, st);
  launch_l2_bounds(g.starts, l3, dc->bounds, st);
  launch_l2_fill_all(as_const(g.left), l3, as_const(g.right), g.boff, g.order, r2, none, n, g.starts, g.raw, st,
                     &dp->t2, 9 * g.cap_l2);
  Segments seg{};
  launch_canon_small(as_const(g.raw), seg, 9, g.l2all, dc->kept9, st, dc->bounds, &dc->overflow,
                     9 * g.cap_l2);
  // L2 -> L1: three ternary joins on the projected quotient
  const uint32_t b1 = std::min(r1, r2 + 32);
  const uint32_t qbits = b1 - r2;
  const uint64_t vary0 = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  const uint64_t vary1 = n > 64 ? ((1ull << (n - 64)) - 1ull) : 0ull;
  for (int grp = 0; grp < 3; ++grp) {
    JoinWork jw{};
    for (int l = 0; l < 3; ++l) {
      const int li = 3 * grp + l;
      launch_l2_quotients(as_const(g.l2all), Count(g.cap_l2, &dc->kept9[li]), b1, r2, 0, 0, l == 2, 0,
                          g.keys[l], st, &dc->bounds[li], dp->q[li]);
      jw.key_lo[l] = g.keys[l];
      jw.key_hi[l] = nullptr;
      jw.id[l] = nullptr;
      jw.count[l] = Count(g.cap_l2, &dc->kept9[li]);
    }
    jw.quotient_bits = qbits;
    jw.cells = nullptr;
    jw.shard = 0;
    jw.shards = 1;
    jw.cap = g.cap_t;
    jw.main_sweep = true;
    jw.projected_bits = 0;
    jw.cancel = g.cancel;
    enqueue_join(g.jb, jw, g.tu_l2, nullptr, st, &launches);
    launch_copy_count(&g.jb.counters[kTriples], &dc->l2_triples[grp], st);
    launch_l1_parents(g.jb.triples, Count(g.cap_t, &g.jb.counters[kTriples]), as_const(g.l2all),
                      as_const(g.l2all), as_const(g.l2all), n, n / 6, g.cand, &dc->ncand[grp], st,
                      &dc->bounds[3 * grp], dc->l1rej[grp]);
    radix_sort_entries(as_const(g.cand), Count(g.cap_t, &dc->ncand[grp]), vary0, vary1, g.perm,
                       g.sort_scratch, st);
    launch_gather_unique(as_const(g.cand), g.perm, Count(g.cap_t, &dc->ncand[grp]), g.l1[grp], g.flags,
                         g.starts2, g.scan2, &dc->l1[grp], st);
  }
  // root: records, device keys, join, authority
  JoinWork jr{};
  for (int l = 0; l < 3; ++l) {
    launch_pack_records(as_const(g.l1[l]), Count(g.cap_t, &dc->l1[l]), n, g.recs[l], st);
    RecordKeyArgs ka{};
    ka.records = g.recs[l];
    ka.count = Count(g.cap_t, &dc->l1[l]);
    ka.record_bytes = rb;
    ka.res_offset = 16 * w64;
    ka.words32 = w32;
    ka.n = n;
    ka.r1 = r1;
    ka.qbits = n - r1;
    ka.negate = l == 2;
    ka.key_lo = g.rk_lo[l];
    ka.key_hi = g.rk_hi[l];
    ka.dvals = dp->rk[l];
    launch_record_keys(ka, st);
    jr.key_lo[l] = g.rk_lo[l];
    jr.key_hi[l] = g.rk_hi[l];
    jr.id[l] = nullptr;
    jr.count[l] = Count(g.cap_t, &dc->l1[l]);
  }
  jr.quotient_bits = n - r1;
  jr.cells = nullptr;
  jr.shard = 0;
  jr.shards = 1;
  jr.cap = g.cap_r;
  jr.main_sweep = true;
  jr.projected_bits = 0;
  jr.cancel = g.cancel;
  enqueue_join(g.jb, jr, g.tu_root, nullptr, st, &launches);
  check(cudaMemsetAsync(dc->auth, 0, sizeof dc->auth, st), "memset");
  AuthorityArgs au{};
  for (int l = 0; l < 3; ++l) au.records[l] = g.recs[l];
  au.record_bytes = rb;
  au.res_offset = 16 * w64;
  au.words32 = w32;
  au.words64 = w64;
  au.n = n;
  au.droot = dp->root;
  au.triples = g.jb.triples;
  au.count = Count(g.cap_r, &g.jb.counters[kTriples]);
  au.flags = g.aflags;
  au.counters = dc->auth;
  launch_authority(au, st);
  check(cudaMemcpyAsync(dc->root_counters, g.jb.counters, sizeof dc->root_counters,
                        cudaMemcpyDeviceToDevice, st), "counters");
  // results to the pinned host copies
  check(cudaMemcpyAsync(g.h_counts, dc, sizeof(GraphCounts), cudaMemcpyDeviceToHost, st), "counts");
  check(cudaMemcpyAsync(g.h_triples, g.jb.triples, g.cap_r * 12, cudaMemcpyDeviceToHost, st), "triples");
  check(cudaMemcpyAsync(g.h_aflags, g.aflags, g.cap_r, cudaMemcpyDeviceToHost, st), "flags");
  check(cudaGetLastError(), "graph capture");
}

bool graph_shape(uint32_t n) { return n == 36 || n == 72; }

// The plan's fixed capacities, tunings and device buffers, carved from g->base
// (without a base: only their byte count, which the preflight adds to its
// prediction).
void size_plan(GraphPlan* g, uint32_t n, uint32_t r1, uint32_t r2, uint64_t l3) {
  g->n = n;
  g->r1 = r1;
  g->r2 = r2;
  g->l3 = l3;
  g->cap_l2 = kCanonSmallCap;
  const double l1 = expected_l1(l3, r1, r2);
  g->cap_t = n == 36 ? 4096 : (1u << 18);
  g->cap_r = 4096;
  const uint32_t b1 = std::min(r1, r2 + 32);
  const uint32_t qbits = b1 - r2;
  const uint32_t fb_l2 = std::max<uint32_t>(6, qbits > 17 ? qbits - 17 : 6);
  const uint32_t filt_l2 = std::clamp<uint32_t>(qbits - fb_l2, 10, 20);
  const double l2 = (double)l3 * l3 / std::ldexp(1.0, r2);  // expected L2 list size
  g->tu_l2 = choose_tuning(g->cap_l2, g->cap_l2, qbits, 0, fb_l2, filt_l2, 0, 1, (uint64_t)l2);
  const uint32_t qroot = n - r1;
  g->tu_root = choose_tuning((uint64_t)l1, (uint64_t)l1, std::min<uint32_t>(qroot, 64), 0, 0, 0, 0, 1,
                             (uint64_t)l1);
  const uint32_t w64 = (n + 63) / 64, w32 = (n + 31) / 32;
  const uint32_t rb = 16 * w64 + 4 * w32;
  const uint32_t nbk = 1u << r2;
  // buffers (fixed capacities)
  g->d_weights = g->alloc<uint64_t>(2 * n);
  g->left = g->entries(l3);
  g->right = g->entries(l3);
  g->bcnt = g->alloc<uint32_t>(nbk + 16);
  g->boff = g->alloc<uint32_t>(nbk + 16);
  g->bcur = g->alloc<uint32_t>(2ull * nbk + 64);
  g->order = g->alloc<uint32_t>(l3 + 16);
  g->counts = g->alloc<uint32_t>(9 * l3 + 16);
  g->starts = g->alloc<uint32_t>(9 * l3 + 16);
  g->scan = g->alloc<uint32_t>(9 * l3 / 2048 + 64);
  g->raw = g->entries(9 * g->cap_l2);
  g->l2all = g->entries(9 * g->cap_l2);
  for (int l = 0; l < 3; ++l) g->keys[l] = g->alloc<uint64_t>(g->cap_l2 + 16);
  const uint64_t jcap = std::max<uint64_t>(g->cap_l2, g->cap_t);
  const uint32_t nfam = 1u << std::max(g->tu_l2.fb, g->tu_root.fb);
  for (int l = 0; l < 3; ++l) {
    const uint64_t slots = jcap + nfam + 16;
    g->jb.res[l] = g->alloc<uint64_t>(slots);
    g->jb.hi[l] = g->alloc<uint8_t>(slots);
    g->jb.id[l] = g->alloc<uint32_t>(slots);
    g->jb.cnt[l] = g->alloc<uint32_t>(nfam + 1);
    g->jb.off[l] = g->alloc<uint32_t>(nfam + 1);
    g->jb.cur[l] = g->alloc<uint32_t>(nfam + 1);
  }
  g->jb.counters = g->alloc<unsigned long long>(kCounters);
  g->jb.triples = g->alloc<uint32_t>(3 * std::max(g->cap_t, g->cap_r));
  if (g->tu_root.variant == 4 && std::min<uint32_t>(qroot, 64) - g->tu_root.fb >= 32) {
    // the root's v4 sweep: A windows and the B lane-slot layout
    const uint32_t nf4 = 1u << g->tu_root.fb;
    const uint64_t s4 = v4_slots(g->cap_t, g->tu_root.fb);
    g->jb.qwin = g->alloc<uint32_t>(g->cap_t + nf4 + 16);
    g->jb.res4 = g->alloc<uint64_t>(s4);
    g->jb.hi4 = g->alloc<uint8_t>(s4);
    g->jb.id4 = g->alloc<uint32_t>(s4);
    g->jb.win4 = g->alloc<uint32_t>(s4);
    g->jb.cnt4 = g->alloc<uint32_t>(nf4 + 1);
    g->jb.off4 = g->alloc<uint32_t>(nf4 + 1);
    g->jb.cur4 = g->alloc<uint32_t>(nf4 + 1);
  }
  g->cand = g->entries(g->cap_t);
  g->sort_scratch = g->alloc<uint32_t>(radix_scratch_words(g->cap_t));
  g->perm = g->alloc<uint32_t>(g->cap_t + 16);
  g->flags = g->alloc<uint32_t>(g->cap_t + 16);
  g->starts2 = g->alloc<uint32_t>(g->cap_t + 16);
  g->scan2 = g->alloc<uint32_t>(g->cap_t / 2048 + 64);
  for (int l = 0; l < 3; ++l) {
    g->l1[l] = g->entries(g->cap_t);
    g->recs[l] = g->alloc<uint8_t>((g->cap_t + 16) * rb);
    g->rk_lo[l] = g->alloc<uint64_t>(g->cap_t + 16);
    g->rk_hi[l] = g->alloc<uint8_t>(g->cap_t + 16);
  }
  g->aflags = g->alloc<uint8_t>(g->cap_r + 16);
  g->d_params = g->alloc<GraphParams>(1);
  g->d_counts = g->alloc<GraphCounts>(1);
}

uint64_t plan_bytes(uint32_t n, uint32_t r1, uint32_t r2, uint64_t l3) {
  GraphPlan g;
  size_plan(&g, n, r1, r2, l3);
  return g.bytes;
}

// The plan of workspace `w` for shape n (built and captured on first use), or
// null when the shape runs stage by stage.
GraphPlan* graph_plan(Workspace& w, uint32_t n, uint32_t r1, uint32_t r2, uint64_t l3, cudaStream_t st) {
  if (!graph_shape(n)) return nullptr;
  auto it = w.plans.find(n);
  if (it != w.plans.end()) return static_cast<GraphPlan*>(it->second.get());
  auto g = std::make_shared<GraphPlan>();
  const uint64_t total = plan_bytes(n, r1, r2, l3);
  check(cudaMalloc(&g->base, total), "cudaMalloc");
  size_plan(g.get(), n, r1, r2, l3);
  check(cudaMallocHost(&g->h_params, sizeof(GraphParams)), "cudaMallocHost");
  check(cudaMallocHost(&g->h_counts, sizeof(GraphCounts)), "cudaMallocHost");
  check(cudaMallocHost(&g->h_triples, g->cap_r * 12), "cudaMallocHost");
  check(cudaMallocHost(&g->h_aflags, g->cap_r), "cudaMallocHost");
  // capture (the kernels' shared-memory limits are set before, outside the capture).
  // The graph's sweeps take no cancel word: an attempt at these sizes lasts
  // milliseconds, so the checks between stages suffice, and a read of host-mapped
  // memory in every captured sweep costs the batched path several times its time
  g->cancel = nullptr;
  prepare_root_kernels();
  prepare_attempt_kernels();
  check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
  try {
    capture_attempt(*g, st);
  } catch (...) {
    cudaGraph_t dropped = nullptr;
    cudaStreamEndCapture(st, &dropped);
    if (dropped) cudaGraphDestroy(dropped);
    throw;
  }
  check(cudaStreamEndCapture(st, &g->graph), "capture");
  check(cudaGraphInstantiate(&g->exec, g->graph, 0), "graph instantiate");
  w.plans[n] = g;
  return g.get();
}

// Level 3 of the call's instance into the plan's buffers (direct launches).
void graph_level3(GraphPlan& g, const std::vector<uint64_t>& weights, cudaStream_t st) {
  check(cudaMemcpyAsync(g.d_weights, weights.data(), weights.size() * 8, cudaMemcpyHostToDevice, st), "weights");
  launch_enumerate_half(g.d_weights, g.n, 0, g.l3, g.left, st);
  launch_enumerate_half(g.d_weights, g.n, 1, g.l3, g.right, st);
  launch_bucket_right(as_const(g.right), g.l3, g.r2, g.bcnt, g.boff, g.bcur, g.order, st);
  check(cudaGetLastError(), "level 3");
}

// One attempt through the graph.  False when a capacity overflowed (the
// attempt then runs stage by stage); else stats and the valid parents.
bool graph_attempt(GraphPlan& g, Workspace& w, const Targets& tg, u128 T, uint32_t policy,
                   tergpu_attempt_stats* stat, RootOutcome* root, cudaStream_t st) {
  const uint32_t n = g.n, r1 = g.r1, r2 = g.r2;
  const uint32_t b1 = std::min(r1, r2 + 32);
  const u128 m1 = mask128(b1), m2 = mask128(r2), nmask = mask128(n);
  GraphParams& hp = *g.h_params;
  std::memset(&hp, 0, sizeof hp);
  for (int i = 0; i < 9; ++i) hp.t2.t[i] = (uint64_t)(tg.t2[i] & m2);
  for (int grp = 0; grp < 3; ++grp) {
    const u128 ta = tg.t2[3 * grp] & m2, tb = tg.t2[3 * grp + 1] & m2, t1 = tg.t1[grp] & m1;
    const u128 tc = (t1 - ta - tb) & m2;
    if (tc != (tg.t2[3 * grp + 2] & m2)) {
      t_error = "derived third L2 target disagrees with the stored target";
      throw Failure{TERGPU_INVARIANT_VIOLATION};
    }
    const uint64_t tau = (uint64_t)((((t1 - ta - tb - tc) & m1) >> r2));
    const u128 tt[3] = {ta, tb, tc};
    for (int l = 0; l < 3; ++l) {
      hp.q[3 * grp + l][0] = (uint64_t)tt[l];
      hp.q[3 * grp + l][1] = (uint64_t)(tt[l] >> 64);
      hp.q[3 * grp + l][2] = tau;
    }
  }
  u128 tau_res = T;
  for (int l = 0; l < 3; ++l) tau_res = (tau_res - tg.t1[l]) & nmask;
  const uint32_t Q = n - r1;
  const u128 tau = (tau_res >> r1) & mask128(Q);
  for (int l = 0; l < 3; ++l) {
    hp.rk[l][0] = (uint64_t)tg.t1[l];
    hp.rk[l][1] = (uint64_t)(tg.t1[l] >> 64);
    hp.rk[l][2] = (uint64_t)tau;
    hp.rk[l][3] = (uint64_t)(tau >> 64);
  }
  hp.root[0] = (uint64_t)T;
  hp.root[1] = (uint64_t)(T >> 64);
  check(cudaMemcpyAsync(g.d_params, g.h_params, sizeof(GraphParams), cudaMemcpyHostToDevice, st), "params");
  check(cudaGraphLaunch(g.exec, st), "graph launch");
  sync_stream(w, st, "graph");
  const GraphCounts& c = *g.h_counts;
  bool overflow = c.overflow != 0 || c.root_counters[kTriples] > g.cap_r;
  for (int grp = 0; grp < 3; ++grp) overflow = overflow || c.l2_triples[grp] > g.cap_t;
  if (overflow) return false;
  for (int i = 0; i < 9; ++i) stat->level2_sizes[i] = c.kept9[i];
  stat->l3_modular = c.bounds[9];
  stat->l3_survivors = c.bounds[9];
  stat->l2_modular = c.l2_triples[0] + c.l2_triples[1] + c.l2_triples[2];
  for (int grp = 0; grp < 3; ++grp) {
    if (c.kept9[3 * grp + 2] != 0) stat->l2_pairs += c.kept9[3 * grp] * c.kept9[3 * grp + 1];
    stat->l2_structural_rejects += c.l1rej[grp][0];
    stat->l2_distribution_rejects += c.l1rej[grp][1];
    stat->l2_survivors += c.ncand[grp];
  }
  for (int l = 0; l < 3; ++l) stat->level1_sizes[l] = c.l1[l];
  stat->root_pairs = c.l1[0] * c.l1[1];
  const uint32_t w64 = (n + 63) / 64, w32 = (n + 31) / 32;
  const uint32_t rb = 16 * w64 + 4 * w32;
  *root = pick_root(w, st, n, n - r1, policy, g.h_triples, g.h_aflags, c.root_counters[kTriples], g.rk_lo[0],
                    g.rk_lo[1], g.recs, rb);
  return true;
}

// FullTerTelemetry::fingerprint (src/full_ter.cpp:2532-2577): the witness's
// digits when one was found, the run's fields, then every attempt's.  l3 is 0
// for a run that stopped before level 3 (the reference leaves its physical
// level-3 sizes unset there).
uint64_t run_fingerprint(const uint8_t* witness, uint32_t n, uint64_t seed, bool fixture, uint32_t r1,
                         uint32_t r2, uint64_t l3, const std::vector<tergpu_attempt_stats>& run) {
  Fnv64 f;
  if (witness != nullptr)
    for (uint32_t i = 0; i < n; ++i) f.mix((uint64_t)witness[i] + 1u);
  f.mix(seed);
  f.mix(n);
  f.mix(n);  // modulus bits: the full TER modulus is 2^n
  f.mix(fixture ? 1 : 0);  // TerExecutionMode: FullTer 0, FixtureTer 1 (include/ter/types.hpp:25-28)
  f.mix(0);  // ShapeFamily::FiniteSanity
  f.mix(r1);
  f.mix(r2);
  f.mix(l3);
  f.mix(l3);
  f.mix(run.size());
  for (const auto& a : run) {
    f.mix(a.attempt_seed);
    f.mix(a.attempt);
    f.mix((uint64_t)a.status);
    for (int i = 0; i < 9; ++i) f.mix(a.level2_sizes[i]);
    for (int i = 0; i < 3; ++i) f.mix(a.level1_sizes[i]);
    f.mix(a.level0_size);
    f.mix(a.l3_modular);
    f.mix(a.l2_modular);
    f.mix(a.root_modular);
    f.mix(a.root_quotient_bits);
    f.mix(a.root_prefilter_bits);
    f.mix(a.root_low_prefilter);
    f.mix(a.root_full_quotient_rejects);
    f.mix(0);  // pair_records: the root materializes no pair records
    f.mix(a.l2_fingerprint);
    f.mix(a.l1_fingerprint);
    f.mix(a.l0_fingerprint);
  }
  return f.h;
}

}  // namespace

// One attempt range on `own` (a private workspace of the batch engine) or, when
// null, on the device's shared workspace.
int attempt_body(const tergpu_attempt_in* in, tergpu_attempt_out* out, Workspace* own) {
  const auto t_call = std::chrono::steady_clock::now();
  const uint32_t n = in->n;
  if (n == 0 || n % 36 != 0 || n > 108) {
    // the reference's message where it refuses the shape too (src/full_ter.cpp:2589)
    t_error = n == 0 || n % 36 != 0 ? "full TER requires n divisible by 36 and 0 < modulus_bits <= n"
                                    : "full TER on the device requires n in {36, 72, 108}";
    return TERGPU_INVALID_CONFIGURATION;
  }
  // solve_full_ter refuses CountOnly, since a SAT result must keep a verifiable
  // witness (src/full_ter.cpp:2945-2957); the root reports count instead
  if (in->root_policy != TERGPU_ROOT_POLICY_FIRST_WITNESS &&
      in->root_policy != TERGPU_ROOT_POLICY_FULL_CANONICAL) {
    t_error = "root_policy must be FirstWitness (0) or FullCanonicalOutput (2); solve_full_ter refuses CountOnly";
    return TERGPU_INVALID_CONFIGURATION;
  }
  const bool preflight = (in->flags & TERGPU_ATTEMPT_PREFLIGHT) != 0;
  constexpr uint32_t kKnownFlags = TERGPU_ATTEMPT_CAPTURE_ONLY | TERGPU_ATTEMPT_PREFLIGHT | TERGPU_ATTEMPT_NO_GRAPH |
                                   TERGPU_ATTEMPT_TELEMETRY | TERGPU_ATTEMPT_BACKGROUND | TERGPU_ATTEMPT_AUDIT |
                                   TERGPU_ATTEMPT_GUIDED | TERGPU_ATTEMPT_FIXTURE;
  if ((in->flags & ~kKnownFlags) != 0) {
    t_error = "unknown attempt flags";
    return TERGPU_INVALID_CONFIGURATION;
  }
  if (!preflight && (in->values_le == nullptr || in->target_le == nullptr)) {
    t_error = "instance missing";
    return TERGPU_INVALID_INPUT;
  }
  // an empty attempt budget is a configuration the reference refuses
  // (runtime_limit_supported, src/full_ter.cpp:2945-2957)
  if (!preflight && in->attempt_count == 0) {
    t_error = "full TER solver configuration or instance is invalid";
    return TERGPU_INVALID_CONFIGURATION;
  }
  const uint32_t r1 = floor_log2_multinomial3(n / 2, n / 6) / 2;
  const uint32_t r2 = floor_log2_multinomial3(n / 6, n / 18) / 2;
  out->r1 = r1;
  out->r2 = r2;
  if (r2 == 0 || r2 >= r1 || r1 >= n || r1 - r2 > 32) {
    t_error = "finite representation counts do not yield a supported 0 < r2 < r1 < n";
    return TERGPU_INVALID_CONFIGURATION;
  }
  const uint32_t w64 = (n + 63) / 64, w32 = (n + 31) / 32;
  const u128 nmask = mask128(n);
  // FixtureTer: each level-3 half is its first fixture_level3_limit subsets
  const bool fixture = (in->flags & TERGPU_ATTEMPT_FIXTURE) != 0;
  if (fixture && in->fixture_level3_limit == 0) {
    t_error = "level-3 generation configuration is invalid";
    return TERGPU_INVALID_CONFIGURATION;
  }
  const uint64_t l3 = fixture ? std::min<uint64_t>(binom_host(n / 2, n / 36), in->fixture_level3_limit)
                              : binom_host(n / 2, n / 36);
  out->level3_size = l3;
  // a call cancelled before it starts returns before level 3, as the
  // reference's does (src/full_ter.cpp:2979-2985), with the run fingerprint of
  // no attempts and no level-3 lists
  if (!preflight && in->cancel != nullptr && *in->cancel != 0) {
    t_error = "full TER execution was cancelled";
    if ((in->flags & TERGPU_ATTEMPT_TELEMETRY) != 0)
      out->fingerprint = run_fingerprint(nullptr, n, in->seed, fixture, r1, r2, 0, {});
    out->total_ms = ms_since(t_call);
    return TERGPU_CANCELLED;
  }

  // Preflight against the ceiling, from the expected level sizes (2x margin).
  const double l2_est = (double)l3 * l3 / std::ldexp(1.0, r2) * 1.3 + 64;
  const double cand_est = std::pow(l2_est, 3) / std::ldexp(1.0, r1 - r2) * 1.3 + 64;
  const double l1_est = cand_est * 0.6;
  const double rec = 16.0 * w64 + 4.0 * w32;
  double predicted = 2.0 * (2 * l3 * 32.0 + 9 * l2_est * 32 + l2_est * 120 + cand_est * (32 + 12 + 60) +
                            3 * l1_est * (32 + rec + 40) + l1_est * 13);  // + the staged scatter's temp copy
  // the graph plan's fixed buffers sit beside the stage-by-stage ones (its fallback)
  if (graph_shape(n) && (in->flags & TERGPU_ATTEMPT_NO_GRAPH) == 0) predicted += (double)plan_bytes(n, r1, r2, l3);
  out->device_bytes = (uint64_t)predicted;
  if (in->memory_limit_bytes != 0 && predicted > (double)in->memory_limit_bytes) {
    t_error = "predicted device bytes exceed the declared ceiling";
    return TERGPU_RESOURCE_LIMIT;
  }
  if (preflight) return TERGPU_COMPLETED;
  u128 T = in->target_le[0];
  if (w64 > 1) T |= (u128)in->target_le[1] << 64;
  T &= nmask;
  // GuidedPlanted: every attempt takes the planted root's targets
  const bool guided = (in->flags & TERGPU_ATTEMPT_GUIDED) != 0;
  Targets guided_tg{};
  std::vector<std::vector<uint8_t>> guided_l2;
  if (guided && !guided_targets(in->planted_root, n, r1, r2, in->values_le, &guided_tg, &guided_l2)) {
    t_error = "guided TER requires a planted binary root balanced across both halves";
    return TERGPU_INVALID_CONFIGURATION;
  }

  Workspace& w = own != nullptr ? *own : workspace(in->device);
  std::lock_guard<std::mutex> lock(w.mu);
  // on every exit: the bytes the workspace holds for this call (grow-only
  // within it): its stage buffers and the graph plan the call used
  struct Held {
    Workspace& w;
    tergpu_attempt_out* o;
    const GraphPlan* plan = nullptr;
    ~Held() {
      uint64_t bytes = plan != nullptr ? plan->bytes : 0;
      for (const auto& kv : w.buf) bytes += kv.second.bytes;
      o->device_bytes_held = bytes;
    }
  } held{w, out};
  check(cudaSetDevice(w.device), "cudaSetDevice");
  cudaStream_t st = (in->flags & TERGPU_ATTEMPT_BACKGROUND) != 0 && w.stream_low != nullptr ? w.stream_low
                                                                                             : w.stream;
  w.alloc_stream = st;
  // the sweeps read the cancel word only when the caller can cancel
  const volatile int* dcancel = nullptr;
  if (in->cancel != nullptr) {
    cancel_word(w);
    dcancel = w.cancel_dev;
  }
  const CancelMirror mirror(in->cancel, w.cancel_host);
  const bool background = (in->flags & TERGPU_ATTEMPT_BACKGROUND) != 0;

  // ---- level 3 (once per call): both halves, lexicographic k-subsets
  std::vector<uint64_t> weights(2 * n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    weights[2 * i] = in->values_le[i * w64];
    weights[2 * i + 1] = w64 > 1 ? in->values_le[i * w64 + 1] : 0;
  }
  // n = 36 and 72: each attempt as one captured graph (not for L1 exports)
  const bool exporting = (in->flags & TERGPU_ATTEMPT_CAPTURE_ONLY) != 0 || out->l1_records[0] != nullptr ||
                         out->l1_records[1] != nullptr || out->l1_records[2] != nullptr;
  const bool telemetry = (in->flags & TERGPU_ATTEMPT_TELEMETRY) != 0;
  // audit: every stage checked against the scalar oracles where they fit (the
  // root then reports FullCanonicalOutput, as the reference's audit does)
  const bool audit = (in->flags & TERGPU_ATTEMPT_AUDIT) != 0;
  const uint32_t policy = audit ? TERGPU_ROOT_POLICY_FULL_CANONICAL : in->root_policy;
  const auto t_l3 = std::chrono::steady_clock::now();
  GraphPlan* plan = nullptr;
  if (!exporting && !telemetry && !audit && !fixture && (in->flags & TERGPU_ATTEMPT_NO_GRAPH) == 0) {
    plan = graph_plan(w, n, r1, r2, l3, st);
    held.plan = plan;
    if (plan != nullptr) graph_level3(*plan, weights, st);
  }
  // the stage-by-stage path's level 3 (at once without a graph, else on the
  // first attempt that overflows a graph capacity)
  EntryArrays left{}, right{};
  uint32_t *boff = nullptr, *order = nullptr;
  auto dynamic_level3 = [&]() {
    if (boff != nullptr) return;
    uint64_t* d_weights = ensure<uint64_t>(w, S_WEIGHTS, weights.size() * 8);
    check(cudaMemcpyAsync(d_weights, weights.data(), weights.size() * 8, cudaMemcpyHostToDevice, st),
          "weights");
    left = entry_slot(w, S_L3, l3);
    right = entry_slot(w, S_L3 + 4, l3);
    launch_enumerate_half(d_weights, n, 0, l3, left, st);
    launch_enumerate_half(d_weights, n, 1, l3, right, st);
    if (fixture && guided) {
      // the guided level-2 vectors' halves first, then the first subsets up to
      // the limit (include_guided_halves, src/full_ter.cpp:2319-2362)
      for (int side = 0; side < 2; ++side) {
        const EntryArrays& dst = side == 0 ? left : right;
        const std::vector<HostEntry> original = host_entries(w, dst, l3, st);
        std::vector<HostEntry> keep;
        for (const auto& leaf : guided_l2) {
          HostEntry e{0, 0, 0};
          for (uint32_t c = side * n / 2; c < (side + 1) * n / 2; ++c) {
            if (leaf[c] == 0) continue;
            if (c < 64) e.p0 |= 1ull << c; else e.p1 |= 1ull << (c - 64);
            u128 wgt = weights[2 * c];
            wgt |= (u128)weights[2 * c + 1] << 64;
            e.res = (e.res + wgt) & nmask;
          }
          keep.push_back(e);
        }
        keep = canonical_entries(std::move(keep));
        if (keep.size() > in->fixture_level3_limit) {
          t_error = "fixture limit is too small for guided level-3 halves";
          throw Failure{TERGPU_RESOURCE_LIMIT};
        }
        for (const HostEntry& cand : original) {
          if (keep.size() >= in->fixture_level3_limit) break;
          if (!std::binary_search(keep.begin(), keep.end(), cand)) {
            keep.push_back(cand);
            std::sort(keep.begin(), keep.end());
          }
        }
        if (keep.size() != l3) {
          t_error = "guided fixture halves disagree in size";
          throw Failure{TERGPU_INVARIANT_VIOLATION};
        }
        std::vector<uint64_t> a(l3), b(l3), c(l3), d(l3);
        for (uint64_t i = 0; i < l3; ++i) {
          a[i] = keep[i].p0;
          b[i] = keep[i].p1;
          c[i] = (uint64_t)keep[i].res;
          d[i] = (uint64_t)(keep[i].res >> 64);
        }
        check(cudaMemcpyAsync(dst.pos0, a.data(), l3 * 8, cudaMemcpyHostToDevice, st), "fixture upload");
        check(cudaMemcpyAsync(dst.pos1, b.data(), l3 * 8, cudaMemcpyHostToDevice, st), "fixture upload");
        check(cudaMemcpyAsync(dst.res_lo, c.data(), l3 * 8, cudaMemcpyHostToDevice, st), "fixture upload");
        check(cudaMemcpyAsync(dst.res_hi, d.data(), l3 * 8, cudaMemcpyHostToDevice, st), "fixture upload");
        sync_stream(w, st, "fixture upload");
      }
    }
    const uint32_t nbk = 1u << r2;
    uint32_t* bcnt = ensure<uint32_t>(w, S_BCNT, (nbk + 16) * 4ull);
    boff = ensure<uint32_t>(w, S_BOFF, (nbk + 16) * 4ull);
    uint32_t* bcur = ensure<uint32_t>(w, S_BCUR, (2ull * nbk + 64) * 4);
    order = ensure<uint32_t>(w, S_ORDER, (l3 + 16) * 4);
    launch_bucket_right(as_const(right), l3, r2, bcnt, boff, bcur, order, st);
    check(cudaGetLastError(), "level 3");
  };
  if (plan == nullptr) dynamic_level3();
  if (telemetry) {  // the level-3 time of the reference's row (one more wait)
    sync_stream(w, st, "level 3");
    out->level3_ms = ms_since(t_l3);
  }
  std::vector<tergpu_attempt_stats> run;  // every attempt's stats (the run fingerprint)

  int status = TERGPU_ATTEMPT_LIMIT_REACHED;
  out->attempts_run = 0;
  for (uint32_t k = 0; k < in->attempt_count; ++k) {
    const uint32_t attempt = in->attempt_first + k;
    cancelled_check(in);
    const auto t_att = std::chrono::steady_clock::now();
    tergpu_attempt_stats stat;
    std::memset(&stat, 0, sizeof stat);
    stat.attempt = attempt;
    const Targets tg = guided ? guided_tg : random_targets(in->seed + attempt, r1, r2, T);
    RootOutcome root;
    bool graphed = false;
    if (plan != nullptr) {
      graphed = graph_attempt(*plan, w, tg, T, policy, &stat, &root, st);
      cancelled_check(in);  // a cancel during the graph cut its sweeps short
      if (!graphed) {  // a capacity overflowed: this attempt runs stage by stage
        root = RootOutcome{};
        std::memset(&stat, 0, sizeof stat);
        stat.attempt = attempt;
        dynamic_level3();
      }
    }
    if (!graphed) {
    // ---- L3 -> L2: the nine binary merges in single launches (count, scan,
    // fill), the raw lists back to back, then each list in canonical order
    // (one CTA per list in shared memory when every list is small)
    std::array<EntryArrays, 9> l2;
    std::array<uint64_t, 9> l2n{};
    MergeTargets mt{};
    for (int i = 0; i < 9; ++i) mt.t[i] = (uint64_t)(tg.t2[i] & mask128(r2));
    uint32_t* counts = ensure<uint32_t>(w, S_L2CNT, (9 * l3 + 16) * 4);
    uint32_t* starts = ensure<uint32_t>(w, S_L2START, (9 * l3 + 16) * 4);
    uint32_t* scan = ensure<uint32_t>(w, S_SCAN, (9 * l3 / 2048 + 64) * 4);
    uint32_t* bounds = ensure<uint32_t>(w, S_BOUNDS, 64);
    launch_l2_count_all(as_const(left), l3, boff, r2, mt, counts, st);
    launch_scan_u32(counts, 9 * l3, starts, scan, st);
    launch_l2_bounds(starts, l3, bounds, st);
    uint32_t hb[10];
    download(w, hb, bounds, 10, st);
    const uint64_t total_raw = hb[9];
    EntryArrays raw = entry_slot(w, S_L2RAW, total_raw);
    launch_l2_fill_all(as_const(left), l3, as_const(right), boff, order, r2, mt, n, starts, raw, st);
    EntryArrays l2all = entry_slot(w, S_L2, total_raw);
    Segments sg{};
    uint32_t maxseg = 0;
    for (int i = 0; i < 9; ++i) {
      sg.off[i] = hb[i];
      sg.cnt[i] = hb[i + 1] - hb[i];
      maxseg = std::max(maxseg, sg.cnt[i]);
      stat.l3_modular += sg.cnt[i];
      l2[i] = view(l2all, hb[i]);
    }
    if (maxseg <= kCanonSmallCap) {
      unsigned long long* kept = ensure<unsigned long long>(w, S_KEPT9, 16 * 8);
      launch_canon_small(as_const(raw), sg, 9, l2all, kept, st);
      unsigned long long hk[9];
      download(w, hk, kept, 9, st);
      for (int i = 0; i < 9; ++i) l2n[i] = hk[i];
    } else {
      for (int i = 0; i < 9; ++i) l2n[i] = canonicalize(w, view(raw, hb[i]), sg.cnt[i], l2[i], st);
    }
    for (int i = 0; i < 9; ++i) stat.level2_sizes[i] = l2n[i];
    stat.l3_survivors = stat.l3_modular;
    if (audit && l3 * l3 <= kAuditCap) {
      const std::vector<HostEntry> hl = host_entries(w, left, l3, st), hr = host_entries(w, right, l3, st);
      for (int i = 0; i < 9; ++i) {
        audit_binary(n, r2, tg.t2[i] & mask128(r2), hl, hr, host_entries(w, view(raw, hb[i]), sg.cnt[i], st),
                     host_entries(w, l2[i], l2n[i], st));
        ++stat.audited_stages;
      }
    }
    check(cudaGetLastError(), "L3 -> L2");
    if (telemetry) stat.l2_fingerprint = lists_fingerprint(w, n, l2.data(), l2n.data(), 9, st);
    stat.l2_ms = ms_since(t_att);
    cancelled_check(in);

    // ---- L2 -> L1: three ternary merges on the projected quotient
    const auto t_l1 = std::chrono::steady_clock::now();
    const uint32_t b1 = std::min(r1, r2 + 32);
    const uint32_t qbits = b1 - r2;
    std::array<EntryArrays, 3> l1;
    std::array<uint64_t, 3> l1n{};
    for (int g = 0; g < 3; ++g) {
      const u128 m1 = mask128(b1), m2 = mask128(r2);
      const u128 ta = tg.t2[3 * g] & m2, tb = tg.t2[3 * g + 1] & m2, t1 = tg.t1[g] & m1;
      const u128 tc = (t1 - ta - tb) & m2;
      if (tc != (tg.t2[3 * g + 2] & m2)) {
        t_error = "derived third L2 target disagrees with the stored target";
        return TERGPU_INVARIANT_VIOLATION;
      }
      const uint64_t tau = (uint64_t)((((t1 - ta - tb - tc) & m1) >> r2));
      uint64_t* keys[3];
      const u128 tt[3] = {ta, tb, tc};
      for (int l = 0; l < 3; ++l) {
        keys[l] = ensure<uint64_t>(w, S_KEYS + l, (l2n[3 * g + l] + 16) * 8);
        launch_l2_quotients(as_const(l2[3 * g + l]), l2n[3 * g + l], b1, r2, (uint64_t)tt[l],
                            (uint64_t)(tt[l] >> 64), l == 2, tau, keys[l], st);
      }
      JoinInput j{};
      j.quotient_bits = qbits;
      for (int l = 0; l < 3; ++l) {
        j.count[l] = l2n[3 * g + l];
        j.key_lo[l] = keys[l];
        j.key_hi[l] = nullptr;
        j.id[l] = nullptr;
      }
      // families so that at most 17 residual bits remain: the filter is exact
      j.family_bits = std::max<uint32_t>(6, qbits > 17 ? qbits - 17 : 6);
      if (j.family_bits + 2 > qbits) j.family_bits = 6;
      j.filter_bits = std::clamp<uint32_t>(qbits - j.family_bits, 10, 20);
      j.stream = st;
      const double est = (double)j.count[0] * j.count[1] * j.count[2] / std::ldexp(1.0, qbits);
      j.capacity = (uint64_t)(est * 1.25) + 4096;
      j.cancel = dcancel;
      j.background = background;
      JoinResult jr = run_join(w, j, 0);
      cancelled_check(in);
      if (jr.triples > j.capacity) {
        j.capacity = jr.triples + 16;
        jr = run_join(w, j, 0);
        cancelled_check(in);
      }
      stat.l2_modular += jr.triples;
      EntryArrays cand = entry_slot(w, S_CAND, jr.triples);
      unsigned long long* acc = ensure<unsigned long long>(w, S_ACC, 64);
      launch_l1_parents(jr.d_triples, jr.triples, as_const(l2[3 * g]), as_const(l2[3 * g + 1]),
                        as_const(l2[3 * g + 2]), n, n / 6, cand, acc + 4, st, nullptr, acc + 6);
      unsigned long long lc[4] = {0, 0, 0, 0};  // kept, (unused), structural, distribution rejects
      download(w, lc, acc + 4, 4, st);
      const unsigned long long ncand = lc[0];
      // the reference's ternary merge counts nothing when a list is empty
      // (src/full_ter.cpp:1153-1156)
      if (l2n[3 * g + 2] != 0) stat.l2_pairs += l2n[3 * g] * l2n[3 * g + 1];
      stat.l2_structural_rejects += lc[2];
      stat.l2_distribution_rejects += lc[3];
      stat.l2_survivors += ncand;
      l1[g] = entry_slot(w, S_L1 + 4 * g, ncand);
      l1n[g] = canonicalize(w, cand, ncand, l1[g], st);
      stat.level1_sizes[g] = l1n[g];
      if (audit && cubic_fits(l2n[3 * g], l2n[3 * g + 1], l2n[3 * g + 2])) {
        const TernaryOracle o =
            ternary_oracle(n, b1, t1, n / 6, host_entries(w, l2[3 * g], l2n[3 * g], st),
                           host_entries(w, l2[3 * g + 1], l2n[3 * g + 1], st),
                           host_entries(w, l2[3 * g + 2], l2n[3 * g + 2], st));
        std::vector<uint32_t> ht(jr.triples * 3);
        if (jr.triples != 0) download(w, ht.data(), jr.d_triples, ht.size(), st);
        std::vector<Triple> dev(jr.triples), want = o.candidates;
        for (uint64_t i = 0; i < jr.triples; ++i) dev[i] = Triple{ht[3 * i], ht[3 * i + 1], ht[3 * i + 2]};
        std::sort(dev.begin(), dev.end());
        std::sort(want.begin(), want.end());
        if (dev != want) audit_failed("an L2 -> L1 merge's candidate triples (provenance)");
        const uint64_t s_rej = std::count(o.decision.begin(), o.decision.end(), 1);
        const uint64_t d_rej = std::count(o.decision.begin(), o.decision.end(), 2);
        if (s_rej != lc[2] || d_rej != lc[3]) audit_failed("an L2 -> L1 merge's rejects");
        if (canonical_entries(o.parents) != host_entries(w, l1[g], l1n[g], st)) audit_failed("an L1 list");
        ++stat.audited_stages;
      }
    }
    check(cudaGetLastError(), "L2 -> L1");
    if (telemetry) stat.l1_fingerprint = lists_fingerprint(w, n, l1.data(), l1n.data(), 3, st);
    stat.l1_ms = ms_since(t_l1);
    cancelled_check(in);

    // ---- root: records, device keys, join, authority
    const auto t_root = std::chrono::steady_clock::now();
    const uint32_t rb = 16 * w64 + 4 * w32;
    uint8_t* recs[3];
    for (int l = 0; l < 3; ++l) {
      recs[l] = ensure<uint8_t>(w, S_REC + l, (l1n[l] + 16) * rb);
      launch_pack_records(as_const(l1[l]), l1n[l], n, recs[l], st);
    }
    auto export_l1 = [&]() {
      for (int l = 0; l < 3; ++l) {
        for (uint32_t q = 0; q < 4; ++q) out->child_targets[l][q] = q < w32 ? (uint32_t)(tg.t1[l] >> (32 * q)) : 0u;
        if (out->l1_records[l] != nullptr && out->l1_capacity[l] >= l1n[l] && l1n[l] != 0) {
          check(cudaMemcpyAsync(out->l1_records[l], recs[l], l1n[l] * rb, cudaMemcpyDeviceToHost, st), "export");
        }
        out->l1_capacity[l] = l1n[l];
      }
      for (uint32_t q = 0; q < 4; ++q) out->root_target[q] = q < w32 ? (uint32_t)(T >> (32 * q)) : 0u;
      sync_stream(w, st, "export");
    };
    if (in->flags & TERGPU_ATTEMPT_CAPTURE_ONLY) {
      stat.status = TERGPU_NO_WITNESS_THIS_ATTEMPT;
      stat.total_ms = ms_since(t_att);
      if (out->stats != nullptr) out->stats[k] = stat;
      out->attempts_run = k + 1;
      export_l1();
      continue;
    }
    const uint32_t Q = n - r1;
    u128 tau_res = T;
    for (int l = 0; l < 3; ++l) tau_res = (tau_res - tg.t1[l]) & nmask;
    const u128 tau = (tau_res >> r1) & mask128(Q);
    JoinInput j{};
    j.quotient_bits = Q;
    for (int l = 0; l < 3; ++l) {
      uint64_t* klo = ensure<uint64_t>(w, S_RKLO + l, (l1n[l] + 16) * 8);
      uint8_t* khi = ensure<uint8_t>(w, S_RKHI + l, l1n[l] + 16);
      RecordKeyArgs ka{};
      ka.records = recs[l];
      ka.count = l1n[l];
      ka.record_bytes = rb;
      ka.res_offset = 16 * w64;
      ka.words32 = w32;
      ka.n = n;
      ka.r1 = r1;
      ka.qbits = Q;
      ka.child_lo = (uint64_t)tg.t1[l];
      ka.child_hi = (uint64_t)(tg.t1[l] >> 64);
      ka.tau_lo = (uint64_t)tau;
      ka.tau_hi = (uint64_t)(tau >> 64);
      ka.negate = l == 2;
      ka.key_lo = klo;
      ka.key_hi = khi;
      launch_record_keys(ka, st);
      j.count[l] = l1n[l];
      j.key_lo[l] = klo;
      j.key_hi[l] = khi;
      j.id[l] = nullptr;
    }
    j.stream = st;
    j.capacity = 4096;
    j.cancel = dcancel;
    j.background = background;
    JoinResult jr = run_join(w, j, 0);
    cancelled_check(in);  // a cancel during the sweep cut it short: nothing is reported
    if (jr.triples > j.capacity) {
      j.capacity = jr.triples + 16;
      jr = run_join(w, j, 0);
      cancelled_check(in);
    }
    stat.root_pairs = jr.pairs;
    std::vector<uint32_t> htrip;
    std::vector<uint8_t> hflags;
    if (jr.triples != 0) {
      uint8_t* dflags = ensure<uint8_t>(w, S_AFLAGS, jr.triples + 16);
      unsigned long long* acount = ensure<unsigned long long>(w, S_ACOUNT, 64);
      check(cudaMemsetAsync(acount, 0, 64, st), "memset");
      AuthorityArgs au{};
      for (int l = 0; l < 3; ++l) au.records[l] = recs[l];
      au.record_bytes = rb;
      au.res_offset = 16 * w64;
      au.words32 = w32;
      au.words64 = w64;
      au.n = n;
      au.root_lo = (uint64_t)T;
      au.root_hi = (uint64_t)(T >> 64);
      au.triples = jr.d_triples;
      au.count = jr.triples;
      au.flags = dflags;
      au.counters = acount;
      launch_authority(au, st);
      check(cudaGetLastError(), "authority");
      htrip.resize(jr.triples * 3);
      hflags.resize(jr.triples);
      check(cudaMemcpyAsync(htrip.data(), jr.d_triples, jr.triples * 12, cudaMemcpyDeviceToHost, st), "d2h");
      check(cudaMemcpyAsync(hflags.data(), dflags, jr.triples, cudaMemcpyDeviceToHost, st), "d2h");
      sync_stream(w, st, "sync");
    }
    root = pick_root(w, st, n, Q, policy, htrip.data(), hflags.data(), jr.triples, j.key_lo[0], j.key_lo[1], recs,
                     rb);
    if (audit && cubic_fits(l1n[0], l1n[1], l1n[2])) {
      const TernaryOracle o = ternary_oracle(n, n, T & nmask, n / 2, host_entries(w, l1[0], l1n[0], st),
                                             host_entries(w, l1[1], l1n[1], st), host_entries(w, l1[2], l1n[2], st));
      std::vector<std::pair<Triple, uint8_t>> dev, want;
      for (uint64_t i = 0; i < jr.triples; ++i) {
        if ((hflags[i] & 1) == 0) continue;
        const uint8_t d = (hflags[i] & 8) != 0 ? 1 : (hflags[i] & 16) != 0 ? 2 : (hflags[i] & 4) != 0 ? 0 : 3;
        dev.push_back({Triple{htrip[3 * i], htrip[3 * i + 1], htrip[3 * i + 2]}, d});
      }
      for (size_t i = 0; i < o.candidates.size(); ++i) want.push_back({o.candidates[i], o.decision[i]});
      auto by_triple = [](const std::pair<Triple, uint8_t>& x, const std::pair<Triple, uint8_t>& y) {
        return x.first < y.first || (x.first == y.first && x.second < y.second);
      };
      std::sort(dev.begin(), dev.end(), by_triple);
      std::sort(want.begin(), want.end(), by_triple);
      if (dev != want) audit_failed("the root's residue-exact triples or their decisions (provenance)");
      std::vector<std::array<uint64_t, 2>> parents;
      for (const HostEntry& e : canonical_entries(o.parents)) parents.push_back({e.p0, e.p1});
      if (parents != root.parents) audit_failed("the root's parents");
      ++stat.audited_stages;
    }
    if (telemetry) {
      // the reporter's low-prefilter candidates: triples equal on the low p
      // bits, counted up to the FirstWitness stop when there is one
      const uint32_t pbits = root_prefilter_bits(Q);
      JoinInput jp = j;
      jp.projected_bits = pbits;
      jp.count_only = true;
      jp.capacity = 0;
      if (root.stopped) {
        jp.visit = VisitBound{1u, pbits, root_tile_bits(pbits), root.stop.m, root.stop.i, root.stop.a,
                              root.stop.b, root.stop.c};
      }
      const JoinResult pr = run_join(w, jp, 0);
      cancelled_check(in);
      stat.root_low_prefilter = pr.projected + (root.stopped ? 1 : 0);
    }
    stat.root_ms = ms_since(t_root);
    // L1 export of the attempt (records + targets), when the caller asked for it
    export_l1();
    }  // stage by stage
    // the root's counters under the policy and the retained parents (level 0)
    const uint32_t Qr = n - r1;
    const auto& parents = root.parents;
    stat.attempt_seed = in->seed + attempt;
    stat.l3_pairs = 9ull * l3 * l3;  // every L3 -> L2 merge pairs the two halves
    // the halves cover disjoint coordinates and hold n/36 ones each, so every
    // L3 -> L2 parent is binary with n/18 ones: add_three rejects none
    stat.l3_structural_rejects = 0;
    stat.l3_distribution_rejects = 0;
    stat.root_modular = root.modular;
    stat.root_structural_rejects = root.structural;
    stat.root_distribution_rejects = root.distribution;
    stat.valid_roots = root.valid;
    stat.root_quotient_bits = Qr;
    stat.root_prefilter_bits = root_prefilter_bits(Qr);
    stat.root_policy = policy;
    stat.root_early_stopped = root.stopped ? 1u : 0u;
    if (telemetry) {
      stat.root_full_quotient_rejects = stat.root_low_prefilter - stat.root_modular;
      stat.l0_fingerprint = l0_fingerprint(n, parents, T);
    }
    if (stat.level1_sizes[0] == 0 || stat.level1_sizes[1] == 0 || stat.level1_sizes[2] == 0) {
      // the reference's tiled root returns before it records anything when a
      // level-1 list is empty (src/full_ter.cpp:1644-1647): its stage telemetry
      // keeps its defaults, FullCanonicalOutput among them
      stat.root_pairs = 0;
      stat.root_quotient_bits = 0;
      stat.root_prefilter_bits = 0;
      stat.root_low_prefilter = 0;
      stat.root_full_quotient_rejects = 0;
      stat.root_policy = TERGPU_ROOT_POLICY_FULL_CANONICAL;
      stat.root_early_stopped = 0;
    }
    stat.level0_size = parents.size();
    stat.status = parents.empty() ? TERGPU_NO_WITNESS_THIS_ATTEMPT : TERGPU_FOUND;
    out->attempts_run = k + 1;

    if (!parents.empty()) {
      // verify the retained parent (the policy's witness): binary digits,
      // weight n/2, weights sum to the target (src/full_ter.cpp:2879-2908)
      const auto t_ver = std::chrono::steady_clock::now();
      const auto& p = parents.front();
      u128 acc = 0;
      uint32_t weight = 0;
      std::memset(out->witness, 0, sizeof out->witness);
      for (uint32_t i = 0; i < n; ++i) {
        const bool on = ((i < 64 ? p[0] >> i : p[1] >> (i - 64)) & 1) != 0;
        if (!on) continue;
        out->witness[i] = 1;
        ++weight;
        acc = (acc + ((u128)weights[2 * i + 1] << 64 | weights[2 * i])) & nmask;
      }
      stat.verification_ms = ms_since(t_ver);
      if (weight != n / 2 || acc != T) {
        t_error = "root witness fails verification";
        return TERGPU_INVARIANT_VIOLATION;
      }
      out->found_attempt = attempt;
      status = TERGPU_FOUND;
    }
    stat.total_ms = ms_since(t_att);
    if (out->stats != nullptr) out->stats[k] = stat;
    run.push_back(stat);
    if (status == TERGPU_FOUND) break;
  }
  if (status == TERGPU_ATTEMPT_LIMIT_REACHED) t_error = "deterministic TER attempts exhausted without proving UNSAT";
  if (telemetry) out->fingerprint = run_fingerprint(status == TERGPU_FOUND ? out->witness : nullptr, n, in->seed,
                                                    fixture, r1, r2, l3, run);
  out->status = status;
  out->total_ms = ms_since(t_call);
  return status;
}

}  // namespace tergpu

extern "C" int tergpu_attempt_run(const tergpu_attempt_in* in, tergpu_attempt_out* out) {
  using namespace tergpu;
  t_error.clear();
  if (in == nullptr || out == nullptr) {
    t_error = "null argument";
    return TERGPU_INVALID_INPUT;
  }
  try {
    const int st = attempt_body(in, out, nullptr);
    out->status = st;
    return st;
  } catch (const Failure& f) {
    out->status = f.status;
    return f.status;
  } catch (const std::bad_alloc&) {
    t_error = "host allocation failed";
    out->status = TERGPU_RESOURCE_LIMIT;
    return TERGPU_RESOURCE_LIMIT;
  } catch (const std::exception& e) {
    t_error = std::string("unexpected exception: ") + e.what();
    out->status = TERGPU_DEVICE_ERROR;
    return TERGPU_DEVICE_ERROR;
  } catch (...) {
    t_error = "unexpected exception";
    out->status = TERGPU_DEVICE_ERROR;
    return TERGPU_DEVICE_ERROR;
  }
}
