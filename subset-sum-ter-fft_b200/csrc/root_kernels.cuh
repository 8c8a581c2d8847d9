// Device side of the B200 root join (L1 -> L0 of the depth-3 TER attempt).
//
// Problem: lists A (q), B (x), D (d = tau - q_C) of Q-bit keys; report every
// (a, b, c) with key_a + key_b == key_c (mod 2^Q), with multiplicity.
//
// Layout in HBM after the partition (per list, structure of arrays):
//   res[i]  uint64  residual key = (key_lo mod 2^F) >> fb      F = min(Q, 64)
//   hi[i]   uint8   key bits [64, Q)
//   id[i]   uint32  EntryId reported in triples
// entries grouped by family f = key_lo mod 2^fb; family f occupies
// [off[f], off[f] + cnt[f]), off[f] even so two residuals load as one 16-byte word.
//
// A cell (s, t) pairs A family s with B family t; its sums land in D family
// u = (s + t) mod 2^fb with carry kappa = (s + t) >> fb into the residual.
#pragma once

#include <cstdint>

#include "count.cuh"

namespace tergpu {

constexpr int kSweepThreads = 256;
constexpr int kSweepWarps = kSweepThreads / 32;
constexpr int kQueueCap = 128;         // survivor slots per warp
constexpr uint32_t kYHashBits = 13;    // shared exact-lookup table: 8192 slots of 16 bits
constexpr uint32_t kYCap = 4096;       // D-family entries the shared table takes
constexpr uint32_t kSortCap = 4096;    // B-family entries the in-family sort takes
// v3: one CTA of 24 warps per SM, so a 2^15-word filter (20 filter bits, 128 KiB)
// fits beside the queues (measured at n=108: 8.0 s against 8.76 s for two CTAs
// of 12 warps with 19 filter bits: half the false passes, same warps per SM),
// and a 4096-slot exact-lookup table (D families of up to 2048 entries; the
// tuning aims at about 1,700, larger families fall back to a scan of the family)
constexpr int kSweep3Threads = 768;
constexpr int kSweep3Warps = kSweep3Threads / 32;
constexpr uint32_t kY3HashBits = 12;
constexpr uint32_t kY3Cap = 2048;

// v4: one CTA of 24 warps per SM.  The probe table covers the low kW4Bits bits
// of the residuals: word v (2^15 + 1 of them) is 1 when v or v - 1 is the sum
// window of a D entry (each D entry sets four words), so a probe is an add, one
// shared load and a shift-add of the loaded 0/1 into the test mask.
constexpr uint32_t kW4Bits = 14;
constexpr uint32_t kT4Words = (1u << (kW4Bits + 1)) + 32;
constexpr int kSweep4Threads = 768;
constexpr int kSweep4Warps = kSweep4Threads / 32;
constexpr uint32_t kY4HashBits = 11;
constexpr uint32_t kY4Cap = 1024;
// A entries whose 32-bit windows a warp stages at once (its buffer holds 16 more:
// the last mask of a segment reads up to 15 entries past it)
constexpr uint32_t kA4Seg = 256;
// table survivors a warp collects before resolving them (one per 32-bit record)
constexpr uint32_t kS4Cap = 256;
// B families of up to kArrange4Cap entries are laid out one bank per lane (at
// most kArrange4ExtraRows rows beyond the minimum); larger ones stay in order.
constexpr uint32_t kArrange4Cap = 4096;
constexpr uint32_t kArrange4ExtraRows = 2;
constexpr uint32_t kHole4 = 0xFFFFFFFFu;  // window of an empty lane slot

struct ListView {
  const uint64_t* res;
  const uint8_t* hi;
  const uint32_t* id;
  const uint32_t* off;
  const uint32_t* cnt;
  const uint32_t* win = nullptr;  // v4: 4 * (probe window [+ bank offset]) per entry, or null
};

// Counting bound in the order the reference's tiled reporter visits the
// prefilter candidates of a root (src/tiled_q3report.cpp:365-410, with lists
// fed in EntryId order, src/full_ter.cpp:1785-1810): a triple (a, b, c) whose
// low-p-bit keys are k_a, k_b is visited at (m, i, id_a, id_b, -id_c) with
// i = k_a >> tb, m = i + (k_b >> tb); the C entries of one window slot are
// visited by descending EntryId.  With `on` set, a projected sweep counts only
// the triples visited before (m, i, a, b, c).
struct VisitBound {
  uint32_t on;
  uint32_t pbits;   // p, the prefilter width (<= 32)
  uint32_t tb;      // tile bits
  uint32_t m, i, a, b, c;
};

struct SweepArgs {
  ListView q, x, y;
  const uint8_t* cells;     // 4096 bytes over the low 6 key bits, or null
  uint32_t fb;              // family bits
  uint32_t s_split;         // CTAs per target family
  uint32_t shard;           // this call joins the target families u == shard (mod shards)
  uint32_t shards;          // power of two, 1..64 (1: the whole root)
  uint32_t wb;              // log2 of filter words (filter bits = wb + 5)
  uint32_t mrb;             // residual bits compared exactly
  uint32_t rb;              // full residual width (carry into the high byte)
  uint32_t hi_bits;         // key bits above 64 (0 when Q <= 64)
  uint32_t project;         // 1: count triples on mrb residual bits only
  VisitBound visit;         // projected counts: only triples visited before this bound
  uint32_t two;             // 2, as an opaque operand (v4 keeps its mask shift-add an IMAD)
  const volatile int* cancel;  // device-visible word (host-mapped) or null: when it reads
                               // nonzero, warps stop taking work items (the counts are then
                               // incomplete and the caller discards them).  Each read crosses
                               // PCIe: pass it only to long sweeps a caller may cancel
  uint32_t* triples;        // 3 * cap
  unsigned long long cap;
  unsigned long long* counters;  // [0] triples [1] survivors [2] fast [3] projected [4] fallback
};

// counters[kMaxQ] holds the largest A family (set by launch_max_family before
// the sweep reads it), so no host round trip separates partition and sweep.
enum Counter {
  kTriples = 0, kSurvivors = 1, kFast = 2, kProjected = 3, kFallback = 4, kMaxQ = 5, kMaxX = 6,
  kCounters = 8
};

// Allows a kernel the device's whole opt-in dynamic shared memory, once per
// device and kernel (root_kernels.cu); launchers call it before a launch that
// needs more than the default 48 KB.
void allow_max_smem(const void* kernel);
// allow_max_smem for every root kernel that needs it (before a graph capture).
void prepare_root_kernels();

// Host-callable launchers (root_kernels.cu).
void launch_hist(const uint64_t* key, Count n, uint32_t fmask, uint32_t* cnt, cudaStream_t st);
void launch_scan(const uint32_t* cnt, uint32_t nfam, uint32_t* off, uint32_t* cursor,
                 cudaStream_t st);
void launch_scatter(const uint64_t* key_lo, const uint8_t* key_hi, const uint32_t* id, Count n,
                    uint32_t fb, uint64_t fast_mask, uint32_t hi_mask, uint32_t* cursor,
                    uint64_t* res, uint8_t* hi, uint32_t* out_id, cudaStream_t st);
void launch_max_family(const uint32_t* cnt, uint32_t nfam, unsigned long long* counters, int slot,
                       cudaStream_t st);

// Staged two-pass scatter for long lists with a host count (staged_partition):
// pass 1 moves every entry into the bucket of its high family digit (a temp
// copy of the list), pass 2 moves it from there into its family; each pass
// sorts a tile of kStageTile entries by digit in shared memory first, so every
// store is part of a run of consecutive entries.  The temp arrays hold
// count + 2^fb + 16 slots like the output arrays; the table holds
// staged_table_words(fb) words.
constexpr uint32_t kStageThreads = 256;
constexpr uint32_t kStagePer = 16;
constexpr uint32_t kStageTile = kStageThreads * kStagePer;
struct StageBuffers {
  uint64_t* key = nullptr;
  uint8_t* hi = nullptr;
  uint32_t* id = nullptr;
  uint32_t* table = nullptr;
};
bool staged_partition(const Count& n, uint32_t fb);
uint32_t staged_table_words(uint32_t fb);
// Family digits of the second staged pass (all fb digits when one pass does).
uint32_t staged_low_bits(uint32_t fb);
// launch_scan that also fills the staged scatter's bucket table (tmp.table).
void launch_scan_staged(const uint32_t* cnt, uint32_t nfam, uint32_t* off, uint32_t* cursor, uint32_t fb,
                        uint32_t* table, cudaStream_t st);
// The scatter of launch_scatter through the staged passes (cursor and the
// bucket table as launch_scan_staged left them).  Returns the kernels launched.
uint32_t launch_scatter_staged(const uint64_t* key_lo, const uint8_t* key_hi, const uint32_t* id, Count n,
                               uint32_t fb, uint64_t fast_mask, uint32_t hi_mask, uint32_t* cursor,
                               const StageBuffers& tmp, uint64_t* res, uint8_t* hi, uint32_t* out_id,
                               cudaStream_t st);
size_t sweep_smem_bytes(uint32_t wb);
// v1: A windows in registers, B broadcast (any family order).
void launch_sweep(const SweepArgs& a, bool aligned, cudaStream_t st);
// v2: B windows in registers (32 consecutive entries per lane slot), A broadcast.
// Exact for any family order; conflict-free filter probes once every B family
// is sorted by the filter's word bits (launch_family_sort).
void launch_sweep2(const SweepArgs& a, bool aligned, cudaStream_t st);
// v3 (needs mrb >= 32): the filter word is picked by the low bits of the probe
// value, so the bank is borrow-free; conflict-free once every B family is laid
// out by launch_family_arrange.  Exact for any family order.
void launch_sweep3(const SweepArgs& a, cudaStream_t st);
// v4 (needs mrb >= 32): probe table of 0/1 words over 14-bit windows, B in the
// lane-per-bank layout of launch_arrange4 (a.x = that layout, a.x.win its
// windows), A windows in a.q.win.  Exact for any layout.
void launch_sweep4(const SweepArgs& a, cudaStream_t st);
size_t sweep4_smem_bytes();
// win[i] = 4 * (res[i] mod 2^kW4Bits) for the n slots of a partitioned list.
void launch_window4(const uint64_t* res, Count n, uint32_t* win, cudaStream_t st);
// v4 layout of the B list, in two launches around a scan: rows4 writes cnt4[f] =
// 32 * (the rows family f takes); arrange4 writes family f at off4[f] as rows of
// 32 lane slots where the entry in lane b probes bank b (its residual class c
// shifted by o in {0, 1}, o folded into its window, so c + o == b mod 32), and
// marks the empty slots with the window kHole4.  Families above kArrange4Cap, or
// whose classes do not balance within kArrange4ExtraRows more rows, keep their
// order (same results, more bank conflicts).
void launch_rows4(const uint64_t* res, const uint32_t* off, const uint32_t* cnt, uint32_t nfam,
                  uint32_t* cnt4, cudaStream_t st);
void launch_arrange4(const uint64_t* res, const uint8_t* hi, const uint32_t* id, const uint32_t* off,
                     const uint32_t* cnt, const uint32_t* off4, const uint32_t* cnt4, uint32_t nfam,
                     uint64_t* res4, uint8_t* hi4, uint32_t* id4, uint32_t* win4, cudaStream_t st);

// Lays every B family (of at most kSortCap entries) out in lane slots of 32
// entries with distinct residual classes mod 32 wherever the counts allow.
void launch_family_arrange(uint64_t* res, uint8_t* hi, uint32_t* id, const uint32_t* off,
                           const uint32_t* cnt, uint32_t nfam, uint64_t mean_family, cudaStream_t st);
// Sorts every family of one partitioned list (of at most kSortCap entries) by
// the top `sb` bits of its sweep window, in place; larger families stay as they are.
void launch_family_sort(uint64_t* res, uint8_t* hi, uint32_t* id, const uint32_t* off,
                        const uint32_t* cnt, uint32_t nfam, uint32_t mrb, uint32_t sb,
                        cudaStream_t st);

// Keys from captured L1 records: q = ((R - c) mod 2^n) >> r1 over Q bits,
// list 2 turned into d = tau - q_C.
struct RecordKeyArgs {
  const uint8_t* records;
  Count count;
  uint32_t record_bytes;
  uint32_t res_offset;     // 16 * W64
  uint32_t words32;
  uint32_t n, r1, qbits;
  uint64_t child_lo, child_hi;
  uint64_t tau_lo, tau_hi;
  int negate;              // list 2
  uint64_t* key_lo;
  uint8_t* key_hi;
  const uint64_t* dvals;   // device {child_lo, child_hi, tau_lo, tau_hi} replacing the fields
                           // above when not null (a captured graph's per-attempt values)
};
void launch_record_keys(const RecordKeyArgs& a, cudaStream_t st);

// Authority chain for the emitted triples: residue sum == T, FiniteSanity
// structural count, root rule (binary parent of weight n/2).  Flags per triple:
// bit0 residue-exact; of those, bit1 FiniteSanity structural (the RootSink count),
// bit2 valid root, bit3 add_three structural reject (invalid digits), bit4
// add_three distribution reject (digit counts other than the root's).
struct AuthorityArgs {
  const uint8_t* records[3];
  uint32_t record_bytes, res_offset, words32, words64, n;
  uint64_t root_lo, root_hi;
  const uint64_t* droot;   // device {lo, hi} replacing root_lo / root_hi when not null
  const uint32_t* triples;
  Count count;
  uint8_t* flags;
  unsigned long long* counters;  // [0] residue [1] structural [2] root rule
};
void launch_authority(const AuthorityArgs& a, cudaStream_t st);

}  // namespace tergpu
