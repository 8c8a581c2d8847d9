// Device kernels of the attempt pipeline below the root: level-3 enumeration,
// the L3 -> L2 binary merge, parent construction of the L2 -> L1 ternary merge,
// and the canonical order (stable LSD radix sort on the packed digit words,
// then duplicate removal) that every level's EntryIds are defined by.
//
// Entry layout at every level (structure of arrays, one index per entry):
//   pos0, pos1  uint64  positive-digit mask words (coordinates 0..63, 64..127)
//   res_lo, res_hi uint64 residue mod 2^n (n <= 128)
// Negative masks are zero throughout: the FiniteSanity shapes of the attempt
// have no -1 digits at any level (every epsilon is zero).
#pragma once

#include <cstdint>

#include "count.cuh"

namespace tergpu {

struct EntryArrays {
  uint64_t* pos0;
  uint64_t* pos1;
  uint64_t* res_lo;
  uint64_t* res_hi;
};

struct ConstEntryArrays {
  const uint64_t* pos0;
  const uint64_t* pos1;
  const uint64_t* res_lo;
  const uint64_t* res_hi;
};

// All k-subsets of the half's n/2 coordinates in lexicographic order, k = n/36;
// residue = sum of the chosen weights mod 2^n.  weights: n x 2 words (lo, hi).
void launch_enumerate_half(const uint64_t* weights, uint32_t n, uint32_t second_half,
                           uint64_t count, EntryArrays out, cudaStream_t st);

// Counting sort of the right list by residue mod 2^r2: bucket offsets (2^r2 + 1)
// and the permuted right indices.
void launch_bucket_right(ConstEntryArrays right, uint64_t nr, uint32_t r2, uint32_t* bucket_cnt,
                         uint32_t* bucket_off, uint32_t* bucket_cur, uint32_t* order, cudaStream_t st);

// L2 = {(l, r) : R_l + R_r == t (mod 2^r2)}: per-left match counts, then the fill
// (counts are scanned on the device; total written to *total).
void launch_l2_count(ConstEntryArrays left, uint64_t nl, const uint32_t* bucket_off, uint32_t r2,
                     uint64_t t_lo, uint32_t* counts, cudaStream_t st);
void launch_l2_fill(ConstEntryArrays left, uint64_t nl, ConstEntryArrays right,
                    const uint32_t* bucket_off, const uint32_t* order, uint32_t r2, uint64_t t_lo,
                    uint32_t n, const uint32_t* starts, EntryArrays out, cudaStream_t st);

// The nine L3 -> L2 merges of one attempt in single launches: merge m pairs
// the left half with the right half on target t[m].  Counts go to
// counts[m * nl + l]; after their scan (starts, total at starts[9 * nl]) the fill
// writes merge m's raw entries at starts[m * nl + l], i.e. the nine raw lists
// back to back; bounds[m] = starts[m * nl] (m = 0..9) give the list boundaries.
struct MergeTargets {
  uint64_t t[9];
};
// dt (device targets, may be null) replaces t: the captured graph's per-attempt
// values; cap bounds the fill's writes (the graph's fixed buffers).
void launch_l2_count_all(ConstEntryArrays left, uint64_t nl, const uint32_t* bucket_off, uint32_t r2,
                         const MergeTargets& t, uint32_t* counts, cudaStream_t st,
                         const MergeTargets* dt = nullptr);
void launch_l2_bounds(const uint32_t* starts, uint64_t nl, uint32_t* bounds, cudaStream_t st);
void launch_l2_fill_all(ConstEntryArrays left, uint64_t nl, ConstEntryArrays right,
                        const uint32_t* bucket_off, const uint32_t* order, uint32_t r2,
                        const MergeTargets& t, uint32_t n, const uint32_t* starts, EntryArrays out,
                        cudaStream_t st, const MergeTargets* dt = nullptr, uint64_t cap = ~0ull);

// Canonical order (sort by (pos0, pos1), drop repeats) of up to 9 segments of at
// most kCanonSmallCap entries each, one CTA per segment, entirely in shared
// memory: segment s of `raw` [off[s], off[s] + cnt[s]) goes to `out` at the same
// offset, kept[s] receives its kept count.
constexpr uint32_t kCanonSmallCap = 4096;
struct Segments {
  uint32_t off[9];
  uint32_t cnt[9];
};
// dbounds (device, may be null): segments from the boundaries dbounds[0..nseg]
// instead of seg; a segment above kCanonSmallCap or reaching past `cap` entries
// of raw / out then sets *overflow and keeps 0.
void launch_canon_small(ConstEntryArrays raw, const Segments& seg, uint32_t nseg, EntryArrays out,
                        unsigned long long* kept, cudaStream_t st, const uint32_t* dbounds = nullptr,
                        unsigned int* overflow = nullptr, uint64_t cap = ~0ull);

// Sets the shared-memory limits of the attempt kernels (before a graph capture).
void prepare_attempt_kernels();

// Exclusive scan of n uint32 counts into uint32 starts; the total lands in
// starts[n].  Scratch: ceil(n / 2048) + 1 words.  One launch when n <= 65536.
void launch_scan_u32(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* scratch,
                     cudaStream_t st);

// Root-style keys of one L2 list for the ternary merge: the projected quotient
// ((R mod 2^b1) - t) mod 2^b1 >> r2, optionally turned into d = tau - q.
// doff (device, may be null): the list starts doff[0] entries after `l`;
// dvals (device, may be null): {t_lo, t_hi, tau} replacing the by-value targets.
void launch_l2_quotients(ConstEntryArrays l, Count count, uint32_t b1, uint32_t r2,
                         uint64_t t_lo, uint64_t t_hi, int negate, uint64_t tau, uint64_t* key,
                         cudaStream_t st, const uint32_t* doff = nullptr,
                         const uint64_t* dvals = nullptr);

// Parent of every (x, y, z) triple: digits must stay binary and disjoint with
// exactly n/6 ones; valid parents are written compacted (order irrelevant: the
// canonical sort follows).  *count receives the number written.
// doff (device, may be null): x, y, z start doff[0], doff[1], doff[2] entries in.
// rejects (device, may be null): [0] += triples whose children overlap (add_three's
// structural rejects), [1] += disjoint triples with the wrong digit count (its
// distribution rejects); cleared first.
void launch_l1_parents(const uint32_t* triples, Count ntriples, ConstEntryArrays x,
                       ConstEntryArrays y, ConstEntryArrays z, uint32_t n, uint32_t expected_ones,
                       EntryArrays out, unsigned long long* count, cudaStream_t st,
                       const uint32_t* doff = nullptr, unsigned long long* rejects = nullptr);

// Stable LSD radix sort of `count` entries by (pos0, pos1) as one 128-bit key
// with pos0 most significant (the reference's packed_less on the word vector),
// 8-bit digits, only the bits that vary.  Sorts an index permutation in
// ping-pong buffers; `perm_out` receives the sorted order.  Scratch words:
// radix_scratch_words(count).
uint64_t radix_scratch_words(uint64_t count);
void radix_sort_entries(ConstEntryArrays in, Count count, uint64_t vary_pos0, uint64_t vary_pos1,
                        uint32_t* perm_out, uint32_t* scratch, cudaStream_t st);

// Gathers entries in permutation order and drops adjacent repeats of the digit
// words (canonicalize: sort + unique).  *count receives the kept count.
void launch_gather_unique(ConstEntryArrays in, const uint32_t* perm, Count count,
                          EntryArrays out, uint32_t* flags, uint32_t* starts, uint32_t* scratch,
                          unsigned long long* kept, cudaStream_t st);

// OR of all pos0 / pos1 words (to find the varying sort bits).
void launch_or_reduce(ConstEntryArrays in, uint64_t count, unsigned long long* acc, cudaStream_t st);

// dst[0] = *src (one device count saved before a later kernel overwrites it).
void launch_copy_count(const unsigned long long* src, unsigned long long* dst, cudaStream_t st);

// Snapshot records (pos[W64] | neg[W64] | residue[W32]) from entry arrays.
void launch_pack_records(ConstEntryArrays in, Count count, uint32_t n, uint8_t* records,
                         cudaStream_t st);

}  // namespace tergpu
