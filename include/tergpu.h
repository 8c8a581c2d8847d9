/*
 * tergpu.h -- C ABI of the B200 root backend for the exact depth-3 TER attempt.
 *
 * Plain pointers and sizes only.  Every entry point is synchronous from the
 * caller's view: inputs are host buffers (read only), the call uploads them,
 * runs the device kernels on one CUDA stream of its own and copies the results
 * back before it returns.  The library holds a per-device workspace between
 * calls; tergpu_release() frees it.
 *
 * Status values 0..11 are the numeric values of ter::Status
 * (reference include/ter/types.hpp:10-23).  Values from 64 up are this ABI's
 * own and never collide with ter::Status.
 */
#ifndef TERGPU_H
#define TERGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: tergpu_root_in / tergpu_root_records_in gained shard_index and shard_count.
 * 3: tergpu_attempt_in gained root_policy, tergpu_attempt_stats the reference's
 *    per-stage counters and output fingerprints, tergpu_attempt_out the run
 *    fingerprint and the level-3 time.
 * 4: tergpu_attempt_stats gained audited_stages (TERGPU_ATTEMPT_AUDIT).
 * 5: tergpu_attempt_in gained planted_root (TERGPU_ATTEMPT_GUIDED) and fixture_level3_limit
 *    (TERGPU_ATTEMPT_FIXTURE).
 * Callers compiled against another version must not call in (the adapter checks). */
#define TERGPU_ABI_VERSION 5

enum tergpu_status {
  TERGPU_COMPLETED = 0,
  TERGPU_FOUND = 1,
  TERGPU_NO_WITNESS_THIS_ATTEMPT = 2,
  TERGPU_ATTEMPT_LIMIT_REACHED = 3,
  TERGPU_INVALID_CONFIGURATION = 4,
  TERGPU_INVALID_SHAPE = 5,
  TERGPU_GENERATION_INCOMPLETE = 6,
  TERGPU_RESOURCE_LIMIT = 7,
  TERGPU_CANCELLED = 8,
  TERGPU_INVARIANT_VIOLATION = 9,
  TERGPU_NOT_APPLICABLE = 10,
  TERGPU_UNSUPPORTED_WIDTH = 11,
  /* ABI-specific */
  TERGPU_OUTPUT_OVERFLOW = 64, /* more triples than capacity: nothing was emitted,
                                  out->triples_count holds the exact count */
  TERGPU_DEVICE_ERROR = 65,    /* no CUDA device, or a CUDA call failed */
  TERGPU_INVALID_INPUT = 66    /* malformed arguments (null pointers, widths) */
};

/* Largest root quotient width the backend accepts: bits [64, Q) travel in one
 * byte per entry, like the reference's FamilyKeys::hi. */
#define TERGPU_MAX_QUOTIENT_BITS 72u

/* tergpu_root_in.flags */
#define TERGPU_ROOT_COUNT_ONLY 1u    /* count triples, write none */
#define TERGPU_ROOT_DEVICE_INPUTS 2u /* key_lo / key_hi / id / cells are device pointers of
                                        `device`, already resident: nothing is uploaded */
#define TERGPU_ROOT_SWEEP_V1 4u      /* sweep variant 1: A in registers, B broadcast */
#define TERGPU_ROOT_AUTOTUNE 16u     /* family bits, filter bits and sweep variant picked per root
                                        shape by timing the neighbours of the size-based choice
                                        on 1/64 of the target families (cached per shape for the
                                        process; ignored when family_bits, filter_bits or a
                                        variant flag is given); same results */
#define TERGPU_ROOT_SWEEP_V2 8u      /* sweep variant 2: B in registers (families sorted by
                                        window), A broadcast.  Same results */
#define TERGPU_ROOT_SWEEP_V4 32u     /* sweep variant 4: a table of 0/1 words over the low 14
                                        residual bits probed with one add, one shared load
                                        and one shift-add per pair, B families laid out one
                                        bank per lane; its table passes about 2.5 % of the
                                        pairs (the default's filter 0.16 %), which makes it
                                        slower at n = 108.  Default (no variant flag):
                                        variant 3, variant 2 with B families laid out in
                                        lane slots of distinct residual classes and filter
                                        words picked by the low probe bits (bank-free
                                        shared-memory probes).  Variants 3 and 4 need 32 or
                                        more residual bits, else variant 2 runs.  Same
                                        results */
#define TERGPU_ROOT_PARTITION_ONE_PASS 64u /* lists of 2^20 or more entries go to their families
                                        in one pass of scattered stores, as shorter lists
                                        always do.  Default: two staged passes (high family
                                        digit into buckets, then low digit into families),
                                        each sorting a tile of 4,096 entries by digit in
                                        shared memory so stores form runs.  Same results */

/*
 * One L1 -> L0 root on full quotient keys.
 *
 * Replaces the body of a frozen root backend: the C ABI a run_gpu_root adapter
 * with the signature of run_hash_join
 * (reference ter2_root/campaign/ter_hash_join_root.hpp:38-40) calls after
 * flattening mr8::Dataset + a64::FamilyKeys
 * (ter2_root/frozen/ter_microreport8_dataset.hpp:60-64,
 *  ter2_root/frozen/ter_a64_chqr.hpp:55-63).
 *
 * List 0 holds q_A, list 1 q_B and list 2 d = tau - q_C, all mod 2^Q, so a
 * full-Q triple is (a, b, c) with key_a + key_b == key_c (mod 2^Q).  key_lo
 * holds bits [0, min(Q, 64)), key_hi bits [64, Q) (may be NULL when Q <= 64).
 * id maps an entry to the EntryId reported in triples (NULL: the index).
 * cells (4096 bytes, index s * 64 + t with s, t the low 6 key bits of the A
 * and B entries) restricts the pairs exactly like RootIndex::selected
 * (ter2_root/frozen/ter_root_queue_kernels.hpp:63-67); NULL selects all.
 */
typedef struct {
  uint32_t quotient_bits;      /* Q, 1..TERGPU_MAX_QUOTIENT_BITS */
  uint32_t flags;              /* TERGPU_ROOT_* */
  uint64_t count[3];
  const uint64_t *key_lo[3];
  const uint8_t *key_hi[3];
  const uint32_t *id[3];
  const uint8_t *cells;
  uint32_t projected_bits;     /* > 0: also count triples equal on key bits [0, k), k <= 64 */
  int32_t device;              /* CUDA device ordinal */
  uint64_t memory_limit_bytes; /* device bytes the call may hold; 0: no ceiling */
  uint32_t family_bits;        /* 0: autotuned; else the device partition radix (6..16) */
  uint32_t filter_bits;        /* 0: autotuned; else log2 of the filter bitmap bits (10..20) */
  void *stream;                /* cudaStream_t to launch on; NULL: the library's own */
  uint32_t shard_index;        /* join only the pairs whose sum key_a + key_b is */
  uint32_t shard_count;        /* == shard_index (mod shard_count), i.e. the D entries with
                                  key_d == shard_index (mod shard_count); shard_count 0 or 1:
                                  the whole root, else a power of two <= 64.  The shards of
                                  one root are disjoint and together give the whole root
                                  (the multi-GPU split: one shard per GPU) */
} tergpu_root_in;

typedef struct {
  uint32_t *triples;        /* capacity * 3 EntryIds: (a, b, c) per full-Q triple */
  uint64_t capacity;
  uint64_t triples_count;   /* full-Q triples, with multiplicity */
  uint64_t logical_pairs;   /* sum over selected cells of |A_s| * |B_t| */
  uint64_t filter_survivors;/* pairs that passed the on-chip filter */
  uint64_t fast_hits;       /* triples equal on the low min(Q, 64) bits */
  uint64_t projected_hits;  /* triples equal on the low projected_bits bits */
  uint64_t device_bytes;    /* device workspace held by the call */
  double join_ms;           /* device time of the partition + join kernels */
  double partition_ms;      /* device time of the partition kernels alone */
  double sweep_ms;          /* device time of the sweep kernel(s) alone */
  double total_ms;          /* wall time of the call */
  uint32_t family_bits;     /* tuning the call ran with */
  uint32_t filter_bits;
  uint32_t kernel_launches; /* device kernels this call launched */
  uint32_t sweep_variant;   /* sweep variant the join ran (1, 2 or 3) */
  double tune_ms;           /* device time the autotuner spent (0: no tuning or cached shape) */
} tergpu_root_out;

/* Replaces: run_hash_join / run_arwlf / run_k2_wide bodies
 * (ter2_root/campaign/ter_hash_join_root.cpp:73-215,
 *  ter2_root/frozen/ter_arwlf.cpp:256-418, ter2_root/frozen/ter_a64_chqr.cpp:329-416). */
int tergpu_root_run(const tergpu_root_in *in, tergpu_root_out *out);

/*
 * One L1 -> L0 root straight from the three captured L1 lists, with the final
 * decision on the original residue words on the device.
 *
 * Records use the layout of the reference's FullTerRootStream / .snap record
 * (include/ter/full_ter.hpp:297-303, ter2_root/frozen/ter_root_snapshot.hpp:9-11):
 *   uint64 pos[W64] | uint64 neg[W64] | uint32 residue[W32]
 * with W64 = ceil(n/64), W32 = ceil(n/32).  EntryId = record index.
 * The device derives q_L = ((R - c_L) mod 2^n) >> r1 over Q = n - r1 bits and
 * d = tau - q_C with tau = ((T - c_0 - c_1 - c_2) mod 2^n) >> r1, exactly as
 * load_snapshot_workload (ter2_root/frozen/ter_root_generalization_workload.cpp:630-702)
 * and ternary_tiled_l1_to_l0 (src/full_ter.cpp:1747-1763) do.
 *
 * For every full-Q triple the device then applies the authority chain of
 * RootSink::emit_triple (ter2_root/frozen/ter_root_queue_kernels.cpp:165-195):
 * residue sum == T (mod 2^n) over all residue words, the FiniteSanity
 * structural count, and the root rule of solve_attempt
 * (ter2_root/campaign/ter_arwlf_solve.cpp:100-114): the parent digit sum is
 * binary with weight n/2 (the design-B root's valid roots, src/full_ter.cpp:1576-1598).
 */
typedef struct {
  uint32_t n;                  /* 36 | n, n <= 128 */
  uint32_t r1;
  uint32_t flags;
  uint32_t record_bytes;       /* 16 * W64 + 4 * W32 */
  uint64_t count[3];
  const uint8_t *records[3];
  const uint32_t *child_target[3]; /* W32 words each, little endian */
  const uint32_t *root_target;     /* W32 words */
  const uint8_t *cells;
  uint32_t projected_bits;
  int32_t device;
  uint64_t memory_limit_bytes;
  uint32_t family_bits;
  uint32_t filter_bits;
  uint32_t shard_index;        /* as tergpu_root_in.shard_index / shard_count */
  uint32_t shard_count;
} tergpu_root_records_in;

typedef struct {
  tergpu_root_out root;        /* triples, counts and timing of the join */
  uint8_t *triple_flags;       /* capacity bytes (may be NULL): bit0 residue-exact,
                                  bit1 FiniteSanity structural, bit2 root rule */
  uint64_t residue_exact;      /* triples whose residues sum to T */
  uint64_t structural;         /* ... that also pass the FiniteSanity structural count */
  uint64_t valid_roots;        /* ... residue-exact with a binary weight-n/2 parent */
  uint64_t tau_lo;             /* the root quotient target */
  uint64_t tau_hi;
} tergpu_root_records_out;

/* Replaces: ternary_tiled_l1_to_l0 + full_ter_root_tiled_visitor
 * (src/full_ter.cpp:1537-1925) and the root pass of solve_attempt
 * (ter2_root/campaign/ter_arwlf_solve.cpp:41-178). */
int tergpu_root_run_records(const tergpu_root_records_in *in, tergpu_root_records_out *out);

/*
 * Exact depth-3 TER attempts on the device: the attempt loop of solve_full_ter
 * (reference src/full_ter.cpp:2933-3521, FiniteSanity shape, Random targets).
 *
 * Per attempt a in [attempt_first, attempt_first + attempt_count): targets from
 * SplitMix64(seed + a) (src/full_ter.cpp:2364-2386), nine L3 -> L2 binary merges
 * (src/full_ter.cpp:827-933), three L2 -> L1 ternary merges on the projected
 * quotient (src/full_ter.cpp:1138-1356), each level in the reference's canonical
 * order (sorted by packed digit words, duplicates dropped), then the root with
 * the device authority (as tergpu_root_run_records).  A valid root stops the
 * loop: the lowest parent in canonical order is verified on the host (binary,
 * weight n/2, sum of the chosen weights == target mod 2^n,
 * src/full_ter.cpp:2879-2908) and returned as the witness.
 *
 * Statuses: TERGPU_FOUND, TERGPU_ATTEMPT_LIMIT_REACHED (budget spent, never UNSAT),
 * TERGPU_CANCELLED (*cancel != 0 when the call starts -- returned before level 3
 * and any device work, with the run fingerprint of no attempts under
 * TERGPU_ATTEMPT_TELEMETRY, as the reference's pre-cancelled solve -- or before
 * an attempt or stage, or inside a sweep), TERGPU_RESOURCE_LIMIT (the predicted
 * device bytes exceed memory_limit_bytes, refused before any allocation),
 * TERGPU_INVALID_CONFIGURATION (36 does not divide n or n > 108, attempt_count
 * 0, root_policy CountOnly or unknown, flag bits outside TERGPU_ATTEMPT_*, an
 * unbalanced planted root under TERGPU_ATTEMPT_GUIDED, fixture limit 0; all
 * before any device work), TERGPU_INVARIANT_VIOLATION (a witness that fails
 * verification, or an audited stage that disagrees with its scalar oracle).
 */
typedef struct {
  uint32_t attempt;
  int32_t status;              /* TERGPU_FOUND or TERGPU_NO_WITNESS_THIS_ATTEMPT */
  uint64_t level2_sizes[9];
  uint64_t level1_sizes[3];
  uint64_t level0_size;        /* parents the root policy retains (FirstWitness: 0 or 1) */
  uint64_t l3_modular;         /* L3 -> L2 pairs meeting the congruence */
  uint64_t l2_modular;         /* L2 -> L1 triples meeting the quotient congruence */
  uint64_t root_modular;       /* root triples passing the full quotient (and, for Q > 64,
                                  the residue words): FirstWitness counts up to the stop */
  uint64_t valid_roots;        /* ... with a binary weight-n/2 parent, pre-dedup (the
                                  reference's valid_root_count for the policy) */
  uint64_t root_pairs;         /* |L1_0| * |L1_1| */
  double l2_ms, l1_ms, root_ms, total_ms;
  /* The reference's FullTerStageTelemetry counters (include/ter/full_ter.hpp:111-146)
   * for level3_to_level2 (l3_*), level2_to_level1 (l2_*) and level1_to_level0 (root_*).
   * Filled on every attempt; the root's low-prefilter count and the output
   * fingerprints need TERGPU_ATTEMPT_TELEMETRY (0 without it). */
  uint64_t attempt_seed;       /* seed + attempt */
  uint64_t l3_pairs, l3_structural_rejects, l3_distribution_rejects, l3_survivors;
  uint64_t l2_pairs, l2_structural_rejects, l2_distribution_rejects, l2_survivors;
  uint64_t root_structural_rejects, root_distribution_rejects;
  uint64_t root_low_prefilter;         /* triples equal on the low root_prefilter_bits */
  uint64_t root_full_quotient_rejects; /* ... failing the full quotient / residue words */
  uint32_t root_quotient_bits, root_prefilter_bits;
  uint32_t root_policy;        /* the policy the root ran with (TERGPU_ROOT_POLICY_*) */
  uint32_t root_early_stopped; /* FirstWitness stopped at a valid root */
  uint64_t l2_fingerprint;     /* stage_fingerprint of the nine L2 lists */
  uint64_t l1_fingerprint;     /* ... of the three L1 lists */
  uint64_t l0_fingerprint;     /* ... of the retained L0 parents */
  double verification_ms;      /* host verification of the witness */
  uint32_t audited_stages;     /* TERGPU_ATTEMPT_AUDIT: stages checked against the scalar
                                  oracles (the nine L3 -> L2 merges, the three L2 -> L1
                                  merges and the root, where the oracle's work is at most
                                  10^6 pairs or triples) */
  uint32_t reserved_audit;
} tergpu_attempt_stats;

/* tergpu_attempt_in.flags */
#define TERGPU_ATTEMPT_CAPTURE_ONLY 1u /* stop after L1 (export only): the device
                                          counterpart of stream_full_ter_root_lists */
#define TERGPU_ATTEMPT_NO_GRAPH 4u     /* n = 36 and 72 run each attempt as one captured CUDA
                                          graph (fixed capacities, counts kept on the device);
                                          this flag runs the stage-by-stage path instead.
                                          Same results */
#define TERGPU_ATTEMPT_TELEMETRY 8u    /* the reference's full attempt telemetry: the root's
                                          low-prefilter count (one more count-only root
                                          join), every stage's output_fingerprint (the
                                          canonical lists are downloaded and hashed on the
                                          host) and out->fingerprint.  Runs stage by stage */
#define TERGPU_ATTEMPT_BACKGROUND 16u  /* run on the workspace's lowest-priority stream, so
                                          work of higher priority on the device (the other
                                          slots of tergpu_attempt_batch, which sets this flag
                                          for n >= 108) takes SMs first as this attempt's
                                          sweep blocks finish; its joins use blocks of about
                                          2^25 pairs (about 2 ms of one SM) instead of 2^29,
                                          so SMs come free often.  Same results */
#define TERGPU_ATTEMPT_AUDIT 32u      /* the reference's audit mode (FullTerConfig::audit,
                                          src/full_ter.cpp:3186-3222, 3318-3334, 3449-3465):
                                          every stage whose scalar oracle needs at most 10^6
                                          pairs or triples (every stage at n = 36, the
                                          L3 -> L2 merges at n = 72) is recomputed on the host
                                          by plain enumeration and compared with the device's
                                          output and provenance; a difference returns
                                          TERGPU_INVARIANT_VIOLATION.  Runs stage by stage and
                                          reports the root as FullCanonicalOutput, as the
                                          reference's audit does */
#define TERGPU_ATTEMPT_GUIDED 64u     /* the reference's GuidedPlanted targets
                                          (TerTargetMode::GuidedPlanted, src/full_ter.cpp:
                                          2281-2317, 2412-2428): planted_root, which must hold
                                          n/4 ones in each half, is split into three level-1
                                          and nine level-2 vectors, each half's ones dealt out
                                          in order, and every attempt's targets are those
                                          vectors' residues (masked to r1 / r2 bits) instead
                                          of SplitMix64 draws; an unbalanced or missing
                                          planted root is TERGPU_INVALID_CONFIGURATION */
#define TERGPU_ATTEMPT_FIXTURE 128u   /* the reference's FixtureTer execution
                                          (TerExecutionMode::FixtureTer, src/full_ter.cpp:
                                          2785-2845, 2319-2362): each level-3 half is its first
                                          min(C(n/2, n/36), fixture_level3_limit) k-subsets in
                                          enumeration order; with TERGPU_ATTEMPT_GUIDED the
                                          halves of the nine guided level-2 vectors come first
                                          and the first subsets fill up to the limit, in
                                          canonical order (a limit below the guided halves is
                                          TERGPU_RESOURCE_LIMIT).  Runs stage by stage */
#define TERGPU_ATTEMPT_PREFLIGHT 2u    /* derive r1, r2, the level-3 size and the predicted
                                          device bytes (out->device_bytes), check them
                                          against memory_limit_bytes and return
                                          TERGPU_COMPLETED without device work; the
                                          instance may be NULL (ter_full_bench --preflight).
                                          The shape, policy, flag and fixture-limit
                                          refusals are the call's own; the budget, cancel
                                          flag and guided root are not checked */

typedef struct {
  uint32_t n;                  /* 36, 72 or 108 */
  uint32_t flags;
  const uint64_t *values_le;   /* n * ceil(n/64) words: the weights */
  const uint64_t *target_le;   /* ceil(n/64) words */
  uint64_t seed;               /* attempt a draws its targets from seed + a */
  uint32_t attempt_first;
  uint32_t attempt_count;
  uint64_t memory_limit_bytes; /* 0: no ceiling */
  const volatile int32_t *cancel; /* host flag, polled between stages and inside the root
                                     and L2 -> L1 sweeps (mirrored into a device-visible word
                                     every 200 us; each warp reads it every eighth work item),
                                     so a running n = 108 sweep stops within milliseconds:
                                     TERGPU_CANCELLED.  May be NULL */
  int32_t device;
  uint32_t root_policy;        /* TERGPU_ROOT_POLICY_* (the numerics of ter::RootOutputPolicy,
                                  include/ter/full_ter.hpp:79-83) */
  const uint8_t *planted_root; /* TERGPU_ATTEMPT_GUIDED: the instance's planted solution, n digits
                                  of 0 or 1 (Instance::planted_root); NULL otherwise */
  uint64_t fixture_level3_limit; /* TERGPU_ATTEMPT_FIXTURE: level-3 entries per half (> 0) */
} tergpu_attempt_in;

/* tergpu_attempt_in.root_policy.  FirstWitness (the reference's default): the
 * root stops at the first valid triple in the order the reference's tiled
 * reporter visits triples (src/tiled_q3report.cpp:365-410: window m = i + j of
 * the prefilter buckets, bucket i of A, then A's and B's EntryIds, then C's
 * EntryId descending); that triple's parent is the witness and the root's
 * counters stop there.  FullCanonicalOutput: every valid parent, sorted and
 * deduplicated; the witness is the first of them.  CountOnly is refused with
 * TERGPU_INVALID_CONFIGURATION before any work, as solve_full_ter refuses it (a
 * SAT result must keep a verifiable witness; src/full_ter.cpp:2945-2957): the
 * root reports count without retaining (report_full_ter_root /
 * count_full_ter_root over tergpu_root_run_records). */
#define TERGPU_ROOT_POLICY_FIRST_WITNESS 0u
#define TERGPU_ROOT_POLICY_COUNT_ONLY 1u
#define TERGPU_ROOT_POLICY_FULL_CANONICAL 2u

typedef struct {
  int32_t status;
  uint32_t r1, r2;
  uint64_t level3_size;        /* entries per half */
  uint32_t attempts_run;
  uint32_t found_attempt;
  uint8_t witness[128];        /* digits 0/1 of the verified witness when FOUND */
  tergpu_attempt_stats *stats; /* attempt_count entries (may be NULL) */
  uint8_t *l1_records[3];      /* optional: L1 lists of the last attempt run, as
                                  .snap records (capacity l1_capacity[l] records) */
  uint64_t l1_capacity[3];
  uint32_t child_targets[3][4];/* the last attempt's L1 targets (words32) */
  uint32_t root_target[4];
  uint64_t device_bytes;        /* predicted device bytes (the preflight's admission figure) */
  double total_ms;
  uint64_t device_bytes_held;   /* device bytes the call's workspace held at its end (its peak:
                                   buffers only grow within a call; the shared workspace keeps
                                   buffers of earlier calls, a batch request starts empty) */
  uint64_t fingerprint;         /* TERGPU_ATTEMPT_TELEMETRY: FullTerTelemetry::fingerprint
                                   (src/full_ter.cpp:2532-2577) over the attempts this call ran
                                   and the witness; the reference's value when attempt_first = 0 */
  double level3_ms;             /* TERGPU_ATTEMPT_TELEMETRY: wall time of the level-3
                                   enumeration (0 without it) */
} tergpu_attempt_out;

/* Replaces: solve_full_ter's attempt loop (src/full_ter.cpp:3125-3515) and
 * stream_full_ter_root_lists (src/full_ter.cpp:3926-4195) for the L1 export. */
int tergpu_attempt_run(const tergpu_attempt_in *in, tergpu_attempt_out *out);

/*
 * Many independent attempt ranges on one device at once: the batched and served
 * paths (continuous batching).  No counterpart in the reference, whose solver
 * runs one attempt at a time on one thread.
 *
 * Request i is jobs[i] (its device field is ignored: the batch's device is used)
 * and its result outs[i], exactly what tergpu_attempt_run(&jobs[i], &outs[i])
 * returns when called alone (status, attempts_run, stats, witness, found_attempt,
 * r1, r2, level3_size); outs[i].status carries the status.  The unit of work is
 * one attempt: `slots` attempts run concurrently, each on a host thread with its
 * own CUDA stream and device workspace, and a request is decided by its lowest
 * attempt that is not NoWitnessThisAttempt (attempts above it are not started);
 * L1 exports (outs[i].l1_records) are not produced in a batch.  A request becomes eligible at arrival_ms[i]
 * after the call starts (NULL: all at once); eligible requests are admitted in
 * arrival order while a slot is free and the predicted device bytes of the
 * running requests (each request's preflight) stay within memory_budget_bytes;
 * a request that does not fit yet waits and later requests that fit go ahead.
 * Requests the preflight refuses (InvalidConfiguration; ResourceLimit against
 * their own ceiling or above the whole budget) complete immediately with that
 * status, before any device work.  admit_ms / finish_ms (optional) receive each
 * request's start on a slot and completion, in ms after the call started.
 * Returns TERGPU_COMPLETED when every request has a result.
 */
typedef struct {
  const tergpu_attempt_in *jobs;
  tergpu_attempt_out *outs;     /* outs[i].stats (attempt_count entries) as in tergpu_attempt_run */
  uint64_t count;
  const double *arrival_ms;     /* may be NULL */
  uint32_t slots;               /* concurrent attempt pipelines; 0: 8 */
  int32_t device;
  uint64_t memory_budget_bytes; /* 0: 90% of the device's free memory at the start */
  double *admit_ms;             /* may be NULL */
  double *finish_ms;            /* may be NULL */
} tergpu_batch_in;

typedef struct {
  double total_ms;              /* wall time from the start to the last result */
  uint64_t peak_predicted_bytes;/* largest predicted bytes of the requests running at once */
  uint32_t peak_running;        /* most requests running at once */
  uint64_t refused;             /* requests completed at admission by the preflight */
} tergpu_batch_out;

/* The slots run two streams each (TERGPU_ATTEMPT_BACKGROUND for n >= 108 on the lower-priority
 * one).  CUDA maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware work queues (8 unless
 * set), so with more streams than queues a short request's kernel can wait behind a long one
 * queued earlier on another slot's stream.  Loading this library sets the variable to 32 when
 * the caller has not set it; it takes effect only for a CUDA context created afterwards, so a
 * caller that initializes CUDA first should set it itself. */
int tergpu_attempt_batch(const tergpu_batch_in *in, tergpu_batch_out *out);

/*
 * The root join for callers that cannot allocate device memory.  This entry
 * has no counterpart in the reference: it exists for callers such as a host
 * framework that owns every device allocation through its own pool, a process
 * whose device memory is reserved up front, or a service loop that must not
 * risk an allocation's synchronization or failure.
 *
 * The caller passes device-resident inputs (flags must include
 * TERGPU_ROOT_DEVICE_INPUTS; key_lo / key_hi / id / cells are device pointers)
 * and a DEVICE buffer out->triples of out->capacity triples.  All
 * intermediates live in one fixed 32 MiB device array inside the library
 * (held by every GPU that loads the library until the process exits); a root
 * whose intermediates do not fit (about 2.4 million key entries over the three
 * lists) is refused with TERGPU_RESOURCE_LIMIT.  Projected counts are not
 * offered here; family bits are limited to 6..10.
 *
 * The first call on a device looks up the array's device address (a lookup,
 * not an allocation).  Every call waits for its stream to finish (it reads the
 * counters back), so a call on a stream under capture is refused with
 * TERGPU_INVALID_INPUT.  The call leaves the caller's current device as it
 * found it.  Every call reuses the same array, so calls whose work overlaps on
 * the GPU race: issue them one after another.  join_ms / partition_ms /
 * sweep_ms are not measured (no events are created) and read 0.
 */
int tergpu_root_run_noalloc(const tergpu_root_in *in, tergpu_root_out *out);

/* Error text of the calling thread's last tergpu_root_run_noalloc call. */
const char *tergpu_noalloc_last_error(void);

/* FNV-1a-64 over size bytes starting from state (0xcbf29ce484222325 for a fresh
 * hash): the list and header checksums of the .snap format
 * (reference ter2_root/frozen/ter_root_snapshot.cpp:94-101).  Host code only. */
uint64_t tergpu_fnv1a(const void *bytes, uint64_t size, uint64_t state);

/* Number of CUDA devices visible to the library (0 when none). */
int tergpu_device_count(void);

/* ABI version compiled into the library. */
int tergpu_abi_version(void);

/* Frees every per-device workspace the library holds. */
void tergpu_release(void);

/* Last error text of the calling thread ("" when none). */
const char *tergpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TERGPU_H */
