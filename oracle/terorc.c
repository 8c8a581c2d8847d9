/*
 * ORACLE -- test infrastructure, never part of the product.
 *
 * A plain-C restatement of the reference's exact depth-3 TER attempt and of its
 * L1 -> L0 root join, used only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py, and there only as the checker.  Nothing in the
 * GPU product links or calls this file.
 *
 * Parity is pinned against the reference itself: tests compare every function
 * here with the reference's own compiled code (oracle/_ref, built from the
 * reference sources by oracle/Makefile) and with golden vectors that the
 * reference's tests and published records hold (tests/golden/).
 *
 * Restated reference behaviour (file:line in the reference project):
 *   SplitMix64 instance generator ........ src/instance.cpp:14-120
 *   benchmark (authentic) instance ....... ter2_root/frozen/ter_root_generalization_workload.cpp:27-65
 *   FiniteSanity parameters r1, r2 ....... src/full_ter.cpp:2581-2767
 *   level-3 half enumeration ............. src/full_ter.cpp:540-617
 *   random targets ....................... src/full_ter.cpp:519-532, 2364-2386
 *   binary L3 -> L2 merge ................ src/full_ter.cpp:827-933
 *   ternary add of packed masks .......... src/packed.cpp:15-38, src/full_ter.cpp:732-790
 *   L2 -> L1 quotient arithmetic ......... src/arithmetic.cpp:9-53, src/full_ter.cpp:1170-1356
 *   canonical order (packed_less) ........ src/full_ter.cpp:320-326, 624-633
 *   design-B root ........................ src/full_ter.cpp:1537-1925
 *   attempt loop and witness check ....... src/full_ter.cpp:2879-2908, 3125-3521
 *   RootSink digest and authority chain .. ter2_root/frozen/ter_root_queue_kernels.cpp:165-195,
 *                                          ter2_root/frozen/ter_translated_tag_dataset.cpp:176-230
 *   synthetic roots with plants .......... ter2_root/tests/ter_synthetic_root.hpp:44-186
 *
 * Scope: ShapeFamily::FiniteSanity (every epsilon zero), n divisible by 36,
 * n <= 128 so a residue fits one unsigned __int128.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* Generators                                                                  */
/* ------------------------------------------------------------------------- */

static uint64_t sm_next(uint64_t *state) {
  uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

uint64_t orc_mix64(uint64_t v) {
  v += 0x9E3779B97F4A7C15ULL;
  v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
  v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
  return v ^ (v >> 31);
}

static uint64_t sm_bounded(uint64_t *state, uint64_t bound) {
  if (bound <= 1) return 0;
  uint64_t threshold = (0 - bound) % bound;
  for (;;) {
    uint64_t v = sm_next(state);
    if (v >= threshold) return v % bound;
  }
}

static u128 mask128(unsigned bits) {
  if (bits >= 128) return ~(u128)0;
  return (((u128)1) << bits) - 1;
}

/*
 * kind 0: build_instance(n, b1, seed) -- uniform n-bit weights and a uniformly
 *         random n/2-subset target (src/instance.cpp:61-120).
 * kind 1: the benchmark / authentic instance -- the same weights with the
 *         planted support fixed to the first n/4 coordinates of each half
 *         (ter_root_generalization_workload.cpp:41-65).
 * values_le: n * W64 words, target_le: W64 words, planted: n bytes.
 */
int orc_build_instance(uint32_t n, uint32_t b1, uint64_t seed, int kind,
                       uint64_t *values_le, uint64_t *target_le, uint8_t *planted) {
  if (n == 0 || n % 2 != 0 || n > 128 || b1 == 0 || b1 >= 64 || b1 >= n) return 1;
  const uint32_t w = (n + 63) / 64;
  uint64_t state = seed;
  const uint32_t high_bits = n % 64;
  const uint64_t high_mask = high_bits == 0 ? ~0ULL : ((1ULL << high_bits) - 1);
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t k = 0; k < w; ++k) values_le[i * w + k] = sm_next(&state);
    values_le[i * w + w - 1] &= high_mask;
  }
  uint32_t perm[128];
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  for (uint32_t remaining = n; remaining > 1; --remaining) {
    uint32_t sel = (uint32_t)sm_bounded(&state, remaining);
    uint32_t tmp = perm[remaining - 1];
    perm[remaining - 1] = perm[sel];
    perm[sel] = tmp;
  }
  memset(planted, 0, n);
  if (kind == 0) {
    for (uint32_t p = 0; p < n / 2; ++p) planted[perm[p]] = 1;
  } else {
    for (uint32_t half = 0; half < 2; ++half)
      for (uint32_t off = 0; off < n / 4; ++off) planted[half * (n / 2) + off] = 1;
  }
  /* target = sum of planted weights, word-wise with carry, top word masked */
  uint64_t acc[2] = {0, 0};
  for (uint32_t i = 0; i < n; ++i) {
    if (!planted[i]) continue;
    uint64_t carry = 0;
    for (uint32_t k = 0; k < w; ++k) {
      uint64_t orig = acc[k];
      uint64_t first = orig + values_le[i * w + k];
      uint64_t c1 = first < orig;
      uint64_t second = first + carry;
      uint64_t c2 = second < first;
      acc[k] = second;
      carry = c1 | c2;
    }
  }
  acc[w - 1] &= high_mask;
  for (uint32_t k = 0; k < w; ++k) target_le[k] = acc[k];
  return 0;
}

/* ------------------------------------------------------------------------- */
/* FiniteSanity parameters: R1 = (n/2)! / (n/6)!^3, R2 = (n/6)! / (n/18)!^3,   */
/* r = floor(log2 R) / 2 (src/full_ter.cpp:2699-2759 with every epsilon 0).    */
/* ------------------------------------------------------------------------- */

typedef struct { uint32_t w[16]; int len; } big_t;

static void big_set(big_t *b, uint32_t v) { memset(b, 0, sizeof *b); b->w[0] = v; b->len = 1; }
static void big_mul(big_t *b, uint32_t m) {
  uint64_t carry = 0;
  for (int i = 0; i < b->len; ++i) {
    uint64_t t = (uint64_t)b->w[i] * m + carry;
    b->w[i] = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry) b->w[b->len++] = (uint32_t)carry;
}
static void big_div(big_t *b, uint32_t d) {
  uint64_t rem = 0;
  for (int i = b->len - 1; i >= 0; --i) {
    uint64_t cur = (rem << 32) | b->w[i];
    b->w[i] = (uint32_t)(cur / d);
    rem = cur % d;
  }
  while (b->len > 1 && b->w[b->len - 1] == 0) --b->len;
}
static uint32_t big_floor_log2(const big_t *b) {
  int top = b->len - 1;
  uint32_t v = b->w[top];
  uint32_t bits = 0;
  while (v >>= 1) ++bits;
  return (uint32_t)top * 32 + bits;
}

/* (total)! / (part!)^3 computed as a product with exact intermediate divisions. */
static uint32_t log2_multinomial3(uint32_t total, uint32_t part) {
  big_t b;
  big_set(&b, 1);
  for (uint32_t i = 2; i <= total; ++i) big_mul(&b, i);
  for (int copy = 0; copy < 3; ++copy)
    for (uint32_t i = 2; i <= part; ++i) big_div(&b, i);
  return big_floor_log2(&b);
}

int orc_params(uint32_t n, uint32_t *r1, uint32_t *r2) {
  if (n == 0 || n % 36 != 0 || n > 128) return 1;
  *r1 = log2_multinomial3(n / 2, n / 6) / 2;
  *r2 = log2_multinomial3(n / 6, n / 18) / 2;
  if (*r2 == 0 || *r2 >= *r1 || *r1 >= n) return 1;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Entries: residue mod 2^n plus packed pos/neg masks (two 64-bit words each). */
/* ------------------------------------------------------------------------- */

typedef struct {
  uint64_t pos[2];
  uint64_t neg[2];
  u128 res;
} entry_t;

static int packed_cmp(const entry_t *a, const entry_t *b) {
  /* words vector = pos[0..W) then neg[0..W), compared lexicographically */
  const uint64_t wa[4] = {a->pos[0], a->pos[1], a->neg[0], a->neg[1]};
  const uint64_t wb[4] = {b->pos[0], b->pos[1], b->neg[0], b->neg[1]};
  for (int i = 0; i < 4; ++i) {
    if (wa[i] != wb[i]) return wa[i] < wb[i] ? -1 : 1;
  }
  return 0;
}
static int packed_cmp_qsort(const void *a, const void *b) { return packed_cmp(a, b); }

/* sort by packed digits and drop repeated digit vectors */
static size_t canonicalize(entry_t *e, size_t count) {
  if (count == 0) return 0;
  qsort(e, count, sizeof *e, packed_cmp_qsort);
  size_t out = 1;
  for (size_t i = 1; i < count; ++i) {
    if (packed_cmp(&e[i], &e[out - 1]) != 0) e[out++] = e[i];
  }
  return out;
}

/* Three-way add of ternary masks: returns 0 when a digit leaves {-1,0,1}
 * (src/packed.cpp:15-38).  The caller checks the digit counts. */
static int add_three(const entry_t *a, const entry_t *b, const entry_t *c, uint32_t n,
                     uint64_t out_pos[2], uint64_t out_neg[2], uint32_t *npos, uint32_t *nneg) {
  uint32_t pc = 0, nc = 0;
  const uint32_t w = (n + 63) / 64;
  for (uint32_t k = 0; k < 2; ++k) {
    out_pos[k] = 0;
    out_neg[k] = 0;
  }
  for (uint32_t k = 0; k < w; ++k) {
    uint64_t ap = a->pos[k], an = a->neg[k], bp = b->pos[k], bn = b->neg[k];
    uint64_t cp = c ? c->pos[k] : 0, cn = c ? c->neg[k] : 0;
    uint64_t pany = ap | bp | cp, nany = an | bn | cn;
    uint64_t ptwo = (ap & bp) | (ap & cp) | (bp & cp);
    uint64_t ntwo = (an & bn) | (an & cn) | (bn & cn);
    uint64_t invalid = (ptwo & ~nany) | (ntwo & ~pany);
    uint64_t one_p = pany & ~ptwo, one_n = nany & ~ntwo;
    uint64_t pp = (one_p & ~nany) | (ptwo & nany);
    uint64_t pn = (one_n & ~pany) | (ntwo & pany);
    uint64_t valid = ~0ULL;
    if (k + 1 == w && n % 64 != 0) valid = (1ULL << (n % 64)) - 1;
    if ((invalid & valid) != 0 || ((pp | pn) & ~valid) != 0) return 0;
    out_pos[k] = pp & valid;
    out_neg[k] = pn & valid;
    pc += (uint32_t)__builtin_popcountll(pp & valid);
    nc += (uint32_t)__builtin_popcountll(pn & valid);
  }
  *npos = pc;
  *nneg = nc;
  return 1;
}

/* One 64-digit word of the packed ternary add (add_packed_word,
 * src/packed.cpp:15-38): 0 when a digit of a + b + c leaves {-1, 0, 1}, else 1
 * with the sum's positive and negative masks. */
int orc_add_packed_word(uint64_t ap, uint64_t an, uint64_t bp, uint64_t bn, uint64_t cp, uint64_t cn,
                        uint64_t *pos, uint64_t *neg) {
  entry_t a = {{ap, 0}, {an, 0}, 0}, b = {{bp, 0}, {bn, 0}, 0}, c = {{cp, 0}, {cn, 0}, 0};
  uint64_t out_pos[2], out_neg[2];
  uint32_t np, nn;
  const int ok = add_three(&a, &b, &c, 64, out_pos, out_neg, &np, &nn);
  *pos = ok ? out_pos[0] : 0;
  *neg = ok ? out_neg[0] : 0;
  return ok;
}

/* ------------------------------------------------------------------------- */
/* Attempt pipeline                                                           */
/* ------------------------------------------------------------------------- */

static u128 instance_coeff(const uint64_t *values_le, uint32_t n, uint32_t i) {
  const uint32_t w = (n + 63) / 64;
  u128 v = values_le[i * w];
  if (w > 1) v |= ((u128)values_le[i * w + 1]) << 64;
  return v;
}

static u128 instance_target(const uint64_t *target_le, uint32_t n) {
  const uint32_t w = (n + 63) / 64;
  u128 v = target_le[0];
  if (w > 1) v |= ((u128)target_le[1]) << 64;
  return v & mask128(n);
}

/* All k-subsets of {0..m-1} in lexicographic order (src/full_ter.cpp:540-578). */
static size_t enumerate_half(uint32_t n, int second, const uint64_t *values_le, entry_t *out) {
  const uint32_t half = n / 2, k = n / 36;
  uint32_t comb[8];
  for (uint32_t i = 0; i < k; ++i) comb[i] = i;
  size_t count = 0;
  const u128 m = mask128(n);
  for (;;) {
    entry_t e;
    memset(&e, 0, sizeof e);
    for (uint32_t i = 0; i < k; ++i) {
      uint32_t coord = comb[i] + (second ? half : 0);
      e.pos[coord / 64] |= 1ULL << (coord % 64);
      e.res = (e.res + instance_coeff(values_le, n, coord)) & m;
    }
    out[count++] = e;
    int idx = (int)k - 1;
    while (idx >= 0 && comb[idx] >= half - (k - (uint32_t)idx)) --idx;
    if (idx < 0) break;
    ++comb[idx];
    for (uint32_t t = (uint32_t)idx + 1; t < k; ++t) comb[t] = comb[t - 1] + 1;
  }
  return count;
}

/* One 32-bit word per SplitMix64 draw: even word -> low half, odd -> high half
 * (src/full_ter.cpp:519-532). */
static u128 sample_residue(uint64_t *state, uint32_t bits) {
  const uint32_t words = (bits + 31) / 32;
  u128 v = 0;
  for (uint32_t i = 0; i < words; ++i) {
    uint64_t r = sm_next(state);
    uint32_t word = (uint32_t)(i % 2 == 0 ? r : r >> 32);
    v |= ((u128)word) << (32 * i);
  }
  return v & mask128(bits);
}

typedef struct {
  u128 t1[3];
  u128 t2[9];
} targets_t;

static void random_targets(uint64_t seed, uint32_t r1, uint32_t r2, u128 T, targets_t *tg) {
  uint64_t state = seed;
  tg->t1[0] = sample_residue(&state, r1);
  tg->t1[1] = sample_residue(&state, r1);
  tg->t1[2] = (T - tg->t1[0] - tg->t1[1]) & mask128(r1);
  for (int g = 0; g < 3; ++g) {
    tg->t2[3 * g] = sample_residue(&state, r2);
    tg->t2[3 * g + 1] = sample_residue(&state, r2);
    tg->t2[3 * g + 2] = (tg->t1[g] - tg->t2[3 * g] - tg->t2[3 * g + 1]) & mask128(r2);
  }
}

typedef struct { uint64_t key; uint32_t id; } keyed_t;
static int keyed_cmp(const void *a, const void *b) {
  const keyed_t *x = a, *y = b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->id < y->id ? -1 : (x->id > y->id);
}
static size_t keyed_lower(const keyed_t *arr, size_t n, uint64_t key) {
  size_t lo = 0, hi = n;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (arr[mid].key < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* binary L3 -> L2 merge: R_l + R_r = t (mod 2^r2), src/full_ter.cpp:827-933 */
static size_t binary_merge(const entry_t *left, size_t nl, const entry_t *right, size_t nr,
                           u128 target, uint32_t r2, uint32_t n, entry_t *out, size_t cap,
                           uint64_t *modular_candidates) {
  keyed_t *idx = malloc(nr * sizeof *idx);
  const u128 m2 = mask128(r2);
  for (size_t i = 0; i < nr; ++i) {
    idx[i].key = (uint64_t)(right[i].res & m2);
    idx[i].id = (uint32_t)i;
  }
  qsort(idx, nr, sizeof *idx, keyed_cmp);
  size_t count = 0;
  for (size_t l = 0; l < nl; ++l) {
    uint64_t need = (uint64_t)((target - left[l].res) & m2);
    for (size_t at = keyed_lower(idx, nr, need); at < nr && idx[at].key == need; ++at) {
      ++*modular_candidates;
      entry_t e;
      uint32_t np, nn;
      if (!add_three(&left[l], &right[idx[at].id], NULL, n, e.pos, e.neg, &np, &nn)) continue;
      if (nn != 0 || np != n / 18) continue; /* level-2 counts {0, n - n/18, n/18} */
      if (count >= cap) { free(idx); return (size_t)-1; }
      e.res = (left[l].res + right[idx[at].id].res) & mask128(n);
      out[count++] = e;
    }
  }
  free(idx);
  return canonicalize(out, count);
}

/* L2 -> L1 ternary merge on the projected quotient (src/full_ter.cpp:1138-1356) */
static size_t ternary_l2_l1(const entry_t *x, size_t nx, const entry_t *y, size_t ny,
                            const entry_t *z, size_t nz, const targets_t *tg, int g,
                            uint32_t n, uint32_t r1, uint32_t r2, entry_t *out, size_t cap,
                            uint64_t *modular_candidates) {
  const uint32_t b1 = r1 < r2 + 32 ? r1 : r2 + 32;
  const u128 m1 = mask128(b1);
  const uint64_t qmask = (1ULL << (b1 - r2)) - 1;
  const u128 ta = tg->t2[3 * g] & mask128(r2), tb = tg->t2[3 * g + 1] & mask128(r2);
  const u128 tc = (tg->t1[g] - ta - tb) & mask128(r2);
  const uint64_t tau = (uint64_t)(((tg->t1[g] - ta - tb - tc) & m1) >> r2);
  const int decisive = (r1 - r2) <= 32;
  uint64_t *qx = malloc(nx * 8), *qy = malloc(ny * 8);
  keyed_t *qz = malloc(nz * sizeof *qz);
  for (size_t i = 0; i < nx; ++i) qx[i] = (uint64_t)((((x[i].res & m1) - ta) & m1) >> r2);
  for (size_t i = 0; i < ny; ++i) qy[i] = (uint64_t)((((y[i].res & m1) - tb) & m1) >> r2);
  for (size_t i = 0; i < nz; ++i) {
    qz[i].key = (uint64_t)((((z[i].res & m1) - tc) & m1) >> r2);
    qz[i].id = (uint32_t)i;
  }
  qsort(qz, nz, sizeof *qz, keyed_cmp);
  size_t count = 0;
  for (size_t i = 0; i < nx; ++i) {
    for (size_t j = 0; j < ny; ++j) {
      uint64_t need = (tau - qx[i] - qy[j]) & qmask;
      for (size_t at = keyed_lower(qz, nz, need); at < nz && qz[at].key == need; ++at) {
        ++*modular_candidates;
        const entry_t *c = &z[qz[at].id];
        entry_t e;
        uint32_t np, nn;
        if (!add_three(&x[i], &y[j], c, n, e.pos, e.neg, &np, &nn)) continue;
        if (nn != 0 || np != n / 6) continue; /* level-1 counts {0, 5n/6, n/6} */
        e.res = (x[i].res + y[j].res + c->res) & mask128(n);
        if (!decisive && ((e.res - tg->t1[g]) & mask128(r1)) != 0) continue;
        if (count >= cap) { free(qx); free(qy); free(qz); return (size_t)-1; }
        out[count++] = e;
      }
    }
  }
  free(qx);
  free(qy);
  free(qz);
  return canonicalize(out, count);
}

/*
 * Result of one attempt.  Level sizes, root candidate accounting and the
 * canonical level-0 parents (pos/neg mask words per parent).
 */
typedef struct {
  int32_t status;            /* 0 NoWitness, 1 Found, <0 error */
  uint32_t r1, r2;
  uint64_t level2_sizes[9];
  uint64_t level1_sizes[3];
  uint64_t level0_size;      /* canonical, after dedup */
  uint64_t l3_modular;       /* L3->L2 modular candidates */
  uint64_t l2_modular;       /* L2->L1 modular candidates */
  uint64_t root_prefilter_candidates; /* low-min(24,Q) quotient matches */
  uint64_t root_full_quotient_rejects;
  uint64_t root_modular_candidates;   /* full-quotient triples */
  uint64_t valid_root_count;          /* accepted before dedup */
  uint64_t witness_pos[2];
  uint64_t witness_neg[2];
  int32_t witness_verified;
} orc_attempt_t;

/* Optional L1 export: per list, residues (lo, hi) and pos/neg masks. */
typedef struct {
  uint64_t *res_lo[3];
  uint64_t *res_hi[3];
  uint64_t *pos0[3];
  uint64_t *pos1[3];
  uint64_t *neg0[3];
  uint64_t *neg1[3];
  uint64_t cap;
  uint64_t t1_lo[3], t1_hi[3];
  uint64_t root_lo, root_hi;
} orc_l1_export_t;

int orc_attempt(uint32_t n, const uint64_t *values_le, const uint64_t *target_le,
                uint64_t attempt_seed, orc_attempt_t *out, orc_l1_export_t *l1x) {
  memset(out, 0, sizeof *out);
  uint32_t r1, r2;
  if (orc_params(n, &r1, &r2) != 0) { out->status = -1; return 1; }
  out->r1 = r1;
  out->r2 = r2;
  const u128 T = instance_target(target_le, n);
  const u128 mn = mask128(n);
  /* level 3: C(n/2, n/36) per half */
  size_t l3cap = 1;
  {
    uint64_t c = 1;
    for (uint32_t i = 0; i < n / 36; ++i) c = c * (n / 2 - i) / (i + 1);
    l3cap = (size_t)c;
  }
  entry_t *left = malloc(l3cap * sizeof(entry_t)), *right = malloc(l3cap * sizeof(entry_t));
  size_t nl = enumerate_half(n, 0, values_le, left);
  size_t nr = enumerate_half(n, 1, values_le, right);
  targets_t tg;
  random_targets(attempt_seed, r1, r2, T, &tg);

  entry_t *l2[9];
  size_t l2n[9];
  size_t l2cap = nl * 8 + 1024;
  for (int i = 0; i < 9; ++i) {
    l2[i] = malloc(l2cap * sizeof(entry_t));
    l2n[i] = binary_merge(left, nl, right, nr, tg.t2[i], r2, n, l2[i], l2cap, &out->l3_modular);
    if (l2n[i] == (size_t)-1) { out->status = -2; return 2; }
    out->level2_sizes[i] = l2n[i];
  }
  entry_t *l1[3];
  size_t l1n[3];
  for (int g = 0; g < 3; ++g) {
    size_t cap = l2n[3 * g] * 64 + 4096;
    cap = cap < 64u * 1024 * 1024 ? cap : 64u * 1024 * 1024;
    l1[g] = malloc(cap * sizeof(entry_t));
    l1n[g] = ternary_l2_l1(l2[3 * g], l2n[3 * g], l2[3 * g + 1], l2n[3 * g + 1], l2[3 * g + 2],
                           l2n[3 * g + 2], &tg, g, n, r1, r2, l1[g], cap, &out->l2_modular);
    if (l1n[g] == (size_t)-1) { out->status = -3; return 3; }
    out->level1_sizes[g] = l1n[g];
  }
  if (l1x != NULL) {
    for (int g = 0; g < 3; ++g) {
      l1x->t1_lo[g] = (uint64_t)tg.t1[g];
      l1x->t1_hi[g] = (uint64_t)(tg.t1[g] >> 64);
      if (l1x->res_lo[g] == NULL || l1n[g] > l1x->cap) continue;
      for (size_t i = 0; i < l1n[g]; ++i) {
        l1x->res_lo[g][i] = (uint64_t)l1[g][i].res;
        l1x->res_hi[g][i] = (uint64_t)(l1[g][i].res >> 64);
        l1x->pos0[g][i] = l1[g][i].pos[0];
        l1x->pos1[g][i] = l1[g][i].pos[1];
        l1x->neg0[g][i] = l1[g][i].neg[0];
        l1x->neg1[g][i] = l1[g][i].neg[1];
      }
    }
    l1x->root_lo = (uint64_t)T;
    l1x->root_hi = (uint64_t)(T >> 64);
  }

  /* design-B root (src/full_ter.cpp:1624-1925) over full quotients */
  const uint32_t Q = n - r1;
  const uint32_t F = Q < 64 ? Q : 64;
  const uint64_t fmask = F == 64 ? ~0ULL : ((1ULL << F) - 1);
  const uint32_t pre = Q < 24 ? Q : 24;
  const uint64_t pmask = (1ULL << pre) - 1;
  u128 tau_res = T;
  for (int g = 0; g < 3; ++g) tau_res = (tau_res - tg.t1[g]) & mn;
  const uint64_t tau = (uint64_t)(tau_res >> r1) & fmask;
  uint64_t *qa = malloc((l1n[0] + 1) * 8), *qb = malloc((l1n[1] + 1) * 8);
  keyed_t *qc = malloc((l1n[2] + 1) * sizeof(keyed_t));
  keyed_t *pc = malloc((l1n[2] + 1) * sizeof(keyed_t));
  for (size_t i = 0; i < l1n[0]; ++i) qa[i] = (uint64_t)(((l1[0][i].res - tg.t1[0]) & mn) >> r1) & fmask;
  for (size_t i = 0; i < l1n[1]; ++i) qb[i] = (uint64_t)(((l1[1][i].res - tg.t1[1]) & mn) >> r1) & fmask;
  for (size_t i = 0; i < l1n[2]; ++i) {
    qc[i].key = (uint64_t)(((l1[2][i].res - tg.t1[2]) & mn) >> r1) & fmask;
    qc[i].id = (uint32_t)i;
    pc[i].key = qc[i].key & pmask;
    pc[i].id = (uint32_t)i;
  }
  qsort(qc, l1n[2], sizeof *qc, keyed_cmp);
  qsort(pc, l1n[2], sizeof *pc, keyed_cmp);
  size_t rcap = 1024, rcount = 0;
  entry_t *roots = malloc(rcap * sizeof(entry_t));
  for (size_t a = 0; a < l1n[0]; ++a) {
    for (size_t b = 0; b < l1n[1]; ++b) {
      uint64_t pneed = (tau - qa[a] - qb[b]) & pmask;
      size_t lo = keyed_lower(pc, l1n[2], pneed), hi = lo;
      while (hi < l1n[2] && pc[hi].key == pneed) ++hi;
      out->root_prefilter_candidates += hi - lo;
      if (hi == lo) continue;
      uint64_t need = (tau - qa[a] - qb[b]) & fmask;
      size_t full = 0;
      for (size_t at = keyed_lower(qc, l1n[2], need); at < l1n[2] && qc[at].key == need; ++at) {
        const entry_t *c = &l1[2][qc[at].id];
        u128 sum = (l1[0][a].res + l1[1][b].res + c->res) & mn;
        if (Q > 64 && sum != T) continue;
        ++full;
        ++out->root_modular_candidates;
        entry_t e;
        uint32_t np, nn;
        if (!add_three(&l1[0][a], &l1[1][b], c, n, e.pos, e.neg, &np, &nn)) continue;
        if (nn != 0 || np != n / 2) continue; /* root counts {0, n/2, n/2} */
        e.res = sum;
        ++out->valid_root_count;
        if (rcount == rcap) {
          rcap *= 2;
          roots = realloc(roots, rcap * sizeof(entry_t));
        }
        roots[rcount++] = e;
      }
      out->root_full_quotient_rejects += (hi - lo) - full;
    }
  }
  rcount = canonicalize(roots, rcount);
  out->level0_size = rcount;
  out->status = 0;
  if (rcount > 0) {
    out->status = 1;
    out->witness_pos[0] = roots[0].pos[0];
    out->witness_pos[1] = roots[0].pos[1];
    out->witness_neg[0] = roots[0].neg[0];
    out->witness_neg[1] = roots[0].neg[1];
    /* verify: binary, weight n/2, inner product equals the target */
    u128 acc = 0;
    uint32_t weight = 0;
    int binary = (roots[0].neg[0] | roots[0].neg[1]) == 0;
    for (uint32_t i = 0; i < n; ++i) {
      if ((roots[0].pos[i / 64] >> (i % 64)) & 1) {
        acc = (acc + instance_coeff(values_le, n, i)) & mn;
        ++weight;
      }
    }
    out->witness_verified = binary && weight == n / 2 && acc == T;
  }
  free(qa); free(qb); free(qc); free(pc); free(roots);
  for (int i = 0; i < 9; ++i) free(l2[i]);
  for (int g = 0; g < 3; ++g) free(l1[g]);
  free(left); free(right);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Root join on full quotient keys and the RootSink digest                     */
/* ------------------------------------------------------------------------- */

typedef struct {
  uint64_t triples;
  uint64_t triple_sum;
  uint64_t triple_xor;
  uint64_t triple_sum2;
  uint64_t full_q;
  uint64_t residue;
  uint64_t residue_sum;
  uint64_t structural;
} orc_digest_t;

/* The sink's order-independent triple hash (ter_root_queue_kernels.cpp:165-175). */
void orc_digest_add(orc_digest_t *d, uint32_t a, uint32_t b, uint32_t c) {
  uint64_t first = orc_mix64((((uint64_t)a << 32) | b) ^ orc_mix64(c));
  uint64_t second = orc_mix64((((uint64_t)c << 32) | a) ^ orc_mix64((uint64_t)b + 0x632BE59BD9B4E019ULL));
  d->triples += 1;
  d->triple_sum += first;
  d->triple_xor ^= first;
  d->triple_sum2 += second;
}

typedef struct {
  uint64_t *slot_key;
  uint32_t *slot_head;
  uint32_t *next;
  uint64_t mask;
} ktable_t;

static void ktable_build(ktable_t *t, const uint64_t *lo, size_t count) {
  uint64_t slots = 16;
  while (slots < 2 * count) slots <<= 1;
  t->mask = slots - 1;
  t->slot_key = malloc(slots * 8);
  t->slot_head = malloc(slots * 4);
  t->next = malloc((count + 1) * 4);
  for (uint64_t s = 0; s < slots; ++s) t->slot_head[s] = UINT32_MAX;
  for (size_t i = count; i-- > 0;) {
    uint64_t h = orc_mix64(lo[i]) & t->mask;
    while (t->slot_head[h] != UINT32_MAX && t->slot_key[h] != lo[i]) h = (h + 1) & t->mask;
    t->slot_key[h] = lo[i];
    t->next[i] = t->slot_head[h];
    t->slot_head[h] = (uint32_t)i;
  }
}
static uint32_t ktable_find(const ktable_t *t, uint64_t key) {
  uint64_t h = orc_mix64(key) & t->mask;
  while (t->slot_head[h] != UINT32_MAX) {
    if (t->slot_key[h] == key) return t->slot_head[h];
    h = (h + 1) & t->mask;
  }
  return UINT32_MAX;
}
static void ktable_free(ktable_t *t) { free(t->slot_key); free(t->slot_head); free(t->next); }

/*
 * Every (a, b, c) with key_a + key_b == key_c (mod 2^bits), bits <= 128, where
 * list 2 already holds d = tau - q_C.  Keys are (lo = bits [0,64), hi = bits
 * [64, bits)).  cells (4096 bytes, index s*64+t over the low 6 key bits) may
 * restrict the pairs like RootIndex::selected; NULL selects all.  Emits into
 * the digest and, up to cap, into triples[3*i].  Returns the triple count.
 */
uint64_t orc_root_join(uint32_t bits, uint64_t na, const uint64_t *a_lo, const uint64_t *a_hi,
                       uint64_t nb, const uint64_t *b_lo, const uint64_t *b_hi, uint64_t nc,
                       const uint64_t *c_lo, const uint64_t *c_hi, const uint8_t *cells,
                       orc_digest_t *digest, uint32_t *triples, uint64_t cap) {
  const uint64_t lo_mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
  const uint64_t hi_mask = bits <= 64 ? 0 : (bits >= 128 ? ~0ULL : ((1ULL << (bits - 64)) - 1));
  ktable_t t;
  ktable_build(&t, c_lo, nc);
  uint64_t count = 0;
  for (uint64_t a = 0; a < na; ++a) {
    for (uint64_t b = 0; b < nb; ++b) {
      if (cells && !cells[(a_lo[a] & 63) * 64 + (b_lo[b] & 63)]) continue;
      uint64_t lo = a_lo[a] + b_lo[b];
      uint64_t carry = lo < a_lo[a];
      uint64_t hi = (a_hi[a] + b_hi[b] + carry) & hi_mask;
      lo &= lo_mask;
      for (uint32_t c = ktable_find(&t, lo); c != UINT32_MAX; c = t.next[c]) {
        if ((c_hi[c] & hi_mask) != hi) continue;
        orc_digest_add(digest, (uint32_t)a, (uint32_t)b, c);
        if (triples && count < cap) {
          triples[3 * count] = (uint32_t)a;
          triples[3 * count + 1] = (uint32_t)b;
          triples[3 * count + 2] = c;
        }
        ++count;
      }
    }
  }
  ktable_free(&t);
  return count;
}

/* Triples agreeing on the low k key bits (k <= 64): ARWLF's projected hits. */
uint64_t orc_projected_count(uint32_t k, uint64_t na, const uint64_t *a_lo, uint64_t nb,
                             const uint64_t *b_lo, uint64_t nc, const uint64_t *c_lo,
                             const uint8_t *cells) {
  const uint64_t m = k >= 64 ? ~0ULL : ((1ULL << k) - 1);
  uint64_t *cm = malloc((nc + 1) * 8);
  for (uint64_t i = 0; i < nc; ++i) cm[i] = c_lo[i] & m;
  ktable_t t;
  ktable_build(&t, cm, nc);
  uint64_t count = 0;
  for (uint64_t a = 0; a < na; ++a)
    for (uint64_t b = 0; b < nb; ++b) {
      if (cells && !cells[(a_lo[a] & 63) * 64 + (b_lo[b] & 63)]) continue;
      for (uint32_t c = ktable_find(&t, (a_lo[a] + b_lo[b]) & m); c != UINT32_MAX; c = t.next[c]) ++count;
    }
  ktable_free(&t);
  free(cm);
  return count;
}

/*
 * The authority chain of the sink for one emitted triple
 * (ter_root_queue_kernels.cpp:176-195): low-32 quotient sum, then the residue
 * sum mod 2^n against the root target, then the FiniteSanity structural count
 * (parent counts {2, n - 4 - n/6, 2 + n/6} from src/shape.cpp:181-207).
 * res: per list residue words (words32 each), q32: per list low-32 quotient
 * (list 2 carries q_C, not d).  pos/neg: per list W64 words each.
 */
void orc_authority(orc_digest_t *d, uint32_t n, uint32_t words32, uint32_t tau_low32,
                   const uint32_t *root_target, const uint32_t *const q32[3],
                   const uint32_t *const res[3], const uint64_t *const pos[3],
                   const uint64_t *const neg[3], uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t ids[3] = {a, b, c};
  if (q32[0][a] + q32[1][b] + q32[2][c] != tau_low32) return;
  d->full_q += 1;
  uint64_t carry = 0;
  for (uint32_t w = 0; w < words32; ++w) {
    uint64_t total = carry + res[0][(uint64_t)a * words32 + w] + res[1][(uint64_t)b * words32 + w] +
                     res[2][(uint64_t)c * words32 + w];
    uint32_t v = (uint32_t)total;
    carry = total >> 32;
    if (w + 1 == words32 && n % 32 != 0) v &= (1u << (n % 32)) - 1;
    if (v != root_target[w]) return;
  }
  d->residue += 1;
  uint64_t first = orc_mix64((((uint64_t)a << 32) | b) ^ orc_mix64(c));
  d->residue_sum += first;
  const uint32_t w64 = (n + 63) / 64;
  uint32_t npos = 0, nneg = 0;
  for (uint32_t w = 0; w < w64; ++w) {
    uint64_t p[3], m[3];
    for (int l = 0; l < 3; ++l) {
      p[l] = pos[l][(uint64_t)ids[l] * w64 + w];
      m[l] = neg[l][(uint64_t)ids[l] * w64 + w];
    }
    /* per coordinate digit sum in {-1, 0, 1} */
    for (uint32_t bit = 0; bit < 64 && w * 64 + bit < n; ++bit) {
      int s = 0;
      for (int l = 0; l < 3; ++l) s += (int)((p[l] >> bit) & 1) - (int)((m[l] >> bit) & 1);
      if (s < -1 || s > 1) return;
      if (s > 0) ++npos;
      if (s < 0) ++nneg;
    }
  }
  if (nneg == 2 && npos == 2 + n / 6) d->structural += 1;
}

/* ------------------------------------------------------------------------- */
/* Synthetic roots (ter2_root/tests/ter_synthetic_root.hpp:113-186)            */
/* ------------------------------------------------------------------------- */

typedef struct { uint64_t lo, hi; } val_t;

static val_t vmask(val_t v, uint32_t bits) {
  if (bits < 64) { v.lo &= (1ULL << bits) - 1; v.hi = 0; return v; }
  v.hi &= (1ULL << (bits - 64)) - 1;
  return v;
}
static val_t vadd(val_t a, val_t b, uint32_t bits) {
  val_t r;
  r.lo = a.lo + b.lo;
  uint64_t carry = r.lo < a.lo;
  r.hi = a.hi + b.hi + carry;
  return vmask(r, bits);
}

typedef struct {
  uint64_t state;
  uint64_t lows[64];
  uint32_t pool;
  uint32_t bits;
} synth_rng_t;

static uint64_t srng_next(synth_rng_t *r) { return orc_mix64(r->state++); }
static val_t srng_value(synth_rng_t *r) {
  val_t v;
  v.lo = srng_next(r);
  v.hi = srng_next(r);
  v = vmask(v, r->bits);
  if (r->pool) v.lo = (v.lo & ~0x7FFFFULL) | r->lows[srng_next(r) % r->pool];
  return v;
}

/*
 * Fills lists (lo/hi arrays, list 2 = d) of a synthetic root with `size`
 * random values per list plus the reference's plants.  Returns the per-list
 * length (identical for all three lists), or 0 when cap is too small.
 */
uint64_t orc_synthetic_root(uint32_t bits, uint64_t seed, uint64_t size, uint32_t pool,
                            uint64_t cap, uint64_t *lo[3], uint64_t *hi[3]) {
  synth_rng_t r;
  memset(&r, 0, sizeof r);
  r.state = seed;
  r.bits = bits;
  r.pool = pool;
  for (uint32_t i = 0; i < pool && i < 64; ++i) r.lows[i] = srng_next(&r) & 0x7FFFFULL;
  uint64_t count = 0;
  const uint64_t needed = size + 40 + 3 + 5 + 3 + (bits > 64 ? 20 : 0);
  if (cap < needed) return 0;
#define PUT(list, v) do { lo[list][count_##list] = (v).lo; hi[list][count_##list] = (v).hi; ++count_##list; } while (0)
  uint64_t count_0 = 0, count_1 = 0, count_2 = 0;
  val_t all_ones = vmask((val_t){~0ULL, ~0ULL}, bits);
  for (int list = 0; list < 3; ++list) {
    for (uint64_t i = 0; i < size; ++i) {
      val_t v = srng_value(&r);
      if (list == 0) PUT(0, v); else if (list == 1) PUT(1, v); else PUT(2, v);
    }
  }
#define PLANT(a, b) do { val_t pa = (a), pb = (b); PUT(0, pa); PUT(1, pb); val_t pd = vadd(pa, pb, bits); PUT(2, pd); } while (0)
  /* The reference writes plant(random_value(), random_value()); C++ leaves the
   * order of the two calls unspecified and the GCC build of the reference (the
   * one that pins this oracle) evaluates the second argument first. */
  for (int i = 0; i < 40; ++i) {
    val_t b = srng_value(&r);
    val_t a = srng_value(&r);
    PLANT(a, b);
  }
  PLANT(all_ones, ((val_t){1, 0}));
  PLANT(all_ones, all_ones);
  PLANT(vmask((val_t){~0ULL, 0}, bits), ((val_t){1, 0}));
  const uint32_t boundaries[5] = {6, 19, 32, 45, 58};
  const uint32_t fast = bits < 64 ? bits : 64;
  for (int i = 0; i < 5; ++i) {
    uint32_t bd = boundaries[i];
    if (bd >= fast) continue;
    uint64_t low = (1ULL << bd) - 1;
    uint64_t x1 = srng_next(&r);
    uint64_t x2 = srng_next(&r);
    PLANT(vmask(((val_t){low | (x1 << bd), x2}), bits), ((val_t){1, 0}));
  }
  {
    val_t a = srng_value(&r);
    val_t b = srng_value(&r);
    for (int copy = 0; copy < 3; ++copy) PLANT(a, b);
  }
  if (bits > 64) {
    for (int i = 0; i < 20; ++i) {
      val_t a = srng_value(&r);
      val_t b = srng_value(&r);
      val_t d = vadd(a, b, bits);
      d.hi ^= 1ULL + (uint64_t)(i % 31);
      d = vmask(d, bits);
      PUT(0, a);
      PUT(1, b);
      PUT(2, d);
    }
  }
  count = count_0;
#undef PUT
#undef PLANT
  return (count_0 == count_1 && count_1 == count_2) ? count : 0;
}
