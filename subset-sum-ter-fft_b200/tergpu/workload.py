"""Seeded root workloads and the sink's order-independent triple digest.

synthetic_root(): three lists of uniform Q-bit keys with the list sizes of an
authentic root (the keys of an authentic root are quotients of uniform residues,
hence uniform themselves), plus planted full-Q triples so a whole-root run has
known outputs.  Generation is counter-based SplitMix64, so any host produces
the same lists for the same seed.

digest(): RootSink's multiset hashes over (a, b, c) EntryIds
(reference ter2_root/frozen/ter_root_queue_kernels.cpp:165-175), vectorized.
"""
from __future__ import annotations

import numpy as np

from .root import RootKeys

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)

# L1 sizes of the n=108 root of seed 0x1001, attempt 0 (3,650,689 x 6,900,048 pairs
# against 6,896,564 targets, 69-bit root quotient).
N108_SIZES = (3_650_689, 6_900_048, 6_896_564)
N108_QUOTIENT_BITS = 69


def mix64(v: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        v = np.asarray(v, dtype=np.uint64) + GOLDEN
        v = (v ^ (v >> np.uint64(30))) * _M1
        v = (v ^ (v >> np.uint64(27))) * _M2
        return v ^ (v >> np.uint64(31))


def splitmix_stream(seed: int, start: int, count: int) -> np.ndarray:
    """Outputs start .. start+count-1 of SplitMix64 seeded with `seed`."""
    with np.errstate(over="ignore"):
        idx = np.arange(start + 1, start + 1 + count, dtype=np.uint64)
        state = np.uint64(seed & (2**64 - 1)) + idx * GOLDEN
        z = (state ^ (state >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def digest(triples: np.ndarray) -> dict:
    t = np.asarray(triples, dtype=np.uint64).reshape(-1, 3)
    a, b, c = t[:, 0], t[:, 1], t[:, 2]
    with np.errstate(over="ignore"):
        first = mix64(((a << np.uint64(32)) | b) ^ mix64(c))
        second = mix64(((c << np.uint64(32)) | a) ^ mix64(b + np.uint64(0x632BE59BD9B4E019)))
        s = int(first.sum(dtype=np.uint64)) if len(t) else 0
        x = int(np.bitwise_xor.reduce(first)) if len(t) else 0
        s2 = int(second.sum(dtype=np.uint64)) if len(t) else 0
    return {"triples": len(t), "triple_sum": s, "triple_xor": x, "triple_sum2": s2}


def synthetic_root(sizes=N108_SIZES, quotient_bits: int = N108_QUOTIENT_BITS, seed: int = 0x1001,
                   planted: int = 8) -> RootKeys:
    """Uniform keys; the last `planted` entries of each list form full-Q
    triples (a_i, b_i, a_i + b_i).  Returns RootKeys (ids = index)."""
    Q = quotient_bits
    lo_mask = np.uint64((1 << min(Q, 64)) - 1) if Q < 64 else np.uint64(2**64 - 1)
    hi_bits = max(0, Q - 64)
    hi_mask = np.uint64((1 << hi_bits) - 1)
    lo, hi = [], []
    offset = 0
    for l in range(3):
        n = sizes[l]
        raw = splitmix_stream(seed, offset, 2 * n)
        offset += 2 * n
        lo.append(raw[0::2] & lo_mask)
        hi.append((raw[1::2] & hi_mask).astype(np.uint8))
    k = min(planted, *sizes)
    for i in range(k):
        a_lo, a_hi = int(lo[0][-1 - i]), int(hi[0][-1 - i])
        b_lo, b_hi = int(lo[1][-1 - i]), int(hi[1][-1 - i])
        v = (((a_hi << 64) | a_lo) + ((b_hi << 64) | b_lo)) & ((1 << Q) - 1)
        lo[2][-1 - i] = np.uint64(v & (2**64 - 1) & int(lo_mask))
        hi[2][-1 - i] = np.uint8(v >> 64)
    return RootKeys(quotient_bits=Q, lo=lo, hi=hi, ids=None)
