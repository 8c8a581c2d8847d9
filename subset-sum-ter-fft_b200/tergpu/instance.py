"""Seeded density-one Subset Sum instances (the reference's generators).

build_instance(n, seed): weights uniform n-bit from SplitMix64 (each word one
draw, the top word masked), then a Fisher-Yates permutation whose first n/2
entries form the planted subset; target = their sum mod 2^n
(reference src/instance.cpp:14-120, b1 = 10).
benchmark_instance(n, seed): the same weights with the planted support fixed
to the first n/4 coordinates of each half -- the instance every authentic
capture and published root of the reference uses
(ter2_root/frozen/ter_root_generalization_workload.cpp:27-65).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

M64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & M64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def bounded(self, bound: int) -> int:
        if bound <= 1:
            return 0
        threshold = ((1 << 64) - bound) % bound
        while True:
            v = self.next()
            if v >= threshold:
                return v % bound


@dataclass
class Instance:
    n: int
    seed: int
    values_le: np.ndarray   # uint64 [n, ceil(n/64)]
    target_le: np.ndarray   # uint64 [ceil(n/64)]
    planted: np.ndarray     # uint8 [n]

    def weight(self, i: int) -> int:
        return sum(int(w) << (64 * k) for k, w in enumerate(self.values_le[i]))

    @property
    def target(self) -> int:
        return sum(int(w) << (64 * k) for k, w in enumerate(self.target_le)) & ((1 << self.n) - 1)


def _generate(n: int, seed: int, fixed_support: bool) -> Instance:
    if n <= 0 or n % 2 != 0 or n > 128:
        raise ValueError("instance requires positive even n <= 128")
    w = (n + 63) // 64
    rng = SplitMix64(seed)
    high_bits = n % 64
    high_mask = M64 if high_bits == 0 else (1 << high_bits) - 1
    values = np.zeros((n, w), dtype=np.uint64)
    for i in range(n):
        for k in range(w):
            values[i, k] = rng.next()
        values[i, w - 1] = int(values[i, w - 1]) & high_mask
    perm = list(range(n))
    for remaining in range(n, 1, -1):
        sel = rng.bounded(remaining)
        perm[remaining - 1], perm[sel] = perm[sel], perm[remaining - 1]
    planted = np.zeros(n, dtype=np.uint8)
    if fixed_support:
        for half in range(2):
            planted[half * (n // 2): half * (n // 2) + n // 4] = 1
    else:
        planted[perm[: n // 2]] = 1
    total = 0
    for i in range(n):
        if planted[i]:
            total += sum(int(values[i, k]) << (64 * k) for k in range(w))
    total &= (1 << n) - 1
    target = np.array([(total >> (64 * k)) & M64 for k in range(w)], dtype=np.uint64)
    return Instance(n=n, seed=seed, values_le=values, target_le=target, planted=planted)


def build_instance(n: int, seed: int) -> Instance:
    return _generate(n, seed, fixed_support=False)


def benchmark_instance(n: int, seed: int) -> Instance:
    return _generate(n, seed, fixed_support=True)


def verify_witness(instance: Instance, witness) -> bool:
    """verify_full_ter_witness (src/full_ter.cpp:2879-2908): binary digits,
    Hamming weight n/2, and the chosen weights sum to the target mod 2^n."""
    digits = [int(d) for d in witness]
    if len(digits) != instance.n or any(d not in (0, 1) for d in digits):
        return False
    if sum(digits) != instance.n // 2:
        return False
    total = sum(instance.weight(i) for i, d in enumerate(digits) if d) & ((1 << instance.n) - 1)
    return total == instance.target
