"""Root report and count on a captured L1 root: the GPU counterparts of the
reference's report_full_ter_root / count_full_ter_root
(include/ter/full_ter.hpp:195-213, 258-265; src/full_ter.cpp:3722-3865).

The capture is a tergpu.snapshot.Snapshot (a .snap file of the reference, or
the device attempt pipeline's capture).  The device runs the whole root with
its authority chain (tergpu_root_run_records): every full-Q triple, then the
residue sum == T check and the root rule (parent digits binary with weight
n/2).  The policies then read as the reference defines them:

* CountOnly: valid_root_count = the pre-dedup multiplicity of accepted
  triples; no parent is retained.
* FullCanonicalOutput: the same count; the distinct parents are retained in
  canonical order (sorted by packed digit words, word 0 most significant).
* FirstWitness: the reference stops at its first accepted triple, so its count
  is min(1, accepted) and it retains at most one parent; the device reports
  the same numbers and retains the lowest parent in canonical order.

Statuses follow the reference: Completed with the counts, ResourceLimit when
the device refuses the declared ceiling, InvalidConfiguration for a capture
that is not a FiniteSanity root the device runs or that breaks the capture
invariants the reference checks (targets and residues below 2^n, residues
congruent to their child target modulo 2^r1), before any device work.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .root import Config, Telemetry, TergpuError, run_gpu_root_records


class RootOutputPolicy(enum.IntEnum):
    """include/ter/full_ter.hpp:79-83 (same numeric values)."""
    FIRST_WITNESS = 0
    COUNT_ONLY = 1
    FULL_CANONICAL_OUTPUT = 2


@dataclass
class FullTerRootReportResult:
    status: int = _abi.INVALID_CONFIGURATION
    effective_root_output_policy: RootOutputPolicy = RootOutputPolicy.COUNT_ONLY
    valid_root_count: int = 0
    retained_root_count: int = 0
    parents: list = field(default_factory=list)   # uint8[n] digit vectors (0/1), canonical order
    telemetry: Telemetry = field(default_factory=Telemetry)
    message: str = ""


@dataclass
class FullTerRootCountResult:
    status: int = _abi.INVALID_CONFIGURATION
    valid_root_count: int = 0
    telemetry: Telemetry = field(default_factory=Telemetry)
    message: str = ""


def _parents(snap, triples: np.ndarray) -> list[tuple[int, ...]]:
    """Parent pos-mask words (disjoint children: the OR of the three masks)."""
    masks = [snap.masks(l)[0] for l in range(3)]
    out = []
    for a, b, c in triples.tolist():
        out.append(tuple(int(masks[0][a, k]) | int(masks[1][b, k]) | int(masks[2][c, k])
                         for k in range(snap.words64)))
    return out


def _digits(words: tuple[int, ...], n: int) -> np.ndarray:
    return np.array([(words[i // 64] >> (i % 64)) & 1 for i in range(n)], dtype=np.uint8)


def _capture_refusal(snap) -> str | None:
    """The capture checks report_full_ter_root makes before its root
    (src/full_ter.cpp:3772-3803), with the reference's messages: every target
    below 2^n, and every residue below 2^n and congruent to its list's child
    target modulo 2^r1.  None when the capture passes."""
    from .snapshot import words_to_int

    n, r1 = snap.n, snap.r1
    targets = [words_to_int(t) for t in snap.child_targets]
    if any(t >> n for t in targets):
        return "root count child target exceeds the captured modulus"
    if words_to_int(snap.root_target) >> n:
        return "root count target exceeds the captured modulus"
    top_bits = n - 32 * (snap.words32 - 1)  # bits of the top residue word below 2^n
    low_mask = np.uint64((1 << r1) - 1)
    for l in range(3):
        res = snap.residues(l)
        if len(res) == 0:
            continue
        low = res[:, 0].astype(np.uint64) | (res[:, 1].astype(np.uint64) << np.uint64(32))
        above = top_bits < 32 and bool((res[:, -1] >> np.uint32(top_bits)).any())
        if above or bool(((low & low_mask) != (np.uint64(targets[l] & (2**64 - 1)) & low_mask)).any()):
            return "root report capture violates the child target invariant"
    return None


def report_full_ter_root(snap, policy: RootOutputPolicy = RootOutputPolicy.FIRST_WITNESS,
                         config: Config | None = None, cancel=None) -> FullTerRootReportResult:
    """report_full_ter_root on a captured root (see the module docstring).
    `cancel` (a ctypes.c_int32 or None) is the reference's config.cancellation:
    set before the call, the report returns Cancelled without device work.  An
    unknown policy or a capture that is not a FiniteSanity root is refused
    with the reference's message (src/full_ter.cpp:3727-3743)."""
    config = config or Config()
    try:
        policy = RootOutputPolicy(policy)
    except ValueError:
        policy = None
    if policy is None or snap.n == 0 or snap.n % 36 != 0 or snap.r1 >= snap.n:
        return FullTerRootReportResult(
            message="root report requires a completed native root capture and valid tiled limits")
    if cancel is not None and cancel.value != 0:
        return FullTerRootReportResult(status=_abi.CANCELLED, message="root report was cancelled")
    refusal = _capture_refusal(snap)
    if refusal is not None:
        return FullTerRootReportResult(status=_abi.INVALID_CONFIGURATION, message=refusal)
    try:
        res = run_gpu_root_records(snap, Config(memory_limit_bytes=config.memory_limit_bytes,
                                                device=config.device,
                                                family_bits=config.family_bits,
                                                filter_bits=config.filter_bits,
                                                capacity=config.capacity))
    except TergpuError as e:
        if e.status in (_abi.RESOURCE_LIMIT, _abi.INVALID_CONFIGURATION, _abi.UNSUPPORTED_WIDTH):
            return FullTerRootReportResult(status=e.status, message=str(e))
        raise
    accepted = res.triples[(res.flags & 5) == 5] if len(res.triples) else res.triples
    total = int(len(accepted))
    if total != res.valid_roots:
        return FullTerRootReportResult(status=_abi.INVARIANT_VIOLATION,
                                       message="accepted triples disagree with the device count")
    out = FullTerRootReportResult(status=_abi.COMPLETED, effective_root_output_policy=policy,
                                  telemetry=res.telemetry)
    distinct = sorted(set(_parents(snap, accepted)), key=lambda w: w)
    if policy == RootOutputPolicy.COUNT_ONLY:
        out.valid_root_count = total
    elif policy == RootOutputPolicy.FULL_CANONICAL_OUTPUT:
        out.valid_root_count = total
        out.parents = [_digits(w, snap.n) for w in distinct]
    else:
        out.valid_root_count = min(total, 1)
        out.parents = [_digits(w, snap.n) for w in distinct[:1]]
    out.retained_root_count = len(out.parents)
    return out


def count_full_ter_root(snap, config: Config | None = None, cancel=None) -> FullTerRootCountResult:
    """count_full_ter_root: the CountOnly projection of the report."""
    r = report_full_ter_root(snap, RootOutputPolicy.COUNT_ONLY, config, cancel)
    return FullTerRootCountResult(status=r.status, valid_root_count=r.valid_root_count,
                                  telemetry=r.telemetry, message=r.message)
