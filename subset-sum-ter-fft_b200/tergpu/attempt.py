"""Full TER attempts on the device: the host mirror of solve_full_ter's attempt loop.

`solve_full_ter(instance, config)` mirrors the reference's entry point
(include/ter/full_ter.hpp:255-256, src/full_ter.cpp:2933-3521) for the
FiniteSanity shape: random targets (attempt a draws from SplitMix64(seed + a))
or the planted root's guided targets, complete (FullTer) or truncated
(FixtureTer) level 3.  The result carries the status, the reference's message
for it, the verified witness and per-attempt telemetry (level sizes, stage
counters, fingerprints).  `preflight(instance, config)` makes the same call's
checks and prediction without device work.  `instance` comes from
tergpu.instance.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .root import TergpuError


class AttemptStats(ctypes.Structure):
    _fields_ = [
        ("attempt", ctypes.c_uint32), ("status", ctypes.c_int32),
        ("level2_sizes", ctypes.c_uint64 * 9), ("level1_sizes", ctypes.c_uint64 * 3),
        ("level0_size", ctypes.c_uint64), ("l3_modular", ctypes.c_uint64),
        ("l2_modular", ctypes.c_uint64), ("root_modular", ctypes.c_uint64),
        ("valid_roots", ctypes.c_uint64), ("root_pairs", ctypes.c_uint64),
        ("l2_ms", ctypes.c_double), ("l1_ms", ctypes.c_double), ("root_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("attempt_seed", ctypes.c_uint64),
        ("l3_pairs", ctypes.c_uint64), ("l3_structural_rejects", ctypes.c_uint64),
        ("l3_distribution_rejects", ctypes.c_uint64), ("l3_survivors", ctypes.c_uint64),
        ("l2_pairs", ctypes.c_uint64), ("l2_structural_rejects", ctypes.c_uint64),
        ("l2_distribution_rejects", ctypes.c_uint64), ("l2_survivors", ctypes.c_uint64),
        ("root_structural_rejects", ctypes.c_uint64), ("root_distribution_rejects", ctypes.c_uint64),
        ("root_low_prefilter", ctypes.c_uint64), ("root_full_quotient_rejects", ctypes.c_uint64),
        ("root_quotient_bits", ctypes.c_uint32), ("root_prefilter_bits", ctypes.c_uint32),
        ("root_policy", ctypes.c_uint32), ("root_early_stopped", ctypes.c_uint32),
        ("l2_fingerprint", ctypes.c_uint64), ("l1_fingerprint", ctypes.c_uint64),
        ("l0_fingerprint", ctypes.c_uint64), ("verification_ms", ctypes.c_double),
        ("audited_stages", ctypes.c_uint32), ("reserved_audit", ctypes.c_uint32),
    ]


class AttemptIn(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("values_le", ctypes.POINTER(ctypes.c_uint64)), ("target_le", ctypes.POINTER(ctypes.c_uint64)),
        ("seed", ctypes.c_uint64), ("attempt_first", ctypes.c_uint32),
        ("attempt_count", ctypes.c_uint32), ("memory_limit_bytes", ctypes.c_uint64),
        ("cancel", ctypes.POINTER(ctypes.c_int32)), ("device", ctypes.c_int32),
        ("root_policy", ctypes.c_uint32), ("planted_root", ctypes.POINTER(ctypes.c_uint8)),
        ("fixture_level3_limit", ctypes.c_uint64),
    ]


class AttemptOut(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("r1", ctypes.c_uint32), ("r2", ctypes.c_uint32),
        ("level3_size", ctypes.c_uint64), ("attempts_run", ctypes.c_uint32),
        ("found_attempt", ctypes.c_uint32), ("witness", ctypes.c_uint8 * 128),
        ("stats", ctypes.POINTER(AttemptStats)), ("l1_records", ctypes.POINTER(ctypes.c_uint8) * 3),
        ("l1_capacity", ctypes.c_uint64 * 3), ("child_targets", (ctypes.c_uint32 * 4) * 3),
        ("root_target", ctypes.c_uint32 * 4), ("device_bytes", ctypes.c_uint64),
        ("total_ms", ctypes.c_double), ("device_bytes_held", ctypes.c_uint64),
        ("fingerprint", ctypes.c_uint64), ("level3_ms", ctypes.c_double),
    ]


@dataclass
class FullTerConfig:
    """The fields of the reference's FullTerConfig this path honours."""
    seed: int = 1
    attempt_limit: int = 1
    attempt_first: int = 0
    memory_limit_bytes: int = 0
    device: int = 0
    export_l1_capacity: int = 0   # > 0: return the last attempt's L1 lists as a Snapshot
    capture_only: bool = False    # stop after L1 (the device stream_full_ter_root_lists)
    no_graph: bool = False        # n = 36 / 72: run stage by stage instead of one graph per attempt
    # RootOutputPolicy (include/ter/full_ter.hpp:79-83); FirstWitness is the reference's default
    root_policy: int = _abi.ROOT_POLICY_FIRST_WITNESS
    telemetry: bool = False       # the reference's full telemetry: prefilter counts, fingerprints
    audit: bool = False           # FullTerConfig::audit: stages checked against the scalar oracles
    guided: bool = False          # TerTargetMode::GuidedPlanted: targets from the planted root
    fixture_limit: int = 0        # > 0: TerExecutionMode::FixtureTer with this level-3 limit


@dataclass
class FullTerResult:
    status: int
    r1: int = 0
    r2: int = 0
    level3_size: int = 0
    witness: np.ndarray | None = None
    found_attempt: int | None = None
    attempts: list = field(default_factory=list)
    snapshot: object | None = None
    total_ms: float = 0.0
    device_bytes: int = 0        # the preflight's predicted bytes
    device_bytes_held: int = 0   # bytes the workspace held at the end of the call
    message: str = ""            # FullTerResult::message: why the call ended short of Found
    fingerprint: int = 0         # FullTerTelemetry::fingerprint (telemetry runs)
    level3_ms: float = 0.0

    @property
    def status_name(self) -> str:
        return _abi.STATUS_NAMES.get(self.status, str(self.status))


_STAT_INTS = ("attempt_seed", "l3_pairs", "l3_structural_rejects", "l3_distribution_rejects",
              "l3_survivors", "l2_pairs", "l2_structural_rejects", "l2_distribution_rejects",
              "l2_survivors", "root_structural_rejects", "root_distribution_rejects",
              "root_low_prefilter", "root_full_quotient_rejects", "root_quotient_bits",
              "root_prefilter_bits", "root_policy", "root_early_stopped", "l2_fingerprint",
              "l1_fingerprint", "l0_fingerprint")


def _stats_dict(s: AttemptStats) -> dict:
    d = {
        "attempt": int(s.attempt), "status": int(s.status),
        "level2": [int(v) for v in s.level2_sizes], "level1": [int(v) for v in s.level1_sizes],
        "level0": int(s.level0_size), "l3_modular": int(s.l3_modular),
        "l2_modular": int(s.l2_modular), "root_modular": int(s.root_modular),
        "valid_roots": int(s.valid_roots), "root_pairs": int(s.root_pairs),
        "l2_ms": float(s.l2_ms), "l1_ms": float(s.l1_ms), "root_ms": float(s.root_ms),
        "total_ms": float(s.total_ms), "verification_ms": float(s.verification_ms),
        "audited_stages": int(s.audited_stages),
    }
    for name in _STAT_INTS:
        d[name] = int(getattr(s, name))
    return d


def _result(st: int, out: AttemptOut, stats, n: int) -> FullTerResult:
    res = FullTerResult(status=st, r1=int(out.r1), r2=int(out.r2), level3_size=int(out.level3_size),
                        total_ms=float(out.total_ms), device_bytes=int(out.device_bytes),
                        device_bytes_held=int(out.device_bytes_held),
                        fingerprint=int(out.fingerprint), level3_ms=float(out.level3_ms),
                        attempts=[_stats_dict(stats[i]) for i in range(int(out.attempts_run))])
    if st == _abi.FOUND:
        res.witness = np.array(out.witness[:n], dtype=np.uint8)
        res.found_attempt = int(out.found_attempt)
    return res


def make_request(instance, config: FullTerConfig, cancel=None):
    """The C structs of one request: (AttemptIn, AttemptOut, keep-alive buffers)."""
    values = np.ascontiguousarray(instance.values_le, dtype=np.uint64).reshape(-1)
    target = np.ascontiguousarray(instance.target_le, dtype=np.uint64)
    ain = AttemptIn()
    ain.n = instance.n
    ain.flags = ((_abi.ATTEMPT_CAPTURE_ONLY if config.capture_only else 0)
                 | (_abi.ATTEMPT_NO_GRAPH if config.no_graph else 0)
                 | (_abi.ATTEMPT_TELEMETRY if config.telemetry else 0)
                 | (_abi.ATTEMPT_AUDIT if config.audit else 0)
                 | (_abi.ATTEMPT_GUIDED if config.guided else 0)
                 | (_abi.ATTEMPT_FIXTURE if config.fixture_limit else 0))
    ain.fixture_level3_limit = config.fixture_limit
    planted = np.ascontiguousarray(instance.planted, dtype=np.uint8)
    if config.guided:
        ain.planted_root = planted.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    ain.values_le = values.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    ain.target_le = target.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    ain.seed = config.seed & (2**64 - 1)
    ain.attempt_first = config.attempt_first
    ain.attempt_count = config.attempt_limit
    ain.memory_limit_bytes = config.memory_limit_bytes
    ain.cancel = ctypes.pointer(cancel) if cancel is not None else None
    ain.device = config.device
    ain.root_policy = config.root_policy
    stats = (AttemptStats * max(1, config.attempt_limit))()
    out = AttemptOut()
    out.stats = ctypes.cast(stats, ctypes.POINTER(AttemptStats))
    return ain, out, (values, target, stats, planted)


def preflight(instance, config: FullTerConfig | None = None) -> FullTerResult:
    """The checks and prediction solve_full_ter makes before any device work, as
    ter_full_bench --preflight reports them (bench/ter_full_bench.cpp:594-680):
    r1, r2, the level-3 size per half and the predicted device bytes with status
    Completed, or the refusal the call would return (InvalidConfiguration,
    ResourceLimit against memory_limit_bytes).  Touches no device."""
    config = config or FullTerConfig()
    lib = _abi.load()
    lib.tergpu_attempt_run.argtypes = [ctypes.POINTER(AttemptIn), ctypes.POINTER(AttemptOut)]
    lib.tergpu_attempt_run.restype = ctypes.c_int
    ain, out, (_values, _target, stats, _planted) = make_request(instance, config)
    ain.flags |= _abi.ATTEMPT_PREFLIGHT
    st = lib.tergpu_attempt_run(ctypes.byref(ain), ctypes.byref(out))
    if st not in (_abi.COMPLETED, _abi.RESOURCE_LIMIT, _abi.INVALID_CONFIGURATION):
        raise TergpuError(st, _abi.last_error())
    res = _result(st, out, stats, instance.n)
    res.message = _abi.last_error() if st != _abi.COMPLETED else ""
    return res


def solve_full_ter(instance, config: FullTerConfig | None = None, cancel=None) -> FullTerResult:
    """Runs attempts [attempt_first, attempt_first + attempt_limit) on the device.

    `cancel` may be a ctypes.c_int32 whose value the caller sets from another
    thread; the loop stops with Cancelled at the next stage boundary."""
    config = config or FullTerConfig()
    lib = _abi.load()
    lib.tergpu_attempt_run.argtypes = [ctypes.POINTER(AttemptIn), ctypes.POINTER(AttemptOut)]
    lib.tergpu_attempt_run.restype = ctypes.c_int
    ain, out, (_values, _target, stats, _planted) = make_request(instance, config, cancel)
    w64, w32 = (instance.n + 63) // 64, (instance.n + 31) // 32
    rb = 16 * w64 + 4 * w32
    bufs = []
    if config.export_l1_capacity > 0:
        for l in range(3):
            b = np.zeros(config.export_l1_capacity * rb, dtype=np.uint8)
            bufs.append(b)
            out.l1_records[l] = b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
            out.l1_capacity[l] = config.export_l1_capacity
    st = lib.tergpu_attempt_run(ctypes.byref(ain), ctypes.byref(out))
    if st not in (_abi.FOUND, _abi.ATTEMPT_LIMIT_REACHED, _abi.CANCELLED, _abi.RESOURCE_LIMIT,
                  _abi.INVALID_CONFIGURATION):
        raise TergpuError(st, _abi.last_error())
    res = _result(st, out, stats, instance.n)
    res.message = _abi.last_error() if st != _abi.FOUND else ""
    if bufs and out.attempts_run > 0:
        from .snapshot import Snapshot

        sizes = [int(out.l1_capacity[l]) for l in range(3)]
        if all(sizes[l] <= config.export_l1_capacity for l in range(3)):
            last = res.attempts[-1]
            res.snapshot = Snapshot(
                n=instance.n, r1=res.r1, r2=res.r2, attempt=last["attempt"], seed=config.seed,
                attempt_seed=(config.seed + last["attempt"]) & (2**64 - 1),
                records=[bufs[l][: sizes[l] * rb].copy() for l in range(3)],
                child_targets=[np.array(out.child_targets[l][:w32], dtype=np.uint32) for l in range(3)],
                root_target=np.array(out.root_target[:w32], dtype=np.uint32),
                level2_sizes=last["level2"])
    return res
