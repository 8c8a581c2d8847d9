"""Host-side mirror of the reference's ter2_root backend interface for the GPU root.

`run_gpu_root(keys, config)` plays the role of run_hash_join / run_arwlf
(reference ter2_root/campaign/ter_hash_join_root.hpp:38-40,
ter2_root/frozen/ter_arwlf.hpp:145-147): it takes the three key lists of one
root and returns every full-Q triple with the backend telemetry.  The work
runs in libtergpu.so; this module only marshals arrays.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi


class TergpuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


@dataclass
class RootKeys:
    """Full quotient keys of one root: list 0 = q_A, 1 = q_B, 2 = d = tau - q_C (mod 2^Q).

    lo[l]: uint64 bits [0, min(Q, 64)); hi[l]: uint8 bits [64, Q) (zeros when Q <= 64);
    ids[l]: uint32 EntryIds or None (the index)."""
    quotient_bits: int
    lo: list
    hi: list
    ids: list | None = None

    def sizes(self):
        return [len(a) for a in self.lo]


@dataclass
class Config:
    """Mirror of the backends' Config: memory ceiling plus the device tuning."""
    memory_limit_bytes: int = 0
    device: int = 0
    projected_bits: int = 0
    family_bits: int = 0
    filter_bits: int = 0
    count_only: bool = False
    capacity: int = 1 << 16
    sweep_v1: bool = False  # sweep variant 1 (A in registers)
    sweep_v2: bool = False  # sweep variant 2 (B in registers, windows sorted); default: variant 3
    sweep_v4: bool = False  # sweep variant 4 (0/1 probe table, one bank per lane)
    autotune: bool = False  # pick fb / filter bits / variant per shape by timing a 1/64 sample
    one_pass_partition: bool = False  # long lists: one scattered pass instead of two staged ones
    shard_index: int = 0
    shard_count: int = 1  # power of two <= 64: join only D entries with key_d == index (mod count)


@dataclass
class Telemetry:
    logical_pairs: int = 0
    filter_survivors: int = 0
    fast_hits: int = 0
    full_hits: int = 0
    projected_hits: int = 0
    device_bytes: int = 0
    join_ms: float = 0.0
    partition_ms: float = 0.0
    sweep_ms: float = 0.0
    total_ms: float = 0.0
    kernel_launches: int = 0
    family_bits: int = 0
    filter_bits: int = 0
    sweep_variant: int = 0
    tune_ms: float = 0.0


@dataclass
class RootResult:
    status: int
    triples: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), dtype=np.uint32))
    telemetry: Telemetry = field(default_factory=Telemetry)
    residue_exact: int = 0
    structural: int = 0
    valid_roots: int = 0
    flags: np.ndarray | None = None
    tau: int = 0


def _p(a, t):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


def _telemetry(out: _abi.RootOut) -> Telemetry:
    return Telemetry(
        logical_pairs=int(out.logical_pairs), filter_survivors=int(out.filter_survivors),
        fast_hits=int(out.fast_hits), full_hits=int(out.triples_count),
        projected_hits=int(out.projected_hits), device_bytes=int(out.device_bytes),
        join_ms=float(out.join_ms), partition_ms=float(out.partition_ms),
        sweep_ms=float(out.sweep_ms), total_ms=float(out.total_ms),
        kernel_launches=int(out.kernel_launches),
        family_bits=int(out.family_bits), filter_bits=int(out.filter_bits),
        sweep_variant=int(out.sweep_variant), tune_ms=float(out.tune_ms))


def run_gpu_root(keys: RootKeys, config: Config | None = None,
                 cells: np.ndarray | None = None) -> RootResult:
    """Every full-Q triple (a, b, c) with key_a + key_b == key_c (mod 2^Q).

    Output-capacity overflow is retried once with the exact count, so the
    result is always complete; other failures raise TergpuError."""
    config = config or Config()
    lib = _abi.load()
    lo = [np.ascontiguousarray(a, dtype=np.uint64) for a in keys.lo]
    hi = [np.ascontiguousarray(a, dtype=np.uint8) for a in keys.hi] if keys.hi is not None else None
    ids = ([None if a is None else np.ascontiguousarray(a, dtype=np.uint32) for a in keys.ids]
           if keys.ids is not None else [None, None, None])
    cells_arr = None if cells is None else np.ascontiguousarray(cells, dtype=np.uint8)
    if cells_arr is not None and cells_arr.size != 4096:
        raise ValueError("cells must hold 4096 bytes")
    rin = _abi.RootIn()
    rin.quotient_bits = keys.quotient_bits
    rin.flags = (_abi.ROOT_COUNT_ONLY if config.count_only else 0) | \
        (_abi.ROOT_SWEEP_V1 if config.sweep_v1 else 0) | \
        (_abi.ROOT_SWEEP_V2 if config.sweep_v2 else 0) | \
        (_abi.ROOT_SWEEP_V4 if config.sweep_v4 else 0) | \
        (_abi.ROOT_AUTOTUNE if config.autotune else 0) | \
        (_abi.ROOT_PARTITION_ONE_PASS if config.one_pass_partition else 0)
    for l in range(3):
        rin.count[l] = len(lo[l])
        rin.key_lo[l] = _p(lo[l], ctypes.c_uint64)
        rin.key_hi[l] = _p(hi[l], ctypes.c_uint8) if hi is not None else None
        rin.id[l] = _p(ids[l], ctypes.c_uint32)
    rin.cells = _p(cells_arr, ctypes.c_uint8)
    rin.projected_bits = config.projected_bits
    rin.device = config.device
    rin.memory_limit_bytes = config.memory_limit_bytes
    rin.family_bits = config.family_bits
    rin.filter_bits = config.filter_bits
    rin.shard_index = config.shard_index
    rin.shard_count = config.shard_count
    capacity = max(1, config.capacity)
    for _ in range(2):
        buf = np.zeros(capacity * 3, dtype=np.uint32)
        out = _abi.RootOut()
        out.triples = _p(buf, ctypes.c_uint32)
        out.capacity = 0 if config.count_only else capacity
        st = lib.tergpu_root_run(ctypes.byref(rin), ctypes.byref(out))
        if st == _abi.OUTPUT_OVERFLOW:
            capacity = int(out.triples_count)
            continue
        if st != _abi.COMPLETED:
            raise TergpuError(st, _abi.last_error())
        n = 0 if config.count_only else int(out.triples_count)
        return RootResult(status=st, triples=buf[: 3 * n].reshape(-1, 3), telemetry=_telemetry(out))
    raise TergpuError(_abi.OUTPUT_OVERFLOW, "output grew between two identical runs")


def run_gpu_root_records(snap, config: Config | None = None,
                         cells: np.ndarray | None = None) -> RootResult:
    """One root straight from captured L1 records (a tergpu.snapshot.Snapshot),
    with the residue / structural / root-rule decision on the device."""
    config = config or Config()
    lib = _abi.load()
    rin = _abi.RootRecordsIn()
    rin.n = snap.n
    rin.r1 = snap.r1
    rin.flags = (_abi.ROOT_COUNT_ONLY if config.count_only else 0) | \
        (_abi.ROOT_SWEEP_V1 if config.sweep_v1 else 0) | \
        (_abi.ROOT_SWEEP_V2 if config.sweep_v2 else 0) | \
        (_abi.ROOT_SWEEP_V4 if config.sweep_v4 else 0) | \
        (_abi.ROOT_AUTOTUNE if config.autotune else 0) | \
        (_abi.ROOT_PARTITION_ONE_PASS if config.one_pass_partition else 0)
    rin.record_bytes = snap.record_bytes
    recs = [np.ascontiguousarray(r, dtype=np.uint8) for r in snap.records]
    targets = [np.ascontiguousarray(t, dtype=np.uint32) for t in snap.child_targets]
    root_t = np.ascontiguousarray(snap.root_target, dtype=np.uint32)
    for l in range(3):
        rin.count[l] = snap.entries[l]
        rin.records[l] = _p(recs[l], ctypes.c_uint8)
        rin.child_target[l] = _p(targets[l], ctypes.c_uint32)
    rin.root_target = _p(root_t, ctypes.c_uint32)
    cells_arr = None if cells is None else np.ascontiguousarray(cells, dtype=np.uint8)
    rin.cells = _p(cells_arr, ctypes.c_uint8)
    rin.projected_bits = config.projected_bits
    rin.device = config.device
    rin.memory_limit_bytes = config.memory_limit_bytes
    rin.family_bits = config.family_bits
    rin.filter_bits = config.filter_bits
    rin.shard_index = config.shard_index
    rin.shard_count = config.shard_count
    capacity = max(1, config.capacity)
    for _ in range(2):
        buf = np.zeros(capacity * 3, dtype=np.uint32)
        flags = np.zeros(capacity, dtype=np.uint8)
        out = _abi.RootRecordsOut()
        out.root.triples = _p(buf, ctypes.c_uint32)
        out.root.capacity = 0 if config.count_only else capacity
        out.triple_flags = _p(flags, ctypes.c_uint8)
        st = lib.tergpu_root_run_records(ctypes.byref(rin), ctypes.byref(out))
        if st == _abi.OUTPUT_OVERFLOW:
            capacity = int(out.root.triples_count)
            continue
        if st != _abi.COMPLETED:
            raise TergpuError(st, _abi.last_error())
        n = 0 if config.count_only else int(out.root.triples_count)
        return RootResult(status=st, triples=buf[: 3 * n].reshape(-1, 3),
                          telemetry=_telemetry(out.root), residue_exact=int(out.residue_exact),
                          structural=int(out.structural), valid_roots=int(out.valid_roots),
                          flags=flags[:n].copy(), tau=int(out.tau_lo) | (int(out.tau_hi) << 64))
    raise TergpuError(_abi.OUTPUT_OVERFLOW, "output grew between two identical runs")


def device_count() -> int:
    return int(_abi.load().tergpu_device_count())


def release() -> None:
    _abi.load().tergpu_release()
