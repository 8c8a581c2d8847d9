"""Byte-compatible reader/writer of the reference's packed root snapshot (.snap).

Layout (reference ter2_root/frozen/ter_root_snapshot.hpp:1-57): a 424-byte
header, then the three L1 lists as fixed-width records
    uint64 pos[W64] | uint64 neg[W64] | uint32 residue[W32]
with EntryId = record index.  The header carries its own FNV-1a-64 checksum
(computed with the checksum field zeroed) and one FNV-1a-64 per list
(ter_root_snapshot.cpp:22-25, 94-101, 226-246).  A writer produces
<path>.partial and renames it once the header is final.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _abi

MAGIC = b"TERRSNP1"
LAYOUT_VERSION = 1
MAX_WORDS32 = 8

HEADER_DTYPE = np.dtype([
    ("magic", "S8"), ("layout_version", "<u4"), ("header_bytes", "<u4"), ("n", "<u4"),
    ("r1", "<u4"), ("r2", "<u4"), ("words64", "<u4"), ("words32", "<u4"),
    ("record_bytes", "<u4"), ("attempt", "<u4"), ("reserved", "<u4"), ("seed", "<u8"),
    ("attempt_seed", "<u8"), ("entries", "<u8", 3), ("offset", "<u8", 3),
    ("checksum", "<u8", 3), ("child_target", "<u4", (3, MAX_WORDS32)),
    ("root_target", "<u4", MAX_WORDS32), ("level2_sizes", "<u8", 9),
    ("memory_limit_bytes", "<u8"), ("declared_peak_bytes", "<u8"),
    ("process_peak_working_set", "<u8"), ("capture_elapsed_ns", "<u8"),
    ("git_commit", "S48"), ("header_checksum", "<u8"),
])
assert HEADER_DTYPE.itemsize == 424

FNV_OFFSET = 0xcbf29ce484222325


class SnapshotError(ValueError):
    pass


def fnv1a(data, state: int = FNV_OFFSET) -> int:
    """FNV-1a-64 over a byte buffer (computed in libtergpu.so's host code)."""
    buf = np.frombuffer(memoryview(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    lib = _abi.load()
    lib.tergpu_fnv1a.restype = ctypes.c_uint64
    lib.tergpu_fnv1a.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
    return int(lib.tergpu_fnv1a(buf.ctypes.data, buf.size, state))


@dataclass
class Snapshot:
    n: int
    r1: int
    r2: int
    attempt: int
    seed: int
    attempt_seed: int
    records: list                 # three uint8 arrays, entries * record_bytes
    child_targets: list           # three uint32 arrays of words32
    root_target: np.ndarray       # uint32[words32]
    level2_sizes: list = field(default_factory=lambda: [0] * 9)
    header: np.ndarray | None = None

    @property
    def words64(self) -> int:
        return (self.n + 63) // 64

    @property
    def words32(self) -> int:
        return (self.n + 31) // 32

    @property
    def record_bytes(self) -> int:
        return 16 * self.words64 + 4 * self.words32

    @property
    def entries(self):
        return [len(r) // self.record_bytes for r in self.records]

    def residues(self, l: int) -> np.ndarray:
        """uint32[entries, words32] residue words of list l."""
        rb = self.record_bytes
        rec = self.records[l].reshape(-1, rb)
        return rec[:, 16 * self.words64:].copy().view("<u4").reshape(-1, self.words32)

    def masks(self, l: int):
        """(pos, neg) uint64[entries, words64]."""
        rb = self.record_bytes
        rec = self.records[l].reshape(-1, rb)
        w = rec[:, : 16 * self.words64].copy().view("<u8").reshape(-1, 2 * self.words64)
        return w[:, : self.words64], w[:, self.words64:]


def load(path: os.PathLike | str, verify_checksums: bool = True) -> Snapshot:
    """Loads and validates a snapshot exactly as root_snapshot::load does
    (ter2_root/frozen/ter_root_snapshot.cpp:213-272)."""
    raw = Path(path).read_bytes()
    if len(raw) < HEADER_DTYPE.itemsize:
        raise SnapshotError("truncated snapshot header")
    h = np.frombuffer(raw[: HEADER_DTYPE.itemsize], dtype=HEADER_DTYPE)[0]
    if bytes(h["magic"]) != MAGIC or int(h["layout_version"]) != LAYOUT_VERSION or \
            int(h["header_bytes"]) != HEADER_DTYPE.itemsize:
        raise SnapshotError("not a layout-1 root snapshot")
    if verify_checksums:
        zeroed = np.frombuffer(raw[: HEADER_DTYPE.itemsize], dtype=HEADER_DTYPE).copy()
        zeroed["header_checksum"] = 0
        if fnv1a(zeroed.tobytes()) != int(h["header_checksum"]):
            raise SnapshotError("snapshot header checksum mismatch")
    n = int(h["n"])
    w64, w32 = (n + 63) // 64, (n + 31) // 32
    rb = 16 * w64 + 4 * w32
    if n == 0 or int(h["words64"]) != w64 or int(h["words32"]) != w32 or w32 > MAX_WORDS32 or \
            int(h["record_bytes"]) != rb:
        raise SnapshotError("snapshot dimensions are inconsistent")
    offset = HEADER_DTYPE.itemsize
    records = []
    for l in range(3):
        if int(h["offset"][l]) != offset:
            raise SnapshotError("snapshot list offsets are inconsistent")
        size = int(h["entries"][l]) * rb
        if offset + size > len(raw):
            raise SnapshotError(f"truncated snapshot list {l}")
        rec = np.frombuffer(raw, dtype=np.uint8, count=size, offset=offset).copy()
        if verify_checksums and fnv1a(rec) != int(h["checksum"][l]):
            raise SnapshotError(f"snapshot list {l} checksum mismatch")
        records.append(rec)
        offset += size
    if offset != len(raw):
        raise SnapshotError("trailing bytes after the last snapshot list")
    snap = Snapshot(n=n, r1=int(h["r1"]), r2=int(h["r2"]), attempt=int(h["attempt"]),
                    seed=int(h["seed"]), attempt_seed=int(h["attempt_seed"]), records=records,
                    child_targets=[np.array(h["child_target"][l][:w32], dtype=np.uint32)
                                   for l in range(3)],
                    root_target=np.array(h["root_target"][:w32], dtype=np.uint32),
                    level2_sizes=[int(v) for v in h["level2_sizes"]], header=h)
    # structural validation: disjoint masks, nothing above n bits
    top64 = n % 64
    top32 = n % 32
    for l in range(3):
        pos, neg = snap.masks(l)
        if np.any(pos & neg):
            raise SnapshotError("snapshot entry has overlapping or out-of-width ternary masks")
        if top64:
            allowed = np.uint64((1 << top64) - 1)
            if np.any((pos[:, -1] | neg[:, -1]) & ~allowed):
                raise SnapshotError("snapshot entry has overlapping or out-of-width ternary masks")
        if top32:
            res = snap.residues(l)
            if np.any(res[:, -1] & ~np.uint32((1 << top32) - 1)):
                raise SnapshotError("snapshot entry residue exceeds n bits")
    return snap


def save(snap: Snapshot, path: os.PathLike | str, git_commit: str = "tergpu") -> int:
    """Writes <path>.partial, then renames it to <path>.  Returns the file size."""
    h = np.zeros(1, dtype=HEADER_DTYPE)
    h["magic"] = MAGIC
    h["layout_version"] = LAYOUT_VERSION
    h["header_bytes"] = HEADER_DTYPE.itemsize
    h["n"] = snap.n
    h["r1"] = snap.r1
    h["r2"] = snap.r2
    h["words64"] = snap.words64
    h["words32"] = snap.words32
    h["record_bytes"] = snap.record_bytes
    h["attempt"] = snap.attempt
    h["seed"] = snap.seed
    h["attempt_seed"] = snap.attempt_seed
    offset = HEADER_DTYPE.itemsize
    for l in range(3):
        rec = np.ascontiguousarray(snap.records[l], dtype=np.uint8)
        h["entries"][0, l] = rec.size // snap.record_bytes
        h["offset"][0, l] = offset
        h["checksum"][0, l] = fnv1a(rec)
        ct = np.zeros(MAX_WORDS32, dtype=np.uint32)
        ct[: snap.words32] = snap.child_targets[l][: snap.words32]
        h["child_target"][0, l] = ct
        offset += rec.size
    rt = np.zeros(MAX_WORDS32, dtype=np.uint32)
    rt[: snap.words32] = snap.root_target[: snap.words32]
    h["root_target"] = rt
    h["level2_sizes"] = np.array(snap.level2_sizes[:9] + [0] * (9 - len(snap.level2_sizes[:9])),
                                 dtype=np.uint64)
    h["git_commit"] = git_commit.encode()[:47]
    h["header_checksum"] = 0
    h["header_checksum"] = fnv1a(h.tobytes())
    partial = Path(str(path) + ".partial")
    with open(partial, "wb") as f:
        f.write(h.tobytes())
        for l in range(3):
            f.write(np.ascontiguousarray(snap.records[l], dtype=np.uint8).tobytes())
    os.replace(partial, path)
    return offset


def words_to_int(words) -> int:
    """Little-endian 32-bit words (a residue or a target) as one integer."""
    v = 0
    for k, w in enumerate(words):
        v |= int(w) << (32 * k)
    return v


def root_keys(snap: Snapshot):
    """Host derivation of the full quotient keys (the device does the same in
    tergpu_root_run_records): q_L = ((R - c_L) mod 2^n) >> r1 over Q = n - r1
    bits, list 2 turned into d = tau - q_C with tau = ((T - c0 - c1 - c2) mod
    2^n) >> r1 (reference ter_root_generalization_workload.cpp:668-702).
    Returns (Q, lo[3], hi[3], tau)."""
    n, r1 = snap.n, snap.r1
    Q = n - r1
    nmask = (1 << n) - 1
    qmask = (1 << Q) - 1
    T = words_to_int(snap.root_target) & nmask
    c = [words_to_int(t) & nmask for t in snap.child_targets]
    tau = (((T - c[0] - c[1] - c[2]) & nmask) >> r1) & qmask
    lo_out, hi_out = [], []
    for l in range(3):
        res = snap.residues(l).astype(np.uint64)
        w32 = snap.words32
        r_lo = res[:, 0] | (res[:, 1] << np.uint64(32)) if w32 > 1 else res[:, 0].copy()
        r_hi = np.zeros_like(r_lo)
        if w32 > 2:
            r_hi = res[:, 2] | ((res[:, 3] << np.uint64(32)) if w32 > 3 else np.uint64(0))
        c_lo, c_hi = np.uint64(c[l] & (2**64 - 1)), np.uint64(c[l] >> 64)
        d_lo = r_lo - c_lo
        borrow = (r_lo < c_lo).astype(np.uint64)
        d_hi = r_hi - c_hi - borrow
        if n < 128:
            d_hi &= np.uint64((1 << (n - 64)) - 1) if n > 64 else np.uint64(0)
            if n <= 64:
                d_lo &= np.uint64(nmask)
        # shift right by r1 across 128 bits
        if r1 < 64:
            q_lo = (d_lo >> np.uint64(r1)) | ((d_hi << np.uint64(64 - r1)) if r1 > 0 else np.uint64(0))
            q_hi = d_hi >> np.uint64(r1)
        else:
            q_lo = d_hi >> np.uint64(r1 - 64)
            q_hi = np.zeros_like(d_hi)
        if Q < 64:
            q_lo &= np.uint64(qmask)
            q_hi[:] = 0
        else:
            q_hi &= np.uint64((1 << (Q - 64)) - 1)
        if l == 2:
            t_lo, t_hi = np.uint64(tau & (2**64 - 1)), np.uint64(tau >> 64)
            n_lo = t_lo - q_lo
            b = (t_lo < q_lo).astype(np.uint64)
            n_hi = t_hi - q_hi - b
            if Q < 64:
                n_lo &= np.uint64(qmask)
                n_hi[:] = 0
            else:
                n_hi &= np.uint64((1 << (Q - 64)) - 1)
            q_lo, q_hi = n_lo, n_hi
        lo_out.append(q_lo.astype(np.uint64))
        hi_out.append(q_hi.astype(np.uint8))
    return Q, lo_out, hi_out, tau
