"""ORACLE -- test infrastructure, never part of the product.

ctypes view of the C restatement in oracle/terorc.c (liboracle.so) and of the
reference harness (oracle/_ref/terref).  Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline / reference legs import this module, and only to
check or to time the reference's own CPU path.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "terref"

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class Digest(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "triples", "triple_sum", "triple_xor", "triple_sum2",
        "full_q", "residue", "residue_sum", "structural")]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class Attempt(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("r1", ctypes.c_uint32), ("r2", ctypes.c_uint32),
        ("level2_sizes", ctypes.c_uint64 * 9), ("level1_sizes", ctypes.c_uint64 * 3),
        ("level0_size", ctypes.c_uint64), ("l3_modular", ctypes.c_uint64),
        ("l2_modular", ctypes.c_uint64), ("root_prefilter_candidates", ctypes.c_uint64),
        ("root_full_quotient_rejects", ctypes.c_uint64),
        ("root_modular_candidates", ctypes.c_uint64), ("valid_root_count", ctypes.c_uint64),
        ("witness_pos", ctypes.c_uint64 * 2), ("witness_neg", ctypes.c_uint64 * 2),
        ("witness_verified", ctypes.c_int32),
    ]


class L1Export(ctypes.Structure):
    _fields_ = [
        ("res_lo", _u64p * 3), ("res_hi", _u64p * 3), ("pos0", _u64p * 3), ("pos1", _u64p * 3),
        ("neg0", _u64p * 3), ("neg1", _u64p * 3), ("cap", ctypes.c_uint64),
        ("t1_lo", ctypes.c_uint64 * 3), ("t1_hi", ctypes.c_uint64 * 3),
        ("root_lo", ctypes.c_uint64), ("root_hi", ctypes.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run __graft_entry__.build())")
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_mix64.restype = ctypes.c_uint64
        L.orc_mix64.argtypes = [ctypes.c_uint64]
        L.orc_add_packed_word.restype = ctypes.c_int
        L.orc_add_packed_word.argtypes = [ctypes.c_uint64] * 6 + [ctypes.POINTER(ctypes.c_uint64)] * 2
        L.orc_build_instance.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                         ctypes.c_int, _u64p, _u64p, _u8p]
        L.orc_params.argtypes = [ctypes.c_uint32, _u32p, _u32p]
        L.orc_attempt.argtypes = [ctypes.c_uint32, _u64p, _u64p, ctypes.c_uint64,
                                  ctypes.POINTER(Attempt), ctypes.POINTER(L1Export)]
        L.orc_root_join.restype = ctypes.c_uint64
        L.orc_root_join.argtypes = [ctypes.c_uint32,
                                    ctypes.c_uint64, _u64p, _u64p,
                                    ctypes.c_uint64, _u64p, _u64p,
                                    ctypes.c_uint64, _u64p, _u64p,
                                    _u8p, ctypes.POINTER(Digest), _u32p, ctypes.c_uint64]
        L.orc_projected_count.restype = ctypes.c_uint64
        L.orc_projected_count.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u64p,
                                          ctypes.c_uint64, _u64p, ctypes.c_uint64, _u64p, _u8p]
        L.orc_synthetic_root.restype = ctypes.c_uint64
        L.orc_synthetic_root.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                         ctypes.c_uint32, ctypes.c_uint64,
                                         ctypes.POINTER(_u64p), ctypes.POINTER(_u64p)]
        L.orc_digest_add.argtypes = [ctypes.POINTER(Digest), ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint32]
        _lib = L
    return _lib


def _p64(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def _p8(a):
    return None if a is None else a.ctypes.data_as(_u8p)


def add_packed_word(ap: int, an: int, bp: int, bn: int, cp: int, cn: int):
    """(valid, positive mask, negative mask) of one word of a + b + c."""
    pos, neg = ctypes.c_uint64(), ctypes.c_uint64()
    ok = lib().orc_add_packed_word(ap, an, bp, bn, cp, cn, ctypes.byref(pos), ctypes.byref(neg))
    return bool(ok), int(pos.value), int(neg.value)


def mix64(v: int) -> int:
    return int(lib().orc_mix64(v))


def build_instance(n: int, seed: int, kind: str = "auth", b1: int = 10):
    """(values_le uint64[n, W64], target_le uint64[W64], planted uint8[n])."""
    w = (n + 63) // 64
    values = np.zeros(n * w, dtype=np.uint64)
    target = np.zeros(w, dtype=np.uint64)
    planted = np.zeros(n, dtype=np.uint8)
    rc = lib().orc_build_instance(n, b1, seed, 1 if kind == "auth" else 0,
                                  _p64(values), _p64(target), planted.ctypes.data_as(_u8p))
    if rc != 0:
        raise ValueError(f"instance rejected: n={n}")
    return values.reshape(n, w), target, planted


def params(n: int):
    r1 = ctypes.c_uint32()
    r2 = ctypes.c_uint32()
    if lib().orc_params(n, ctypes.byref(r1), ctypes.byref(r2)) != 0:
        return None
    return int(r1.value), int(r2.value)


def attempt(n: int, seed: int, attempt_index: int, kind: str = "auth", export_l1: bool = False,
            l1_cap: int = 1 << 20):
    values, target, _ = build_instance(n, seed, kind)
    out = Attempt()
    x = None
    arrays = None
    if export_l1:
        x = L1Export()
        x.cap = l1_cap
        arrays = {k: [np.zeros(l1_cap, dtype=np.uint64) for _ in range(3)]
                  for k in ("res_lo", "res_hi", "pos0", "pos1", "neg0", "neg1")}
        for k, lists in arrays.items():
            for g in range(3):
                getattr(x, k)[g] = _p64(lists[g])
    rc = lib().orc_attempt(n, _p64(values.reshape(-1)), _p64(target),
                           seed + attempt_index, ctypes.byref(out),
                           ctypes.byref(x) if x is not None else None)
    if rc != 0:
        raise RuntimeError(f"oracle attempt failed rc={rc}")
    result = {
        "status": int(out.status), "r1": int(out.r1), "r2": int(out.r2),
        "level2": [int(v) for v in out.level2_sizes], "level1": [int(v) for v in out.level1_sizes],
        "level0": int(out.level0_size), "l3_modular": int(out.l3_modular),
        "l2_modular": int(out.l2_modular), "root_prefilter": int(out.root_prefilter_candidates),
        "root_quotient_rejects": int(out.root_full_quotient_rejects),
        "root_modular": int(out.root_modular_candidates), "valid_roots": int(out.valid_root_count),
        "witness_pos": [int(v) for v in out.witness_pos],
        "witness_verified": int(out.witness_verified),
    }
    if export_l1:
        sizes = result["level1"]
        result["l1"] = {k: [lists[g][: sizes[g]].copy() for g in range(3)]
                        for k, lists in arrays.items()}
        result["t1"] = [int(x.t1_lo[g]) | (int(x.t1_hi[g]) << 64) for g in range(3)]
        result["root_target"] = int(x.root_lo) | (int(x.root_hi) << 64)
    return result


def synthetic_root(bits: int, seed: int, size: int, pool: int = 0):
    """Lists (lo[3], hi[3]) of the reference's synthetic root; list 2 holds d."""
    cap = size + 128
    lo = [np.zeros(cap, dtype=np.uint64) for _ in range(3)]
    hi = [np.zeros(cap, dtype=np.uint64) for _ in range(3)]
    lo_p = (_u64p * 3)(*[_p64(a) for a in lo])
    hi_p = (_u64p * 3)(*[_p64(a) for a in hi])
    count = lib().orc_synthetic_root(bits, seed, size, pool, cap, lo_p, hi_p)
    if count == 0:
        raise RuntimeError("synthetic root generation failed")
    return [a[:count].copy() for a in lo], [a[:count].copy() for a in hi]


def root_join(bits: int, lo, hi, cells: np.ndarray | None = None, capacity: int = 0):
    """Every full-Q triple of key lists (list 2 = d): (digest dict, triples array)."""
    d = Digest()
    his = [np.ascontiguousarray(h, dtype=np.uint64) for h in hi]
    los = [np.ascontiguousarray(v, dtype=np.uint64) for v in lo]
    trip = np.zeros(max(capacity, 1) * 3, dtype=np.uint32)
    count = lib().orc_root_join(bits, len(los[0]), _p64(los[0]), _p64(his[0]),
                                len(los[1]), _p64(los[1]), _p64(his[1]),
                                len(los[2]), _p64(los[2]), _p64(his[2]),
                                _p8(cells), ctypes.byref(d), _p32(trip), capacity)
    n_out = min(int(count), capacity)
    return d.as_dict(), trip[: 3 * n_out].reshape(-1, 3)


def projected_count(k: int, lo, cells: np.ndarray | None = None) -> int:
    los = [np.ascontiguousarray(v, dtype=np.uint64) for v in lo]
    return int(lib().orc_projected_count(k, len(los[0]), _p64(los[0]), len(los[1]), _p64(los[1]),
                                         len(los[2]), _p64(los[2]), _p8(cells)))


def digest_of(triples) -> dict:
    d = Digest()
    for a, b, c in triples:
        lib().orc_digest_add(ctypes.byref(d), int(a), int(b), int(c))
    return d.as_dict()


def select_cells(count: int) -> np.ndarray:
    """The reference's declared microproblem subsample (select_microproblems,
    ter2_root/frozen/ter_root_queue_kernels.cpp:112-133): Fisher-Yates over the
    4096 cells with mix64(0x5EED5EED + i)."""
    sel = np.zeros(4096, dtype=np.uint8)
    if count >= 4096:
        sel[:] = 1
        return sel
    order = list(range(4096))
    state = 0x5EED5EED
    for at in range(4095, 0, -1):
        pick = mix64(state) % (at + 1)
        state += 1
        order[at], order[pick] = order[pick], order[at]
    for at in range(count):
        sel[order[at]] = 1
    return sel


# --------------------------------------------------------------------------
# The reference harness (compiled reference code), when it was built here.
# --------------------------------------------------------------------------

def ref_available() -> bool:
    return REF_BIN.exists()


def ref_run(*args, timeout: float = 600.0, env: dict | None = None) -> list[dict]:
    e = dict(os.environ)
    pkg_lib = HERE.parent / "subset-sum-ter-fft_b200" / "libtergpu.so"
    e.setdefault("TERGPU_LIBRARY", str(pkg_lib))
    if env:
        e.update(env)
    proc = subprocess.run([str(REF_BIN), *[str(a) for a in args]], capture_output=True,
                          text=True, timeout=timeout, env=e)
    if proc.returncode != 0:
        raise RuntimeError(f"terref {args} failed rc={proc.returncode}: {proc.stderr}{proc.stdout}")
    return [json.loads(line) for line in proc.stdout.splitlines() if line.startswith("{")]
