"""ctypes mirror of include/tergpu.h and the loader of libtergpu.so.

The library is built in-tree (the package directory).  There is no fallback:
a missing library raises, so no computation can silently run elsewhere.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_DIR / "libtergpu.so"

COMPLETED = 0
FOUND = 1
NO_WITNESS_THIS_ATTEMPT = 2
ATTEMPT_LIMIT_REACHED = 3
INVALID_CONFIGURATION = 4
INVALID_SHAPE = 5
GENERATION_INCOMPLETE = 6
RESOURCE_LIMIT = 7
CANCELLED = 8
INVARIANT_VIOLATION = 9
NOT_APPLICABLE = 10
UNSUPPORTED_WIDTH = 11
OUTPUT_OVERFLOW = 64
DEVICE_ERROR = 65
INVALID_INPUT = 66

STATUS_NAMES = {
    0: "Completed", 1: "Found", 2: "NoWitnessThisAttempt", 3: "AttemptLimitReached",
    4: "InvalidConfiguration", 5: "InvalidShape", 6: "GenerationIncomplete", 7: "ResourceLimit",
    8: "Cancelled", 9: "InvariantViolation", 10: "NotApplicable", 11: "UnsupportedWidth",
    64: "OutputOverflow", 65: "DeviceError", 66: "InvalidInput",
}

ROOT_COUNT_ONLY = 1
ROOT_DEVICE_INPUTS = 2
ABI_VERSION = 5  # include/tergpu.h TERGPU_ABI_VERSION: the struct layouts below
ROOT_SWEEP_V1 = 4
ROOT_SWEEP_V2 = 8
ROOT_AUTOTUNE = 16
ROOT_SWEEP_V4 = 32
ROOT_PARTITION_ONE_PASS = 64
MAX_QUOTIENT_BITS = 72
# tergpu_attempt_in.root_policy: the numerics of ter::RootOutputPolicy
ROOT_POLICY_FIRST_WITNESS = 0
ROOT_POLICY_COUNT_ONLY = 1
ROOT_POLICY_FULL_CANONICAL = 2
ATTEMPT_CAPTURE_ONLY = 1
ATTEMPT_PREFLIGHT = 2
ATTEMPT_NO_GRAPH = 4
ATTEMPT_TELEMETRY = 8
ATTEMPT_BACKGROUND = 16
ATTEMPT_AUDIT = 32
ATTEMPT_GUIDED = 64
ATTEMPT_FIXTURE = 128

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class RootIn(ctypes.Structure):
    _fields_ = [
        ("quotient_bits", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("count", ctypes.c_uint64 * 3), ("key_lo", _u64p * 3), ("key_hi", _u8p * 3),
        ("id", _u32p * 3), ("cells", _u8p), ("projected_bits", ctypes.c_uint32),
        ("device", ctypes.c_int32), ("memory_limit_bytes", ctypes.c_uint64),
        ("family_bits", ctypes.c_uint32), ("filter_bits", ctypes.c_uint32),
        ("stream", ctypes.c_void_p), ("shard_index", ctypes.c_uint32),
        ("shard_count", ctypes.c_uint32),
    ]


class RootOut(ctypes.Structure):
    _fields_ = [
        ("triples", _u32p), ("capacity", ctypes.c_uint64), ("triples_count", ctypes.c_uint64),
        ("logical_pairs", ctypes.c_uint64), ("filter_survivors", ctypes.c_uint64),
        ("fast_hits", ctypes.c_uint64), ("projected_hits", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64), ("join_ms", ctypes.c_double),
        ("partition_ms", ctypes.c_double), ("sweep_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double), ("family_bits", ctypes.c_uint32),
        ("filter_bits", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
        ("sweep_variant", ctypes.c_uint32), ("tune_ms", ctypes.c_double),
    ]


class RootRecordsIn(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32), ("r1", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("record_bytes", ctypes.c_uint32), ("count", ctypes.c_uint64 * 3),
        ("records", _u8p * 3), ("child_target", _u32p * 3), ("root_target", _u32p),
        ("cells", _u8p), ("projected_bits", ctypes.c_uint32), ("device", ctypes.c_int32),
        ("memory_limit_bytes", ctypes.c_uint64), ("family_bits", ctypes.c_uint32),
        ("filter_bits", ctypes.c_uint32), ("shard_index", ctypes.c_uint32),
        ("shard_count", ctypes.c_uint32),
    ]


class RootRecordsOut(ctypes.Structure):
    _fields_ = [
        ("root", RootOut), ("triple_flags", _u8p), ("residue_exact", ctypes.c_uint64),
        ("structural", ctypes.c_uint64), ("valid_roots", ctypes.c_uint64),
        ("tau_lo", ctypes.c_uint64), ("tau_hi", ctypes.c_uint64),
    ]


EXPORTED = (
    "tergpu_root_run", "tergpu_root_run_records", "tergpu_device_count", "tergpu_abi_version",
    "tergpu_release", "tergpu_last_error", "tergpu_fnv1a", "tergpu_root_run_noalloc",
    "tergpu_noalloc_last_error",
)

_lib = None


def load(path: os.PathLike | str | None = None):
    """Load libtergpu.so (raises when it was not built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"libtergpu.so not built: {p} (run __graft_entry__.build())")
    lib = ctypes.CDLL(str(p))
    lib.tergpu_root_run.argtypes = [ctypes.POINTER(RootIn), ctypes.POINTER(RootOut)]
    lib.tergpu_root_run.restype = ctypes.c_int
    lib.tergpu_root_run_records.argtypes = [ctypes.POINTER(RootRecordsIn),
                                            ctypes.POINTER(RootRecordsOut)]
    lib.tergpu_root_run_records.restype = ctypes.c_int
    lib.tergpu_device_count.restype = ctypes.c_int
    lib.tergpu_abi_version.restype = ctypes.c_int
    lib.tergpu_last_error.restype = ctypes.c_char_p
    lib.tergpu_release.restype = None
    lib.tergpu_root_run_noalloc.argtypes = [ctypes.POINTER(RootIn), ctypes.POINTER(RootOut)]
    lib.tergpu_root_run_noalloc.restype = ctypes.c_int
    lib.tergpu_noalloc_last_error.restype = ctypes.c_char_p
    if lib.tergpu_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{p} implements ABI {lib.tergpu_abi_version()}, this package "
                           f"ABI {ABI_VERSION}: rebuild it (__graft_entry__.build())")
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    return load().tergpu_last_error().decode(errors="replace")
