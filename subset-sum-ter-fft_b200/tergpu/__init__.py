"""tergpu: the B200 root backend of the exact depth-3 TER attempt (host side).

The computation lives in libtergpu.so (hand-written sm_100a CUDA behind the C
ABI in include/tergpu.h); this package marshals arrays, reads and writes the
reference's .snap format and builds seeded workloads.
"""
from . import _abi
from .root import (Config, RootKeys, RootResult, Telemetry, TergpuError, device_count, release,
                   run_gpu_root, run_gpu_root_records)

__all__ = [
    "Config", "RootKeys", "RootResult", "Telemetry", "TergpuError", "device_count", "release",
    "run_gpu_root", "run_gpu_root_records", "_abi",
]
