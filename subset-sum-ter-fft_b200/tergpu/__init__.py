"""tergpu: the B200 root backend of the exact depth-3 TER attempt (host side).

The computation lives in libtergpu.so (hand-written sm_100a CUDA behind the C
ABI in include/tergpu.h); this package marshals arrays, reads and writes the
reference's .snap format and builds seeded workloads.
"""
import os as _os

# Hardware work queues of the CUDA context this process creates: CUDA maps every
# stream onto CUDA_DEVICE_MAX_CONNECTIONS of them (8 by default), in order, so
# with more streams than queues a short kernel can wait behind a long one queued
# earlier on another stream (the batch engine runs two streams per slot, and an
# n=108 sweep is seconds).  32 is the most CUDA takes.  Read when the context is
# created: this import must come before the process's first CUDA call, and a
# value the caller set is kept.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import _abi  # noqa: E402
from .root import (Config, RootKeys, RootResult, Telemetry, TergpuError, device_count, release,
                   run_gpu_root, run_gpu_root_records)

__all__ = [
    "Config", "RootKeys", "RootResult", "Telemetry", "TergpuError", "device_count", "release",
    "run_gpu_root", "run_gpu_root_records", "_abi",
]
