"""Batched and served attempts: many independent requests on one device at once.

`solve_batch(requests, slots, memory_budget_bytes)` hands the whole set to
tergpu_attempt_batch (include/tergpu.h), the library's continuous-batching
engine: `slots` attempt pipelines run concurrently (a host thread, a CUDA
stream and a device workspace each); requests are admitted in arrival order
while a slot is free and the predicted device bytes of the running requests
stay within the budget; requests the preflight refuses (36 does not divide n,
or more bytes than the budget) complete at once.  With arrival times set the
same call is a served stream: a request becomes eligible at its arrival and
its latency runs from arrival to completion.

Each request's result is exactly tergpu_attempt_run's for that request alone
(the same device code on a private workspace); only the timing differs.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .attempt import AttemptIn, AttemptOut, FullTerConfig, FullTerResult, _result, make_request
from .root import TergpuError


class BatchIn(ctypes.Structure):
    _fields_ = [
        ("jobs", ctypes.POINTER(AttemptIn)), ("outs", ctypes.POINTER(AttemptOut)),
        ("count", ctypes.c_uint64), ("arrival_ms", ctypes.POINTER(ctypes.c_double)),
        ("slots", ctypes.c_uint32), ("device", ctypes.c_int32),
        ("memory_budget_bytes", ctypes.c_uint64),
        ("admit_ms", ctypes.POINTER(ctypes.c_double)), ("finish_ms", ctypes.POINTER(ctypes.c_double)),
    ]


class BatchOut(ctypes.Structure):
    _fields_ = [
        ("total_ms", ctypes.c_double), ("peak_predicted_bytes", ctypes.c_uint64),
        ("peak_running", ctypes.c_uint32), ("refused", ctypes.c_uint64),
    ]


@dataclass
class Request:
    instance: object              # tergpu.instance.Instance
    config: FullTerConfig
    arrival_ms: float = 0.0


@dataclass
class BatchResult:
    results: list                 # FullTerResult per request, in request order
    admit_ms: np.ndarray
    finish_ms: np.ndarray
    arrival_ms: np.ndarray
    total_ms: float = 0.0
    peak_running: int = 0
    peak_predicted_bytes: int = 0
    refused: int = 0
    latency_ms: np.ndarray = field(default_factory=lambda: np.zeros(0))  # finish - arrival


def solve_batch(requests: list[Request], slots: int = 8, memory_budget_bytes: int = 0,
                device: int = 0, served: bool = False) -> BatchResult:
    """Runs every request through the library's batch engine (see the module
    docstring).  served=True passes the arrival times (a served stream);
    otherwise every request is eligible at once."""
    lib = _abi.load()
    lib.tergpu_attempt_batch.argtypes = [ctypes.POINTER(BatchIn), ctypes.POINTER(BatchOut)]
    lib.tergpu_attempt_batch.restype = ctypes.c_int
    count = len(requests)
    jobs = (AttemptIn * max(1, count))()
    outs = (AttemptOut * max(1, count))()
    keep = []
    for i, r in enumerate(requests):
        ain, aout, bufs = make_request(r.instance, r.config)
        jobs[i] = ain
        outs[i] = aout
        keep.append(bufs)
    arrival = np.ascontiguousarray([r.arrival_ms for r in requests], dtype=np.float64)
    admit = np.zeros(count, dtype=np.float64)
    finish = np.zeros(count, dtype=np.float64)
    bin_ = BatchIn()
    bin_.jobs = ctypes.cast(jobs, ctypes.POINTER(AttemptIn))
    bin_.outs = ctypes.cast(outs, ctypes.POINTER(AttemptOut))
    bin_.count = count
    bin_.arrival_ms = arrival.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if served else None
    bin_.slots = slots
    bin_.device = device
    bin_.memory_budget_bytes = memory_budget_bytes
    bin_.admit_ms = admit.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    bin_.finish_ms = finish.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    bout = BatchOut()
    st = lib.tergpu_attempt_batch(ctypes.byref(bin_), ctypes.byref(bout))
    if st != _abi.COMPLETED:
        raise TergpuError(st, _abi.last_error())
    results = []
    for i, r in enumerate(requests):
        stats = keep[i][2]
        results.append(_result(int(outs[i].status), outs[i], stats, r.instance.n))
    if not served:
        arrival = np.zeros(count, dtype=np.float64)
    return BatchResult(results=results, admit_ms=admit, finish_ms=finish, arrival_ms=arrival,
                       total_ms=float(bout.total_ms), peak_running=int(bout.peak_running),
                       peak_predicted_bytes=int(bout.peak_predicted_bytes),
                       refused=int(bout.refused), latency_ms=finish - arrival)


def same_result(a: FullTerResult, b: FullTerResult) -> bool:
    """Bit-exact equality of two results of the same request: status, witness,
    found attempt and every attempt's level sizes and candidate counts."""
    if a.status != b.status or a.found_attempt != b.found_attempt:
        return False
    if (a.witness is None) != (b.witness is None):
        return False
    if a.witness is not None and not np.array_equal(a.witness, b.witness):
        return False
    keys = ("attempt", "status", "level2", "level1", "level0", "l3_modular", "l2_modular",
            "root_modular", "valid_roots", "root_pairs")
    if len(a.attempts) != len(b.attempts):
        return False
    return all(x[k] == y[k] for x, y in zip(a.attempts, b.attempts) for k in keys)
