"""tergpu_root_run_noalloc through the C ABI: the same triples and counts as
tergpu_root_run, on two calls in a row.

The no-allocation entry is for callers that may not allocate device memory
themselves (a host framework whose pool owns all device memory, a process that
reserved its memory up front, a service loop that must not risk an allocation).
It keeps its intermediates in a fixed 32 MiB device array inside the library,
so this test hands it device-resident keys and a device output buffer (made
here with torch: the test may allocate, the entry point may not).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(torch, keys):
    lo = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()
          for a in keys.lo]
    hi = [torch.from_numpy(np.ascontiguousarray(h, dtype=np.uint8)).cuda() for h in keys.hi]
    return lo, hi


def _noalloc_call(lib, _abi, torch, keys, lo, hi, capacity, flags=0, cells=None, family_bits=0,
                  filter_bits=0, stream=None):
    rin = _abi.RootIn()
    rin.quotient_bits = keys.quotient_bits
    rin.flags = _abi.ROOT_DEVICE_INPUTS | flags
    for l in range(3):
        rin.count[l] = lo[l].numel()
        rin.key_lo[l] = ctypes.cast(lo[l].data_ptr(), _abi._u64p)
        rin.key_hi[l] = ctypes.cast(hi[l].data_ptr(), _abi._u8p)
        rin.id[l] = None
    rin.cells = None if cells is None else ctypes.cast(cells.data_ptr(), _abi._u8p)
    rin.family_bits = family_bits
    rin.filter_bits = filter_bits
    rin.device = torch.cuda.current_device()
    stream = stream or torch.cuda.current_stream()
    rin.stream = ctypes.c_void_p(stream.cuda_stream)
    out_dev = torch.zeros(capacity * 3, dtype=torch.int32, device="cuda")
    out = _abi.RootOut()
    out.triples = ctypes.cast(out_dev.data_ptr(), _abi._u32p)
    out.capacity = capacity
    torch.cuda.synchronize()
    status = lib.tergpu_root_run_noalloc(ctypes.byref(rin), ctypes.byref(out))
    torch.cuda.synchronize()
    n = int(out.triples_count)
    trip = out_dev[: 3 * min(n, capacity)].cpu().numpy().view(np.uint32).reshape(-1, 3)
    return status, out, trip


def _sorted(t):
    return sorted(map(tuple, np.asarray(t).reshape(-1, 3).tolist()))


@pytest.mark.parametrize("which", ["synthetic_q69", "planted_q47"])
def test_noalloc_matches_existing_entry_twice(which):
    import torch

    import tergpu
    from tergpu import _abi, workload

    if which == "synthetic_q69":
        import oracle

        lo, hi = oracle.synthetic_root(69, 0x1234, 2000, 0)
        keys = tergpu.RootKeys(quotient_bits=69, lo=lo, hi=[h.astype(np.uint8) for h in hi])
    else:
        keys = _planted_q47()
    expected = tergpu.run_gpu_root(keys)
    lib = _abi.load()
    lo_d, hi_d = _device_inputs(torch, keys)
    for _ in range(2):
        status, out, trip = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=4096)
        assert status == _abi.COMPLETED, lib.tergpu_noalloc_last_error()
        assert int(out.triples_count) == expected.telemetry.full_hits
        assert int(out.logical_pairs) == expected.telemetry.logical_pairs
        assert _sorted(trip) == _sorted(expected.triples)
        if which == "synthetic_q69":
            # and the oracle's multiset digest of the same root, directly
            from tergpu import workload as wl

            digest, _ = oracle.root_join(69, lo, hi)
            got = wl.digest(trip)
            for k in ("triples", "triple_sum", "triple_xor", "triple_sum2"):
                assert got[k] == digest[k], k


def _planted_q47():
    from tergpu import workload

    return workload.synthetic_root(sizes=(60_000, 120_000, 120_000), quotient_bits=47, seed=0x5EED,
                                   planted=16)


def test_noalloc_cells_count_only_and_tuning_limits():
    """The device cell mask, count-only calls and the family / filter limits
    (10 and 20 bits) give what tergpu_root_run gives on the same keys."""
    import torch

    import tergpu
    from tergpu import _abi

    keys = _planted_q47()
    lib = _abi.load()
    lo_d, hi_d = _device_inputs(torch, keys)
    rng = np.random.default_rng(7)
    cells = (rng.random(4096) < 0.4).astype(np.uint8)
    want = tergpu.run_gpu_root(keys, cells=cells)
    status, out, trip = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=4096,
                                      cells=torch.from_numpy(cells).cuda())
    assert status == _abi.COMPLETED, lib.tergpu_noalloc_last_error()
    assert int(out.logical_pairs) == want.telemetry.logical_pairs
    assert _sorted(trip) == _sorted(want.triples)
    whole = tergpu.run_gpu_root(keys)
    status, out, _ = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=0,
                                   flags=_abi.ROOT_COUNT_ONLY)
    assert status == _abi.COMPLETED and int(out.triples_count) == whole.telemetry.full_hits
    status, out, trip = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=4096,
                                      family_bits=10, filter_bits=20)
    assert status == _abi.COMPLETED, lib.tergpu_noalloc_last_error()
    assert (int(out.family_bits), int(out.filter_bits)) == (10, 20)
    assert _sorted(trip) == _sorted(whole.triples)


def test_noalloc_output_overflow_reports_the_exact_count():
    """A capacity below the true triple count: OUTPUT_OVERFLOW, the exact count,
    and `capacity` of the root's triples written."""
    import torch

    import tergpu
    from tergpu import _abi

    keys = _planted_q47()
    whole = _sorted(tergpu.run_gpu_root(keys).triples)
    assert len(whole) > 4
    lib = _abi.load()
    lo_d, hi_d = _device_inputs(torch, keys)
    cap = len(whole) - 3
    status, out, trip = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=cap)
    assert status == _abi.OUTPUT_OVERFLOW
    assert int(out.triples_count) == len(whole)
    got = _sorted(trip)
    assert len(got) == cap and set(got) <= set(whole)


def test_noalloc_refuses_a_capturing_stream_and_restores_the_device():
    """The entry waits for its stream, so on a stream under capture it returns
    INVALID_INPUT without touching the capture; it leaves the caller's current
    device as it found it."""
    import torch

    from tergpu import _abi

    keys = _planted_q47()
    lib = _abi.load()
    lo_d, hi_d = _device_inputs(torch, keys)
    status, _, _ = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=4096)
    assert status == _abi.COMPLETED  # the first call on the device does its set-up here
    side = torch.cuda.Stream()
    x = torch.zeros(16, device="cuda")
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        graph.capture_begin()
        x.add_(1)
        rin = _abi.RootIn()
        rin.quotient_bits = keys.quotient_bits
        rin.flags = _abi.ROOT_DEVICE_INPUTS
        for l in range(3):
            rin.count[l] = lo_d[l].numel()
            rin.key_lo[l] = ctypes.cast(lo_d[l].data_ptr(), _abi._u64p)
            rin.key_hi[l] = ctypes.cast(hi_d[l].data_ptr(), _abi._u8p)
        rin.device = torch.cuda.current_device()
        rin.stream = ctypes.c_void_p(side.cuda_stream)
        out = _abi.RootOut()
        status = lib.tergpu_root_run_noalloc(ctypes.byref(rin), ctypes.byref(out))
        graph.capture_end()
    assert status == _abi.INVALID_INPUT
    assert b"capturing" in lib.tergpu_noalloc_last_error()
    graph.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 16.0
    before = torch.cuda.current_device()
    status, _, _ = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=4096)
    assert status == _abi.COMPLETED and torch.cuda.current_device() == before


def test_noalloc_refuses_roots_beyond_its_scratch():
    import torch

    from tergpu import _abi, workload

    # 3 x 2.5M entries need ~100 MB of intermediates, over the 32 MiB array; the
    # inputs are real device buffers of that size, so nothing reads past them.
    keys = workload.synthetic_root(sizes=(2_500_000, 2_500_000, 2_500_000), quotient_bits=69,
                                   seed=1, planted=0)
    lib = _abi.load()
    lo_d, hi_d = _device_inputs(torch, keys)
    status, out, _ = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=16)
    assert status == _abi.RESOURCE_LIMIT
    assert b"32 MiB" in lib.tergpu_noalloc_last_error()
