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


def _noalloc_call(lib, _abi, torch, keys, lo, hi, capacity):
    rin = _abi.RootIn()
    rin.quotient_bits = keys.quotient_bits
    rin.flags = _abi.ROOT_DEVICE_INPUTS
    for l in range(3):
        rin.count[l] = lo[l].numel()
        rin.key_lo[l] = ctypes.cast(lo[l].data_ptr(), _abi._u64p)
        rin.key_hi[l] = ctypes.cast(hi[l].data_ptr(), _abi._u8p)
        rin.id[l] = None
    rin.cells = None
    rin.device = torch.cuda.current_device()
    rin.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
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
        keys = workload.synthetic_root(sizes=(60_000, 120_000, 120_000), quotient_bits=47,
                                       seed=0x5EED, planted=16)
    expected = tergpu.run_gpu_root(keys)
    lib = _abi.load()
    lo_d, hi_d = _device_inputs(torch, keys)
    for _ in range(2):
        status, out, trip = _noalloc_call(lib, _abi, torch, keys, lo_d, hi_d, capacity=4096)
        assert status == _abi.COMPLETED, lib.tergpu_noalloc_last_error()
        assert int(out.triples_count) == expected.telemetry.full_hits
        assert int(out.logical_pairs) == expected.telemetry.logical_pairs
        assert _sorted(trip) == _sorted(expected.triples)


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
