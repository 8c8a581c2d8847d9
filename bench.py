#!/usr/bin/env python
"""Benchmark of the B200 root join: n=108 root logical pairs/s.

Workload: one whole authentic n=108 root -- the three L1 lists of the
reference's benchmark instance, seed 0x1001, attempt 0 (3,650,689 x 6,900,048
logical pairs against 6,896,564 targets, 69-bit root quotient), produced on the
device by this library's attempt pipeline (level sizes equal the reference's
published capture).  --synthetic swaps in uniform seeded keys of the same sizes
with 8 planted full-Q triples.  A step = one full pass of the hot path (device
radix partition of all three lists + the sweep over all 2.5e13 pairs + exact
resolution).  Inputs (226 MB) exceed L2 (126 MB), so no flush is needed.

  value  : pairs/s with keys already resident in HBM (CUDA events on the
           launching stream, max over ranks).
  e2e    : the same pairs/s through the public C ABI with pinned HOST key
           buffers: upload, partition, sweep, result download per step.
  --impl reference : the reference's own CPU path on the box's host cores: its
           capture of the same root (stream_full_ter_root_lists, untimed), then
           its frozen ARWLF over successive windows of its shuffled cell order,
           one pinned process per host core (no part of this library runs).

Multi-GPU: one process per GPU (torchrun); each rank runs its own independent
root (seed + rank) -- weak scaling, no data-path collective.  --shard-root
splits ONE root over the ranks instead (rank r joins the D entries with
key_d == r (mod G), G the power of two >= N; each step ends with one all-gather
of the triples) -- strong scaling.
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "subset-sum-ter-fft_b200"))
# 32 hardware work queues for this process's CUDA context (the batch / serve
# measurements run 32 streams; with CUDA's default of 8 a short request's kernel
# waits behind a long sweep queued on another stream); before any CUDA call
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "n=108 root pairs/s"
UNIT = "pairs/s"
SIZES = (3_650_689, 6_900_048, 6_896_564)
QBITS = 69
PLANTED = 8
# The sweep's roofline: 2 INT32 ops per logical pair (one add forming the sum, one
# test), the algorithmic minimum, against 148 SMs x 128 INT32 lanes x the SM clock.
OPS_PER_PAIR = 2
INT32_LANES = 148 * 128
# secondary view: the instructions per pair of the kernel's probe design
DESIGN_OPS_PER_PAIR = 5
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one default-variant sweep
# launch on the default workload (the whole authentic n=108 root of seed 0x1001), from one
# ncu capture of that launch; other workloads and variants report null
SWEEP_DRAM_BYTES = {"k_sweep3": 2.571e9 + 355.7e6}
# The reference's published whole-root ARWLF run of this root (seed 0x1001, attempt 0,
# all 4096 cells, 25,189,929,333,072 logical pairs) took 3,575,458 ms on one core
# (results/arwlf/whole-root-20261003/summary.md:10 in the reference): its pairs/s.
PUBLISHED_ARWLF_PAIRS_PER_S = 25_189_929_333_072 / 3575.458


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tergpu", choices=["tergpu", "reference"])
    p.add_argument("--seed", type=lambda s: int(s, 0), default=0x1001)
    p.add_argument("--scale", type=float, default=1.0, help="list-size multiplier (smaller runs)")
    p.add_argument("--family-bits", type=int, default=0)
    p.add_argument("--filter-bits", type=int, default=0)
    p.add_argument("--sweep-v1", action="store_true", help="sweep variant 1 (A/B runs)")
    p.add_argument("--sweep-v2", action="store_true", help="sweep variant 2 (A/B runs)")
    p.add_argument("--sweep-v4", action="store_true", help="sweep variant 4 (A/B runs)")
    p.add_argument("--partition-one-pass", action="store_true",
                   help="one scattered pass per list instead of the staged two (A/B runs)")
    p.add_argument("--cpu-cells", type=int, default=1,
                   help="cells per timed pass of the reference's CPU legs (per process)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batch", action="store_true",
                   help="leave the batch / serve sub-measurements out of the root line")
    p.add_argument("--batch", action="store_true",
                   help="batched attempts (256 instances, n from {36,48,60,72}, 1-16 attempts): "
                        "solves/s batched vs one at a time")
    p.add_argument("--serve", action="store_true",
                   help="served solve stream: Poisson arrivals, continuous batching, p50/p99")
    p.add_argument("--requests", type=int, default=256, help="--batch / --serve request count")
    p.add_argument("--slots", type=int, default=16, help="--batch / --serve concurrent pipelines")
    p.add_argument("--rate", type=float, default=40.0, help="--serve arrivals per second")
    p.add_argument("--serve-n", default="36,48,60,72,84,96",
                   help="--serve dimensions (108 makes one attempt ~9 s; add it explicitly)")
    p.add_argument("--max-attempts", type=int, default=0,
                   help="attempt budgets uniform in [1, max]: 16 for --batch, 64 for --serve")
    p.add_argument("--max-attempts-108", type=int, default=0,
                   help="--serve: budgets of n=108 requests uniform in [1, max] (one n=108 attempt "
                        "holds the device for ~7.7 s; 0 = the same as --max-attempts)")
    p.add_argument("--shard-root", action="store_true",
                   help="N>1: split one root over the ranks (strong scaling) instead of replicas")
    p.add_argument("--n72", action="store_true",
                   help="config 2: the n=72 whole roots (anchor, 0x7201 / 0x7203 / 0x7207 attempt 0) on "
                        "the device against the reference's K2, K2_WIDE, ARWLF and DISPATCH on one core")
    p.add_argument("--synthetic", action="store_true",
                   help="uniform seeded keys (+8 planted triples) instead of the authentic root")
    return p.parse_args()


def sizes_for(args):
    return tuple(max(1, int(round(s * args.scale))) for s in SIZES)


def workload_name(sizes, synthetic=True, seed=0x1001):
    if synthetic:
        return (f"n=108 whole root: {sizes[0]} x {sizes[1]} logical pairs against {sizes[2]} "
                f"targets, Q={QBITS}, uniform seeded keys + {PLANTED} planted full-Q triples")
    return (f"n=108 whole authentic root (benchmark instance seed {seed:#x}, attempt 0): "
            f"{sizes[0]} x {sizes[1]} logical pairs against {sizes[2]} targets, Q={QBITS}")


def authentic_root(seed: int):
    """L1 lists of attempt 0 of the n=108 benchmark instance, from the device
    attempt pipeline, as root keys (list 2 = tau - q_C)."""
    import tergpu
    from tergpu import attempt, instance, snapshot

    t0 = time.perf_counter()
    inst = instance.benchmark_instance(108, seed)
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=seed, attempt_limit=1,
                                                             capture_only=True,
                                                             export_l1_capacity=7_500_000))
    if res.snapshot is None:
        raise RuntimeError(f"attempt pipeline failed: {res.status_name}")
    capture_ms = res.attempts[0]["total_ms"]
    q, lo, hi, _ = snapshot.root_keys(res.snapshot)
    keys = tergpu.RootKeys(quotient_bits=q, lo=lo, hi=hi)
    return keys, {"capture_ms": capture_ms, "level2": res.attempts[0]["level2"],
                  "level1": res.attempts[0]["level1"], "setup_s": time.perf_counter() - t0}, \
        res.snapshot


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if self.proc is None or self.path is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def run_tergpu(args):
    import torch
    import torch.distributed as dist

    import tergpu
    from tergpu import _abi, workload

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from tergpu.shard import shard_count_for, shards_of_rank

    sharded = args.shard_root and world > 1
    my_shards = shards_of_rank(rank, world) if sharded else [0]
    shard_count = shard_count_for(world) if sharded else 1
    root_seed = args.seed if sharded else args.seed + rank
    capture = snap_obj = None
    if args.synthetic:
        sizes = sizes_for(args)
        keys = workload.synthetic_root(sizes=sizes, quotient_bits=QBITS, seed=root_seed,
                                       planted=PLANTED)
        planted = {(sizes[0] - 1 - i, sizes[1] - 1 - i, sizes[2] - 1 - i) for i in range(PLANTED)}
    else:
        keys, capture, snap_obj = authentic_root(root_seed)
        sizes = tuple(len(a) for a in keys.lo)
        planted = set()
    lib = _abi.load()
    first_triples = []

    # device-resident keys (torch is only the allocator here)
    d_lo = [torch.from_numpy(k.view(np.int64)).cuda() for k in keys.lo]
    d_hi = [torch.from_numpy(h).cuda() for h in keys.hi]
    stream = torch.cuda.current_stream()
    cap = 4096
    host_trip = np.zeros(cap * 3, dtype=np.uint32)

    def make_in(resident: bool, lo_src, hi_src, shard: int = 0):
        rin = _abi.RootIn()
        rin.quotient_bits = QBITS
        rin.flags = (_abi.ROOT_DEVICE_INPUTS if resident else 0) | \
            (_abi.ROOT_SWEEP_V1 if args.sweep_v1 else 0) | \
            (_abi.ROOT_SWEEP_V2 if args.sweep_v2 else 0) | \
            (_abi.ROOT_SWEEP_V4 if args.sweep_v4 else 0) | \
            (_abi.ROOT_PARTITION_ONE_PASS if args.partition_one_pass else 0)
        for l in range(3):
            rin.count[l] = sizes[l]
            if resident:
                rin.key_lo[l] = ctypes.cast(lo_src[l].data_ptr(), _abi._u64p)
                rin.key_hi[l] = ctypes.cast(hi_src[l].data_ptr(), _abi._u8p)
            else:
                rin.key_lo[l] = ctypes.cast(lo_src[l].data_ptr(), _abi._u64p)
                rin.key_hi[l] = ctypes.cast(hi_src[l].data_ptr(), _abi._u8p)
            rin.id[l] = None
        rin.cells = None
        rin.device = local
        rin.family_bits = args.family_bits
        rin.filter_bits = args.filter_bits
        rin.stream = ctypes.c_void_p(stream.cuda_stream)
        rin.shard_index = shard
        rin.shard_count = shard_count
        return rin

    def gather(got):
        """One all-gather of this rank's triples (count + 12-byte records)."""
        if not sharded:
            return got
        mine = torch.tensor(got, dtype=torch.int64, device="cuda").reshape(-1, 3)
        counts = [torch.zeros(1, dtype=torch.int64, device="cuda") for _ in range(world)]
        dist.all_gather(counts, torch.tensor([len(got)], dtype=torch.int64, device="cuda"))
        width = max(1, max(int(c.item()) for c in counts))
        pad = torch.zeros((width, 3), dtype=torch.int64, device="cuda")
        pad[: len(got)] = mine
        bufs = [torch.zeros_like(pad) for _ in range(world)]
        dist.all_gather(bufs, pad)
        return sorted(tuple(t) for b, c in zip(bufs, counts) for t in b[: int(c.item())].tolist())

    def call(rins):
        """One step: this rank's shard(s) of the root, then the gather."""
        got, outs_ = [], []
        for rin in rins:
            out = _abi.RootOut()
            out.triples = host_trip.ctypes.data_as(_abi._u32p)
            out.capacity = cap
            st = lib.tergpu_root_run(ctypes.byref(rin), ctypes.byref(out))
            if st != _abi.COMPLETED:
                raise RuntimeError(f"tergpu_root_run status {st}: {_abi.last_error()}")
            n = int(out.triples_count)
            got += [tuple(t) for t in host_trip[: 3 * n].reshape(-1, 3).tolist()]
            outs_.append(out)
        got = gather(sorted(got))
        if not planted <= set(got):
            raise RuntimeError("a planted full-Q triple is missing")
        if not first_triples:
            first_triples.append(got)
        elif got != first_triples[0]:
            raise RuntimeError("two passes over the same root reported different triples")
        out = outs_[0]
        for o in outs_[1:]:
            for f in ("logical_pairs", "filter_survivors", "triples_count", "kernel_launches"):
                setattr(out, f, getattr(out, f) + getattr(o, f))
            for f in ("sweep_ms", "partition_ms", "join_ms"):
                setattr(out, f, getattr(out, f) + getattr(o, f))
        return out

    def barrier():
        if world > 1:
            dist.barrier()

    rin = [make_in(True, d_lo, d_hi, i) for i in my_shards]
    for _ in range(max(3, args.warmup)):
        out = call(rin)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    outs = []
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            outs.append(call(rin))
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    sweep_ms = statistics.median(o.sweep_ms for o in outs)
    part_ms = statistics.median(o.partition_ms for o in outs)
    pairs = local_pairs = int(outs[-1].logical_pairs)
    launches = sum(int(o.kernel_launches) for o in outs)
    survivors = int(outs[-1].filter_survivors)
    triples = int(outs[-1].triples_count)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        # whole-job pairs: the shards of one root, or every rank's own root
        t = torch.tensor([pairs], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        pairs = int(t.item())

    # e2e: pinned host keys through the C ABI, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        h_lo = [torch.from_numpy(k.view(np.int64)).pin_memory() for k in keys.lo]
        h_hi = [torch.from_numpy(h).pin_memory() for h in keys.hi]
        rin_h = [make_in(False, h_lo, h_hi, i) for i in my_shards]
        call(rin_h)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_outs = [call(rin_h) for _ in range(args.steps)]
        torch.cuda.synchronize()
        e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
        if world > 1:
            t = torch.tensor([e_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        h2d = sum(s * 9 for s in sizes) * len(my_shards)
        d2h = triples * 12 + 8 * 8 + 2 * 4 * (1 << e_outs[-1].family_bits)
        e2e = {"value": pairs / (e_ms / 1000.0), "unit": UNIT, "ms_per_step": e_ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    result = None
    if rank == 0:
        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = json.loads(pk.read_text())
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        clk = clocks.summary()
        sm_mhz = clk.get("sm_mhz") or 1965.0
        # algorithmic HBM bytes of one sweep launch: each partitioned list read once (8 B keys)
        sweep_bytes = sum(sizes) * 8
        sweep_kernel = {1: "k_sweep", 2: "k_sweep2", 3: "k_sweep3", 4: "k_sweep4"}.get(
            int(outs[-1].sweep_variant), "k_sweep3")
        # algorithmic partition bytes: every entry read once (8 B key + 1 B high byte) and
        # written once in its family (8 B residual, 1 B high byte, 4 B id), and the B list
        # read and written once more by the lane-slot arrangement of its families
        part_bytes = sum(sizes) * (9 + 13) + sizes[1] * 26
        int32_peak = INT32_LANES * sm_mhz * 1e6  # INT32 ops/s
        sweep_pairs_s = local_pairs / (sweep_ms / 1000.0)
        design_peak = INT32_LANES * sm_mhz * 1e6 / DESIGN_OPS_PER_PAIR
        result = {
            "metric": METRIC, "value": pairs / (ms / 1000.0), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak",
            "vs_baseline": (pairs / (ms / 1000.0) / PUBLISHED_ARWLF_PAIRS_PER_S
                            if not args.synthetic and args.seed == 0x1001 else None),
            "dtype": "u64",
            "data": ("synthetic" if args.synthetic else
                     "authentic: L1 lists generated on the device by this library's attempt "
                     "pipeline from the reference's benchmark instance (sizes equal its published capture)"),
            "config": {"workload": workload_name(sizes, args.synthetic, args.seed), "seed": args.seed,
                       "capture": capture,
                       "l2_flush": "inputs (226 MB) larger than L2 (126 MB)",
                       "family_bits": int(outs[-1].family_bits),
                       "filter_bits": int(outs[-1].filter_bits),
                       "partition_ms": part_ms, "sweep_ms": sweep_ms,
                       "filter_survivors": survivors, "full_q_triples": triples,
                       "parallelism": (f"shards{shard_count}-over-{world}" if sharded
                                       else f"replicas{world}")},
            # the sweep is neither HBM- nor tensor-bound: its roofline is INT32 issue
            # at the algorithmic 2 ops per logical pair
            "roofline": {"bound": "int32", "kernel": sweep_kernel,
                         "achieved": sweep_pairs_s * OPS_PER_PAIR / 1e9, "peak": int32_peak / 1e9,
                         "unit": "Gop/s", "frac": sweep_pairs_s * OPS_PER_PAIR / int32_peak,
                         "ops_per_pair": OPS_PER_PAIR,
                         "peak_source": f"148 SMs x 128 INT32 lanes x {sm_mhz:.0f} MHz (the SM clock "
                                        "sampled during the timed region)",
                         "traffic": (SWEEP_DRAM_BYTES.get(sweep_kernel)
                                     if not args.synthetic and args.seed == 0x1001 else None),
                         "algorithmic_bytes": sweep_bytes},
            "hbm_roofline": {"bound": "hbm", "kernel": sweep_kernel,
                             "achieved": sweep_bytes / (sweep_ms / 1000.0) / 1e9, "peak": hbm,
                             "unit": "GB/s", "frac": sweep_bytes / (sweep_ms / 1000.0) / 1e9 / hbm,
                             "peak_source": peak_src},
            "issue_roofline": {"bound": "int32-issue", "kernel": sweep_kernel, "unit": "pairs/s",
                               "achieved": sweep_pairs_s, "peak": design_peak,
                               "frac": sweep_pairs_s / design_peak,
                               "ops_per_pair": DESIGN_OPS_PER_PAIR, "sm_mhz": sm_mhz,
                               "note": "secondary: the probe design's instructions per pair"},
            "partition_roofline": {"bound": "hbm", "unit": "GB/s",
                                   "kernels": "histogram, scan, scatter (staged two-pass unless "
                                              "--partition-one-pass), family maxima, B arrangement",
                                   "achieved": part_bytes / (part_ms / 1000.0) / 1e9, "peak": hbm,
                                   "frac": part_bytes / (part_ms / 1000.0) / 1e9 / hbm,
                                   "algorithmic_bytes": part_bytes, "partition_ms": part_ms,
                                   "one_pass": bool(args.partition_one_pass),
                                   "peak_source": peak_src},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if e2e is not None:
            result["e2e"] = e2e
    # the reference's CPU path on this host, rank 0 at N=1 only
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if snap_obj is None:
            result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                                      "sample": "the reference's root path runs on captured "
                                                "authentic roots only (not --synthetic)"}
        else:
            result["cpu_baseline"] = cpu_baseline(snap_obj, args)
    # configs 4 and 5 beside the root line (N=1 only): batched and served
    # admitted solves/s against one-at-a-time GPU solves
    if rank == 0 and world == 1 and not args.no_batch:
        result["batch"] = batch_measure(args, False, 256, args.rate, args.serve_n)
        result["serve"] = batch_measure(args, True, 400, 200.0, "36,48,60,72,84,96")
        result["serve"]["note"] = ("without n = 108: see serve_n108 for a mix with it")
        # the same 400 requests (the rate scales only the seeded arrival gaps) arriving at
        # 5,000/s, faster than either engine serves them: the served ratio at saturation
        try:
            result["serve_saturated"] = batch_measure(args, True, 400, 5000.0, "36,48,60,72,84,96")
            result["serve_saturated"]["note"] = ("the serve stream's requests arriving at 5,000/s, so "
                                                 "both the batched engine and one at a time run saturated")
        except RuntimeError as e:  # recorded in its own object; the root line above stands
            result["serve_saturated"] = {"error": str(e)}
        # config 5 with n = 108 in the mix: 28 requests at 4/s over n = 36 ... 108; n = 108
        # budgets capped at one attempt (one holds the device for ~7.7 s), the others 1-64
        result["serve_n108"] = batch_measure(args, True, 28, 4.0, "36,48,60,72,84,96,108",
                                             max_attempts_108=1)
        result["serve_n108"]["note"] = ("n = 108 requests with a budget of 1 attempt (the config's "
                                        "1-64 would make one such request minutes of whole-GPU "
                                        "sweep); per-n latency, admission wait and service time "
                                        "in config.by_n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def ref_binary(have=None, ref=None):
    """The reference harness for timing: the widest of its builds whose CPU flags
    this host has (`have`, default /proc/cpuinfo's) -- -march=native (the CPU
    that built it), then x86-64-v4 (AVX-512), then the portable x86-64-v3."""
    ref = Path(ref) if ref is not None else ROOT / "oracle" / "_ref"
    if have is None:
        have = set()
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                have = set(line.split(":", 1)[1].split())
                break
    skipped = []
    for exe, flags, name in (("terref_native", "native_flags.txt", "native"),
                             ("terref_v4", "v4_flags.txt", "x86-64-v4")):
        if (ref / exe).exists() and (ref / flags).exists():
            missing = set((ref / flags).read_text().split()) - have
            if not missing:
                note = f" (native build lacks: {skipped[0]})" if skipped else ""
                return ref / exe, f"g++ -O2 -march={name}{note}"
            skipped.append(" ".join(sorted(missing)[:8]))
    note = f" (wider builds need CPU flags this host lacks: {'; '.join(skipped)})" if skipped else ""
    return ref / "terref", f"g++ -O2 -march=x86-64-v3{note}"


def cpu_model() -> str:
    for line in Path("/proc/cpuinfo").read_text().splitlines():
        if line.startswith("model name"):
            return line.split(":", 1)[1].strip()
    return "unknown"


def snaptime(binary, snap, backend, cells, reps, first, stride, core=None, timeout=3600):
    """The reference's own root path on one core: load_snapshot_workload of SNAP
    (untimed), then `reps` timed passes of `backend` over successive windows of
    its shuffled cell order (oracle/ref_harness.cpp, snaptime)."""
    cmd = [str(binary), "snaptime", str(snap), backend, "0", str(cells), str(reps), str(first),
           str(stride)]
    if core is not None:
        cmd = ["taskset", "-c", str(core)] + cmd
    return subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)


def rows_of(proc, timeout=3600):
    out, err = proc.communicate(timeout=timeout)
    rows = [json.loads(x) for x in out.splitlines() if x.startswith("{")]
    if proc.returncode != 0 or not rows or "error" in rows[0]:
        raise RuntimeError(f"reference harness failed: {err[-300:]} {out[-300:]}")
    return rows


def target_families(cells) -> int:
    """Distinct target families u = (s + t) mod 64 of cells s * 64 + t."""
    return len({((c >> 6) + (c & 63)) & 63 for c in cells})


def cpu_baseline(snapshot_obj, args):
    """The reference's frozen ARWLF on one pinned host core over the same root,
    read through the reference's own load_snapshot_workload: 3 warm-up and 7 timed
    passes over successive cells of its shuffled cell order, the median (the
    protocol of TER_L1_to_L0_ARWLF_Architecture_v1.0.md:138-142), and K2_WIDE
    timed beside it on one cell."""
    from tergpu import snapshot

    binary, build = ref_binary()
    if not binary.exists():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/terref was not built"}
    cells = max(1, args.cpu_cells)
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "root.snap"
        snapshot.save(snapshot_obj, path, git_commit="reference")
        arwlf = rows_of(snaptime(binary, path, "arwlf", cells, 10, 0, cells, core=0))
        wide = rows_of(snaptime(binary, path, "k2wide", cells, 1, 10 * cells, cells, core=0))
    timed = arwlf[3:]
    rates = [r["pairs"] / (r["ms"] / 1000.0) for r in timed]
    v = statistics.median(rates)
    k2w = wide[0]
    return {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "host_cores": os.cpu_count(),
            "cpu": cpu_model(), "build": build,
            "sample": (f"frozen ARWLF (reference sources, {build}) on 1 pinned core over the same "
                       f"root loaded by the reference's load_snapshot_workload: 3 warm-up + 7 timed "
                       f"passes of {cells} cell(s) each, successive windows of its shuffled cell "
                       f"order ({sum(r['pairs'] for r in timed)} timed pairs), median"),
            "pass_ms": [r["ms"] for r in timed], "pass_pairs": [r["pairs"] for r in timed],
            "k2_wide": {"value": k2w["pairs"] / (k2w["ms"] / 1000.0), "unit": UNIT, "cores": 1,
                        "pairs": k2w["pairs"], "ms": k2w["ms"],
                        "sample": f"frozen K2_WIDE, one pass over {cells} cell(s)"}}


def run_reference(args):
    """The reference's own CPU path only: its capture of the root, its workload
    loader and its frozen ARWLF (oracle/_ref/terref, compiled from its sources);
    nothing of this library is imported or run here."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sizes = sizes_for(args)
    binary, build = ref_binary()
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": workload_name(sizes, args.synthetic, args.seed), "seed": args.seed,
                       "parallelism": "host processes"}}
    if not binary.exists():
        base["unavailable"] = "reference harness oracle/_ref/terref was not built on this host"
        print(json.dumps(base), flush=True)
        return
    if args.synthetic:
        base["unavailable"] = "the reference's root path runs on captured authentic roots only"
        print(json.dumps(base), flush=True)
        return
    procs_n = max(1, min(os.cpu_count() or 1, 64))
    # at least 512 distinct timed cells (successive windows of a shuffled order:
    # 63.99 of the 64 target families appear on average; 256 cells left 61 of 64
    # in one run)
    cells = max(1, args.cpu_cells, -(-512 // (procs_n * max(1, args.steps))))
    reps = max(1, args.steps + args.warmup)
    with tempfile.TemporaryDirectory() as d:
        snap = Path(d) / "root.snap"
        t0 = time.perf_counter()
        cap = subprocess.run([str(binary), "capture", "108", str(args.seed), "0", "auth", str(snap)],
                             capture_output=True, text=True, timeout=3600)
        capture_s = time.perf_counter() - t0
        caps = [json.loads(x) for x in cap.stdout.splitlines() if x.startswith("{")]
        if cap.returncode != 0 or not caps:
            base["unavailable"] = f"the reference's capture failed: {cap.stderr[-200:]}"
            print(json.dumps(base), flush=True)
            return
        sizes = tuple(caps[0]["level1"])
        base["config"]["workload"] = workload_name(sizes, False, args.seed)
        # process i, pass r: cells [(r * P + i) * C, +C) of the shuffled order
        procs = [snaptime(binary, snap, "arwlf", cells, reps, i * cells, procs_n * cells, core=i)
                 for i in range(procs_n)]
        per_proc = [rows_of(p) for p in procs]
    values, timed_cells = [], []
    for rep in range(args.warmup, reps):
        pairs = sum(rows[rep]["pairs"] for rows in per_proc)
        ms = max(rows[rep]["ms"] for rows in per_proc)
        values.append(pairs / (ms / 1000.0))
        for rows in per_proc:
            timed_cells += rows[rep]["cell_ids"]
    v = statistics.median(values)
    pairs_step = statistics.median(sum(rows[rep]["pairs"] for rows in per_proc)
                                   for rep in range(args.warmup, reps))
    sample = (f"the reference's capture of the root ({capture_s:.0f} s, untimed), then its frozen "
              f"ARWLF ({build}) in {procs_n} pinned processes, each pass {cells} cell(s) per "
              f"process from successive windows of its shuffled cell order; {len(set(timed_cells))} "
              f"distinct timed cells over {target_families(timed_cells)} of 64 target families; "
              f"per step: pairs of all processes / the slowest process; median over the timed steps")
    base["config"]["sample"] = sample
    base.update({
        "value": v, "ms_per_step": pairs_step / v * 1000.0,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs_n, "kind": "reference",
                         "cpu": cpu_model(), "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(base), flush=True)


N72_ROOTS = ((19797034556212562, 0), (0x7201, 0), (0x7203, 0), (0x7207, 0))


def run_n72(args):
    """Config 2: each n=72 whole root (L1 lists from the device attempt
    pipeline, byte-identical to the reference's capture) joined on the device
    (CUDA events, keys resident) and by the reference's frozen CPU backends on
    one pinned core over the same root read by its load_snapshot_workload
    (1 warm-up + 3 timed passes each, median; backends in rotated order)."""
    import torch

    import tergpu
    from tergpu import _abi, attempt, instance, snapshot

    torch.cuda.set_device(0)
    binary, build = ref_binary()
    lib = _abi.load()
    backends = ["k2", "k2wide", "arwlf", "dispatch"]
    rows = []
    for k, (seed, att) in enumerate(N72_ROOTS):
        inst = instance.benchmark_instance(72, seed)
        res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=seed, attempt_first=att,
                                                                 attempt_limit=1, capture_only=True,
                                                                 export_l1_capacity=200_000))
        snap = res.snapshot
        q, lo, hi, _ = snapshot.root_keys(snap)
        keys = tergpu.RootKeys(quotient_bits=q, lo=lo, hi=hi)
        d_lo = [torch.from_numpy(a.view(np.int64)).cuda() for a in keys.lo]
        d_hi = [torch.from_numpy(h).cuda() for h in keys.hi]
        stream = torch.cuda.current_stream()
        rin = _abi.RootIn()
        rin.quotient_bits = q
        rin.flags = _abi.ROOT_DEVICE_INPUTS
        for l in range(3):
            rin.count[l] = len(keys.lo[l])
            rin.key_lo[l] = ctypes.cast(d_lo[l].data_ptr(), _abi._u64p)
            rin.key_hi[l] = ctypes.cast(d_hi[l].data_ptr(), _abi._u8p)
        rin.device = 0
        rin.stream = ctypes.c_void_p(stream.cuda_stream)
        trip = np.zeros(4096 * 3, dtype=np.uint32)

        def call():
            out = _abi.RootOut()
            out.triples = trip.ctypes.data_as(_abi._u32p)
            out.capacity = 4096
            st = lib.tergpu_root_run(ctypes.byref(rin), ctypes.byref(out))
            if st != _abi.COMPLETED:
                raise RuntimeError(f"tergpu_root_run status {st}: {_abi.last_error()}")
            return out

        def timed(flags):
            rin.flags = _abi.ROOT_DEVICE_INPUTS | flags
            for _ in range(max(3, args.warmup)):
                call()
            torch.cuda.synchronize()
            steps = max(10, args.steps)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            outs = [call() for _ in range(steps)]
            ev1.record(stream)
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1) / steps
            return ms, outs

        ms, outs = timed(0)
        ms_t, outs_t = timed(_abi.ROOT_AUTOTUNE)  # the autotuner's pick (cached per shape)
        pairs = int(outs[-1].logical_pairs)
        row = {"seed": seed, "attempt": att, "level1": [len(a) for a in keys.lo], "pairs": pairs,
               "gpu": {"ms": ms, "pairs_per_s": pairs / (ms / 1000.0),
                       "sweep_ms": statistics.median(o.sweep_ms for o in outs),
                       "partition_ms": statistics.median(o.partition_ms for o in outs),
                       "family_bits": int(outs[-1].family_bits), "full_q_triples": int(outs[-1].triples_count)},
               "gpu_autotuned": {"ms": ms_t, "pairs_per_s": pairs / (ms_t / 1000.0),
                                 "family_bits": int(outs_t[-1].family_bits),
                                 "filter_bits": int(outs_t[-1].filter_bits),
                                 "sweep_variant": int(outs_t[-1].sweep_variant),
                                 "full_q_triples": int(outs_t[-1].triples_count)},
               "cpu": {}}
        if binary.exists():
            with tempfile.TemporaryDirectory() as d:
                path = Path(d) / "root.snap"
                snapshot.save(snap, path, git_commit="reference")
                order = backends[k % 4:] + backends[:k % 4]
                for b in order:
                    r = rows_of(snaptime(binary, path, b, 4096, 4, 0, 0, core=0))
                    t = statistics.median(x["ms"] for x in r[1:])
                    row["cpu"][b] = {"ms": t, "pairs_per_s": pairs / (t / 1000.0),
                                     "full_q": r[-1]["full_q"], "residue": r[-1]["residue"]}
                    if b == "dispatch":
                        row["cpu"][b]["ran"] = r[-1].get("ran")
            best = max(row["cpu"].items(), key=lambda kv: kv[1]["pairs_per_s"])
            row["best_cpu"] = best[0]
            row["gpu_vs_best_cpu_core"] = row["gpu"]["pairs_per_s"] / best[1]["pairs_per_s"]
        rows.append(row)
    line = {"metric": "n=72 root pairs/s", "unit": "pairs/s", "impl": "tergpu", "n_gpus": 1,
            "value": statistics.median(r["gpu"]["pairs_per_s"] for r in rows),
            "config": {"workload": "n=72 whole authentic roots (benchmark instance, attempt 0): "
                                   + ", ".join(f"{s:#x}" for s, _ in N72_ROOTS),
                       "cpu": cpu_model(), "cpu_build": build, "cpu_cores": 1},
            "roots": rows}
    print(json.dumps(line), flush=True)


def solve_requests(args, serve: bool):
    """Seeded request mix of the batch (config 4) or served (config 5) workload."""
    from tergpu import attempt, batch, instance

    rng = np.random.default_rng(args.seed)
    ns = [36, 48, 60, 72] if not serve else [int(v) for v in args.serve_n.split(",")]
    max_att = args.max_attempts or (64 if serve else 16)
    max_108 = getattr(args, "max_attempts_108", 0) or max_att
    reqs, t = [], 0.0
    for _ in range(args.requests):
        n = int(rng.choice(ns))
        seed = int(rng.integers(1, 1 << 62))
        if serve:
            t += float(rng.exponential(1000.0 / args.rate))
        budget = int(rng.integers(1, max_att + 1))
        if n >= 108 and max_108 < max_att:
            budget = 1 + (budget - 1) * max_108 // max_att    # same draw, scaled to [1, max_108]
        reqs.append(batch.Request(instance.build_instance(n, seed),
                                  attempt.FullTerConfig(seed=seed, attempt_limit=budget),
                                  arrival_ms=t))
    return reqs


def batch_measure(args, serve: bool, requests: int, rate: float, serve_n: str,
                  max_attempts_108: int | None = None) -> dict:
    """One batch (config 4) or served (config 5) measurement: the same seeded
    requests one at a time (one pipeline, in order) and through the
    continuous-batching engine; every result must be bit-identical between the
    two.  The headline is admitted solves/s: requests the preflight refuses
    (36 does not divide n) complete at once and are counted apart."""
    from tergpu import batch

    a = argparse.Namespace(**vars(args))
    a.requests, a.rate, a.serve_n = requests, rate, serve_n
    if max_attempts_108 is not None:
        a.max_attempts_108 = max_attempts_108
    reqs = solve_requests(a, serve)
    # warm both paths: module load, and every slot's workspace with its captured
    # attempt graphs (the engine keeps its slots between calls, as a server would);
    # n=108 requests warm with one of them at one attempt (their cost is the sweep)
    big = [r for r in reqs if r.instance.n >= 108]
    warm = [r for r in reqs if r.instance.n < 108]
    if big:
        r0 = big[0]
        warm.append(batch.Request(r0.instance, dataclasses.replace(r0.config, attempt_limit=1)))
    batch.solve_batch(warm, slots=args.slots)
    one = batch.solve_batch(reqs, slots=1, served=serve)
    many = batch.solve_batch(reqs, slots=args.slots, served=serve)
    for i, (x, y) in enumerate(zip(one.results, many.results)):
        if not batch.same_result(x, y):
            print(f"request {i} (n={reqs[i].instance.n}, seed={reqs[i].config.seed:#x}, "
                  f"budget {reqs[i].config.attempt_limit}): one at a time {x.status_name}, "
                  f"batched {y.status_name}", file=sys.stderr)
            raise RuntimeError("a request's result differs between one-at-a-time and batched runs")
    statuses = [r.status for r in many.results]
    found = [i for i, st in enumerate(statuses) if st == 1]
    admitted = [i for i, st in enumerate(statuses) if st in (1, 3)]

    def pct(v, q):
        return float(np.percentile(v, q)) if len(v) else None

    def summary(res):
        lat = res.latency_ms
        return {"admitted_solves_per_s": len(admitted) / (res.total_ms / 1000.0),
                "all_requests_per_s": len(reqs) / (res.total_ms / 1000.0),
                "wall_ms": res.total_ms, "peak_running": res.peak_running,
                "latency_p50_ms": pct(lat[admitted], 50), "latency_p99_ms": pct(lat[admitted], 99),
                "time_to_found_p50_ms": pct(lat[found], 50),
                "time_to_found_p99_ms": pct(lat[found], 99)}

    s1, sb = summary(one), summary(many)
    by_n = {}
    for r, st in zip(reqs, statuses):
        d = by_n.setdefault(str(r.instance.n), {"requests": 0, "found": 0, "refused": 0})
        d["requests"] += 1
        d["found"] += st == 1
        d["refused"] += st not in (1, 3)
    for key, d in by_n.items():
        idx = [i for i in admitted if str(reqs[i].instance.n) == key]
        if idx:
            for name, res in (("batched", many), ("one_at_a_time", one)):
                wait = res.admit_ms[idx] - res.arrival_ms[idx]
                service = res.finish_ms[idx] - res.admit_ms[idx]
                d[name] = {"latency_p50_ms": pct(res.latency_ms[idx], 50),
                           "latency_p99_ms": pct(res.latency_ms[idx], 99),
                           "admit_wait_p50_ms": pct(wait, 50), "service_p50_ms": pct(service, 50)}
    return {
        "metric": "served admitted solves/s" if serve else "batched admitted solves/s",
        "value": sb["admitted_solves_per_s"], "unit": "solves/s",
        "vs_one_at_a_time": sb["admitted_solves_per_s"] / s1["admitted_solves_per_s"],
        "config": {"workload": "served stream (Poisson arrivals)" if serve else "batched attempts",
                   "requests": len(reqs), "admitted": len(admitted), "refused": many.refused,
                   "found": len(found), "slots": args.slots, "seed": args.seed,
                   "n": sorted({r.instance.n for r in reqs}), "by_n": by_n,
                   "max_attempts": args.max_attempts or (64 if serve else 16),
                   "max_attempts_n108": (getattr(a, "max_attempts_108", 0) or None)
                   if any(r.instance.n >= 108 for r in reqs) else None,
                   "arrival_rate_per_s": rate if serve else None,
                   "attempts_run": sum(len(r.attempts) for r in many.results),
                   "identical_results": True},
        "batched": sb, "one_at_a_time": s1,
    }


def run_batch_modes(args):
    """--batch / --serve: one measurement as its own JSON line."""
    import torch

    torch.cuda.set_device(0)
    line = batch_measure(args, args.serve, args.requests, args.rate, args.serve_n)
    line.update({"higher_is_better": True, "n_gpus": 1, "impl": "tergpu"})
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.batch or args.serve:
        run_batch_modes(args)
    elif args.n72:
        run_n72(args)
    else:
        run_tergpu(args)


if __name__ == "__main__":
    main()
