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
  --impl reference : the reference's frozen ARWLF (built from its sources into
           oracle/_ref) on the box's host cores, one process per core over
           disjoint cells of the same root.

Multi-GPU: one process per GPU (torchrun); each rank runs its own independent
root (seed + rank) -- weak scaling, no data-path collective.  --shard-root
splits ONE root over the ranks instead (rank r joins the D entries with
key_d == r (mod G), G the power of two >= N; each step ends with one all-gather
of the triples) -- strong scaling.
"""
from __future__ import annotations

import argparse
import ctypes
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

METRIC = "n=108 root pairs/s"
UNIT = "pairs/s"
SIZES = (3_650_689, 6_900_048, 6_896_564)
QBITS = 69
PLANTED = 8
# per logical pair the sweep issues at least: IADD, LOP (word offset), LDS, 2x SHF.funnel
OPS_PER_PAIR = 5
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
    p.add_argument("--cpu-cells", type=int, default=6,
                   help="cells of the reference's declared subsample timed on one core")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
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
    p.add_argument("--shard-root", action="store_true",
                   help="N>1: split one root over the ranks (strong scaling) instead of replicas")
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
                  "level1": res.attempts[0]["level1"], "setup_s": time.perf_counter() - t0}


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
    capture = None
    if args.synthetic:
        sizes = sizes_for(args)
        keys = workload.synthetic_root(sizes=sizes, quotient_bits=QBITS, seed=root_seed,
                                       planted=PLANTED)
        planted = {(sizes[0] - 1 - i, sizes[1] - 1 - i, sizes[2] - 1 - i) for i in range(PLANTED)}
    else:
        keys, capture = authentic_root(root_seed)
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
            (_abi.ROOT_SWEEP_V2 if args.sweep_v2 else 0)
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
        sweep_kernel = "k_sweep" if args.sweep_v1 else ("k_sweep2" if args.sweep_v2 else "k_sweep3")
        part_bytes = sum(sizes) * (2 * 9 + 8 + 13 + 4)  # hist read, scatter read + write
        issue_peak = 148 * 4 * 32 * sm_mhz * 1e6 / OPS_PER_PAIR
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
            "roofline": {"bound": "hbm", "kernel": sweep_kernel,
                         "achieved": sweep_bytes / (sweep_ms / 1000.0) / 1e9, "peak": hbm,
                         "unit": "GB/s", "frac": sweep_bytes / (sweep_ms / 1000.0) / 1e9 / hbm,
                         "peak_source": peak_src,
                         "traffic": (SWEEP_DRAM_BYTES.get(sweep_kernel)
                                     if not args.synthetic and args.seed == 0x1001 else None),
                         "note": "the sweep is bound on chip (issue, shared-memory probes), not by "
                                 "HBM: see issue_roofline"},
            "issue_roofline": {"bound": "int32-issue", "kernel": sweep_kernel, "unit": "pairs/s",
                               "achieved": local_pairs / (sweep_ms / 1000.0), "peak": issue_peak,
                               "frac": local_pairs / (sweep_ms / 1000.0) / issue_peak,
                               "ops_per_pair": OPS_PER_PAIR, "sm_mhz": sm_mhz},
            "partition_roofline": {"bound": "hbm", "unit": "GB/s",
                                   "achieved": part_bytes / (part_ms / 1000.0) / 1e9, "peak": hbm,
                                   "frac": part_bytes / (part_ms / 1000.0) / 1e9 / hbm,
                                   "peak_source": peak_src},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if e2e is not None:
            result["e2e"] = e2e
    # the reference's CPU path on this host, rank 0 at N=1 only
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(keys, args)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def write_keys(keys, path: Path):
    with open(path, "wb") as f:
        f.write(b"TERKEYS1")
        f.write(np.array([keys.quotient_bits, 0], dtype=np.uint32).tobytes())
        f.write(np.array([len(a) for a in keys.lo], dtype=np.uint64).tobytes())
        for l in range(3):
            f.write(np.ascontiguousarray(keys.lo[l], dtype=np.uint64).tobytes())
            f.write(np.ascontiguousarray(keys.hi[l], dtype=np.uint8).tobytes())
            f.write(b"\0" * ((8 - len(keys.lo[l]) % 8) % 8))


def ref_binary():
    return ROOT / "oracle" / "_ref" / "terref"


def cpu_baseline(keys, args):
    """The reference's frozen ARWLF on one host core over its declared cell subsample."""
    binary = ref_binary()
    if not binary.exists():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/terref was not built"}
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "root.keys"
        write_keys(keys, path)
        proc = subprocess.run(["taskset", "-c", "0", str(binary), "keysroot", str(path), "arwlf",
                               str(args.cpu_cells), "2", "0"], capture_output=True, text=True,
                              timeout=900)
    rows = [json.loads(x) for x in proc.stdout.splitlines() if x.startswith("{")]
    if proc.returncode != 0 or not rows:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"failed: {proc.stderr[-200:]}"}
    row = min(rows, key=lambda r: r["ms"])
    return {"value": row["pairs"] / (row["ms"] / 1000.0), "unit": UNIT, "cores": 1,
            "kind": "reference", "host_cores": os.cpu_count(),
            "sample": (f"frozen ARWLF (reference sources, g++ -O2 -march=x86-64-v3) on the "
                       f"reference's declared subsample of {args.cpu_cells} of 4096 cells of the "
                       f"same root ({row['pairs']} logical pairs), best of 2, 1 pinned core"),
            "ms": row["ms"], "pairs": row["pairs"],
            "digest_triples": row["triples"]}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sizes = sizes_for(args)
    binary = ref_binary()
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": workload_name(sizes, args.synthetic, args.seed), "seed": args.seed,
                       "parallelism": "host processes"}}
    if not binary.exists():
        base["unavailable"] = "reference harness oracle/_ref/terref was not built on this host"
        print(json.dumps(base), flush=True)
        return
    from tergpu import workload

    if args.synthetic:
        keys = workload.synthetic_root(sizes=sizes, quotient_bits=QBITS, seed=args.seed,
                                       planted=PLANTED)
    else:
        # the authentic root's L1 lists come from the device attempt pipeline
        # (bit-identical to the reference's capture); only ARWLF is timed
        keys, _ = authentic_root(args.seed)
        sizes = tuple(len(a) for a in keys.lo)
        base["config"]["workload"] = workload_name(sizes, False, args.seed)
    procs_n = max(1, min(os.cpu_count() or 1, 64))
    cells_per = max(1, args.cpu_cells)
    reps = max(1, args.steps + args.warmup)
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "root.keys"
        write_keys(keys, path)
        procs = []
        for i in range(procs_n):
            procs.append(subprocess.Popen(
                ["taskset", "-c", str(i % (os.cpu_count() or 1)), str(binary), "keysroot", str(path),
                 "arwlf", f"mod:{procs_n}:{i}:{cells_per}", str(reps), "0"],
                stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        outs = [p.communicate(timeout=3600) for p in procs]
    per_rep = [[json.loads(x) for x in o.splitlines() if x.startswith("{")] for o, _ in outs]
    values = []
    for rep in range(args.warmup, reps):
        pairs = sum(rows[rep]["pairs"] for rows in per_rep)
        ms = max(rows[rep]["ms"] for rows in per_rep)
        values.append(pairs / (ms / 1000.0))
    v = statistics.median(values)
    pairs_step = sum(rows[-1]["pairs"] for rows in per_rep)
    base.update({
        "value": v, "ms_per_step": pairs_step / v * 1000.0,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs_n, "kind": "reference",
                         "sample": (f"frozen ARWLF, {procs_n} processes x {cells_per} disjoint "
                                    f"cells of the same root per step ({pairs_step} pairs)")},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(base), flush=True)


def solve_requests(args, serve: bool):
    """Seeded request mix of the batch (config 4) or served (config 5) workload."""
    from tergpu import attempt, batch, instance

    rng = np.random.default_rng(args.seed)
    ns = [36, 48, 60, 72] if not serve else [int(v) for v in args.serve_n.split(",")]
    max_att = args.max_attempts or (64 if serve else 16)
    reqs, t = [], 0.0
    for _ in range(args.requests):
        n = int(rng.choice(ns))
        seed = int(rng.integers(1, 1 << 62))
        if serve:
            t += float(rng.exponential(1000.0 / args.rate))
        reqs.append(batch.Request(instance.build_instance(n, seed),
                                  attempt.FullTerConfig(seed=seed,
                                                        attempt_limit=int(rng.integers(1, max_att + 1))),
                                  arrival_ms=t))
    return reqs


def run_batch_modes(args):
    """--batch / --serve: the same requests one at a time (one pipeline, in
    order) and through the continuous-batching engine; every result must be
    bit-identical between the two; prints one JSON line."""
    import torch

    from tergpu import batch

    torch.cuda.set_device(0)
    serve = args.serve
    reqs = solve_requests(args, serve)
    # warm both paths: module load, and every slot's workspace with its captured
    # attempt graphs (the engine keeps its slots between calls, as a server would)
    batch.solve_batch(reqs, slots=args.slots)
    one = batch.solve_batch(reqs, slots=1, served=serve)
    many = batch.solve_batch(reqs, slots=args.slots, served=serve)
    for i, (a, b) in enumerate(zip(one.results, many.results)):
        if not batch.same_result(a, b):
            print(f"request {i} (n={reqs[i].instance.n}, seed={reqs[i].config.seed:#x}, "
                  f"budget {reqs[i].config.attempt_limit}): one at a time {a.status_name} "
                  f"{[t['level1'] for t in a.attempts][:3]}, batched {b.status_name} "
                  f"{[t['level1'] for t in b.attempts][:3]}", file=sys.stderr)
            raise RuntimeError("a request's result differs between one-at-a-time and batched runs")
    statuses = [r.status for r in many.results]
    found = [i for i, s in enumerate(statuses) if s == 1]
    admitted = [i for i, s in enumerate(statuses) if s in (1, 3)]

    def pct(v, q):
        return float(np.percentile(v, q)) if len(v) else None

    def summary(res):
        lat = res.latency_ms
        return {"solves_per_s": len(reqs) / (res.total_ms / 1000.0),
                "admitted_solves_per_s": len(admitted) / (res.total_ms / 1000.0),
                "wall_ms": res.total_ms, "peak_running": res.peak_running,
                "latency_p50_ms": pct(lat[admitted], 50), "latency_p99_ms": pct(lat[admitted], 99),
                "time_to_found_p50_ms": pct(lat[found], 50),
                "time_to_found_p99_ms": pct(lat[found], 99)}

    s1, sb = summary(one), summary(many)
    attempts = sum(len(r.attempts) for r in many.results)
    line = {
        "metric": "served solves/s" if serve else "batched solves/s",
        "value": sb["solves_per_s"], "unit": "solves/s", "higher_is_better": True,
        "n_gpus": 1, "impl": "tergpu",
        "vs_one_at_a_time": sb["solves_per_s"] / s1["solves_per_s"],
        "config": {"workload": ("served stream" if serve else "batched attempts"),
                   "requests": len(reqs), "slots": args.slots, "seed": args.seed,
                   "n": sorted({r.instance.n for r in reqs}),
                   "max_attempts": args.max_attempts or (64 if serve else 16),
                   "arrival_rate_per_s": args.rate if serve else None,
                   "refused": many.refused, "found": len(found), "attempts_run": attempts,
                   "identical_results": True},
        "batched": sb, "one_at_a_time": s1,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.batch or args.serve:
        run_batch_modes(args)
    else:
        run_tergpu(args)


if __name__ == "__main__":
    main()
