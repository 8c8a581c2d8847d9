"""Run records of the reference's root campaigns, produced by the device root.

The reference keeps its evidence as JSON lines appended by two runners; this
module writes the same rows with the device as the backend ("gpu"), so GPU runs
sit beside the published CPU rows and the reference's summary scripts read both:

* ``whole_root``: one whole authentic root with one planted final output on
  the anchor microproblem, one row per run in ``<out-dir>/runs.jsonl``
  (ter2_root/campaign/ter_arwlf_whole_root_main.cpp:190-417).  A rerun of a
  finished run id does nothing; a run id recorded with another backend or root
  is refused (exit 2).  The planted output must come back exactly: nothing
  missed, nothing extra (exit 4 and an EXACTNESS_FAILURE row otherwise).
* ``solve_attempt``: one Full TER attempt's root stage on a captured root, one
  row appended to ``--out`` (ter2_root/campaign/ter_arwlf_solve_attempt_main.cpp:
  143-185 over ter_arwlf_solve.cpp:41-178): residue-exact triples, the root rule
  (binary parent of weight n/2), the distinct parents rebuilt from the records,
  each verified against the benchmark instance.

``plant_positive`` restates the reference's positive planting
(PlantedTargets, ter2_root/campaign/ter_arwlf_campaign.cpp:400-587) on snapshot
records: a seeded pair (a, b) of the anchor cell's A and B families gets a new
D record whose key is key_a + key_b and whose digits and residue complete the
pair to the root target, appended to list C as EntryId |C|.

Command line:
    python -m tergpu.runs whole-root --snapshot=PATH --out-dir=DIR --run=ID
    python -m tergpu.runs whole-root --n=108 --seed=0x1001 --attempt=0 --out-dir=DIR --run=ID
    python -m tergpu.runs solve-attempt --snapshot=PATH --out=FILE.jsonl
(--n/--seed/--attempt capture the root with the device attempt pipeline instead
of reading a .snap file.)
"""
from __future__ import annotations

import argparse
import json
import os
import resource
import subprocess
import sys
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import snapshot as snapmod
from .root import Config, run_gpu_root_records

FAMILIES = 64                 # target families of a root (rg::kFamilies)
SPLIT_BITS = 6                # family = low 6 key bits (mr8::kSplitBits)
RESIDUAL_MASK = (1 << 19) - 1  # posting value = the next 19 key bits (mr8::kResidualMask)
PLANT_TAG = 0x504C414E54      # "PLANT"
PLANT_SEED = 0xB1A57001       # the whole-root runner's plant seed
_U64 = (1 << 64) - 1


def mix64(v: int) -> int:
    """SplitMix64 finalizer (ter2_root/frozen/ter_root_queue_kernels.hpp:39-44)."""
    v = (v + 0x9E3779B97F4A7C15) & _U64
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & _U64
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & _U64
    return v ^ (v >> 31)


def thinning_hash(root_seed: int, cell: int, tag: int, entry: int, seed: int) -> int:
    """ter2_root/campaign/ter_arwlf_campaign.cpp:232-239."""
    h = seed & _U64
    h = mix64(h ^ (root_seed & _U64))
    h = mix64(h ^ cell)
    h = mix64(h ^ tag)
    return mix64(h ^ (entry & _U64))


def select_cells(count: int) -> np.ndarray:
    """The reference's microproblem sample (select_microproblems,
    ter2_root/frozen/ter_root_queue_kernels.cpp:111-133): a Fisher-Yates order
    of the 4096 cells driven by mix64(0x5EED5EED + i); the first `count` cells."""
    sel = np.zeros(FAMILIES * FAMILIES, dtype=np.uint8)
    if count >= sel.size:
        sel[:] = 1
        return sel
    order = list(range(sel.size))
    state = 0x5EED5EED
    for at in range(sel.size - 1, 0, -1):
        pick = mix64(state) % (at + 1)
        state += 1
        order[at], order[pick] = order[pick], order[at]
    for at in range(count):
        sel[order[at]] = 1
    return sel


def anchor_cell() -> int:
    """The campaign's anchor microproblem: the one cell of a 1-cell sample."""
    return int(np.flatnonzero(select_cells(1))[0])


def _digits(snap, l: int, e: int) -> np.ndarray:
    """int8[n] digits of entry e of list l (+1 pos bit, -1 neg bit)."""
    pos, neg = snap.masks(l)
    out = np.zeros(snap.n, dtype=np.int8)
    for i in range(snap.n):
        w, b = divmod(i, 64)
        out[i] = ((int(pos[e, w]) >> b) & 1) - ((int(neg[e, w]) >> b) & 1)
    return out


def _complete_digits(a: np.ndarray, b: np.ndarray, want: tuple[int, int, int]) -> np.ndarray | None:
    """Digits c with a + b + c in {-1, 0, +1} and `want` = (negative, zero,
    positive) parent digits: forced coordinates (a + b = +-2) first, then the
    free ones in coordinate order (ter_arwlf_campaign.cpp:428-478)."""
    n = len(a)
    s = a.astype(np.int32) + b.astype(np.int32)
    w_neg, w_zero, w_pos = want
    forced_pos, forced_neg = int((s == 2).sum()), int((s == -2).sum())
    ones, minus_ones, zeros = int((s == 1).sum()), int((s == -1).sum()), int((s == 0).sum())
    if w_pos < forced_pos or w_neg < forced_neg or w_pos + w_neg + w_zero != n:
        return None
    pos_from_ones = min(ones, w_pos - forced_pos)
    pos_from_zeros = w_pos - forced_pos - pos_from_ones
    neg_from_minus = min(minus_ones, w_neg - forced_neg)
    neg_from_zeros = w_neg - forced_neg - neg_from_minus
    if pos_from_zeros + neg_from_zeros > zeros:
        return None
    out = np.zeros(n, dtype=np.int8)
    for i in range(n):
        si = int(s[i])
        parent = 0
        if si == 2:
            parent = 1
        elif si == -2:
            parent = -1
        elif si == 1 and pos_from_ones > 0:
            parent, pos_from_ones = 1, pos_from_ones - 1
        elif si == -1 and neg_from_minus > 0:
            parent, neg_from_minus = -1, neg_from_minus - 1
        elif si == 0 and pos_from_zeros > 0:
            parent, pos_from_zeros = 1, pos_from_zeros - 1
        elif si == 0 and neg_from_zeros > 0:
            parent, neg_from_zeros = -1, neg_from_zeros - 1
        out[i] = parent - si
    return out


def structural_parent_counts(n: int) -> tuple[int, int, int]:
    """(negative, zero, positive) digits of a FiniteSanity structural parent at
    the root, the shape the reference's authority tables carry (the device
    authority's structural flag tests the same counts)."""
    return 2, n - 4 - n // 6, 2 + n // 6


@dataclass
class Planted:
    snapshot: object        # the snapshot with the planted records appended to list C
    cell: int
    first_planted: int      # EntryId of the first planted C record
    expected: list          # sorted [a, b, c] witnesses the root must report
    d_lo: list              # planted keys (low 64 bits of the Q-bit d = tau - q_c)
    d_hi: list


def plant_positive(snap, cell: int, count: int = 1, seed: int = PLANT_SEED) -> Planted:
    """PlantedTargets(workload, cell, Plant{Positive, count, seed}) on records."""
    Q, lo, hi, _tau = snapmod.root_keys(snap)
    n, w32 = snap.n, snap.words32
    s, t = cell // FAMILIES, cell % FAMILIES
    u = (s + t) & (FAMILIES - 1)

    def family(l: int, f: int) -> np.ndarray:
        ids = np.flatnonzero((lo[l] & np.uint64(FAMILIES - 1)) == np.uint64(f)).astype(np.uint64)
        vals = (lo[l][ids.astype(np.int64)] >> np.uint64(SPLIT_BITS)) & np.uint64(RESIDUAL_MASK)
        return ids[np.lexsort((ids, vals))]  # the loader's (value, EntryId) posting order

    qs, xs = family(0, s), family(1, t)
    if len(qs) == 0 or len(xs) == 0:
        raise ValueError("positive planting needs a microproblem with work")
    lo_bits = min(Q, 64)
    lo_mask = (1 << lo_bits) - 1
    hi_mask = (1 << (Q - 64)) - 1 if Q > 64 else 0
    nmask = (1 << n) - 1
    root = snapmod.words_to_int(snap.root_target) & nmask
    res = [snap.residues(l) for l in range(2)]
    want = structural_parent_counts(n)
    key_size = snap.entries[2]
    used, planted_recs, expected, d_lo, d_hi = set(), [], [], [], []
    draw, max_draws = 0, 64 * count + 1024
    while len(planted_recs) < count:
        if draw == max_draws:
            raise RuntimeError("could not find enough distinct completable pairs to plant")
        h = thinning_hash(snap.seed, cell, PLANT_TAG, draw, seed)
        draw += 1
        qi, xi = h % len(qs), mix64(h) % len(xs)
        if (qi, xi) in used:
            continue
        a, b = int(qs[qi]), int(xs[xi])
        qa, qb = int(lo[0][a]), int(lo[1][b])
        dl = (qa + qb) & lo_mask
        carry = 1 if lo_bits == 64 and qa + qb > _U64 else 0
        dh = (int(hi[0][a]) + int(hi[1][b]) + carry) & hi_mask
        c_digits = _complete_digits(_digits(snap, 0, a), _digits(snap, 1, b), want)
        if c_digits is None:
            continue
        ra = snapmod.words_to_int(res[0][a]) & nmask
        rb = snapmod.words_to_int(res[1][b]) & nmask
        rc = (root - ra - rb) & nmask
        used.add((qi, xi))
        if (dl & (FAMILIES - 1)) != u:
            raise RuntimeError("planted key left its target family")
        pos = [0] * snap.words64
        neg = [0] * snap.words64
        for i, d in enumerate(c_digits.tolist()):
            if d > 0:
                pos[i // 64] |= 1 << (i % 64)
            elif d < 0:
                neg[i // 64] |= 1 << (i % 64)
        rec = np.concatenate([np.array(pos + neg, dtype="<u8").view(np.uint8),
                              np.array([(rc >> (32 * k)) & 0xFFFFFFFF for k in range(w32)],
                                       dtype="<u4").view(np.uint8)])
        expected.append([a, b, key_size + len(planted_recs)])
        planted_recs.append(rec)
        d_lo.append(dl)
        d_hi.append(dh)
    records = list(snap.records)
    records[2] = np.concatenate([np.asarray(records[2], dtype=np.uint8)] + planted_recs)
    out = snapmod.Snapshot(n=snap.n, r1=snap.r1, r2=snap.r2, attempt=snap.attempt, seed=snap.seed,
                           attempt_seed=snap.attempt_seed, records=records,
                           child_targets=snap.child_targets, root_target=snap.root_target,
                           level2_sizes=list(snap.level2_sizes))
    return Planted(snapshot=out, cell=cell, first_planted=key_size, expected=sorted(expected),
                   d_lo=d_lo, d_hi=d_hi)


# ---------------------------------------------------------------------------
# rows
# ---------------------------------------------------------------------------

def _utc() -> str:
    return time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())


def _git_commit() -> str:
    try:
        return subprocess.run(["git", "rev-parse", "HEAD"], cwd=Path(__file__).resolve().parent,
                              capture_output=True, text=True, timeout=10).stdout.strip() or "unknown"
    except (OSError, subprocess.SubprocessError):
        return "unknown"


def _memory_mib() -> tuple[float, float]:
    peak = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 1024.0  # KiB on Linux
    try:
        with open("/proc/self/statm") as f:
            rss = int(f.read().split()[1]) * os.sysconf("SC_PAGE_SIZE") / 2**20
    except OSError:
        rss = peak
    return round(rss, 1), round(peak, 1)


def _device_name(device: int) -> str:
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:  # noqa: BLE001 - informational field only
        return ""


def _residue_sum(triples: np.ndarray) -> int:
    from .workload import digest

    return digest(triples)["triple_sum"] if len(triples) else 0


def _capture(n: int, seed: int, attempt_index: int, device: int):
    from . import attempt, instance

    inst = instance.benchmark_instance(n, seed)
    cap = {36: 4096, 72: 200_000, 108: 7_500_000}.get(n, 7_500_000)
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=seed, attempt_first=attempt_index,
                                                             attempt_limit=1, capture_only=True,
                                                             export_l1_capacity=cap, device=device))
    if res.snapshot is None:
        raise RuntimeError(f"device capture of n={n} seed={seed:#x} attempt {attempt_index} failed")
    return res.snapshot


def whole_root(snap, root: str, run_id: str, out_dir, device: int = 0, load_ms: float = 0.0,
               plant: bool = True) -> tuple[int, dict | None]:
    """One whole root on the device, appended to <out_dir>/runs.jsonl.
    Returns (exit code, row); the exit codes are the reference runner's."""
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    runs_path = out_dir / "runs.jsonl"
    if runs_path.exists():
        for line in runs_path.read_text().splitlines():
            try:
                r = json.loads(line)
            except ValueError:
                continue
            if r.get("run_id") != run_id:
                continue
            if r.get("backend") != "gpu" or r.get("root") != root:
                print(f"# refused: run {run_id} already recorded with another backend or root")
                return 2, None
            if r.get("status") == "COMPLETED":
                print(f"# run {run_id} already complete")
                return 0, None
    Q = snap.n - snap.r1
    if Q < PROJECTION_BITS:
        # the reference's runner stops at its workload loader with exit 3 and no row
        # (ter2_root/campaign/ter_arwlf_whole_root_main.cpp:234-240)
        print(f"# snapshot {root} : NotApplicable (quotient width Q={Q} is below the 25-bit projection)")
        return 3, None
    cell = anchor_cell()
    t0 = time.perf_counter()
    planted = plant_positive(snap, cell) if plant else None
    plant_ms = (time.perf_counter() - t0) * 1000.0
    work = planted.snapshot if planted else snap
    res = run_gpu_root_records(work, Config(device=device))
    tel = res.telemetry
    exact_rows = res.triples[(res.flags & 1) == 1] if len(res.triples) else res.triples
    witnesses = sorted(map(list, exact_rows.tolist()))
    first = planted.first_planted if planted else snap.entries[2]
    planted_found = [w for w in witnesses if w[2] >= first]
    planted_ok = planted_found == (planted.expected if planted else [])
    exact = planted_ok and len(witnesses) == res.residue_exact
    rss, peak = _memory_mib()
    row = {
        "run_id": run_id, "chunk": "all", "backend": "gpu",
        "status": "COMPLETED" if exact else "EXACTNESS_FAILURE",
        "root": root, "n": snap.n, "root_seed": hex(snap.seed), "Q": Q, "W": min(Q, 64) - SPLIT_BITS,
        "git_commit": _git_commit(), "git_dirty_at_configure": -1,
        "compiler": "nvcc sm_100a", "build": "Release", "pin": "none", "pinned_cpu": -1,
        "anchor_cell": cell, "plant_seed": hex(PLANT_SEED) if plant else "",
        "first_planted": first, "planted": planted.expected if planted else [],
        "setup_load_ms": round(load_ms, 1), "setup_plant_ms": round(plant_ms, 1),
        "setup_keys_ms": 0.0, "setup_index_ms": 0.0, "setup_census_ms": 0.0, "utc": _utc(),
        "cells": FAMILIES * FAMILIES, "logical_pairs": int(tel.logical_pairs),
        "ms": round(float(tel.total_ms), 4), "cpu_start": -1, "cpu_end": -1, "on_pinned_core": False,
        "ac_start": -1, "ac_end": -1,
        "residue_exact": int(res.residue_exact), "structural": int(res.structural),
        "full_q": int(len(res.triples)), "pair_hits": 0,
        "residue_sum": f"{_residue_sum(exact_rows):#018x}",
        "directory_misses": 0, "residual_mismatches": 0, "planted_ok": planted_ok,
        "witnesses": witnesses, "arwlf_status": "", "dispatch_ran": "", "dispatch_probe_ms": 0.0,
        "working_set_mib": rss, "peak_working_set_mib": peak,
        # device-only fields
        "device": _device_name(device), "sweep_ms": round(float(tel.sweep_ms), 4),
        "partition_ms": round(float(tel.partition_ms), 4),
        "filter_survivors": int(tel.filter_survivors), "family_bits": int(tel.family_bits),
        "filter_bits": int(tel.filter_bits),
    }
    with open(runs_path, "a") as f:
        f.write(json.dumps(row, separators=(",", ":")) + "\n")
    print(f"# {run_id} all : {tel.total_ms / 1000.0:.2f} s, {row['cells']} cells, "
          f"{len(witnesses)} outputs" + ("" if exact else "  EXACTNESS FAILURE"))
    return (0 if exact else 4), row


# The reference's workload loader refuses roots below its 25-bit projection
# (ter2_root/frozen/ter_root_generalization_workload.cpp:604-609).
PROJECTION_BITS = 25


def _attempt_row(snapshot_label: str, status: str, message: str, n: int = 0, seed: int = 0, attempt: int = 0,
                 attempt_seed: int = 0, load_ms: float = 0.0, root_ms: float = 0.0, rebuild_ms: float = 0.0,
                 verify_ms: float = 0.0, residue_exact: int = 0, structural_triples: int = 0,
                 parents=(), planted_found: bool = False, device_name: str = "", device_root_ms: float = 0.0) -> dict:
    """One attempts.jsonl row with the fields, in the order, that
    ter_arwlf_solve_attempt writes (ter2_root/campaign/ter_arwlf_solve_attempt_main.cpp:161-177),
    plus the device's name and root time."""
    rss, peak = _memory_mib()
    return {
        "snapshot": snapshot_label, "status": status, "message": message, "n": n, "seed": seed,
        "attempt": attempt, "attempt_seed": attempt_seed, "backend": "gpu",
        "dispatch_ran": "", "load_ms": round(load_ms, 1), "keys_ms": 0.0, "root_ms": round(root_ms, 1),
        "rebuild_ms": round(rebuild_ms, 1), "verify_ms": round(verify_ms, 3),
        "residue_exact": int(residue_exact), "structural_triples": int(structural_triples),
        "unique_parents": len(parents), "planted_found": planted_found,
        "parents": sorted(parents) if status == "Found" else [],
        "pin": "none", "pinned_cpu": -1, "cpu_start": -1, "cpu_end": -1,
        "working_set_mib": rss, "peak_working_set_mib": peak, "build": "Release",
        "git_commit": _git_commit(), "git_dirty_at_configure": -1, "utc": _utc(),
        "device": device_name, "device_root_ms": round(float(device_root_ms), 3),
    }


def _append(out_path, row: dict) -> dict:
    with open(out_path, "a") as f:
        f.write(json.dumps(row, separators=(",", ":")) + "\n")
    return row


def solve_attempt(snap, snapshot_label: str, out_path, device: int = 0, load_ms: float = 0.0) -> dict:
    """One attempt's root stage on the device, appended to `out_path`.  A root
    whose quotient is below the reference's 25-bit projection (n = 36) is
    recorded NotApplicable without device work, as the reference's
    solve_attempt records it (ter2_root/campaign/ter_arwlf_solve.cpp:53-58)."""
    from . import instance as inst_mod

    n = snap.n
    if n - snap.r1 < PROJECTION_BITS:
        return _append(out_path, _attempt_row(
            snapshot_label, "NotApplicable",
            f"quotient width Q={n - snap.r1} is below the 25-bit projection", n=n, seed=snap.seed,
            load_ms=load_ms))
    t0 = time.perf_counter()
    res = run_gpu_root_records(snap, Config(device=device))
    root_ms = (time.perf_counter() - t0) * 1000.0
    exact = res.triples[(res.flags & 1) == 1] if len(res.triples) else res.triples
    accepted = res.triples[(res.flags & 5) == 5] if len(res.triples) else res.triples
    t0 = time.perf_counter()
    parents = set()
    message, status = "", "NoWitnessThisAttempt"
    for a, b, c in accepted.tolist():
        digits = _digits(snap, 0, a).astype(np.int32) + _digits(snap, 1, b) + _digits(snap, 2, c)
        if digits.min() < -1 or digits.max() > 1:
            status, message = "InvariantViolation", "an accepted triple's parent digit leaves {-1, 0, +1}"
            break
        parents.add("".join(str(int(d)) for d in digits))
    rebuild_ms = (time.perf_counter() - t0) * 1000.0
    t0 = time.perf_counter()
    planted_found = False
    if parents and status != "InvariantViolation":
        inst = inst_mod.benchmark_instance(n, snap.seed)
        planted_str = "".join(str(int(d)) for d in inst.planted)
        for p in parents:
            if not inst_mod.verify_witness(inst, [int(ch) for ch in p]):
                status, message = "InvariantViolation", "a root parent failed witness verification"
                break
            planted_found = planted_found or p == planted_str
        else:
            status = "Found"
    verify_ms = (time.perf_counter() - t0) * 1000.0
    return _append(out_path, _attempt_row(
        snapshot_label, status, message, n=n, seed=snap.seed, attempt=snap.attempt,
        attempt_seed=snap.attempt_seed, load_ms=load_ms, root_ms=root_ms, rebuild_ms=rebuild_ms,
        verify_ms=verify_ms, residue_exact=len(exact), structural_triples=len(accepted), parents=parents,
        planted_found=planted_found, device_name=_device_name(device),
        device_root_ms=res.telemetry.total_ms))


def _load(args) -> tuple[object, str, float]:
    t0 = time.perf_counter()
    if args.snapshot:
        snap = snapmod.load(args.snapshot)
        label = Path(args.snapshot).stem
    else:
        snap = _capture(args.n, args.seed, args.attempt, args.device)
        label = f"n{args.n}_s{args.seed:#x}_a{args.attempt}"
    return snap, label, (time.perf_counter() - t0) * 1000.0


def main(argv=None) -> int:
    p = argparse.ArgumentParser(prog="python -m tergpu.runs")
    sub = p.add_subparsers(dest="cmd", required=True)
    for name in ("whole-root", "solve-attempt"):
        s = sub.add_parser(name)
        s.add_argument("--snapshot", default="")
        s.add_argument("--n", type=int, default=0)
        s.add_argument("--seed", type=lambda v: int(v, 0), default=0)
        s.add_argument("--attempt", type=int, default=0)
        s.add_argument("--device", type=int, default=0)
        if name == "whole-root":
            s.add_argument("--out-dir", required=True)
            s.add_argument("--run", required=True)
            s.add_argument("--no-plant", action="store_true")
        else:
            s.add_argument("--out", required=True)
    args = p.parse_args(argv)
    if not args.snapshot and args.n == 0:
        print("usage: --snapshot=PATH or --n/--seed/--attempt", file=sys.stderr)
        return 2
    try:
        snap, label, load_ms = _load(args)
    except (OSError, snapmod.SnapshotError, RuntimeError) as e:
        print(f"# snapshot: {e}")
        if args.cmd == "solve-attempt":
            # recorded, as the reference records an unreadable or damaged snapshot
            # (ter_arwlf_solve.cpp:59-60; exit code 3)
            _append(args.out, _attempt_row(args.snapshot or f"n{args.n}", "InvalidConfiguration", str(e)))
        return 3
    if args.cmd == "whole-root":
        if '"' in args.run:
            print("usage: the run id may not contain a quote", file=sys.stderr)
            return 2
        code, _ = whole_root(snap, label, args.run, args.out_dir, args.device, load_ms,
                             plant=not args.no_plant)
        return code
    row = solve_attempt(snap, args.snapshot or label, args.out, args.device, load_ms)
    print(f"# {row['status']} ({row['unique_parents']} parents)")
    return 0 if row["status"] != "InvariantViolation" else 4


if __name__ == "__main__":
    sys.exit(main())
