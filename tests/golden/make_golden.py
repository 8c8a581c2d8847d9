"""Regenerates tests/golden/ from the reference's own compiled code.

Run on a machine where oracle/_ref/terref was built from the reference sources
(python __graft_entry__.py, then python tests/golden/make_golden.py).  Every
number written here is printed by the reference itself (solve_full_ter,
capture_to_file, the frozen K2 / K2_WIDE / ARWLF backends, the synthetic-root
brute-force oracle of ter2_root/tests/ter_synthetic_root.hpp) or read from the
reference's own published run records (published_runs); nothing is typed in by
hand.
"""
from __future__ import annotations

import contextlib
import fcntl
import json
import os
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
import oracle as O  # noqa: E402

ANCHOR_SEED = 19797034556212562  # the reference's authentic n=72 anchor seed


def n36_attempts():
    out = []
    for kind in ("auth", "build"):
        for seed in (ANCHOR_SEED, 0x1001, 0x2A):
            rows = O.ref_run("solve", 36, seed, 8, kind, "canon", 0)
            out.append({"kind": kind, "seed": seed, "attempts": rows[:-1], "final": rows[-1]})
    return out


def synthetic_roots(tmp: Path):
    out = []
    # the configurations of ter2_root/tests/ter_arwlf_tests.cpp:302-307
    for bits, seed, size, pool in ((69, 0x1234, 2000, 0), (47, 0x5555, 2000, 0),
                                   (69, 0x9876, 600, 16), (47, 0x4242, 600, 16),
                                   (69, 0x3131, 600, 1), (47, 0x2727, 600, 1)):
        path = tmp / f"s{bits}_{seed:x}.keys"
        brute = O.ref_run("synth", bits, seed, size, pool, path)[0]
        arwlf = O.ref_run("keysroot", path, "arwlf", 4096, 1, 0)[0]
        sub = O.ref_run("keysroot", path, "arwlf", 700, 1, 0)[0]
        out.append({"bits": bits, "seed": seed, "size": size, "pool": pool, "sizes": brute["sizes"],
                    "brute": {k: brute[k] for k in ("triples", "triple_sum", "triple_xor", "triple_sum2")},
                    "arwlf": {k: arwlf[k] for k in ("triples", "triple_sum", "triple_xor", "triple_sum2",
                                                    "projected_hits", "projected_bits",
                                                    "logical_pairs")},
                    "subsample700": {k: sub[k] for k in ("triples", "triple_sum", "triple_xor",
                                                         "triple_sum2", "logical_pairs")}})
    return out


def n72_roots(tmp: Path):
    out = []
    for seed, attempt in ((ANCHOR_SEED, 0), (0x7201, 0), (0x7201, 21)):
        snap = tmp / f"n72_{seed:x}_{attempt}.snap"
        cap = O.ref_run("capture", 72, seed, attempt, "auth", snap)[0]
        row = {"seed": seed, "attempt": attempt, "level1": cap["level1"], "level2": cap["level2"],
               "file_bytes": cap["file_bytes"]}
        k2 = O.ref_run("snaproot", snap, "k2", 4096, 0)[0]
        wide = O.ref_run("snaproot", snap, "k2wide", 4096, 0)[0]
        a32 = O.ref_run("snaproot", snap, "arwlf", 4096, 32)[0]
        keep = ("triples", "triple_sum", "triple_xor", "triple_sum2", "full_q", "residue",
                "residue_sum", "structural", "witnesses", "pairs")
        row["k2"] = {k: k2[k] for k in keep}
        row["k2wide"] = {k: wide[k] for k in keep}
        row["k2wide"]["projected_hits_25"] = wide["projected_hits"]
        row["arwlf_k32_projected_hits"] = a32["projected_hits"]
        sub = O.ref_run("snaproot", snap, "k2wide", 512, 0)[0]
        row["k2wide_subsample512"] = {k: sub[k] for k in keep}
        out.append(row)
    return out


def n36_snapshot(tmp: Path):
    path = HERE / "n36_anchor_a0.snap"
    cap = O.ref_run("capture", 36, ANCHOR_SEED, 0, "auth", path)[0]
    return {"path": path.name, "level1": cap["level1"], "level2": cap["level2"],
            "file_bytes": cap["file_bytes"]}


def root_reports(tmp: Path):
    """report_full_ter_root / count_full_ter_root on captured roots, per policy."""
    sys.path.insert(0, str(HERE.parent.parent / "subset-sum-ter-fft_b200"))
    import numpy as np

    from tergpu import snapshot

    out = []
    sources = [("n36_anchor_a0", HERE / "n36_anchor_a0.snap", 36, ANCHOR_SEED, 0, None)]
    for n, seed, attempt in ((36, 358, 0), (72, ANCHOR_SEED, 0), (72, 0x7201, 21)):
        snap = tmp / f"r{n}_{seed:x}_{attempt}.snap"
        O.ref_run("capture", n, seed, attempt, "auth", snap)
        sources.append((f"n{n}_{seed:x}_{attempt}", snap, n, seed, attempt, None))
    # the positive n=72 root with the witness's list-0 record appended once more:
    # two accepted triples, one distinct parent (pre-dedup count vs retained roots)
    s = snapshot.load(tmp / "r72_7201_21.snap")
    rec = s.records[0].reshape(-1, s.record_bytes)
    s.records[0] = np.concatenate([rec, rec[2877:2878]]).reshape(-1)
    snapshot.save(s, tmp / "r72_7201_21_dup.snap", git_commit="reference")
    sources.append(("n72_7201_21_dup0_2877", tmp / "r72_7201_21_dup.snap", 72, 0x7201, 21,
                    {"list": 0, "record": 2877}))
    for name, path, n, seed, attempt, dup in sources:
        row = {"name": name, "n": n, "seed": seed, "attempt": attempt, "duplicate": dup}
        for policy in ("first", "count", "canon"):
            r = O.ref_run("report", path, policy)[0]
            row[policy] = {k: r[k] for k in ("status", "valid_root_count", "retained_root_count",
                                             "count_valid_root_count")}
        out.append(row)
    return out


def whole_root_plants(tmp: Path):
    """The whole-root runner's positive construction (one planted final output,
    seed 0xB1A57001, on the anchor microproblem) on authentic roots: the planted
    D keys and the expected outputs, as the reference computes them.  The n=108
    root is the published 0x1001 attempt-0 capture (about 150 s to capture)."""
    out = []
    for n, seed in ((72, ANCHOR_SEED), (108, 0x1001)):
        snap = tmp / f"w{n}_{seed:x}.snap"
        O.ref_run("capture", n, seed, 0, "auth", snap, timeout=1800)
        p = O.ref_run("plant", snap, 1, 0xB1A57001, timeout=1800)[0]
        out.append({"n": n, "seed": seed, "attempt": 0, "plant_seed": 0xB1A57001,
                    "anchor_cell": p["anchor_cell"], "first_planted": p["first_planted"],
                    "d_lo": [int(v) for v in p["d_lo"]], "d_hi": p["d_hi"],
                    "expected": p["expected"]})
    return out


# Config-3 seeds at n=108: the six published roots (results/arwlf/holdout-snapshots)
# and 26 fresh ones, 0x108001 .. 0x10801a.
PUBLISHED_SEEDS_108 = [0x1001, 0x2003, 0x3007, 0x4001, 0x5003, 0x6007]
FRESH_SEEDS_108 = [0x108000 + k for k in range(1, 27)]
# Unplanted roots the reference's frozen ARWLF runs over all 4096 cells.
WHOLE_ROOT_SEEDS_108 = [0x2003, 0x3007]
WHOLE_ROOT_SLICES = 8
JOBS = int(os.environ.get("TERGPU_GOLDEN_JOBS", max(1, min(7, (os.cpu_count() or 2) - 1))))

_DIGEST_KEEP = ("triples", "triple_sum", "triple_xor", "triple_sum2", "full_q", "residue",
                "residue_sum", "structural", "witnesses", "pairs", "projected_hits")


def _snap_checksums(path: Path) -> list:
    """The three per-list FNV-1a-64 checksums the reference wrote into its
    .snap header (ter2_root/frozen/ter_root_snapshot.cpp:94-101)."""
    sys.path.insert(0, str(HERE.parent.parent / "subset-sum-ter-fft_b200"))
    import numpy as np

    from tergpu import snapshot

    head = np.fromfile(path, dtype=snapshot.HEADER_DTYPE, count=1)[0]
    return [f"0x{int(c):016x}" for c in head["checksum"]]


def _capture_108(tmp: Path, seed: int) -> tuple[Path, dict]:
    snap = tmp / f"s108_{seed:x}.snap"
    cap = O.ref_run("capture", 108, seed, 0, "auth", snap, timeout=3600)[0]
    return snap, cap


@contextlib.contextmanager
def _golden_update():
    """Read-modify-write of the golden file under an exclusive lock: the long
    sections write every finished item at once (several generator processes may
    run side by side), so an interrupted run resumes where it stopped."""
    target = HERE / "reference_golden.json"
    with open(target, "r+") as f:
        fcntl.flock(f, fcntl.LOCK_EX)
        golden = json.loads(f.read())
        yield golden
        f.seek(0)
        f.write(json.dumps(golden, indent=1, sort_keys=True) + "\n")
        f.truncate()


def seed_roots(tmp: Path):
    """Config 3's 32 n=108 roots (benchmark instance, attempt 0): per seed the
    reference's capture sizes, the three L1 list checksums of its .snap header
    and its frozen ARWLF over the declared 16-cell sample with 32-bit projected
    counts (about 17 minutes of one core per seed; seeds run in parallel).  Each
    finished seed is written at once; seeds already written are skipped."""
    from concurrent.futures import ThreadPoolExecutor

    order = PUBLISHED_SEEDS_108 + FRESH_SEEDS_108
    with _golden_update() as g:
        done = {r["seed"] for r in g.get("seed_roots", []) if "checksums" in r}

    def one(seed):
        snap, cap = _capture_108(tmp, seed)
        row = O.ref_run("snaproot", snap, "arwlf", 16, 32, timeout=3600)[0]
        sums = _snap_checksums(snap)
        snap.unlink()
        new = {"seed": seed, "published": seed in PUBLISHED_SEEDS_108, "level1": cap["level1"],
               "level2": cap["level2"], "file_bytes": cap["file_bytes"], "checksums": sums,
               "arwlf16": {k: row[k] for k in _DIGEST_KEEP}}
        with _golden_update() as g:
            rows = [r for r in g.get("seed_roots", []) if r["seed"] != seed] + [new]
            rows.sort(key=lambda r: order.index(r["seed"]) if r["seed"] in order else len(order))
            g["seed_roots"] = rows
        print("seed_roots: wrote seed", hex(seed), flush=True)

    with ThreadPoolExecutor(max_workers=JOBS) as pool:
        list(pool.map(one, [s for s in order if s not in done]))


def merge_digests(rows: list) -> dict:
    """Sink digests of disjoint cell slices combine field by field: counts and
    multiset sums add (mod 2^64), the xor hash xors, witnesses concatenate
    (RootSink::emit_triple, ter2_root/frozen/ter_root_queue_kernels.cpp:165-195)."""
    out = {"triples": 0, "full_q": 0, "residue": 0, "structural": 0, "pairs": 0,
           "projected_hits": 0, "cells": 0, "witnesses": []}
    sums = {"triple_sum": 0, "triple_sum2": 0, "residue_sum": 0}
    xor = 0
    for r in rows:
        for k in ("triples", "full_q", "residue", "structural", "pairs", "projected_hits", "cells"):
            out[k] += int(r[k])
        for k in sums:
            sums[k] = (sums[k] + int(r[k], 16)) % (1 << 64)
        xor ^= int(r["triple_xor"], 16)
        out["witnesses"] += r["witnesses"]
    out["witnesses"].sort()
    for k, v in sums.items():
        out[k] = f"0x{v:016x}"
    out["triple_xor"] = f"0x{xor:016x}"
    return out


_SLICE_KEEP = ("triples", "triple_sum", "triple_xor", "triple_sum2", "full_q", "residue",
               "residue_sum", "structural", "witnesses", "pairs", "projected_hits", "cells",
               "projected_bits", "ms")


def whole_roots(tmp: Path):
    """The reference's frozen ARWLF over every cell of unplanted n=108 roots
    (seeds WHOLE_ROOT_SEEDS_108, attempt 0) at its default projection (its
    check bits give 51-bit projected counts; 32-bit counts cost about 40 s per
    cell, so they are taken on the 16-cell samples of seed_roots): each root
    runs as WHOLE_ROOT_SLICES disjoint cell slices in parallel processes (about
    4 hours of one core per root), merged with merge_digests once all its slices
    are in.  Each finished slice is written at once; slices already written are
    skipped."""
    from concurrent.futures import ThreadPoolExecutor

    with _golden_update() as g:
        have = {e["seed"]: set(e.get("slice_rows", {})) for e in g.get("whole_roots", [])}
    todo = {seed: [i for i in range(WHOLE_ROOT_SLICES) if str(i) not in have.get(seed, set())]
            for seed in WHOLE_ROOT_SEEDS_108}
    todo = {seed: slices for seed, slices in todo.items() if slices}
    if not todo:
        return
    with ThreadPoolExecutor(max_workers=JOBS) as pool:
        captures = dict(zip(todo, pool.map(lambda seed: _capture_108(tmp, seed), todo)))

        def one(job):
            seed, i = job
            snap, cap = captures[seed]
            row = O.ref_run("snaproot", snap, "arwlf", f"mod:{WHOLE_ROOT_SLICES}:{i}:4096", 0,
                            timeout=8 * 3600)[0]
            with _golden_update() as g:
                entries = g.setdefault("whole_roots", [])
                entry = next((e for e in entries if e["seed"] == seed), None)
                if entry is None:
                    entry = {"seed": seed, "attempt": 0, "level1": cap["level1"],
                             "checksums": _snap_checksums(snap), "slices": WHOLE_ROOT_SLICES,
                             "slice_rows": {}}
                    entries.append(entry)
                    entries.sort(key=lambda e: WHOLE_ROOT_SEEDS_108.index(e["seed"]))
                entry["slice_rows"][str(i)] = {k: row[k] for k in _SLICE_KEEP}
                if len(entry["slice_rows"]) == WHOLE_ROOT_SLICES:
                    part = [entry["slice_rows"][str(k)] for k in range(WHOLE_ROOT_SLICES)]
                    entry["projected_bits"] = part[0]["projected_bits"]
                    entry["arwlf"] = merge_digests(part)
            print("whole_roots: wrote seed", hex(seed), "slice", i, flush=True)

        list(pool.map(one, [(seed, i) for seed, slices in todo.items() for i in slices]))
    for snap, _ in captures.values():
        snap.unlink()


def attempt_telemetry(tmp: Path):
    """solve_full_ter's per-attempt telemetry (every stage counter and output
    fingerprint) and the run fingerprint, under FirstWitness (the reference's
    default) and FullCanonicalOutput, for the n=36 cases of both generators and
    the n=72 authentic roots: the anchor's attempt 0 and the 0x7201 solve that is
    Found at attempt 21 (its root counters stop at the first witness)."""
    out = []
    cases = [(36, kind, seed, 8) for kind in ("auth", "build") for seed in (ANCHOR_SEED, 0x1001, 0x2A)]
    cases += [(72, "auth", ANCHOR_SEED, 1), (72, "auth", 0x7201, 22)]
    for n, kind, seed, attempts in cases:
        for policy in ("first", "canon"):
            rows = O.ref_run("solve", n, seed, attempts, kind, policy, 0, timeout=1800)
            out.append({"n": n, "kind": kind, "seed": seed, "attempts": attempts, "policy": policy,
                        "rows": rows[:-1], "final": rows[-1]})
    return out


# (n, instance seed, config seed, modes, policy, audit): the solves of the
# reference's guided tests in tests/full_ter_tests.cpp, at its default root
# prefilter (the device has no prefilter or tile-width knob)
GUIDED_CASES = [
    # test_guided_pipeline_and_replay (:236-350): FullTer and FixtureTer 9, audited
    (36, 0x544552F, 91, "guided", "first", 1),
    (36, 0x544552F, 91, "guided,fixture=9", "first", 1),
    (36, 0x544552F, 91, "guided", "first", 0),
    # test_phase5_root_output_policies (:352-421): audited, FirstWitness, and the
    # deterministic no-root run under random targets
    (36, 0x5048415345355445, 0x5048415345355345, "guided,fixture=9", "first", 1),
    (36, 0x5048415345355445, 0x5048415345355345, "guided,fixture=9", "first", 0),
    (36, 0x5048415345355445, 0x4E4F524F4F543535, "fixture=9", "first", 0),
    # test_authentic_l2_capture_tiled_merge_matches_exact_authorities (:497-527)
    (36, 0x54494C4544434150, 0x4C324C31, "guided", "first", 1),
    # test_m2_root_uses_complete_47_bit_quotients (:562-595): the n=72 root reads
    # quotient bits above 63
    (72, 0x4d32524f4f543732, 0x373242495453, "guided,fixture=9", "first", 1),
]


def guided_replay(tmp: Path):
    """The solves of the reference's guided tests (GUIDED_CASES) on their
    balanced instances (the benchmark instance): every stage's telemetry, the
    run fingerprint, the status and the witness, from the reference's own
    solve_full_ter."""
    out = []
    for n, seed, config_seed, modes, policy, audit in GUIDED_CASES:
        rows = O.ref_run("solve", n, seed, 1, "auth", policy, audit, config_seed, modes)
        out.append({"n": n, "seed": seed, "config_seed": config_seed, "modes": modes, "policy": policy,
                    "audit": audit, "rows": rows[:-1], "final": rows[-1]})
    return out


def failure_semantics(tmp: Path):
    """The solves of the reference's failure-semantics test
    (tests/full_ter_tests.cpp:597-668): its balanced n=36 instance (seed 17),
    config seed 3, FixtureTer with level-3 limit 1, random targets, two
    attempts, the default (audited) config; the same run with its cancellation
    flag set before the call; and an empty attempt budget."""
    out = []
    for name, attempts, modes in (("run", 2, "fixture=1"), ("pre_cancelled", 2, "fixture=1,cancelled"),
                                  ("no_attempts", 0, "fixture=1")):
        rows = O.ref_run("solve", 36, 17, attempts, "auth", "first", 1, 3, modes)
        out.append({"name": name, "n": 36, "seed": 17, "config_seed": 3, "attempts": attempts,
                    "fixture_limit": 1, "audit": 1, "rows": rows[:-1], "final": rows[-1]})
    return out


def full_bench_rows(tmp: Path):
    """The reference's own ter_full_bench (bench/ter_full_bench.cpp, built from its
    sources into oracle/_ref/ter_full_bench): its CSV header and row for the
    device command line to reproduce, with random and with guided (planted-root)
    targets, complete (FullTer) and truncated (FixtureTer) level-3 lists."""
    import subprocess

    binary = HERE.parent.parent / "oracle" / "_ref" / "ter_full_bench"
    out = []
    for n, seed, limit, extra in ((36, ANCHOR_SEED, 8, []), (36, 0x1001, 8, []), (36, 0x2A, 8, []),
                                  (72, ANCHOR_SEED, 1, []), (72, 0x7201, 22, []),
                                  (36, ANCHOR_SEED, 2, ["--guided"]), (72, ANCHOR_SEED, 1, ["--guided"]),
                                  (36, ANCHOR_SEED, 2, ["--fixture"]),
                                  (72, ANCHOR_SEED, 2, ["--fixture", "--fixture-limit=200"]),
                                  (72, ANCHOR_SEED, 2, ["--fixture", "--fixture-limit=100", "--guided"]),
                                  (108, 0x1001, 2, ["--fixture", "--fixture-limit=1500"]),
                                  (108, 0x1001, 2, ["--fixture", "--fixture-limit=600", "--guided"])):
        args = [f"--n={n}", f"--seed={seed}", f"--attempt-limit={limit}", "--warmup=0", "--repeat=1", *extra]
        proc = subprocess.run([str(binary), *args], capture_output=True, text=True, timeout=1800)
        if proc.returncode != 0:
            raise RuntimeError(f"ter_full_bench {args} failed: {proc.stderr}")
        lines = [l for l in proc.stdout.splitlines() if l and not l.startswith("#")]
        out.append({"args": args, "header": lines[0], "row": lines[1]})
    return out


def preflight_text(tmp: Path):
    """The reference's own ter_full_bench --preflight output (geometry,
    representation counts, decisions) at n = 36, 72, 108 and a large ceiling,
    FixtureTer at n = 72, and the refused n = 48."""
    import subprocess

    binary = HERE.parent.parent / "oracle" / "_ref" / "ter_full_bench"
    out = []
    for args in (["--n=36"], ["--n=72"], ["--n=108"], ["--n=72", "--fixture"], ["--n=48"]):
        args = ["--preflight", *args, "--memory-limit-mib=1000000"]
        proc = subprocess.run([str(binary), *args], capture_output=True, text=True, timeout=600)
        out.append({"args": args, "rc": proc.returncode, "lines": proc.stdout.splitlines()})
    return out


REFERENCE = Path(os.environ.get("TER_REFERENCE_DIR", "/root/reference"))


def published_runs(tmp: Path):
    """The reference's own published run records, read from its results tree:
    the whole-root ARWLF row of the n=108 seed 0x1001 root with its planted
    output (results/arwlf/whole-root-20261003/runs.jsonl) and the per-attempt
    rows of the n=72 seed 0x7201 full solve
    (results/arwlf/full-solve-n72-s0x7201-arwlf/attempts.jsonl)."""
    keep_run = ("root", "n", "root_seed", "Q", "W", "anchor_cell", "plant_seed", "first_planted",
                "planted", "cells", "logical_pairs", "residue_exact", "structural", "full_q",
                "residue_sum", "witnesses", "planted_ok", "status")
    runs = [json.loads(line) for line in
            (REFERENCE / "results/arwlf/whole-root-20261003/runs.jsonl").read_text().splitlines() if line]
    arwlf = [r for r in runs if r["backend"] == "arwlf"][0]
    keep_att = ("status", "n", "seed", "attempt", "attempt_seed", "residue_exact", "structural_triples",
                "unique_parents", "planted_found", "parents")
    atts = [json.loads(line) for line in
            (REFERENCE / "results/arwlf/full-solve-n72-s0x7201-arwlf/attempts.jsonl").read_text().splitlines()
            if line]
    return {"whole_root_n108": {k: arwlf[k] for k in keep_run},
            "solve_n72_s0x7201": sorted(({k: a[k] for k in keep_att} for a in atts),
                                        key=lambda a: a["attempt"])}


SECTIONS = {
    "n36_attempts": lambda tmp: n36_attempts(),
    "n36_snapshot": n36_snapshot,
    "synthetic_roots": synthetic_roots,
    "n72_roots": n72_roots,
    "root_reports": root_reports,
    "whole_root_plants": whole_root_plants,
    "seed_roots": seed_roots,
    "whole_roots": whole_roots,
    "attempt_telemetry": attempt_telemetry,
    "guided_replay": guided_replay,
    "failure_semantics": failure_semantics,
    "full_bench_rows": full_bench_rows,
    "preflight_text": preflight_text,
    "published_runs": published_runs,
}


def main():
    """python tests/golden/make_golden.py [SECTION ...]: regenerates the named
    sections (all when none is named) and keeps the others as they are."""
    if not O.ref_available():
        raise SystemExit("oracle/_ref/terref missing: build it where the reference sources exist")
    wanted = sys.argv[1:] or list(SECTIONS)
    target = HERE / "reference_golden.json"
    # TERGPU_GOLDEN_TMP: where captures (0.84 GB each at n=108) are written
    with tempfile.TemporaryDirectory(dir=os.environ.get("TERGPU_GOLDEN_TMP")) as d:
        for name in wanted:
            section = SECTIONS[name](Path(d))
            if section is None:  # written item by item
                print("complete", target, "section", name, flush=True)
                continue
            with _golden_update() as golden:
                golden[name] = section
            print("wrote", target, "section", name, flush=True)


if __name__ == "__main__":
    main()
