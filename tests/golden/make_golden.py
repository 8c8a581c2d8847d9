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

import json
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


def seed_roots(tmp: Path):
    """The six published n=108 roots (benchmark instance, attempt 0): the
    reference's capture sizes and its frozen ARWLF over the declared 16-cell
    sample with 32-bit projected counts (about 3 minutes per seed, in parallel)."""
    from concurrent.futures import ThreadPoolExecutor

    def one(seed):
        snap = tmp / f"s108_{seed:x}.snap"
        cap = O.ref_run("capture", 108, seed, 0, "auth", snap, timeout=3600)[0]
        row = O.ref_run("snaproot", snap, "arwlf", 16, 32, timeout=3600)[0]
        snap.unlink()
        keep = ("triples", "triple_sum", "triple_xor", "triple_sum2", "residue", "residue_sum",
                "structural", "witnesses", "pairs", "projected_hits")
        return {"seed": seed, "level1": cap["level1"], "level2": cap["level2"],
                "arwlf16": {k: row[k] for k in keep}}

    seeds = [0x1001, 0x2003, 0x3007, 0x4001, 0x5003, 0x6007]
    with ThreadPoolExecutor(max_workers=6) as pool:
        return list(pool.map(one, seeds))


REFERENCE = Path("/root/reference")


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
    "published_runs": published_runs,
}


def main():
    """python tests/golden/make_golden.py [SECTION ...]: regenerates the named
    sections (all when none is named) and keeps the others as they are."""
    if not O.ref_available():
        raise SystemExit("oracle/_ref/terref missing: build it where the reference sources exist")
    wanted = sys.argv[1:] or list(SECTIONS)
    target = HERE / "reference_golden.json"
    golden = json.loads(target.read_text()) if target.exists() else {}
    with tempfile.TemporaryDirectory() as d:
        for name in wanted:
            golden[name] = SECTIONS[name](Path(d))
    target.write_text(json.dumps(golden, indent=1, sort_keys=True) + "\n")
    print("wrote", target, "sections", wanted)


if __name__ == "__main__":
    main()
