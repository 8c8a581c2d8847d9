"""Run records from the device root against the reference's published rows.

The reference's whole-root run of the n=108 seed 0x1001 root (ARWLF, one
planted final output on the anchor microproblem) and its per-attempt solve rows
of the n=72 seed 0x7201 instance are golden (published_runs, read from the
reference's results tree).  Here the device attempt pipeline captures the same
roots, tergpu.runs plants and runs them, and every exactness field of the rows
must equal the published ones: the planted output, the residue-exact,
structural and full-Q counts, the residue multiset hash, the logical pairs, and
per attempt the status, counts and rebuilt parents.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

PKG = Path(__file__).resolve().parent.parent / "subset-sum-ter-fft_b200"
RUN_FIELDS = ("root", "n", "root_seed", "Q", "W", "anchor_cell", "plant_seed", "first_planted",
              "planted", "cells", "logical_pairs", "residue_exact", "structural", "full_q",
              "residue_sum", "witnesses", "planted_ok", "status")


def test_whole_root_n108_row_matches_published(golden, tmp_path):
    from tergpu import runs

    pub = golden["published_runs"]["whole_root_n108"]
    snap = runs._capture(108, 0x1001, 0, 0)
    code, row = runs.whole_root(snap, pub["root"], "gpu-1", tmp_path)
    assert code == 0
    for k in RUN_FIELDS:
        assert row[k] == pub[k], k
    # a finished run id is not run again
    assert runs.whole_root(snap, pub["root"], "gpu-1", tmp_path) == (0, None)
    assert len((tmp_path / "runs.jsonl").read_text().splitlines()) == 1


def test_solve_attempt_rows_match_published_n72_full_solve(golden, tmp_path):
    from tergpu import runs

    out = tmp_path / "attempts.jsonl"
    for pub in golden["published_runs"]["solve_n72_s0x7201"]:
        snap = runs._capture(72, pub["seed"], pub["attempt"], 0)
        row = runs.solve_attempt(snap, f"attempt_{pub['attempt']}", out)
        for k in pub:
            assert row[k] == pub[k], (pub["attempt"], k)
    assert len(out.read_text().splitlines()) == len(golden["published_runs"]["solve_n72_s0x7201"])


def test_whole_root_cli_on_the_n72_anchor(golden, tmp_path):
    g = golden["whole_root_plants"][0]
    env = dict(os.environ, PYTHONPATH=str(PKG) + os.pathsep + os.environ.get("PYTHONPATH", ""))
    cmd = [sys.executable, "-m", "tergpu.runs", "whole-root", "--n=72", f"--seed={g['seed']}",
           "--attempt=0", f"--out-dir={tmp_path}", "--run=gpu-cli"]
    first = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    assert first.returncode == 0, first.stdout + first.stderr
    rows = [json.loads(line) for line in (tmp_path / "runs.jsonl").read_text().splitlines()]
    assert len(rows) == 1
    row = rows[0]
    assert row["status"] == "COMPLETED" and row["backend"] == "gpu"
    assert row["witnesses"] == row["planted"] == g["expected"]
    assert row["residue_exact"] == row["structural"] == 1
    assert row["anchor_cell"] == g["anchor_cell"] and row["first_planted"] == g["first_planted"]
    again = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    assert again.returncode == 0 and "already complete" in again.stdout
    assert len((tmp_path / "runs.jsonl").read_text().splitlines()) == 1
