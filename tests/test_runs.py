"""Run records (tergpu.runs) on the CPU: the reference's anchor sample, its
positive planting against the reference's own plant of the n=72 anchor root
(golden whole_root_plants, printed by the reference harness), and the
whole-root runner's resume / refuse rules, which act before any device work."""
import json

import numpy as np

from conftest import GOLDEN_DIR

ANCHOR_SEED = 19797034556212562


def _n72_anchor_snapshot(att):
    from tergpu import snapshot

    l1 = att["l1"]
    recs = []
    for g in range(3):
        pos = np.stack([l1["pos0"][g], l1["pos1"][g]], axis=1)
        neg = np.stack([l1["neg0"][g], l1["neg1"][g]], axis=1)
        res = np.stack([l1["res_lo"][g] & np.uint64(0xFFFFFFFF), l1["res_lo"][g] >> np.uint64(32),
                        l1["res_hi"][g] & np.uint64(0xFFFFFFFF)], axis=1).astype("<u4")
        rec = np.concatenate([pos.astype("<u8").view(np.uint8), neg.astype("<u8").view(np.uint8),
                              res.view(np.uint8)], axis=1)
        recs.append(np.ascontiguousarray(rec).reshape(-1))

    def words(v):
        return np.array([(v >> (32 * k)) & 0xFFFFFFFF for k in range(3)], dtype=np.uint32)

    return snapshot.Snapshot(n=72, r1=att["r1"], r2=att["r2"], attempt=0, seed=ANCHOR_SEED,
                             attempt_seed=ANCHOR_SEED, records=recs,
                             child_targets=[words(t) for t in att["t1"]],
                             root_target=words(att["root_target"]), level2_sizes=att["level2"])


def test_anchor_sample_and_hashes(oracle_mod, golden):
    from tergpu import runs, workload

    assert runs.anchor_cell() == golden["whole_root_plants"][0]["anchor_cell"] == 2730
    assert (runs.select_cells(16) == oracle_mod.select_cells(16)).all()
    vals = np.array([0, 1, 0x5EED5EED, 2**64 - 1], dtype=np.uint64)
    assert [runs.mix64(int(v)) for v in vals] == [int(x) for x in workload.mix64(vals)]


def test_plant_matches_reference_on_n72_anchor_root(n72_anchor_attempt, golden):
    from tergpu import runs, snapshot

    g = golden["whole_root_plants"][0]
    assert g["n"] == 72 and g["seed"] == ANCHOR_SEED
    snap = _n72_anchor_snapshot(n72_anchor_attempt)
    assert snap.entries == [19109, 32496, 33505]
    p = runs.plant_positive(snap, runs.anchor_cell())
    assert p.first_planted == g["first_planted"]
    assert p.expected == g["expected"]
    assert p.d_lo == g["d_lo"] and p.d_hi == g["d_hi"]
    # the planted record derives exactly the planted key and completes the pair
    _, lo, hi, _ = snapshot.root_keys(p.snapshot)
    assert int(lo[2][p.first_planted]) == g["d_lo"][0] and int(hi[2][p.first_planted]) == g["d_hi"][0]
    a, b, c = p.expected[0]
    nmask = (1 << 72) - 1
    res = [snapshot.words_to_int(p.snapshot.residues(l)[e]) for l, e in enumerate((a, b, c))]
    root = snapshot.words_to_int(snap.root_target) & nmask
    assert (res[0] + res[1] + res[2]) & nmask == root
    digits = sum(runs._digits(p.snapshot, l, e).astype(int) for l, e in enumerate((a, b, c)))
    neg, zero, pos = runs.structural_parent_counts(72)
    assert set(digits.tolist()) <= {-1, 0, 1}
    assert ((digits == -1).sum(), (digits == 0).sum(), (digits == 1).sum()) == (neg, zero, pos)


def test_whole_root_resume_and_refusal(tmp_path):
    from tergpu import runs

    rows = [{"run_id": "gpu-1", "chunk": "all", "backend": "gpu", "status": "COMPLETED", "root": "r1"},
            {"run_id": "k2-1", "chunk": "all", "backend": "k2", "status": "COMPLETED", "root": "r1"}]
    (tmp_path / "runs.jsonl").write_text("".join(json.dumps(r) + "\n" for r in rows))
    # a finished run id is not rerun; one recorded with another backend or root is refused
    assert runs.whole_root(None, "r1", "gpu-1", tmp_path) == (0, None)
    assert runs.whole_root(None, "r1", "k2-1", tmp_path) == (2, None)
    assert runs.whole_root(None, "r2", "gpu-1", tmp_path) == (2, None)
    assert len((tmp_path / "runs.jsonl").read_text().splitlines()) == 2


def test_cli_usage_errors(tmp_path):
    import os
    import subprocess
    import sys
    from pathlib import Path

    pkg = Path(__file__).resolve().parent.parent / "subset-sum-ter-fft_b200"
    env = dict(os.environ, PYTHONPATH=str(pkg))
    # neither a snapshot nor an instance to capture: usage, exit 2, nothing written
    r = subprocess.run([sys.executable, "-m", "tergpu.runs", "whole-root", f"--out-dir={tmp_path}",
                        "--run=x"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and not (tmp_path / "runs.jsonl").exists()
    # an unreadable snapshot: recorded InvalidConfiguration, exit 3, as the reference's
    r = subprocess.run([sys.executable, "-m", "tergpu.runs", "solve-attempt",
                        f"--snapshot={tmp_path / 'missing.snap'}", f"--out={tmp_path / 'a.jsonl'}"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 3
    rows = (tmp_path / "a.jsonl").read_text().splitlines()
    assert len(rows) == 1 and json.loads(rows[0])["status"] == "InvalidConfiguration"


def test_solve_attempt_refusals_are_recorded(tmp_path, golden):
    """ter_arwlf_solve_attempt's refusals (ter2_root/tests/ter_arwlf_solve_tests.cpp:66-97),
    recorded without device work: the n=36 root (Q = 24, below the 25-bit
    projection) is NotApplicable with no parents and exit 0; a missing and a
    damaged snapshot are InvalidConfiguration rows with no parents and exit 3."""
    from tergpu import runs

    out = tmp_path / "attempts.jsonl"
    snap = GOLDEN_DIR / golden["n36_snapshot"]["path"]
    assert runs.main(["solve-attempt", f"--snapshot={snap}", f"--out={out}"]) == 0
    assert runs.main(["solve-attempt", f"--snapshot={tmp_path / 'missing.snap'}", f"--out={out}"]) == 3
    damaged = tmp_path / "damaged.snap"
    raw = bytearray(snap.read_bytes())
    raw[-3] ^= 0x10
    damaged.write_bytes(bytes(raw))
    assert runs.main(["solve-attempt", f"--snapshot={damaged}", f"--out={out}"]) == 3
    rows = [json.loads(line) for line in out.read_text().splitlines()]
    assert [r["status"] for r in rows] == ["NotApplicable", "InvalidConfiguration", "InvalidConfiguration"]
    assert rows[0]["message"] == "quotient width Q=24 is below the 25-bit projection"
    assert rows[0]["n"] == 36 and rows[0]["root_ms"] == 0.0
    for r in rows:
        assert r["parents"] == [] and r["unique_parents"] == 0 and r["backend"] == "gpu"


def test_whole_root_below_the_projection_is_refused(tmp_path, golden):
    """The whole-root runner on the n=36 root (Q = 24): the reference's loader
    refuses it, so the run exits 3 and records no row
    (ter2_root/campaign/ter_arwlf_whole_root_main.cpp:234-240), with no device work."""
    from tergpu import runs

    snap = GOLDEN_DIR / golden["n36_snapshot"]["path"]
    code = runs.main(["whole-root", f"--snapshot={snap}", f"--out-dir={tmp_path}", "--run=n36"])
    assert code == 3 and not (tmp_path / "runs.jsonl").exists()
