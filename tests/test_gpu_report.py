"""report_full_ter_root / count_full_ter_root on the device against the
reference's own report on the same captures (golden root_reports): the
pre-dedup accepted count and the retained parents under each output policy,
including a capture with a duplicated child record (two accepted triples, one
distinct parent)."""
import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu

POLICIES = {"first": 0, "count": 1, "canon": 2}


def _capture(row):
    from tergpu import attempt, instance, snapshot

    if row["name"] == "n36_anchor_a0":
        return snapshot.load(GOLDEN_DIR / "n36_anchor_a0.snap"), None
    inst = instance.benchmark_instance(row["n"], row["seed"])
    cfg = attempt.FullTerConfig(seed=row["seed"], attempt_first=row["attempt"], attempt_limit=1,
                                capture_only=True, export_l1_capacity=1 << 20)
    snap = attempt.solve_full_ter(inst, cfg).snapshot
    dup = row.get("duplicate")
    if dup is not None:
        rec = snap.records[dup["list"]].reshape(-1, snap.record_bytes)
        snap.records[dup["list"]] = np.concatenate([rec, rec[dup["record"]:dup["record"] + 1]]).reshape(-1)
    return snap, inst


@pytest.mark.parametrize("index", range(5))
def test_root_report_matches_reference(golden, index):
    from tergpu import instance as I
    from tergpu import report

    row = golden["root_reports"][index]
    snap, inst = _capture(row)
    for name, policy in POLICIES.items():
        got = report.report_full_ter_root(snap, policy)
        want = row[name]
        assert got.status == want["status"] == 0
        assert int(got.effective_root_output_policy) == policy
        assert got.valid_root_count == want["valid_root_count"], name
        assert got.retained_root_count == want["retained_root_count"], name
        for parent in got.parents:
            assert inst is not None and I.verify_witness(inst, parent)
    count = report.count_full_ter_root(snap)
    assert count.status == 0
    assert count.valid_root_count == row["count"]["count_valid_root_count"]


def test_root_report_resource_limit():
    from tergpu import report, snapshot
    from tergpu.root import Config

    snap = snapshot.load(GOLDEN_DIR / "n36_anchor_a0.snap")
    got = report.report_full_ter_root(snap, report.RootOutputPolicy.COUNT_ONLY,
                                      Config(memory_limit_bytes=1024))
    assert got.status == 7 and got.valid_root_count == 0  # ResourceLimit, nothing counted

