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


def test_wide_quotient_root_uses_the_full_key():
    """The reference's Q = 69 truncation fixture (tests/full_ter_tests.cpp:805-838):
    both pairs agree on the low quotient window, the device's full 69-bit key
    keeps one; exactly one valid root under every policy and in the count."""
    from conftest import wide_quotient_capture
    from tergpu import report
    from tergpu.root import Config, run_gpu_root_records

    snap = wide_quotient_capture()
    res = run_gpu_root_records(snap, Config(projected_bits=32))
    assert res.tau == 0 and res.telemetry.logical_pairs == 2
    assert res.telemetry.projected_hits == 2
    assert res.triples.tolist() == [[0, 0, 0]]
    assert res.residue_exact == 1 and res.valid_roots == 1
    for policy in (report.RootOutputPolicy.FULL_CANONICAL_OUTPUT, report.RootOutputPolicy.FIRST_WITNESS):
        got = report.report_full_ter_root(snap, policy)
        assert got.status == 0 and got.valid_root_count == 1 and got.retained_root_count == 1
        assert got.parents[0].tolist() == [0] * 54 + [1] * 54
    count = report.count_full_ter_root(snap)
    assert count.status == 0 and count.valid_root_count == 1


def test_early_root_fixture_report_stops_and_counts():
    """The reference's deterministic root-report fixture
    (tests/full_ter_tests.cpp:423-485): FullCanonicalOutput counts the 64
    pre-dedup roots and retains the 2 distinct parents, FirstWitness counts and
    retains one, CountOnly counts 64."""
    from conftest import early_root_capture
    from tergpu import report

    snap = early_root_capture()
    canon = report.report_full_ter_root(snap, report.RootOutputPolicy.FULL_CANONICAL_OUTPUT)
    assert canon.status == 0 and canon.valid_root_count == 64 and canon.retained_root_count == 2
    first = report.report_full_ter_root(snap, report.RootOutputPolicy.FIRST_WITNESS)
    assert first.status == 0 and first.valid_root_count == 1 and first.retained_root_count == 1
    count = report.count_full_ter_root(snap)
    assert count.status == 0 and count.valid_root_count == 64
