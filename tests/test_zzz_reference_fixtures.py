"""The reference's own test fixtures and solves on the device, against goldens
the reference printed or the numbers its tests assert: the solves of its guided
tests and of its failure-semantics test (every stage counter and fingerprint,
then a replay), its Q = 69 truncation fixture and its deterministic root-report
fixture (tests/full_ter_tests.cpp)."""
import numpy as np
import pytest

from conftest import STAGES, hexint

pytestmark = pytest.mark.gpu


GUIDED_CASES = 8  # golden guided_replay: the solves of the reference's guided tests


@pytest.mark.parametrize("case", range(GUIDED_CASES))
def test_guided_tests_match_reference(golden, case):
    """The solves of the reference's guided tests in tests/full_ter_tests.cpp
    (guided pipeline and replay, root output policies with their no-root run,
    the authentic L2 capture, the n=72 root over 47-bit quotients) on the
    device: their balanced instances with their config seeds, GuidedPlanted or
    random targets, FullTer or FixtureTer at level-3 limit 9, audited or under
    FirstWitness.  The reference's status and witness, every stage counter,
    stage fingerprint and the run fingerprint; a second identical call replays
    them exactly."""
    from tergpu import _abi, attempt, instance

    assert len(golden["guided_replay"]) == GUIDED_CASES
    g = golden["guided_replay"][case]
    inst = instance.benchmark_instance(g["n"], g["seed"])
    fixture = int(g["modes"].split("fixture=")[1]) if "fixture=" in g["modes"] else 0
    cfg = attempt.FullTerConfig(seed=g["config_seed"], attempt_limit=1, guided="guided" in g["modes"],
                                fixture_limit=fixture, audit=bool(g["audit"]), telemetry=True,
                                memory_limit_bytes=128 << 20)
    first = attempt.solve_full_ter(inst, cfg)
    final = g["final"]
    assert first.status == final["status"], (g["modes"], first.status_name, _abi.last_error())
    if first.status == _abi.FOUND:
        assert "".join(str(int(d)) for d in first.witness) == final["witness"]
        assert instance.verify_witness(inst, first.witness)
    else:
        assert first.witness is None
    assert first.fingerprint == hexint(final["fingerprint"]), (g["seed"], g["modes"], g["audit"])
    assert first.level3_size == final["l3"][0]
    (a,), (row,) = first.attempts, g["rows"]
    assert a["attempt_seed"] == row["seed"] and a["status"] == row["status"]
    assert a["level2"] == row["level2"] and a["level1"] == row["level1"] and a["level0"] == row["level0"]
    for stage, fields in STAGES.items():
        for ref_key, dev_key in fields.items():
            want = row[stage][ref_key]
            want = hexint(want) if ref_key == "fingerprint" else want
            assert a[dev_key] == want, (g["seed"], g["modes"], g["audit"], stage, ref_key, a[dev_key], want)
    # the nine L3 -> L2 merges always fit the audit's cap at these level-3 sizes
    assert a["audited_stages"] >= 9 if g["audit"] else a["audited_stages"] == 0
    second = attempt.solve_full_ter(inst, cfg)
    assert second.status == first.status and second.fingerprint == first.fingerprint
    if first.status == _abi.FOUND:
        assert np.array_equal(second.witness, first.witness)


def test_failure_semantics_run_matches_reference(golden):
    """The reference's failure-semantics run (tests/full_ter_tests.cpp:597-628):
    balanced n=36 instance (seed 17), config seed 3, FixtureTer with one level-3
    subset per half, random targets, two audited attempts.  Both attempts have
    empty level-1 lists and the budget is exhausted; every attempt's seed, stage
    counters and fingerprints and the run fingerprint equal the reference's, and
    a second call replays them."""
    from tergpu import _abi, attempt, instance

    g = next(c for c in golden["failure_semantics"] if c["name"] == "run")
    inst = instance.benchmark_instance(g["n"], g["seed"])
    cfg = attempt.FullTerConfig(seed=g["config_seed"], attempt_limit=g["attempts"],
                                fixture_limit=g["fixture_limit"], audit=bool(g["audit"]), telemetry=True,
                                memory_limit_bytes=16 << 20)
    res = attempt.solve_full_ter(inst, cfg)
    assert res.status == g["final"]["status"] == _abi.ATTEMPT_LIMIT_REACHED, _abi.last_error()
    assert res.fingerprint == hexint(g["final"]["fingerprint"])
    assert [a["attempt_seed"] for a in res.attempts] == [r["seed"] for r in g["rows"]] == [3, 4]
    for a, row in zip(res.attempts, g["rows"]):
        assert a["status"] == row["status"] and a["level2"] == row["level2"] and a["level1"] == row["level1"]
        for stage, fields in STAGES.items():
            for ref_key, dev_key in fields.items():
                want = row[stage][ref_key]
                want = hexint(want) if ref_key == "fingerprint" else want
                assert a[dev_key] == want, (row["attempt"], stage, ref_key, a[dev_key], want)
    again = attempt.solve_full_ter(inst, cfg)
    assert again.status == res.status and again.fingerprint == res.fingerprint


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


def test_boundary_roots_on_the_device():
    """The reporter's boundary cases (tests/tiled_q3report_tests.cpp:157-231),
    scaled to the device's key widths 24, 47, 64, 69 and 72: pair sums at 0,
    M - 1, M and 2M - 2 of M = 2^Q, and duplicated keys keeping multiplicity;
    every count equals exact integer arithmetic."""
    import tergpu
    from conftest import boundary_roots

    for Q, lo, hi, want in boundary_roots():
        res = tergpu.run_gpu_root(tergpu.RootKeys(quotient_bits=Q, lo=lo, hi=hi))
        assert len(res.triples) == want, (Q, [int(v[0]) for v in lo], len(res.triples), want)
