"""Full TER attempts on the device against the reference: level cardinalities,
candidate counts, statuses, witnesses, and byte-identical L1 lists."""
import ctypes

import numpy as np
import pytest

from conftest import GOLDEN_DIR, STAGES, hexint

pytestmark = pytest.mark.gpu

ANCHOR_SEED = 19797034556212562


def _attempt(n, seed, first, count, kind="auth", **kw):
    from tergpu import attempt, instance

    inst = instance.benchmark_instance(n, seed) if kind == "auth" else instance.build_instance(n, seed)
    cfg = attempt.FullTerConfig(seed=seed, attempt_first=first, attempt_limit=count, **kw)
    return inst, attempt.solve_full_ter(inst, cfg)


@pytest.mark.parametrize("case", range(6))
def test_n36_attempts_match_reference(golden, case):
    from tergpu import _abi, instance

    g = golden["n36_attempts"][case]  # solve_full_ter with FullCanonicalOutput
    for row in g["attempts"]:
        inst, res = _attempt(36, g["seed"], row["attempt"], 1, kind=g["kind"],
                             root_policy=_abi.ROOT_POLICY_FULL_CANONICAL)
        assert (res.r1, res.r2) == (g["final"]["r1"], g["final"]["r2"])
        a = res.attempts[0]
        for key in ("level2", "level1", "level0", "l3_modular", "l2_modular"):
            assert a[key] == row[key], (g["kind"], g["seed"], row["attempt"], key)
        assert a["root_modular"] == row["root_modular"]
        assert a["valid_roots"] == row["valid_roots"]
        if row["status"] == 1:
            assert res.status == _abi.FOUND and instance.verify_witness(inst, res.witness)
        else:
            assert res.status == _abi.ATTEMPT_LIMIT_REACHED


@pytest.mark.parametrize("case", range(16))
def test_attempt_telemetry_matches_reference(golden, case):
    """Every stage counter, every stage output fingerprint and the run fingerprint
    of solve_full_ter, under FirstWitness and FullCanonicalOutput, on both
    instance generators at n=36 and on the n=72 authentic roots (0x7201 is Found
    at attempt 21: FirstWitness stops its root counters at the reference's first
    witness in the tiled visit order)."""
    from tergpu import _abi

    g = golden["attempt_telemetry"][case]
    policy = (_abi.ROOT_POLICY_FIRST_WITNESS if g["policy"] == "first"
              else _abi.ROOT_POLICY_FULL_CANONICAL)
    _, res = _attempt(g["n"], g["seed"], 0, g["attempts"], kind=g["kind"], root_policy=policy,
                      telemetry=True, memory_limit_bytes=64 << 30)
    final = g["final"]
    assert res.status == final["status"]
    assert res.fingerprint == hexint(final["fingerprint"]), (g["n"], g["kind"], g["seed"], g["policy"])
    assert len(res.attempts) == len(g["rows"])
    if res.status == _abi.FOUND:
        assert "".join(str(int(d)) for d in res.witness) == final["witness"]
    for a, row in zip(res.attempts, g["rows"]):
        assert a["attempt_seed"] == row["seed"] and a["status"] == row["status"]
        assert a["level2"] == row["level2"] and a["level1"] == row["level1"]
        assert a["level0"] == row["level0"]
        for stage, fields in STAGES.items():
            for ref_key, dev_key in fields.items():
                want = row[stage][ref_key]
                want = hexint(want) if ref_key == "fingerprint" else want
                assert a[dev_key] == want, (g["kind"], g["seed"], g["policy"], row["attempt"], stage,
                                            ref_key, a[dev_key], want)
        assert sum(a["level2"]) == row["binary"]["deduplicated"]
        assert sum(a["level1"]) == row["middle"]["deduplicated"]


@pytest.mark.parametrize("case", [i for i in range(16) if i % 2 == 1])
def test_audit_mode_checks_every_stage_and_matches_reference(golden, case):
    """TERGPU_ATTEMPT_AUDIT (the reference's FullTerConfig::audit): every stage
    whose scalar oracle takes at most 10^6 pairs or triples is recomputed on the
    host and compared with the device's output and provenance -- all 13 stages
    at n=36 (nine L3 -> L2 merges, three L2 -> L1 merges, the root), the nine
    L3 -> L2 merges at n=72.  No stage disagrees, and the audited run reports the
    root as FullCanonicalOutput whatever policy was asked for, as the reference's
    audit does: its counters and fingerprints equal the reference's
    FullCanonicalOutput telemetry."""
    from tergpu import _abi

    g = golden["attempt_telemetry"][case]
    assert g["policy"] == "canon"
    _, res = _attempt(g["n"], g["seed"], 0, g["attempts"], kind=g["kind"],
                      root_policy=_abi.ROOT_POLICY_FIRST_WITNESS, telemetry=True, audit=True,
                      memory_limit_bytes=64 << 30)
    final = g["final"]
    assert res.status == final["status"], (res.status_name, _abi.last_error())
    assert res.fingerprint == hexint(final["fingerprint"])
    assert len(res.attempts) == len(g["rows"])
    for a, row in zip(res.attempts, g["rows"]):
        assert a["audited_stages"] == (13 if g["n"] == 36 else 9)
        for stage, fields in STAGES.items():
            for ref_key, dev_key in fields.items():
                want = row[stage][ref_key]
                want = hexint(want) if ref_key == "fingerprint" else want
                assert a[dev_key] == want, (g["n"], g["seed"], row["attempt"], stage, ref_key)


def test_n36_attempt_loop_stops_like_the_reference(golden):
    """The whole loop in one call: the reference's final status and attempt count."""
    from tergpu import _abi

    for g in golden["n36_attempts"]:
        _, res = _attempt(36, g["seed"], 0, 8, kind=g["kind"])
        assert res.status == g["final"]["status"]
        assert len(res.attempts) == len(g["attempts"])


def test_n72_anchor_l1_lists_are_byte_identical(oracle_mod, golden, tmp_path):
    from tergpu import snapshot

    g = golden["n72_roots"][0]
    _, res = _attempt(72, ANCHOR_SEED, 0, 1, export_l1_capacity=40_000, capture_only=True)
    a = res.attempts[0]
    assert a["level1"] == g["level1"] and a["level2"] == g["level2"]
    snap = res.snapshot
    assert snap.entries == g["level1"]
    if oracle_mod.ref_available():
        path = tmp_path / "ref.snap"
        oracle_mod.ref_run("capture", 72, ANCHOR_SEED, 0, "auth", path)
        ref = snapshot.load(path)
        for l in range(3):
            assert np.array_equal(ref.records[l], snap.records[l]), l
            assert np.array_equal(ref.child_targets[l], snap.child_targets[l])
        assert np.array_equal(ref.root_target, snap.root_target)


def test_n72_positive_attempt_found():
    """Seed 0x7201: attempts 0..20 find nothing, attempt 21 finds the planted
    solution (the reference's pinned positive path)."""
    from tergpu import _abi, instance

    inst, res = _attempt(72, 0x7201, 0, 22)
    assert res.status == _abi.FOUND and res.found_attempt == 21
    assert [a["status"] for a in res.attempts[:21]] == [_abi.NO_WITNESS_THIS_ATTEMPT] * 21
    assert res.attempts[21]["level1"] == [36425, 33948, 34773]
    assert instance.verify_witness(inst, res.witness)
    assert np.array_equal(res.witness, inst.planted)


def test_n108_authentic_attempt_matches_published_capture():
    """n=108 seed 0x1001 attempt 0 on the device: the level sizes of the reference's
    published capture (results/root-queue-generalization/snapshots/n108_s0x1001_a0.snap.json)
    and, on its anchor cell 2730, the published logical pairs and projected counts
    (results/arwlf/hash-join-n108-anchor.log: 6,143,192,070 pairs, 1,261,846,123
    triples on 25 bits, 9,856,289 on 32 bits)."""
    import tergpu

    _, res = _attempt(108, 0x1001, 0, 1, export_l1_capacity=7_000_000, capture_only=True)
    a = res.attempts[0]
    assert (res.r1, res.r2) == (39, 12)
    assert a["level2"] == [150329, 150329, 149477, 150611, 150012, 150030, 149933, 150092, 150148]
    assert a["level1"] == [3650689, 6900048, 6896564]
    snap = res.snapshot
    assert sum(len(r) for r in snap.records) + 424 == 837_470_872  # the published file size
    cells = np.zeros(4096, dtype=np.uint8)
    cells[2730] = 1
    r32 = tergpu.run_gpu_root_records(snap, tergpu.Config(projected_bits=32), cells=cells)
    assert r32.telemetry.logical_pairs == 6_143_192_070
    assert r32.telemetry.projected_hits == 9_856_289
    assert r32.telemetry.full_hits == 0 and r32.residue_exact == 0
    r25 = tergpu.run_gpu_root_records(snap, tergpu.Config(projected_bits=25, count_only=True), cells=cells)
    assert r25.telemetry.projected_hits == 1_261_846_123


def test_attempt_statuses():
    from tergpu import _abi, attempt, instance

    inst = instance.benchmark_instance(36, 5)
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=5, attempt_limit=4, memory_limit_bytes=1000))
    assert res.status == _abi.RESOURCE_LIMIT
    flag = ctypes.c_int32(1)
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=5, attempt_limit=4), cancel=flag)
    assert res.status == _abi.CANCELLED
    bad = instance.benchmark_instance(48, 5)
    res = attempt.solve_full_ter(bad, attempt.FullTerConfig(seed=5))
    assert res.status == _abi.INVALID_CONFIGURATION


@pytest.mark.parametrize("n,seed,first,count", [(36, ANCHOR_SEED, 0, 8), (36, 358, 0, 2),
                                               (72, ANCHOR_SEED, 0, 3), (72, 0x7201, 19, 4)])
def test_graph_attempts_equal_stage_by_stage(n, seed, first, count):
    """n = 36 and 72 run each attempt as one captured CUDA graph; the same
    attempts stage by stage give the same levels, counts, status and witness."""
    from tergpu import batch

    inst, graphed = _attempt(n, seed, first, count)
    _, staged = _attempt(n, seed, first, count, no_graph=True)
    assert batch.same_result(graphed, staged)
    assert graphed.attempts and graphed.attempts[0]["level1"] == staged.attempts[0]["level1"]


def test_cancel_reaches_the_running_n108_sweep():
    """A cancel raised while the n=108 root sweep runs (about 7.6 s of device
    work) stops it within a few work items: the attempt returns Cancelled soon
    after the flag is set, with no witness."""
    import ctypes
    import threading
    import time

    from tergpu import _abi, attempt, instance

    inst = instance.benchmark_instance(108, 0x1001)
    flag = ctypes.c_int32(0)
    timer = threading.Timer(1.5, lambda: setattr(flag, "value", 1))
    t0 = time.perf_counter()
    timer.start()
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=0x1001, attempt_limit=1,
                                                             memory_limit_bytes=64 << 30),
                                 cancel=flag)
    elapsed = time.perf_counter() - t0
    timer.cancel()
    assert res.status == _abi.CANCELLED
    assert res.witness is None
    assert elapsed < 4.0, elapsed
