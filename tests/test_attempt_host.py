"""tergpu_attempt_run's host side through the C ABI, with no device work (CPU
only): the preflight's geometry and byte prediction, and the refusals the
reference's solve_full_ter makes before any work (src/full_ter.cpp:2945-2957,
3012-3024)."""
import dataclasses

import numpy as np
import pytest

SHAPES = [(36, 12, 3, 18), (72, 25, 7, 630), (108, 39, 12, 24804)]


@pytest.mark.parametrize("n, r1, r2, l3", SHAPES)
def test_preflight_geometry(n, r1, r2, l3):
    from tergpu import _abi, attempt, instance

    res = attempt.preflight(instance.benchmark_instance(n, 1))
    assert res.status == _abi.COMPLETED
    assert (res.r1, res.r2, res.level3_size) == (r1, r2, l3)
    assert res.device_bytes > 0 and res.attempts == []


def test_preflight_fixture_level3_size():
    """FixtureTer keeps the first min(C(n/2, n/36), limit) subsets per half."""
    from tergpu import _abi, attempt, instance

    for n, limit, want in ((36, 9, 9), (36, 64, 18), (108, 1500, 1500), (108, 10**6, 24804)):
        res = attempt.preflight(instance.benchmark_instance(n, 1), attempt.FullTerConfig(fixture_limit=limit))
        assert res.status == _abi.COMPLETED and res.level3_size == want, (n, limit)
    full = attempt.preflight(instance.benchmark_instance(108, 1))
    small = attempt.preflight(instance.benchmark_instance(108, 1), attempt.FullTerConfig(fixture_limit=1500))
    assert small.device_bytes < full.device_bytes


def test_solve_refuses_count_only_and_unknown_policies():
    """solve_full_ter refuses CountOnly, as a SAT result must keep a verifiable
    witness (the reference's own check: tests/full_ter_tests.cpp:415-418), and
    any policy outside the enum; both before any device work."""
    from tergpu import _abi, attempt, instance

    inst = instance.benchmark_instance(36, 0x5048415345355445)
    for policy in (_abi.ROOT_POLICY_COUNT_ONLY, 3, 255):
        cfg = attempt.FullTerConfig(seed=0x5048415345355345, root_policy=policy)
        assert attempt.solve_full_ter(inst, cfg).status == _abi.INVALID_CONFIGURATION, policy
        assert attempt.preflight(inst, cfg).status == _abi.INVALID_CONFIGURATION, policy
        assert "CountOnly" in _abi.last_error()
    for policy in (_abi.ROOT_POLICY_FIRST_WITNESS, _abi.ROOT_POLICY_FULL_CANONICAL):
        assert attempt.preflight(inst, attempt.FullTerConfig(root_policy=policy)).status == _abi.COMPLETED


def test_solve_refusals_before_device_work():
    """36 not dividing n, a predicted footprint above the declared ceiling, and
    guided targets whose planted root is not balanced across the halves
    (InvalidConfiguration with the reference's message) all return before the
    device is touched."""
    from tergpu import _abi, attempt, instance

    for n in (48, 60, 84, 96):
        res = attempt.solve_full_ter(instance.benchmark_instance(n, 1))
        assert res.status == _abi.INVALID_CONFIGURATION
        assert res.message == "full TER requires n divisible by 36 and 0 < modulus_bits <= n"
    tight = attempt.FullTerConfig(memory_limit_bytes=1 << 20)
    assert attempt.solve_full_ter(instance.benchmark_instance(108, 1), tight).status == _abi.RESOURCE_LIMIT
    inst = instance.benchmark_instance(36, 0x544552F)
    lopsided = np.zeros(36, dtype=np.uint8)
    lopsided[:18] = 1
    bad = dataclasses.replace(inst, planted=lopsided)
    res = attempt.solve_full_ter(bad, attempt.FullTerConfig(seed=91, guided=True))
    assert res.status == _abi.INVALID_CONFIGURATION
    assert _abi.last_error() == "guided TER requires a planted binary root balanced across both halves"


def _failure_case(golden, name):
    from tergpu import attempt, instance

    g = next(c for c in golden["failure_semantics"] if c["name"] == name)
    inst = instance.benchmark_instance(g["n"], g["seed"])
    cfg = attempt.FullTerConfig(seed=g["config_seed"], attempt_limit=g["attempts"],
                                fixture_limit=g["fixture_limit"], audit=bool(g["audit"]), telemetry=True)
    return g, inst, cfg


def test_pre_cancelled_solve_matches_reference(golden):
    """A solve whose cancellation flag is set before the call returns Cancelled
    before level 3, with the reference's run fingerprint (no attempts, no
    level-3 lists): the reference's failure-semantics test
    (tests/full_ter_tests.cpp:636-645), with no device work."""
    import ctypes

    from conftest import hexint
    from tergpu import _abi, attempt

    g, inst, cfg = _failure_case(golden, "pre_cancelled")
    assert g["final"]["status"] == _abi.CANCELLED and g["final"]["l3"] == [0, 0]
    res = attempt.solve_full_ter(inst, cfg, cancel=ctypes.c_int32(1))
    assert res.status == _abi.CANCELLED and res.attempts == []
    assert res.fingerprint == hexint(g["final"]["fingerprint"])
    assert res.message == _abi.last_error() == g["final"]["message"]


def test_empty_budget_and_tiny_ceiling_fail_closed(golden):
    """An empty attempt budget is InvalidConfiguration, as the reference's
    (tests/full_ter_tests.cpp:647-652), and a 1-byte memory ceiling is
    ResourceLimit (:630-633); neither touches the device."""
    from tergpu import _abi, attempt

    g, inst, cfg = _failure_case(golden, "no_attempts")
    assert g["final"]["status"] == _abi.INVALID_CONFIGURATION
    res = attempt.solve_full_ter(inst, cfg)
    assert res.status == _abi.INVALID_CONFIGURATION and res.message == g["final"]["message"]
    _, inst, cfg = _failure_case(golden, "run")
    tight = attempt.FullTerConfig(**{**cfg.__dict__, "memory_limit_bytes": 1})
    assert attempt.solve_full_ter(inst, tight).status == _abi.RESOURCE_LIMIT


def test_unknown_flags_are_refused():
    """Flag bits outside the ABI's set fail closed (the reference refuses
    out-of-range execution-mode values: tests/full_ter_tests.cpp:654-658)."""
    import ctypes

    from tergpu import _abi, attempt, instance

    lib = _abi.load()
    ain, out, keep = attempt.make_request(instance.benchmark_instance(36, 17), attempt.FullTerConfig())
    ain.flags |= 1 << 12
    lib.tergpu_attempt_run.argtypes = [ctypes.POINTER(attempt.AttemptIn), ctypes.POINTER(attempt.AttemptOut)]
    assert lib.tergpu_attempt_run(ctypes.byref(ain), ctypes.byref(out)) == _abi.INVALID_CONFIGURATION
