"""The batch / serving engine (tergpu_attempt_batch): every request's result is
bit-identical to the same request run alone, in a batch and in a served
stream; admission respects the memory budget; the preflight refuses what it
must before any device work; the preflight never predicts fewer bytes than a
request holds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(rng, count, ns=(36, 48, 72), max_attempts=6):
    from tergpu import attempt, batch, instance

    out = []
    for i in range(count):
        n = int(rng.choice(ns))
        seed = int(rng.integers(1, 1 << 40))
        inst = instance.benchmark_instance(n, seed) if n % 36 == 0 else instance.build_instance(n, seed)
        cfg = attempt.FullTerConfig(seed=seed, attempt_limit=int(rng.integers(1, max_attempts + 1)))
        out.append(batch.Request(inst, cfg, arrival_ms=float(i) * 7.0))
    # the reference's positive n=72 attempt inside the mix: Found at attempt 21
    inst = instance.benchmark_instance(72, 0x7201)
    out.append(batch.Request(inst, attempt.FullTerConfig(seed=0x7201, attempt_first=18,
                                                         attempt_limit=6), arrival_ms=3.0))
    return out


def _alone(req):
    from tergpu import attempt

    return attempt.solve_full_ter(req.instance, req.config)


def test_batch_results_equal_alone():
    from tergpu import batch

    reqs = _requests(np.random.default_rng(11), 20)
    alone = [_alone(r) for r in reqs]
    got = batch.solve_batch(reqs, slots=8)
    for r, a, b in zip(reqs, alone, got.results):
        assert batch.same_result(a, b), (r.instance.n, r.config.seed)
    assert got.results[-1].status == 1 and got.results[-1].found_attempt == 21
    assert got.refused == sum(1 for r in reqs if r.instance.n % 36 != 0)
    assert got.peak_running > 1
    for b in got.results:
        if b.status in (1, 3):
            assert 0 < b.device_bytes_held <= b.device_bytes  # the preflight never underestimates


def test_served_stream_results_and_timing():
    from tergpu import batch

    reqs = _requests(np.random.default_rng(12), 16)
    alone = [_alone(r) for r in reqs]
    got = batch.solve_batch(reqs, slots=4, served=True)
    for a, b in zip(alone, got.results):
        assert batch.same_result(a, b)
    arrival = np.array([r.arrival_ms for r in reqs])
    assert np.all(got.admit_ms >= arrival - 1e-6)
    assert np.all(got.finish_ms >= got.admit_ms)
    assert np.allclose(got.latency_ms, got.finish_ms - arrival)


def test_memory_budget_admission_and_refusals():
    from tergpu import attempt, batch, instance

    reqs = _requests(np.random.default_rng(13), 10, ns=(72,), max_attempts=2)
    one = max(_alone(r).device_bytes for r in reqs)
    # room for one n=72 request at a time: the engine must serialize them
    got = batch.solve_batch(reqs, slots=8, memory_budget_bytes=one)
    assert got.peak_predicted_bytes <= one and got.peak_running == 1
    for r, b in zip(reqs, got.results):
        assert batch.same_result(_alone(r), b)
    # a request above the whole budget, one above its own ceiling, and 36 not dividing n
    big = batch.Request(instance.benchmark_instance(72, 5), attempt.FullTerConfig(seed=5))
    small_ceiling = batch.Request(instance.benchmark_instance(36, 5),
                                  attempt.FullTerConfig(seed=5, memory_limit_bytes=1024))
    bad = batch.Request(instance.build_instance(60, 5), attempt.FullTerConfig(seed=5))
    got = batch.solve_batch([big, small_ceiling, bad], slots=2, memory_budget_bytes=1 << 20)
    assert [b.status for b in got.results] == [7, 7, 4]
    assert got.refused == 3
