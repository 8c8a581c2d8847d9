"""bench.py's host logic (CPU only): which reference build times the CPU legs,
and the served request mix: bounded n=108 budgets, the same requests at any rate."""
import argparse
import importlib.util

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_build_is_the_widest_the_host_runs(tmp_path):
    bench = _bench()
    for name in ("terref", "terref_native", "terref_v4"):
        (tmp_path / name).write_text("")
    (tmp_path / "native_flags.txt").write_text("avx2\navx512f\navx512vnni\n")
    (tmp_path / "v4_flags.txt").write_text("avx2\navx512f\n")
    exe, build = bench.ref_binary({"avx2", "avx512f", "avx512vnni", "sse4_2"}, tmp_path)
    assert exe.name == "terref_native" and build == "g++ -O2 -march=native"
    exe, build = bench.ref_binary({"avx2", "avx512f"}, tmp_path)
    assert exe.name == "terref_v4" and "x86-64-v4" in build and "avx512vnni" in build
    exe, build = bench.ref_binary({"avx2"}, tmp_path)
    assert exe.name == "terref" and "x86-64-v3" in build
    (tmp_path / "terref_native").unlink()
    (tmp_path / "terref_v4").unlink()
    exe, build = bench.ref_binary({"avx2"}, tmp_path)
    assert exe.name == "terref" and build == "g++ -O2 -march=x86-64-v3"


def test_served_n108_budgets_are_bounded_and_seeded():
    bench = _bench()
    args = argparse.Namespace(seed=0x1001, requests=56, rate=4.0, serve_n="36,48,60,72,84,96,108",
                              max_attempts=0, max_attempts_108=2)
    reqs = bench.solve_requests(args, True)
    big = [r.config.attempt_limit for r in reqs if r.instance.n == 108]
    small = [r.config.attempt_limit for r in reqs if r.instance.n != 108]
    assert big and all(1 <= b <= 2 for b in big)
    assert max(small) > 2 and all(1 <= b <= 64 for b in small)
    arrivals = [r.arrival_ms for r in reqs]
    assert arrivals == sorted(arrivals) and arrivals[-1] > 0
    again = bench.solve_requests(args, True)
    assert [(r.instance.n, r.config.seed, r.config.attempt_limit) for r in again] == \
        [(r.instance.n, r.config.seed, r.config.attempt_limit) for r in reqs]


def test_saturated_serve_stream_has_the_same_requests():
    """serve_saturated re-times the serve stream: the same seeded requests (n,
    seed, budget), only the arrival gaps shrink with the rate."""
    bench = _bench()

    def stream(rate):
        args = argparse.Namespace(seed=0x1001, requests=400, rate=rate, serve_n="36,48,60,72,84,96",
                                  max_attempts=0)
        return bench.solve_requests(args, True)

    slow, fast = stream(200.0), stream(5000.0)
    assert [(r.instance.n, r.config.seed, r.config.attempt_limit) for r in slow] == \
        [(r.instance.n, r.config.seed, r.config.attempt_limit) for r in fast]
    assert abs(fast[-1].arrival_ms * 25 - slow[-1].arrival_ms) < 1e-6 * slow[-1].arrival_ms
