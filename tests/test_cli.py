"""tergpu_full_bench: ter_full_bench's command line over the device attempt path.

CPU: option handling and --preflight (no device work).  GPU: attempt-cost and
time-to-found rows against the reference's attempts (golden fixtures),
success-curve against the oracle, and the cooperative time limit."""
import json
import subprocess

import pytest

from conftest import GOLDEN_DIR, ROOT

CLI = ROOT / "subset-sum-ter-fft_b200" / "cli" / "tergpu_full_bench"
ANCHOR_SEED = 19797034556212562  # ter_full_bench's default seed (0x46554c4c544552)


def run(*args, timeout=600):
    if not CLI.exists():
        raise RuntimeError(f"{CLI} not built (run __graft_entry__.build())")
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=timeout)


def csv_rows(text):
    lines = [l for l in text.splitlines() if l and not l.startswith("#")]
    header = lines[0].split(",")
    return [dict(zip(header, _split(l))) for l in lines[1:]]


def _split(line):
    out, cur, quoted = [], "", False
    for ch in line:
        if ch == '"':
            quoted = not quoted
        elif ch == "," and not quoted:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    out.append(cur)
    return out


@pytest.mark.parametrize("n,r1,r2,q", [(36, 12, 3, 24), (72, 25, 7, 47), (108, 39, 12, 69)])
def test_preflight_geometry(n, r1, r2, q):
    p = run("--preflight", f"--n={n}", "--memory-limit-mib=1000000")
    assert p.returncode == 0, p.stderr
    assert f"r1={r1} r2={r2} root_Q={q} l2_to_l1_Q={r1 - r2}" in p.stdout
    assert "VERDICT: bounded exact path on both merge stages" in p.stdout


@pytest.mark.parametrize("case", range(5))
def test_preflight_prints_the_reference_lines(case):
    """Every line of the reference's own ter_full_bench --preflight (golden
    preflight_text) appears in the device preflight, with the same exit code:
    geometry, the exact representation counts R1 and R2, the decisions, the
    ceiling and the mode.  The backend lines name the device's own join, and at
    Q > 64 its full-key root decision, so those are left out of the
    comparison."""
    g = json.loads((GOLDEN_DIR / "reference_golden.json").read_text())["preflight_text"][case]
    p = run(*g["args"])
    assert p.returncode == g["rc"], p.stderr
    got = set(p.stdout.splitlines())
    device_worded = ("  l2_to_l1_backend=", "  root_backend=", "  root_decision=low-64")
    for line in g["lines"]:
        if not line.startswith(device_worded):
            assert line in got, line


def test_preflight_refusals():
    p = run("--preflight", "--n=48")
    assert p.returncode == 1 and "InvalidConfiguration" in p.stdout
    p = run("--preflight", "--n=108", "--memory-limit-bytes=1048576")
    assert p.returncode == 1 and "ResourceLimit" in p.stdout


@pytest.mark.parametrize("args,rc,text", [
    (["--mode=bogus"], 1, "invalid --mode value"),
    (["--mode=success-curve", "--repeat=3"], 1, "--repeat does not apply"),
    (["--attempt-limit=0"], 1, "invalid --attempt-limit value"),
    (["--fixture-limit=0"], 1, "invalid --fixture-limit value"),
    (["--family=paper-rounded"], 2, "does not implement"),
    (["--nonsense"], 1, "usage"),
])
def test_option_errors(args, rc, text):
    p = run(*args)
    assert p.returncode == rc
    assert text in p.stderr


@pytest.mark.gpu
def test_attempt_cost_row_matches_reference(golden):
    case = next(c for c in golden["n36_attempts"] if c["kind"] == "auth" and c["seed"] == ANCHOR_SEED)
    p = run("--n=36", "--attempt-limit=3", "--warmup=1", "--repeat=3")
    assert p.returncode == 0, p.stderr
    row = csv_rows(p.stdout)[0]
    last = case["attempts"][2]
    assert row["status"] == "AttemptLimitReached"
    assert (row["r1"], row["r2"]) == ("12", "3")
    assert row["L2_sizes"] == ":".join(map(str, last["level2"]))
    assert row["L1_sizes"] == ":".join(map(str, last["level1"]))
    assert row["attempts_used"] == "3" and row["terminal_attempt_index"] == "2"
    assert int(row["root_modular"]) == last["root_modular"]


# ter_full_bench columns whose values the device row must reproduce exactly; the
# others are timings, the CPU memory model and the tiled reporter's internals.
SHARED_COLUMNS = (
    "status", "n", "r1", "r2", "L3_left", "L3_right", "L2_sizes", "L1_sizes", "L0",
    "binary_pairs", "binary_modular", "binary_structural_rejects", "binary_distribution_rejects",
    "binary_survivors", "binary_deduplicated", "middle_pairs", "middle_modular",
    "middle_structural_rejects", "middle_distribution_rejects", "middle_survivors",
    "middle_deduplicated", "root_pairs", "root_modular", "root_structural_rejects",
    "root_distribution_rejects", "root_survivors", "root_deduplicated", "fingerprint",
    "l2_to_l1_pair_records", "l1_to_l0_pair_records", "l1_to_l0_quotient_bits",
    "l1_to_l0_prefilter_bits", "l1_to_l0_low_prefilter_candidates",
    "l1_to_l0_full_quotient_rejects", "l1_to_l0_root_policy", "l1_to_l0_valid_roots",
    "l1_to_l0_early_stopped", "attempts_used", "terminal_attempt_index", "terminal_attempt_seed",
    "terminal_attempt_status", "total_root_pair_candidates",
)


_ROWS = len(json.loads((GOLDEN_DIR / "reference_golden.json").read_text())["full_bench_rows"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(_ROWS))
def test_row_matches_reference_ter_full_bench(golden, case):
    """The device row against the reference's own ter_full_bench row (built from
    bench/ter_full_bench.cpp): the same header, and every count column plus the
    telemetry fingerprint equal.  The n=72 0x7201 run is Found at attempt 21
    under FirstWitness, so its root counters stop at the reference's first
    witness in its tiled visit order.  The --guided rows take every attempt's
    targets from the planted root (TerTargetMode::GuidedPlanted) and are Found at
    attempt 0."""
    g = golden["full_bench_rows"][case]
    ref = csv_rows(g["header"] + "\n" + g["row"])[0]
    p = run(*g["args"], "--memory-limit-mib=65536", timeout=1200)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l and not l.startswith("#")]
    assert lines[0] == g["header"]
    row = csv_rows(p.stdout)[0]
    for col in SHARED_COLUMNS:
        assert row[col] == ref[col], (g["args"], col, row[col], ref[col])
    for col, v in row.items():
        assert v == "" or v.lstrip("-").replace(".", "").isdigit() or col.endswith("status") \
            or col.endswith("_sizes"), (col, v)


@pytest.mark.gpu
def test_time_to_found_n72_reference_positive_attempt():
    # the reference's positive n=72 attempt: seed 0x7201, Found at attempt 21
    p = run("--n=72", f"--seed={0x7201}", "--mode=time-to-found", "--attempt-limit=32",
            "--warmup=0", "--repeat=1", "--memory-limit-mib=65536", "--require-found")
    assert p.returncode == 0, p.stderr
    row = csv_rows(p.stdout)[0]
    assert row["status"] == "Found" and row["terminal_attempt_index"] == "21"
    assert row["attempts_used"] == "22"


@pytest.mark.gpu
def test_success_curve_matches_oracle(oracle_mod):
    seeds, limit = 4, 16
    p = run("--n=36", "--mode=success-curve", f"--seeds={seeds}", f"--attempt-limit={limit}")
    assert p.returncode == 0, p.stderr
    blocks = p.stdout.split("\n")
    summary = csv_rows("\n".join(l for l in blocks if not l.startswith("#"))[: 10_000])[0]
    expected = []
    for trial in range(seeds):
        seed = (ANCHOR_SEED + trial * 0x9E3779B97F4A7C15) % (1 << 64)
        hit = next((a + 1 for a in range(limit)
                    if oracle_mod.attempt(36, seed, a, kind="auth")["status"] == 1), None)
        expected.append(hit)
    found = [e for e in expected if e is not None]
    assert int(summary["independent_runs"]) == seeds
    assert int(summary["found"]) == len(found)
    assert int(summary["attempt_limit_reached"]) == seeds - len(found)
    text = p.stdout
    per_run = text[text.index("run_index,"):text.index("attempt_budget,")]
    got = [int(r["attempts_to_found"]) for r in csv_rows(per_run)]
    assert got == found


@pytest.mark.gpu
def test_time_limit_cancels():
    p = run("--n=72", "--attempt-limit=100000", "--warmup=0", "--repeat=1", "--time-limit-ms=50",
            "--memory-limit-mib=65536")
    assert p.returncode == 1
    assert "Cancelled" in p.stderr


@pytest.mark.gpu
def test_time_limit_cancels_inside_the_n108_root():
    """--time-limit-ms at n=108 lands inside the root sweep (one launch of about
    7.6 s): the run ends Cancelled within about a second of the limit."""
    import time

    t0 = time.perf_counter()
    p = run("--n=108", "--attempt-limit=1", "--warmup=0", "--repeat=1", "--time-limit-ms=2000",
            "--memory-limit-mib=65536")
    elapsed = time.perf_counter() - t0
    assert p.returncode == 1
    assert "Cancelled" in p.stderr
    assert elapsed < 6.0, elapsed


@pytest.mark.gpu
def test_audit_flag_checks_the_stages(tmp_path):
    """--audit (the reference's audit mode) runs: every stage of the n=36 attempts
    is checked against the scalar oracles and the command succeeds with
    audit=on in its metadata."""
    import subprocess

    proc = subprocess.run([str(CLI), "--n=36", "--attempt-limit=8", "--warmup=0", "--repeat=1", "--audit"],
                          capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr
    assert "audit=on" in proc.stdout
