"""tergpu_full_bench: ter_full_bench's command line over the device attempt path.

CPU: option handling and --preflight (no device work).  GPU: attempt-cost and
time-to-found rows against the reference's attempts (golden fixtures),
success-curve against the oracle, and the cooperative time limit."""
import subprocess

import pytest

from conftest import ROOT

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


def test_preflight_refusals():
    p = run("--preflight", "--n=48")
    assert p.returncode == 1 and "InvalidConfiguration" in p.stdout
    p = run("--preflight", "--n=108", "--memory-limit-bytes=1048576")
    assert p.returncode == 1 and "ResourceLimit" in p.stdout


@pytest.mark.parametrize("args,rc,text", [
    (["--mode=bogus"], 1, "invalid --mode value"),
    (["--mode=success-curve", "--repeat=3"], 1, "--repeat does not apply"),
    (["--attempt-limit=0"], 1, "invalid --attempt-limit value"),
    (["--fixture"], 2, "does not implement"),
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
