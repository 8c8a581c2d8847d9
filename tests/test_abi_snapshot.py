"""C-ABI library loading and the .snap reader/writer (CPU only, no device compute)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN_DIR, ROOT


def test_library_exports_every_declared_symbol():
    from tergpu import _abi

    lib = _abi.load()
    header = (ROOT / "include" / "tergpu.h").read_text()
    declared = set(re.findall(r"^\w[\w \*]*?\b(tergpu_\w+)\s*\(", header, flags=re.M))
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(_abi.EXPORTED) <= declared
    version = re.search(r"#define TERGPU_ABI_VERSION (\d+)", header).group(1)
    assert lib.tergpu_abi_version() == int(version)


def test_python_constants_mirror_every_header_value():
    """Every flag, limit and status value of include/tergpu.h has a constant of
    the same name (less the TERGPU_ prefix) and value in tergpu._abi."""
    from tergpu import _abi

    header = (ROOT / "include" / "tergpu.h").read_text()
    values = {m.group(1): int(m.group(2))
              for m in re.finditer(r"^#define TERGPU_(\w+) (\d+)u?\b", header, flags=re.M)}
    enum = re.search(r"enum tergpu_status \{(.*?)\};", header, flags=re.S).group(1)
    values.update((m.group(1), int(m.group(2)))
                  for m in re.finditer(r"TERGPU_(\w+) = (\d+)", enum))
    assert len(values) > 30 and "ATTEMPT_FIXTURE" in values and "INVALID_INPUT" in values
    for name, value in values.items():
        assert getattr(_abi, name, None) == value, name


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """Every ctypes mirror has the C struct's size and field offsets (a C probe
    compiled against include/tergpu.h prints them)."""
    import subprocess

    from tergpu import _abi, attempt, batch

    mirrors = {"tergpu_root_in": _abi.RootIn, "tergpu_root_out": _abi.RootOut,
               "tergpu_root_records_in": _abi.RootRecordsIn,
               "tergpu_root_records_out": _abi.RootRecordsOut,
               "tergpu_attempt_stats": attempt.AttemptStats, "tergpu_attempt_in": attempt.AttemptIn,
               "tergpu_attempt_out": attempt.AttemptOut, "tergpu_batch_in": batch.BatchIn,
               "tergpu_batch_out": batch.BatchOut}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "tergpu.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    for line in out.splitlines():
        cname, field, value = line.split()
        py = mirrors[cname]
        got = ctypes.sizeof(py) if field == "size" else getattr(py, field).offset
        assert got == int(value), (cname, field, got, value)


def test_fnv1a_known_answers():
    from tergpu import snapshot

    assert snapshot.fnv1a(b"") == 0xcbf29ce484222325
    assert snapshot.fnv1a(b"a") == 0xaf63dc4c8601ec8c
    assert snapshot.fnv1a(b"foobar") == 0x85944171f73967e8


def test_adapter_header_declares_hash_join_signature():
    text = (ROOT / "subset-sum-ter-fft_b200" / "adapter" / "ter_gpu_root.hpp").read_text()
    assert re.search(r"Status run_gpu_root\(const mr8::Dataset& data, const rg::RootIndex& index,\s*"
                     r"const a64::FamilyKeys& keys, const Config& config,\s*"
                     r"rg::RootSink& sink, Telemetry\* telemetry", text)


def test_snapshot_load_matches_reference_capture(golden):
    from tergpu import snapshot

    g = golden["n36_snapshot"]
    snap = snapshot.load(GOLDEN_DIR / g["path"])
    assert snap.entries == g["level1"]
    assert snap.level2_sizes == g["level2"]
    assert snap.n == 36 and snap.r1 == 12 and snap.r2 == 3
    assert (GOLDEN_DIR / g["path"]).stat().st_size == g["file_bytes"]
    pos, neg = snap.masks(0)
    assert not np.any(neg) and all(bin(int(p)).count("1") == 6 for p in pos[:, 0])


def test_snapshot_roundtrip_is_byte_identical(tmp_path, golden):
    from tergpu import snapshot

    src = GOLDEN_DIR / golden["n36_snapshot"]["path"]
    snap = snapshot.load(src)
    out = tmp_path / "copy.snap"
    snapshot.save(snap, out, git_commit="reference")
    a, b = src.read_bytes(), out.read_bytes()
    # identical lists, targets and checksums; the writer does not carry the
    # capture-only telemetry fields (peak bytes, elapsed ns, memory limit)
    assert a[424:] == b[424:]
    ha = np.frombuffer(a[:424], dtype=snapshot.HEADER_DTYPE)[0]
    hb = np.frombuffer(b[:424], dtype=snapshot.HEADER_DTYPE)[0]
    for f in ("n", "r1", "r2", "entries", "offset", "checksum", "child_target", "root_target",
              "level2_sizes", "seed", "attempt_seed", "attempt"):
        assert np.array_equal(ha[f], hb[f]), f
    assert snapshot.load(out).entries == snap.entries


def test_snapshot_damage_is_rejected(tmp_path, golden):
    from tergpu import snapshot

    src = GOLDEN_DIR / golden["n36_snapshot"]["path"]
    raw = bytearray(src.read_bytes())
    for where in (10, 500, len(raw) - 3):
        bad = bytearray(raw)
        bad[where] ^= 0x40
        p = tmp_path / f"bad{where}.snap"
        p.write_bytes(bytes(bad))
        with pytest.raises(snapshot.SnapshotError):
            snapshot.load(p)
    # the reference's own damage cases (ter2_root/tests/ter_root_snapshot_tests.cpp:205-220):
    # a record cut short by two records, a tampered header field, a trailing byte
    off_n = snapshot.HEADER_DTYPE.fields["n"][1]
    tampered = bytearray(raw)
    tampered[off_n] ^= 0x01
    for name, data in (("trunc", raw[:-5]), ("trunc48", raw[:-48]), ("header", tampered),
                       ("trailing", raw + b"\0")):
        p = tmp_path / f"{name}.snap"
        p.write_bytes(bytes(data))
        with pytest.raises(snapshot.SnapshotError):
            snapshot.load(p)
    p = tmp_path / "original.snap"
    p.write_bytes(bytes(raw))
    assert snapshot.load(p).entries == golden["n36_snapshot"]["level1"]


def test_host_key_derivation_matches_oracle_attempt(oracle_mod, golden):
    """Keys from the reference's n=36 capture equal the oracle's quotients."""
    from tergpu import snapshot

    snap = snapshot.load(GOLDEN_DIR / golden["n36_snapshot"]["path"])
    Q, lo, hi, tau = snapshot.root_keys(snap)
    assert Q == 24
    att = oracle_mod.attempt(36, 19797034556212562, 0, export_l1=True)
    r1 = att["r1"]
    for l in range(3):
        res = att["l1"]["res_lo"][l].astype(object) | (att["l1"]["res_hi"][l].astype(object) << 64)
        q = [(((int(r) - att["t1"][l]) % (1 << 36)) >> r1) for r in res]
        if l == 2:
            q = [(tau - v) % (1 << Q) for v in q]
        assert [int(v) for v in lo[l]] == q
    # the oracle's full-Q join over these keys reproduces the reference's root stage
    d, _ = oracle_mod.root_join(Q, lo, [h.astype(np.uint64) for h in hi])
    row = golden["n36_attempts"][0]["attempts"][0]
    assert d["triples"] == row["root_modular"]


def test_root_report_refuses_captures_that_break_the_invariants(golden):
    """report_full_ter_root's capture checks (src/full_ter.cpp:3772-3803), with
    the reference's messages and before any device work: a residue not
    congruent to its child target modulo 2^r1, a residue at or above 2^n, and a
    child or root target at or above 2^n are InvalidConfiguration."""
    import copy

    from tergpu import _abi, report, snapshot

    base = snapshot.load(GOLDEN_DIR / golden["n36_snapshot"]["path"])
    assert report._capture_refusal(base) is None
    invariant = "root report capture violates the child target invariant"
    cases = []
    low = copy.deepcopy(base)
    low.records[1].reshape(-1, low.record_bytes)[3, 16 * low.words64] ^= 1  # residue bit 0
    cases.append((low, invariant))
    high = copy.deepcopy(base)
    high.records[2].reshape(-1, high.record_bytes)[0, 16 * high.words64 + 4] ^= 0x10  # residue bit 36
    cases.append((high, invariant))
    child = copy.deepcopy(base)
    child.child_targets[0] = child.child_targets[0].copy()
    child.child_targets[0][1] |= 1 << 4  # bit 36
    cases.append((child, "root count child target exceeds the captured modulus"))
    root = copy.deepcopy(base)
    root.root_target = root.root_target.copy()
    root.root_target[1] |= 1 << 5
    cases.append((root, "root count target exceeds the captured modulus"))
    for snap, message in cases:
        for policy in report.RootOutputPolicy:
            got = report.report_full_ter_root(snap, policy)
            assert got.status == _abi.INVALID_CONFIGURATION and got.message == message
        counted = report.count_full_ter_root(snap)
        assert counted.status == _abi.INVALID_CONFIGURATION and counted.message == message


def test_root_report_refuses_bad_policy_and_honours_a_set_cancel_flag(golden):
    """report_full_ter_root's first checks (src/full_ter.cpp:3727-3743), before
    any device work: a policy outside the enum is InvalidConfiguration with the
    reference's message, and a cancellation flag already set returns Cancelled
    from the report and the count."""
    from tergpu import _abi, report, snapshot

    snap = snapshot.load(GOLDEN_DIR / golden["n36_snapshot"]["path"])
    bad = report.report_full_ter_root(snap, 7)
    assert bad.status == _abi.INVALID_CONFIGURATION
    assert bad.message == "root report requires a completed native root capture and valid tiled limits"
    flag = ctypes.c_int32(1)
    for policy in report.RootOutputPolicy:
        got = report.report_full_ter_root(snap, policy, cancel=flag)
        assert got.status == _abi.CANCELLED and got.message == "root report was cancelled"
    counted = report.count_full_ter_root(snap, cancel=flag)
    assert counted.status == _abi.CANCELLED and counted.valid_root_count == 0
