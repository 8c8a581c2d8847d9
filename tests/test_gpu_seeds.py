"""n=108 roots of several seeds against the reference's frozen ARWLF.

For every seed the device attempt pipeline makes the authentic attempt-0 L1
lists (the benchmark instance, as the reference's captures), the host derives
the root keys, and both the device root and the reference's ARWLF (compiled
from its sources, oracle/_ref/terref) run the reference's declared 16-cell
sample of the same root: identical full-Q triple multisets (count and the three
sink hashes), identical logical pairs, identical 32-bit projected hits (about
2.5e7 per seed, the strong check: the full-Q outputs are almost always empty).
The six published roots run by default; TERGPU_SEED_SWEEP=32 adds 26 fresh
seeds (the reference's 32-seed configuration).
"""
import json
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import pytest

from conftest import hexint

pytestmark = pytest.mark.gpu

PUBLISHED = [0x1001, 0x2003, 0x3007, 0x4001, 0x5003, 0x6007]
FRESH = [0x9000 + 0x111 * i for i in range(26)]
SEEDS = PUBLISHED + (FRESH if os.environ.get("TERGPU_SEED_SWEEP") == "32" else [])
CELLS = 16


def _write_keys(keys, path: Path):
    with open(path, "wb") as f:
        f.write(b"TERKEYS1")
        f.write(np.array([keys.quotient_bits, 0], dtype=np.uint32).tobytes())
        f.write(np.array([len(a) for a in keys.lo], dtype=np.uint64).tobytes())
        for l in range(3):
            f.write(np.ascontiguousarray(keys.lo[l], dtype=np.uint64).tobytes())
            f.write(np.ascontiguousarray(keys.hi[l], dtype=np.uint8).tobytes())
            f.write(b"\0" * ((8 - len(keys.lo[l]) % 8) % 8))


def _keys(seed):
    import tergpu
    from tergpu import attempt, instance, snapshot

    inst = instance.benchmark_instance(108, seed)
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=seed, attempt_limit=1,
                                                             capture_only=True,
                                                             export_l1_capacity=7_500_000))
    q, lo, hi, _ = snapshot.root_keys(res.snapshot)
    return tergpu.RootKeys(quotient_bits=q, lo=lo, hi=hi), res.attempts[0]["level1"]


def test_seeds_match_reference_arwlf_on_the_declared_sample(oracle_mod):
    import tergpu
    from tergpu import workload

    if not oracle_mod.ref_available():
        raise RuntimeError("the reference harness oracle/_ref/terref is needed for this test")
    cells = oracle_mod.select_cells(CELLS)
    with tempfile.TemporaryDirectory() as d:
        jobs = []
        gpu = {}
        for seed in SEEDS:
            keys, level1 = _keys(seed)
            res = tergpu.run_gpu_root(keys, tergpu.Config(projected_bits=32), cells=cells)
            gpu[seed] = (res, level1)
            path = Path(d) / f"k{seed:x}.keys"
            _write_keys(keys, path)
            jobs.append((seed, path))

        def reference(job):
            seed, path = job
            p = subprocess.run([str(oracle_mod.REF_BIN), "keysroot", str(path), "arwlf", str(CELLS),
                                "1", "32"], capture_output=True, text=True, timeout=3600)
            rows = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
            return seed, rows[0]

        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
            ref = dict(pool.map(reference, jobs))
    for seed in SEEDS:
        res, level1 = gpu[seed]
        row = ref[seed]
        got = workload.digest(res.triples)
        for k in ("triples", "triple_sum", "triple_xor", "triple_sum2"):
            assert got[k] == hexint(row[k]), (hex(seed), k)
        assert res.telemetry.logical_pairs == row["pairs"], hex(seed)
        assert res.telemetry.projected_hits == row["projected_hits"] > 0, hex(seed)
        assert len(level1) == 3 and min(level1) > 3_000_000
