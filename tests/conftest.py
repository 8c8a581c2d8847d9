import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "subset-sum-ter-fft_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN_DIR = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return json.loads((GOLDEN_DIR / "reference_golden.json").read_text())


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    return oracle


@pytest.fixture(scope="session")
def n72_anchor_attempt(oracle_mod):
    """The oracle's attempt 0 of the n=72 anchor instance with its L1 lists
    (about 80 s on one core: computed once per session)."""
    return oracle_mod.attempt(72, 19797034556212562, 0, export_l1=True)


def hexint(v):
    return int(v, 16) if isinstance(v, str) else int(v)


def wide_quotient_capture():
    """The reference's Q = 69 truncation fixture (wide_quotient_root_capture,
    tests/full_ter_tests.cpp:769-803) as a capture: n = 108, r1 = 39; list A
    holds the root parent (ones on coordinates 54..107) twice, with residues 0
    and 2^103; lists B and C hold the zero vector; every target is 0.  Both A
    entries have quotient 0 on the low 64 bits; 2^103 >> 39 = 2^64 sets bit 64
    of the second one's quotient, just outside a 64-bit window."""
    import numpy as np
    from tergpu import snapshot

    n, w64, w32 = 108, 2, 4

    def record(ones, residue_words):
        pos = [0] * w64
        for i in ones:
            pos[i // 64] |= 1 << (i % 64)
        masks = np.array(pos + [0] * w64, dtype="<u8").view(np.uint8)
        return np.concatenate([masks, np.array(residue_words, dtype="<u4").view(np.uint8)])

    parent = range(n // 2, n)
    a = np.concatenate([record(parent, [0, 0, 0, 0]), record(parent, [0, 0, 0, 1 << 7])])
    zero = record([], [0, 0, 0, 0])
    return snapshot.Snapshot(n=n, r1=39, r2=12, attempt=0, seed=0, attempt_seed=0,
                             records=[a, zero.copy(), zero.copy()],
                             child_targets=[np.zeros(w32, dtype=np.uint32) for _ in range(3)],
                             root_target=np.zeros(w32, dtype=np.uint32))
