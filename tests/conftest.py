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


# reference FullTerStageTelemetry field -> device stats field, per stage
STAGES = {
    "binary": {"pairs": "l3_pairs", "modular": "l3_modular", "structural": "l3_structural_rejects",
               "distribution": "l3_distribution_rejects", "survivors": "l3_survivors",
               "fingerprint": "l2_fingerprint"},
    "middle": {"pairs": "l2_pairs", "modular": "l2_modular", "structural": "l2_structural_rejects",
               "distribution": "l2_distribution_rejects", "survivors": "l2_survivors",
               "fingerprint": "l1_fingerprint"},
    "root": {"pairs": "root_pairs", "modular": "root_modular",
             "structural": "root_structural_rejects", "distribution": "root_distribution_rejects",
             "survivors": "valid_roots", "deduplicated": "level0", "quotient_bits": "root_quotient_bits",
             "prefilter_bits": "root_prefilter_bits", "low_prefilter": "root_low_prefilter",
             "full_quotient_rejects": "root_full_quotient_rejects", "valid_roots": "valid_roots",
             "policy": "root_policy", "early_stopped": "root_early_stopped",
             "fingerprint": "l0_fingerprint"},
}


def hexint(v):
    return int(v, 16) if isinstance(v, str) else int(v)


def capture_from_records(n, r1, r2, lists):
    """A snapshot.Snapshot of a hand-built root capture: `lists` holds, per L1
    list, (ones, residue) pairs -- the coordinates whose digit is 1 and the
    residue as an integer mod 2^n; every child and root target is 0."""
    import numpy as np
    from tergpu import snapshot

    w64, w32 = (n + 63) // 64, (n + 31) // 32

    def record(ones, residue):
        pos = [0] * w64
        for i in ones:
            pos[i // 64] |= 1 << (i % 64)
        masks = np.array(pos + [0] * w64, dtype="<u8").view(np.uint8)
        words = [(residue >> (32 * k)) & 0xFFFFFFFF for k in range(w32)]
        return np.concatenate([masks, np.array(words, dtype="<u4").view(np.uint8)])

    records = [np.concatenate([record(o, r) for o, r in entries]) if entries else np.zeros(0, np.uint8)
               for entries in lists]
    return snapshot.Snapshot(n=n, r1=r1, r2=r2, attempt=0, seed=0, attempt_seed=0, records=records,
                             child_targets=[np.zeros(w32, dtype=np.uint32) for _ in range(3)],
                             root_target=np.zeros(w32, dtype=np.uint32))


def wide_quotient_capture():
    """The reference's Q = 69 truncation fixture (wide_quotient_root_capture,
    tests/full_ter_tests.cpp:769-803): n = 108, r1 = 39; list A holds the root
    parent (ones on coordinates 54..107) twice, with residues 0 and 2^103; lists
    B and C hold the zero vector; every target is 0.  Both A entries have
    quotient 0 on the low 64 bits; 2^103 >> 39 = 2^64 sets bit 64 of the second
    one's quotient, just outside a 64-bit window."""
    parent = range(54, 108)
    return capture_from_records(108, 39, 12, [[(parent, 0), (parent, 1 << 103)], [((), 0)], [((), 0)]])


def early_root_capture():
    """The reference's deterministic root-report fixture (early_root_capture,
    tests/full_ter_tests.cpp:423-453): n = 36, r1 = 12; list A holds the parents
    with ones on 18..35 and on 0..17, alternating, four entries; lists B and C
    hold four zero vectors each; residues and targets are 0.  Every one of the
    4 x 4 x 4 triples is an exact root, with two distinct parents."""
    first, second = range(18, 36), range(0, 18)
    zeros = [((), 0)] * 4
    return capture_from_records(36, 12, 3, [[(first, 0), (second, 0), (first, 0), (second, 0)],
                                            zeros, zeros])


def boundary_roots():
    """The tiled reporter's boundary cases (tests/tiled_q3report_tests.cpp:157-231),
    scaled from modulus 64 to 2^Q at
    the device's key widths: singleton lists whose pair sums land on 0, M - 1,
    M and 2M - 2 (M = 2^Q), and duplicated keys that keep their multiplicity.
    Yields (Q, lo[3], hi[3], expected triples) with list 2 holding
    d = tau - q_c, the expected count from exact integer arithmetic."""
    import numpy as np

    def lists(Q, a, b, c, tau):
        M = 1 << Q
        keys = [list(a), list(b), [(tau - v) % M for v in c]]
        lo = [np.array([k & (2**64 - 1) for k in ks], dtype=np.uint64) for ks in keys]
        hi = [np.array([k >> 64 for k in ks], dtype=np.uint8) for ks in keys]
        want = sum(1 for x in keys[0] for y in keys[1] for z in keys[2] if (x + y - z) % M == 0)
        return lo, hi, want

    for Q in (24, 47, 64, 69, 72):
        M = 1 << Q
        for a, b, c, tau in ((0, 0, 0, 0), (0, 0, 1, 0), (M - 1, 0, 1, 0), (M - 1, 1, 0, 0),
                             (M - 1, M - 1, 2, 0), (M - 1, M - 1, 1, M - 1), (M // 2, M // 2, 0, 0),
                             (M // 2, M // 2 - 1, 1, 0)):
            yield (Q,) + lists(Q, [a], [b], [c], tau)
        yield (Q,) + lists(Q, [7] * 3, [9] * 2, [M - 16] * 4, 0)
