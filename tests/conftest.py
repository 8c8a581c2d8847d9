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
