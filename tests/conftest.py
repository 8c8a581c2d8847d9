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


def hexint(v):
    return int(v, 16) if isinstance(v, str) else int(v)
