import json
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU-side parity cases")


def load_golden(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


def hx(value: str) -> int:
    return int(value, 16)


@pytest.fixture(scope="session")
def golden():
    return load_golden
