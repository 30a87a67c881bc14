import shutil
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
TESTS = ROOT / "tests"
GOLDEN = TESTS / "golden"
for p in (str(ROOT), str(TESTS)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    return sorted(p.name for p in GOLDEN.iterdir() if (p / "golden.npz").exists())


@pytest.fixture
def golden_case(tmp_path):
    """Copies tests/golden/<name> (inputs + reference outputs) to a scratch dir."""
    def make(name: str) -> Path:
        dst = tmp_path / name
        shutil.copytree(GOLDEN / name, dst)
        return dst
    return make
