"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on any machine (oracle against the golden fixtures, host
logic, library exports); `-m gpu` needs a CUDA device and checks the CUDA
path through the C ABI against the oracle.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
