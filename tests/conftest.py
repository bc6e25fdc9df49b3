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
    config.addinivalue_line("markers", "late: runs after all other tests (a GPU test that has not "
                                       "yet run on a B200)")


def pytest_collection_modifyitems(config, items):
    """Tests marked `late` run after the others, in their own order, so that
    with -x a failure among them cannot hide the results of the rest."""
    items[:] = ([i for i in items if i.get_closest_marker("late") is None]
                + [i for i in items if i.get_closest_marker("late") is not None])


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
