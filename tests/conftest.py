"""Shared test configuration.

Markers:
  gpu   needs a CUDA device (run with -m gpu on a B200)
  slow  long runs (enable with --runslow)
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_addoption(parser):
    parser.addoption("--runslow", action="store_true", default=False, help="also run slow tests")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long runs (enable with --runslow)")


def pytest_collection_modifyitems(config, items):
    if config.getoption("--runslow"):
        return
    skip = pytest.mark.skip(reason="slow test: use --runslow")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_mod():
    """The oracle (test infrastructure): the C restatement and, where it was
    built, the reference compiled from its own sources."""
    from oracle import oracle
    oracle.port_lib()
    return oracle
