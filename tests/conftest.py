"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on any machine (oracle vs the reference's known answers,
host logic, ABI exports); `-m gpu` needs a B200 and calls the CUDA library
through its C ABI, checking it against the CPU oracle.
"""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a)")


@pytest.fixture(scope="session")
def ctx():
    from cenote_b200 import Context

    c = Context(0)
    yield c
    c.close()
