"""Shared test setup. GPU tests carry @pytest.mark.gpu; everything else runs on a CPU-only host."""
import os
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """The library and the CPU checkers are built in-tree before any test runs."""
    from ssblasex_b200 import build as B
    B.build()
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "-s"], check=True)
    yield


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "golden_cases.npz")
