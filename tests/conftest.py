"""Shared test set-up: the `gpu` marker and session fixtures.

Tests marked `gpu` need a CUDA device (they run the sm_100a kernels through
the C ABI); everything else runs on a CPU-only machine.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def golden_knn():
    data = np.load(GOLDEN / "knn_cases.npz")
    cases = {}
    for name in data["names"]:
        name = str(name)
        cases[name] = {key.split("/", 1)[1]: data[key] for key in data.files
                       if key.startswith(name + "/")}
    return cases


@pytest.fixture(scope="session")
def ctx():
    from photon_mapping_b200 import Context
    c = Context(0)
    yield c
    c.close()
