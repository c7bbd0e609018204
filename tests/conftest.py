"""Shared pytest configuration.

Markers
  gpu : needs a CUDA device (B200, sm_100a); deselect with -m "not gpu".
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O.Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = os.path.join(ROOT, "tests", "golden")
    return {name: dict(np.load(os.path.join(d, f"{name}.npz"))) for name in ("field_16", "field_12", "faces")}
