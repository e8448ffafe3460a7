import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    return load


def rel_err(a, b, floor_frac=1e-6):
    """|a-b| / max(|b|, floor) per element, the floor being floor_frac of the
    column's median magnitude (so exact zeros and sign changes do not
    dominate).  Columns along the last axis."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    med = np.median(np.abs(b), axis=0)
    floor = np.maximum(floor_frac * med, 1e-300)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)
