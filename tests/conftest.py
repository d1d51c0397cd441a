import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")


def load_golden(name):
    return np.load(GOLDEN / f"{name}.npz")


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


def grids_from_golden(d, i):
    kg = {a: d[f"c{i}_k{a}"] for a in "xyz"}
    rk = {"tan": {a: d[f"c{i}_tan_{a}"] for a in "xyz"}, "sin": {a: d[f"c{i}_sin_{a}"] for a in "xyz"}}
    return kg, rk


@pytest.fixture
def golden():
    return load_golden
