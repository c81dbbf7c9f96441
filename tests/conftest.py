import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_cases():
    return json.load(open(os.path.join(GOLDEN, "cases.json")))


def golden_arrays(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def golden_graph(name, case=None):
    import make_golden

    return make_golden.build_graph(make_golden.CASES[name][0])


def f64_hex(x) -> str:
    return "%016x" % np.float64(x).view(np.uint64)


def initial_labels_for(name, case, g):
    """Labels phase 2 starts from in the golden run (phase-1 output, or the stored labels_in)."""
    arr = golden_arrays(name)
    if case["labels_from"] == "phase1":
        return arr["labels1"]
    return arr["labels_in"]
