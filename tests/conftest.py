import gzip
import json
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "x-ted_b200"))

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) device")


def load_golden(name):
    """Golden cases: list of (name, tree_a, tree_b, distance)."""
    from xted.trees import from_parent
    with gzip.open(os.path.join(GOLDEN, name), "rt") as f:
        data = json.load(f)
    out = []
    for c in data["cases"]:
        a = from_parent(c["a"]["labels"], c["a"]["parent"])
        b = from_parent(c["b"]["labels"], c["b"]["parent"])
        out.append((c["name"], a, b, int(c["distance"])))
    return out


@pytest.fixture(scope="session")
def golden_datasets():
    return load_golden("datasets.json.gz")


@pytest.fixture(scope="session")
def golden_synthetic():
    return load_golden("synthetic.json.gz")


@pytest.fixture(scope="session")
def ctx():
    import xted
    c = xted.Context()
    yield c
    c.close()
