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


def load_configs():
    """Reference distances of the benchmark workloads themselves (configs.json.gz,
    made by tests/golden/make_golden.py configs): trees given by generator seed
    plus a hash of their arrays, distances from the reference X-TED_CPU."""
    with gzip.open(os.path.join(GOLDEN, "configs.json.gz"), "rt") as f:
        return json.load(f)


def tree_hash(t):
    """First 16 hex digits of the SHA-256 of a tree's labels | off | idx (int32),
    the hash make_golden.py stores."""
    import hashlib

    import numpy as np
    h = hashlib.sha256()
    for arr in (t.labels, t.off, t.idx):
        h.update(np.ascontiguousarray(arr, dtype=np.int32).tobytes())
    return h.hexdigest()[:16]


def topk_from_distances(dist, k):
    """Exact top-k of one query: ascending distance, ties by lower corpus index."""
    order = sorted(range(len(dist)), key=lambda i: (dist[i], i))[:k]
    return [int(i) for i in order], [int(dist[i]) for i in order]


@pytest.fixture(scope="session")
def golden_configs():
    return load_configs()
