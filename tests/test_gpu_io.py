"""Dataset I/O and the drivers over it, on the GPU: the command-line tools on
reference-format files, the all-pairs matrix, and the bracket-notation pair
against the reference's distance."""
import gzip
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
import xted
from xted import gen, trees

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "x-ted_b200", "bin")


def _write_dataset(path_lab, path_adj, ts, strings):
    with open(path_lab, "w") as f:
        for s in strings:
            f.write("".join(x + " " for x in s) + "\n")
    with open(path_adj, "w") as f:
        for t in ts:
            f.write("[" + ", ".join("[" + ", ".join(str(c) for c in t.idx[t.off[v]:t.off[v + 1]]) + "]"
                                    for v in range(len(t))) + "]\n")


@pytest.fixture(scope="module")
def dataset(tmp_path_factory, golden_datasets):
    d = tmp_path_factory.mktemp("ds")
    name, a, b, dist = next(c for c in golden_datasets if "swissport_nodes_300" in c[0])
    extra = [gen.tree("random", 60, 7, "zipf", 20), gen.tree("deep", 80, 8, "zipf", 20)]
    ts = [a, b] + extra
    strings = [[f"s{x}" for x in t.labels.tolist()] for t in ts]
    _write_dataset(str(d / "n.txt"), str(d / "a.txt"), ts, strings)
    return str(d / "n.txt"), str(d / "a.txt"), ts, dist


def test_cli_gpu_and_cpu_named_tools(dataset):
    lab, adj, ts, dist = dataset
    out = subprocess.run([os.path.join(BIN, "X-TED_GPU"), lab, adj], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    ds = [int(l.split("=")[1]) for l in out.stdout.splitlines() if l.startswith("The distance =")]
    assert ds == [dist] * 20
    assert out.stdout.count("Measured time for total parallel execution =") == 20
    out = subprocess.run([os.path.join(BIN, "X-TED_CPU"), "8", lab, adj], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    ds = [int(l.split("=")[1]) for l in out.stdout.splitlines() if l.startswith("The distance =")]
    assert ds == [dist] * 20
    assert out.stdout.count("Total Time for Parallel Computing =") == 20


def test_cli_matrix(dataset):
    lab, adj, ts, _ = dataset
    out = subprocess.run([os.path.join(BIN, "X-TED_GPU"), "--matrix", lab, adj], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    m = np.array([[int(x) for x in l.split()] for l in out.stdout.splitlines()])
    loaded, _ = trees.load_dataset(lab, adj)
    want = np.array([[oracle.distance(x, y) for y in loaded] for x in loaded])
    assert np.array_equal(m, want)


def test_distance_matrix_chunks():
    ts = [gen.tree(s, n, 100 + k, "zipf", 12) for k, (s, n) in
          enumerate([("random", 40), ("wide", 90), ("deep", 70), ("caterpillar", 55), ("random", 1),
                     ("random", 120), ("wide", 30), ("deep", 64)])]
    ts.append(trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32)))
    want = np.array([[oracle.distance(a, b) for b in ts] for a in ts])
    with xted.Context() as c:
        for budget in (0, 5000):  # one chunk; a chunk every few pairs
            assert np.array_equal(c.distance_matrix(ts, pair_budget=budget), want)


def test_bracket_pair_matches_reference_distance():
    with gzip.open(os.path.join(REPO, "tests", "golden", "bracket.json.gz"), "rt") as f:
        cases = json.load(f)["cases"]
    with xted.Context() as c:
        for case in cases:
            intern = trees.Interner()
            ts = [trees.parse_bracket(l, intern)[0] for l in case["text"].split("\n") if l.strip()]
            assert c.distance(ts[0], ts[1]) == case["distance"], case["name"]
