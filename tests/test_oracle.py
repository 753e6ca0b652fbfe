"""The oracle itself, pinned before it is trusted (CPU only).

* the C restatement (oracle/xted_oracle.c) reproduces every golden distance,
  which were produced by the reference X-TED_CPU built from its own sources;
* the reference library (oracle/_ref) agrees with the restatement;
* the independent brute-force recursion agrees on small trees;
* metric properties of unit-cost TED hold on the restatement.
"""
import random

import numpy as np
import pytest

import oracle
from oracle import brute
from xted import gen, trees


def test_restatement_matches_reference_goldens_datasets(golden_datasets):
    small = [c for c in golden_datasets if max(len(c[1]), len(c[2])) <= 2000]
    assert len(small) >= 35
    for name, a, b, d in small:
        assert oracle.distance(a, b) == d, name


def test_restatement_matches_reference_goldens_synthetic(golden_synthetic):
    assert len(golden_synthetic) > 200
    for name, a, b, d in golden_synthetic:
        assert oracle.distance(a, b) == d, name


def test_goldens_match_reference_cli_values(golden_datasets):
    got = {name: d for name, _, _, d in golden_datasets}
    # tree pair (0,1) of the sampled datasets, as the reference CLI reports them
    assert got["Sampled_Dataset/1_Swissport/swissport_nodes_1000.txt"] == 767
    assert got["Sampled_Dataset/2_Python/python_nodes_1000.txt"] == 1103
    assert got["Sampled_Dataset/4_DBLP/dblp_nodes_900.txt"] == 653
    assert got["Sampled_Dataset/3_Bolzano/bolzano_nodes.txt"] == 1
    assert got["Sampled_Dataset_Extra_Large_Trees/synthetic/6000_nodes/synthetic_nodes_6000.txt"] == 7334


def _rand_tree(rng, n, alpha):
    parent = [-1] + [rng.randrange(0, i) for i in range(1, n)]
    adj = [[] for _ in range(n)]
    for v in range(1, n):
        adj[parent[v]].append(v)
    # random sibling order, then renumber in preorder
    for ch in adj:
        rng.shuffle(ch)
    order, st = [], [0]
    while st:
        v = st.pop()
        order.append(v)
        st.extend(reversed(adj[v]))
    new = {v: k for k, v in enumerate(order)}
    labels = [0] * n
    out = [[] for _ in range(n)]
    for v in range(n):
        labels[new[v]] = rng.randrange(alpha)
        out[new[v]] = [new[c] for c in adj[v]]
    return trees.from_adjacency(labels, out)


def test_brute_force_agrees_small():
    rng = random.Random(11)
    for _ in range(250):
        a = _rand_tree(rng, rng.randint(1, 9), rng.randint(1, 4))
        b = _rand_tree(rng, rng.randint(1, 9), rng.randint(1, 4))
        assert oracle.distance(a, b) == brute.distance(a, b)
    brute.clear_cache()


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_reference_library_agrees_with_restatement():
    rng = random.Random(5)
    for _ in range(40):
        a = _rand_tree(rng, rng.randint(1, 120), rng.randint(1, 30))
        b = _rand_tree(rng, rng.randint(1, 120), rng.randint(1, 30))
        d, _ = oracle.ref_distance(a, b, num_threads=2)
        assert d == oracle.distance(a, b)


def test_empty_tree_rules():
    e = trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))
    t = gen.tree("random", 17, 3)
    assert oracle.distance(e, t) == 17  # X-TED_CPU/TED.cpp:181-183
    assert oracle.distance(t, e) == 17  # X-TED_CPU/TED.cpp:184-186
    assert oracle.distance(e, e) == 0


def test_metric_properties():
    rng = random.Random(9)
    ts = [_rand_tree(rng, rng.randint(1, 40), 5) for _ in range(12)]
    for i, a in enumerate(ts):
        assert oracle.distance(a, a) == 0
        for b in ts[i + 1:]:
            d = oracle.distance(a, b)
            assert d == oracle.distance(b, a)
            assert abs(len(a) - len(b)) <= d <= len(a) + len(b)
            assert d == oracle.distance(trees.mirror(a), trees.mirror(b))
    for a, b, c in zip(ts, ts[1:], ts[2:]):
        assert oracle.distance(a, c) <= oracle.distance(a, b) + oracle.distance(b, c)


def test_batch_matches_single():
    pairs = [(gen.tree("random", 40 + k, k), gen.tree("deep", 30 + 2 * k, 100 + k)) for k in range(8)]
    got = oracle.distance_batch(pairs, nthreads=3)
    assert list(got) == [oracle.distance(a, b) for a, b in pairs]
