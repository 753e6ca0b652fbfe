"""The benchmark workloads are the ones the reference distances were computed on.

tests/golden/configs.json.gz holds reference X-TED_CPU distances for the
1,000-node pair, both 20,000-node pairs, all 4,096 pairs of the mixed batch and
8 serving queries against the 1,000-tree corpus, with a hash of every tree.
These CPU tests require the generators (the C one behind the library and the
pure-Python one the benchmark's reference arm uses) to rebuild exactly those
trees, so the GPU parity tests and the benchmark's parity check compare
against the right numbers.
"""
import numpy as np

from conftest import tree_hash
from xted import gen, synth


def test_single_pairs_hash_to_the_fixture(golden_configs):
    byname = {c["name"]: c for c in golden_configs["singles"]}
    for name, (a, b) in (("single1000", gen.single_pair_1000()),
                         ("single20000_caterpillar", gen.single_pair_20000(shape="caterpillar")),
                         ("single20000_random", gen.single_pair_20000(shape="random"))):
        c = byname[name]
        assert (tree_hash(a), tree_hash(b)) == (c["a"], c["b"]), name
        assert (a.n, b.n) == (c["m"], c["n"])


def test_mixed_batch_hashes_to_the_fixture(golden_configs):
    g = golden_configs["batch4096"]
    pairs = gen.mixed_batch(g["npairs"], seed=g["seed"])
    got = [[tree_hash(a), tree_hash(b)] for a, b in pairs]
    assert got == g["hashes"]
    assert len(g["distances"]) == g["npairs"]


def test_python_generator_rebuilds_sampled_pairs(golden_configs):
    """The reference arm of the benchmark builds its sample with xted.synth
    (no CUDA library): those pairs must be the fixture's pairs."""
    g = golden_configs["batch4096"]
    which = list(range(0, g["npairs"], 128))
    for p, (a, b) in zip(which, synth.mixed_pairs(g["npairs"], g["seed"], which)):
        assert [tree_hash(a), tree_hash(b)] == g["hashes"][p], p


def test_serving_workload_hashes_to_the_fixture(golden_configs):
    s = golden_configs["serve"]
    corpus = gen.corpus(s["ntrees"], seed=s["corpus_seed"])
    queries = gen.corpus(64, seed=s["query_seed"])[:s["nqueries"]]
    assert [tree_hash(t) for t in corpus] == s["corpus_hashes"]
    assert [tree_hash(q) for q in queries] == s["query_hashes"]
    assert np.array(s["distances"]).shape == (s["nqueries"], s["ntrees"])


def test_python_generator_equals_c_generator():
    """Every shape and label kind, sizes 0 to 2,000: identical arrays."""
    for shape in synth.SHAPES:
        for n in (0, 1, 2, 3, 7, 10, 11, 57, 100, 203, 999, 2000):
            for kind, alpha in (("uniform", 26), ("zipf", 1000), ("uniform", 1), ("zipf", 3)):
                a = gen.tree(shape, n, 777 + n, kind, alpha)
                b = synth.tree(shape, n, 777 + n, kind, alpha)
                assert np.array_equal(a.labels, b.labels), (shape, n, kind)
                assert np.array_equal(a.off, b.off), (shape, n, kind)
                assert np.array_equal(a.idx, b.idx), (shape, n, kind)
