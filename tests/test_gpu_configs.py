"""Parity on the benchmark workloads themselves (needs a B200).

Reference X-TED_CPU distances (tests/golden/configs.json.gz) for the
1,000-node wide-shallow vs deep-narrow pair, the 20,000-node random-recursive
and caterpillar pairs (the multi-block path), every one of the 4,096 pairs of
the headline mixed batch, and 8 top-10 serving queries over the 1,000-tree
serving corpus. Integer DP: bit-exact (tolerance 0).
"""
import numpy as np
import pytest

from conftest import topk_from_distances
import xted
from xted import gen

pytestmark = pytest.mark.gpu


def _singles(golden_configs):
    return {c["name"]: c["distance"] for c in golden_configs["singles"]}


def test_pair_1000_wide_vs_deep(ctx, golden_configs):
    a, b = gen.single_pair_1000()
    assert ctx.distance(a, b) == _singles(golden_configs)["single1000"]


def test_pairs_20000_match_reference(golden_configs):
    """Both 20,000-node pairs in one batch, default options (striped
    multi-block units), and the caterpillar pair alone."""
    want = _singles(golden_configs)
    r = gen.single_pair_20000(shape="random")
    c = gen.single_pair_20000(shape="caterpillar")
    with xted.Context() as ctx:
        got = ctx.distance_batch([r, c])
        assert int(got[0]) == want["single20000_random"]
        assert int(got[1]) == want["single20000_caterpillar"]
        assert ctx.distance(*c) == want["single20000_caterpillar"]


def test_mixed_batch_4096_all_pairs(golden_configs):
    g = golden_configs["batch4096"]
    pairs = gen.mixed_batch(g["npairs"], seed=g["seed"])
    want = np.array(g["distances"], np.int32)
    with xted.Context() as ctx:
        got = ctx.distance_batch(pairs)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, [(int(i), int(got[i]), int(want[i])) for i in bad[:8]]
        ctx.prepare_batch(pairs)
        for _ in range(2):  # direct run, then the captured graph's replay
            assert np.array_equal(ctx.run_prepared(), want)


def test_serving_corpus_1000_top10(golden_configs):
    s = golden_configs["serve"]
    corpus = gen.corpus(s["ntrees"], seed=s["corpus_seed"])
    queries = gen.corpus(64, seed=s["query_seed"])[:s["nqueries"]]
    with xted.Context() as ctx:
        ctx.corpus_load(corpus)
        tickets = [ctx.query_submit(q, 10) for q in queries]  # all in flight together
        for qi, t in enumerate(tickets):
            ids, dists, _, _ = ctx.query_wait(t, timeout_s=120.0)
            want_ids, want_d = topk_from_distances(s["distances"][qi], 10)
            assert ids.tolist() == want_ids and dists.tolist() == want_d, qi
        # the batch path on the same pairs: every distance, not only the top 10
        got = ctx.distance_batch([(q, t) for q in queries[:2] for t in corpus])
        assert got.tolist() == s["distances"][0] + s["distances"][1]
