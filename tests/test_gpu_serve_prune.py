"""Serving with exact top-k pruning (label and preorder-sequence bounds, two
rounds per query): the same answers as computing every pair, equal to the
oracle's ranking, with fewer pairs computed. A module of its own, so that it
runs on a fresh serving context after the other serving tests have closed
theirs. All through the C ABI.
"""
import numpy as np
import pytest

import oracle
import xted
from xted import gen, trees

pytestmark = pytest.mark.gpu

SHAPES = ("random", "wide", "deep", "caterpillar")


def _corpus(n, seed, lo=1, hi=150):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(rng.integers(lo, hi + 1))
        out.append(gen.tree(SHAPES[i % 4], size, seed * 1000 + i, "zipf", 12))
    return out


def _exact_topk(q, corpus, k):
    d = np.array([oracle.distance(q, t) for t in corpus])
    order = sorted(range(len(corpus)), key=lambda i: (d[i], i))[:k]
    ids = np.full(k, -1, np.int32)
    ds = np.full(k, -1, np.int32)
    ids[:len(order)] = order
    ds[:len(order)] = d[order]
    return ids, ds


def _relabel(t, frac, seed):
    rng = np.random.default_rng(seed)
    lab = np.array(t.labels, np.int32, copy=True)
    m = rng.random(len(lab)) < frac
    lab[m] = rng.integers(0, 40, int(m.sum()))
    return trees.Tree(lab, np.array(t.off, np.int32), np.array(t.idx, np.int32))


@pytest.mark.timeout(300)
def test_pruned_topk_is_exact():
    """Exact top-k pruning by the label bound: the same answers as computing
    every pair, equal to the oracle's ranking, with fewer pairs computed.
    Queries are near-copies of corpus trees (the case pruning is for), a
    fresh tree, both bounds, and first-round sizes that force a second round."""
    corpus = _corpus(300, 41, 1, 150)
    queries = [_relabel(corpus[i], f, 50 + i) for i, f in ((3, 0.0), (77, 0.05), (150, 0.2), (299, 0.5))]
    queries.append(gen.tree("random", 120, 4242, "zipf", 12))
    with xted.Context(device=0) as ctx:
        ctx.corpus_load(corpus)
        res = {}
        modes = {"full": (0, 0), "label": (1, 0), "pruned": (2, 0), "tight": (2, 1)}
        for mode, (prune, first) in modes.items():
            ctx.serve_options(prune=prune, first_round=first)
            st0 = ctx.serve_stats()
            tickets = [(q, k, ctx.query_submit(q, k)) for q in queries for k in (1, 5, 17)]
            res[mode] = [ctx.query_wait(t, timeout_s=60)[:2] for _, _, t in tickets]
            ctx.serve_drain()
            st1 = ctx.serve_stats()
            res[mode + "_stats"] = {key: st1[key] - st0[key] for key in st1}
        for mode in ("label", "pruned", "tight"):
            for a, b in zip(res["full"], res[mode]):
                assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), mode
        n_q = len(queries) * 3
        assert res["full_stats"]["pairs_pruned"] == 0 and res["full_stats"]["pairs"] == n_q * len(corpus)
        for mode in ("label", "pruned", "tight"):
            assert res[mode + "_stats"]["pairs"] + res[mode + "_stats"]["pairs_pruned"] == n_q * len(corpus)
        assert res["pruned_stats"]["pairs_pruned"] > res["label_stats"]["pairs_pruned"] > 0
        assert res["tight_stats"]["second_rounds"] > 0
        # against the oracle, for one query per k
        for (ids, ds), (q, k) in zip(res["pruned"][::4], [(q, k) for q in queries for k in (1, 5, 17)][::4]):
            want_ids, want_ds = _exact_topk(q, corpus, k)
            assert np.array_equal(ids, want_ids) and np.array_equal(ds, want_ds)
