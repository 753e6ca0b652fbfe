"""Serving: a resident corpus, exact top-k queries, continuous batching.

Every query's top-k is checked against the oracle's distances (exact, ties by
lower corpus index), and each query's result must be the same when it runs
alone as when it runs in a mix with others (continuous batching must not change
an answer). All through the C ABI.
"""
import time

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


def _empty():
    return trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))


def _exact_topk(q, corpus, k):
    d = np.array([oracle.distance(q, t) for t in corpus])
    order = sorted(range(len(corpus)), key=lambda i: (d[i], i))[:k]
    ids = np.full(k, -1, np.int32)
    ds = np.full(k, -1, np.int32)
    ids[:len(order)] = order
    ds[:len(order)] = d[order]
    return ids, ds


@pytest.fixture(scope="module")
def setup():
    corpus = _corpus(23, 3) + [_empty()]
    queries = _corpus(8, 11, 1, 160)
    ctx = xted.Context(device=0)
    ctx.corpus_load(corpus)
    yield ctx, corpus, queries
    ctx.close()


@pytest.mark.timeout(300)
def test_topk_full_ranking_matches_oracle(setup):
    ctx, corpus, queries = setup
    k = len(corpus)  # the whole ranking: every distance is checked
    tickets = [ctx.query_submit(q, k) for q in queries]
    for q, t in zip(queries, tickets):
        ids, ds, _, _ = ctx.query_wait(t, timeout_s=120)
        want_ids, want_ds = _exact_topk(q, corpus, k)
        assert np.array_equal(ds, want_ds)
        assert np.array_equal(ids, want_ids)
    ctx.serve_drain()


@pytest.mark.timeout(300)
def test_alone_equals_in_the_mix(setup):
    ctx, corpus, queries = setup
    alone = []
    for q in queries:
        t = ctx.query_submit(q, 10)
        ids, ds, _, _ = ctx.query_wait(t, timeout_s=120)
        alone.append((ids, ds))
        time.sleep(0.01)  # let the launch go idle between queries: exercises relaunch
    tickets = [ctx.query_submit(q, 10) for q in queries for _ in range(3)]
    mixed = [ctx.query_wait(t, timeout_s=120) for t in tickets]
    for i, (ids, ds, _, _) in enumerate(mixed):
        a_ids, a_ds = alone[i // 3]
        assert np.array_equal(ids, a_ids) and np.array_equal(ds, a_ds)
    st = ctx.serve_stats()
    assert st["launches"] >= 2 and st["queries"] >= len(queries) * 4


@pytest.mark.timeout(300)
def test_more_queries_than_slots(setup):
    ctx, corpus, queries = setup
    qs = _corpus(40, 21, 1, 120)
    tickets = [ctx.query_submit(q, 5) for q in qs]
    got = [ctx.query_wait(t, timeout_s=200) for t in tickets]
    for q, (ids, ds, qms, tms) in zip(qs, got):
        want_ids, want_ds = _exact_topk(q, corpus, 5)
        assert np.array_equal(ids, want_ids) and np.array_equal(ds, want_ds)
        assert 0 <= qms <= tms
    ctx.serve_drain()


@pytest.mark.timeout(120)
def test_edge_queries_and_errors(setup):
    ctx, corpus, _ = setup
    # empty query: distance = corpus tree size
    ids, ds, _, _ = ctx.query_wait(ctx.query_submit(_empty(), 3), timeout_s=60)
    sizes = [len(t) for t in corpus]
    order = sorted(range(len(corpus)), key=lambda i: (sizes[i], i))[:3]
    assert list(ids) == order and list(ds) == [sizes[i] for i in order]
    # k beyond the corpus: trailing -1
    one = gen.tree("random", 1, 5)
    ids, ds, _, _ = ctx.query_wait(ctx.query_submit(one, len(corpus) + 2), timeout_s=60)
    assert list(ids[-2:]) == [-1, -1] and list(ds[-2:]) == [-1, -1]
    with pytest.raises(xted.XtedError) as e:
        ctx.query_submit(gen.tree("random", xted._lib.XTED_SERVE_MAX_QUERY + 1, 1), 3)
    assert e.value.code == xted.XTED_EINVAL
    with pytest.raises(xted.XtedError) as e:
        ctx.query_submit(one, 0)
    assert e.value.code == xted.XTED_EINVAL
    with pytest.raises(xted.XtedError) as e:
        ctx.query_poll(987654321)
    assert e.value.code == xted.XTED_ENOTFOUND


@pytest.mark.timeout(300)
def test_batch_calls_after_serving_and_reload(setup):
    ctx, corpus, queries = setup
    ctx.serve_drain()
    pairs = [(queries[0], corpus[i]) for i in range(5)]
    got = ctx.distance_batch(pairs)
    assert list(got) == [oracle.distance(a, b) for a, b in pairs]
    # a new corpus replaces the old one
    small = _corpus(5, 99, 1, 60)
    ctx.corpus_load(small)
    ids, ds, _, _ = ctx.query_wait(ctx.query_submit(queries[1], 5), timeout_s=60)
    want_ids, want_ds = _exact_topk(queries[1], small, 5)
    assert np.array_equal(ids, want_ids) and np.array_equal(ds, want_ds)
    ctx.corpus_load(corpus)  # restore for any later test of the module

