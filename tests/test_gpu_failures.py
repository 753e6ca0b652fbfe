"""Failure handling (needs a B200): every failure is bounded, reported as an
error code and leaves the context usable. Nothing here faults, traps or hangs
a GPU: the faults are made on the host (xted_test_fault holds one pair's first
level back, so a bounded wait runs out; mem_limit refuses an allocation).

The reference has no such handling: it prints CUDA errors and carries on or
exits (X-TED_GPU/utils/cuda_utils.h:35-41, X-TED_GPU/help.h:6-14), and its
spin barriers wait without bound (X-TED_GPU/parallel_X_TED.cu:68-91, 128-157).
"""
import time

import numpy as np
import pytest

import oracle
import xted
from xted import gen, trees

pytestmark = pytest.mark.gpu


def _pairs(n, seed, hi=300):
    return gen.mixed_batch(n, seed=seed, lo=20, hi=hi)


def test_batch_wait_runs_out_then_context_recovers():
    """A batch whose pair 0 never becomes ready: the persistent launch's
    bounded idle wait (0.3 s) runs out, the call returns XTED_ETIMEOUT in
    bounded time, and the next batch on the same context is exact."""
    pairs = _pairs(24, 901)
    with xted.Context(wait_timeout_s=0.3) as ctx:
        ctx.test_fault(xted.XTED_FAULT_HOLD_PAIR)
        t0 = time.monotonic()
        with pytest.raises(xted.XtedError) as ei:
            ctx.distance_batch(pairs)
        assert ei.value.code == xted.XTED_ETIMEOUT
        assert time.monotonic() - t0 < 30.0
        got = ctx.distance_batch(pairs)
        assert np.array_equal(got, oracle.distance_batch(pairs, nthreads=4))
        # and a prepared batch with its captured graph on the same context
        ctx.prepare_batch(pairs)
        for _ in range(2):
            assert np.array_equal(ctx.run_prepared(), got)


def test_mem_limit_refuses_then_smaller_batch_runs():
    """mem_limit below what a batch's distance tables need: XTED_ENOMEM, no
    launch; a batch that fits the same limit then runs exactly."""
    big = [gen.single_pair_20000(shape="caterpillar")]  # 1.6 GB of tables
    small = _pairs(8, 902, hi=120)
    with xted.Context(mem_limit=256 << 20) as ctx:
        with pytest.raises(xted.XtedError) as ei:
            ctx.distance_batch(big)
        assert ei.value.code == xted.XTED_ENOMEM
        assert np.array_equal(ctx.distance_batch(small), oracle.distance_batch(small, nthreads=4))


def _chain(n, label0):
    """A path of n nodes (labels label0, label0+1, ...)."""
    adj = [[i + 1] for i in range(n - 1)] + [[]]
    return trees.from_adjacency([label0 + i for i in range(n)], adj)


def test_serving_query_too_large_is_refused():
    """Serving admission by distance-table bytes: with mem_limit = 16 MB the
    table pool holds 2 M int32; a 1,200-node query against a corpus of 2,000
    nodes needs 2.4 M and fails with XTED_ENOMEM at admission (pruning off:
    one round over every tree), while a small query on the same context is
    answered exactly."""
    corpus = [gen.tree("random", 100, 700 + i, "zipf", 20) for i in range(20)]
    with xted.Context(mem_limit=16 << 20) as ctx:
        ctx.corpus_load(corpus)
        ctx.serve_options(prune=0)
        big = gen.tree("random", 1200, 77, "zipf", 20)
        with pytest.raises(xted.XtedError) as ei:
            ctx.query_wait(ctx.query_submit(big, 5), timeout_s=60)
        assert ei.value.code == xted.XTED_ENOMEM
        q = gen.tree("wide", 80, 78, "zipf", 20)
        ids, dists, _, _ = ctx.query_wait(ctx.query_submit(q, 5), timeout_s=60)
        d = [oracle.distance(q, t) for t in corpus]
        want = sorted(range(len(corpus)), key=lambda i: (d[i], i))[:5]
        assert ids.tolist() == want and dists.tolist() == [d[i] for i in want]


def test_serving_second_round_that_cannot_fit_fails():
    """Exact top-k pruning runs a query in two rounds; the second covers every
    tree whose bound may still beat the k-th distance found and can need more
    room than the first. Here round 1 (the 40 trees of lowest bound, k = 10)
    fits the 1.5 M-int32 table pool and round 2 (the other 60 trees: every
    distance exceeds the common bound) cannot: the query fails with
    XTED_ENOMEM instead of waiting for room forever, and the next query runs."""
    corpus = [gen.tree("random", 150, 800 + i, "uniform", 30) for i in range(100)]
    q = _chain(200, 1000)  # labels shared with no corpus tree: every label bound is 200
    with xted.Context(mem_limit=12 << 20) as ctx:  # table pool 1.5 M int32
        ctx.corpus_load(corpus)
        ctx.serve_options(prune=1, first_round=1)
        with pytest.raises(xted.XtedError) as ei:
            ctx.query_wait(ctx.query_submit(q, 10), timeout_s=120)
        assert ei.value.code == xted.XTED_ENOMEM
        q2 = corpus[5]
        ids, dists, _, _ = ctx.query_wait(ctx.query_submit(q2, 1), timeout_s=60)
        assert ids.tolist() == [5] and dists.tolist() == [0]


def test_serving_query_whose_work_never_arrives_fails():
    """A serving query with one pair held back: its launch goes idle and
    ends without finishing the query, which then fails with XTED_ETIMEOUT
    instead of waiting forever; the next query on the same context is exact,
    and closing the context returns."""
    corpus = [gen.tree("deep", 60, 900 + i, "zipf", 10) for i in range(30)]
    ctx = xted.Context()
    try:
        ctx.corpus_load(corpus)
        ctx.serve_options(prune=0)
        ctx.test_fault(xted.XTED_FAULT_HOLD_PAIR)
        q = gen.tree("random", 50, 91, "zipf", 10)
        t0 = time.monotonic()
        with pytest.raises(xted.XtedError) as ei:
            ctx.query_wait(ctx.query_submit(q, 3), timeout_s=60)
        assert ei.value.code == xted.XTED_ETIMEOUT
        assert time.monotonic() - t0 < 30.0
        ids, dists, _, _ = ctx.query_wait(ctx.query_submit(q, 3), timeout_s=60)
        d = [oracle.distance(q, t) for t in corpus]
        want = sorted(range(len(corpus)), key=lambda i: (d[i], i))[:3]
        assert ids.tolist() == want and dists.tolist() == [d[i] for i in want]
        with pytest.raises(xted.XtedError) as ei:  # the failure is reported once by drain
            ctx.serve_drain()
        assert ei.value.code == xted.XTED_ETIMEOUT
        ctx.serve_drain()
    finally:
        t0 = time.monotonic()
        ctx.close()
        assert time.monotonic() - t0 < 30.0
