"""General edit costs (needs a B200): delete, insert and rename costs other
than the reference's unit costs, on every executor, against the oracle's C
restatement run with the same costs and against the brute-force forest
recursion. The recurrence sites generalised are those of
X-TED_CPU/parallel_computing.cpp:17-25 (borders) and :31-39 (tree and forest
cells). Integer DP: bit-exact (tolerance 0).
"""
import random

import numpy as np
import pytest

import oracle
from oracle import brute
import xted
from xted import gen, trees

pytestmark = pytest.mark.gpu

COSTS = [(1, 1, 1), (2, 3, 1), (3, 1, 4), (1, 2, 5), (0, 1, 1), (4, 4, 0), (5, 2, 3)]


def _rand_pairs(rng, n, sizes_a, sizes_b, alpha=4):
    shapes = ["random", "wide", "deep", "caterpillar"]
    return [(gen.tree(rng.choice(shapes), rng.choice(sizes_a), rng.randrange(1 << 30), "uniform", alpha),
             gen.tree(rng.choice(shapes), rng.choice(sizes_b), rng.randrange(1 << 30), "uniform", alpha))
            for _ in range(n)]


@pytest.mark.parametrize("costs", COSTS)
def test_costs_brute_force_small(costs):
    rng = random.Random(hash(costs) & 0xffff)
    pairs = _rand_pairs(rng, 120, [0, 1, 2, 3, 5, 8, 10], [0, 1, 2, 4, 7, 9], alpha=3)
    with xted.Context(costs=costs) as c:
        got = c.distance_batch(pairs)
    for (a, b), d in zip(pairs, got):
        assert d == brute.distance(a, b, costs), (costs, a.n, b.n)
    brute.clear_cache()


@pytest.mark.parametrize("costs", COSTS[1:])
@pytest.mark.parametrize("narrow_width,run_rows,half_width", [(0, 5, 0), (7, 3, 100), (32, 64, 0), (256, 17, -1),
                                                              (256, 64, 0)])
def test_costs_every_executor(costs, narrow_width, run_rows, half_width):
    """Warp-narrow of each width class, half-block and whole-block units,
    forced, in both decompositions."""
    rng = random.Random(narrow_width * 31 + run_rows + half_width + costs[0] * 7 + costs[2])
    pairs = _rand_pairs(rng, 16, [1, 2, 30, 90, 200, 420], [1, 3, 50, 130, 300, 700, 1100])
    want = [oracle.distance(a, b, costs) for a, b in pairs]
    for orientation in (xted.ORIENT_RIGHT, xted.ORIENT_LEFT):
        with xted.Context(orientation=orientation, narrow_width=narrow_width, run_rows=run_rows,
                          half_width=half_width, costs=costs) as c:
            assert list(c.distance_batch(pairs)) == want


@pytest.mark.parametrize("costs", [(2, 3, 1), (1, 2, 5)])
def test_costs_wide_and_striped_paths(costs):
    """Column segments wider than 2,048: the generic one-block wide path
    (stripes off) and the striped multi-block path (forced on every wide unit)."""
    a = gen.tree("caterpillar", 2300, 11, "uniform", 8)
    b = gen.tree("caterpillar", 2293, 12, "uniform", 8)
    r = gen.tree("random", 2300, 13, "uniform", 8)
    pairs = [(a, b), (r, a), (b, r)]
    want = [oracle.distance(x, y, costs) for x, y in pairs]
    for smc in (-1, 1):
        with xted.Context(stripe_min_cells=smc, costs=costs) as c:
            assert list(c.distance_batch(pairs)) == want, smc


def test_costs_asymmetric_matrix_and_empty_trees():
    """With delete != insert TED is not symmetric: the all-pairs matrix holds
    both orders; an empty tree costs the other tree's inserts or deletes."""
    costs = (3, 1, 2)
    rng = random.Random(77)
    ts = [gen.tree(rng.choice(["random", "deep"]), rng.randint(1, 60), 500 + i, "uniform", 5) for i in range(7)]
    e = trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))
    ts.append(e)
    with xted.Context(costs=costs) as c:
        M = c.distance_matrix(ts)
        for i in range(len(ts)):
            for j in range(len(ts)):
                assert M[i, j] == (0 if i == j else oracle.distance(ts[i], ts[j], costs)), (i, j)
        assert c.distance(e, ts[0]) == ts[0].n * 1 and c.distance(ts[0], e) == ts[0].n * 3
        # a pair whose weighted size exceeds the row scan's key range is refused
        big = gen.tree("random", 40000, 5)
        with pytest.raises(xted.XtedError) as ei:
            c.distance(big, big)
        assert ei.value.code == xted.XTED_EINVAL


def test_costs_serving_topk():
    """Serving under costs answers TED(query, corpus tree) (delete query
    nodes, insert corpus nodes) with exact top-k, with and without pruning
    (the bounds are scaled to the costs)."""
    costs = (2, 1, 3)
    rng = random.Random(5)
    corpus = [gen.tree(["random", "wide", "deep", "caterpillar"][i % 4], rng.randint(1, 120), 600 + i, "zipf", 9)
              for i in range(60)]
    queries = [gen.tree("random", rng.randint(1, 110), 700 + i, "zipf", 9) for i in range(4)] + [corpus[7]]
    with xted.Context(costs=costs) as c:
        c.corpus_load(corpus)
        for prune in (0, 1, 2):
            c.serve_options(prune=prune, first_round=1)
            tickets = [c.query_submit(q, 6) for q in queries]
            for q, t in zip(queries, tickets):
                ids, dists, _, _ = c.query_wait(t, timeout_s=60)
                d = [oracle.distance(q, x, costs) for x in corpus]
                want = sorted(range(len(corpus)), key=lambda i: (d[i], i))[:6]
                assert ids.tolist() == want and dists.tolist() == [d[i] for i in want], prune
