"""Parity of the CUDA path with the oracle, through the C ABI (needs a B200).

Integer min-plus arithmetic: every distance must match bit-exactly (tolerance 0).
"""
import random

import numpy as np
import pytest

import oracle
from oracle import brute
import xted
from xted import gen, trees

pytestmark = pytest.mark.gpu


def _rand_tree(rng, n, alpha, shape):
    if n == 0:
        return trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))
    adj = [[] for _ in range(n)]
    for i in range(1, n):
        if shape == 0:
            p = rng.randrange(i)
        elif shape == 1:
            p = rng.randrange(min(i, 8))
        else:
            p = max(0, i - 1 - rng.randrange(3))
        if rng.random() < 0.5:
            adj[p].append(i)
        else:
            adj[p].insert(0, i)
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


def test_single_pair_100_matches_oracle(ctx):
    a, b = gen.single_pair_100()
    assert ctx.distance(a, b) == oracle.distance(a, b)


def test_golden_datasets(ctx, golden_datasets):
    pairs = [(a, b) for _, a, b, _ in golden_datasets]
    want = [d for *_, d in golden_datasets]
    got = ctx.distance_batch(pairs)
    bad = [(golden_datasets[i][0], int(got[i]), want[i]) for i in range(len(want)) if got[i] != want[i]]
    assert not bad, bad[:5]


def test_golden_datasets_one_by_one(ctx, golden_datasets):
    for name, a, b, d in golden_datasets[:12]:
        assert ctx.distance(a, b) == d, name


def test_golden_synthetic(ctx, golden_synthetic):
    pairs = [(a, b) for _, a, b, _ in golden_synthetic]
    want = np.array([d for *_, d in golden_synthetic])
    got = ctx.distance_batch(pairs)
    assert np.array_equal(got, want), [(golden_synthetic[i][0], got[i], want[i])
                                       for i in np.nonzero(got != want)[0][:5]]


@pytest.mark.parametrize("orientation", [xted.ORIENT_RIGHT, xted.ORIENT_LEFT, xted.ORIENT_AUTO])
@pytest.mark.parametrize("narrow_width,run_rows,half_width", [(0, 1, -1), (0, 5, 0), (7, 3, 100), (32, 64, 0),
                                                              (256, 17, -1), (256, 64, 0)])
def test_forced_granularities(orientation, narrow_width, run_rows, half_width):
    """Every executor (warp-narrow of each width class, half-block, block-wide)
    and every decomposition, forced, on the same random pairs."""
    rng = random.Random(1000 * orientation + narrow_width + run_rows + half_width)
    pairs = []
    for _ in range(24):
        pairs.append((_rand_tree(rng, rng.choice([0, 1, 2, 5, 30, 90, 200, 420]), rng.randint(1, 6), rng.randrange(3)),
                      _rand_tree(rng, rng.choice([1, 3, 8, 50, 130, 300, 700, 1100]), rng.randint(1, 6),
                                 rng.randrange(3))))
    want = [oracle.distance(a, b) for a, b in pairs]
    with xted.Context(orientation=orientation, narrow_width=narrow_width, run_rows=run_rows,
                      half_width=half_width) as c:
        got = c.distance_batch(pairs)
    assert list(got) == want


def test_runtime_tune_table():
    """xted_set_tune_table: a size-bucket table set on the context plans the
    batches after it (here each bucket with a granularity of the forced cases
    above), the distances stay the oracle's, a malformed table is refused with
    XTED_EINVAL and leaves the table in force, and an empty one restores the
    compiled table."""
    rng = random.Random(4242)
    pairs = []
    for _ in range(24):
        pairs.append((_rand_tree(rng, rng.choice([0, 1, 2, 5, 30, 90, 200, 420]), rng.randint(1, 6), rng.randrange(3)),
                      _rand_tree(rng, rng.choice([1, 3, 8, 50, 130, 300, 700, 1100]), rng.randint(1, 6),
                                 rng.randrange(3))))
    want = [oracle.distance(a, b) for a, b in pairs]
    with xted.Context() as c:
        c.set_tune_table([(40, 3, 7, 100), (300, 1, 0, -1), (1 << 30, 64, 256, 512)])
        assert list(c.distance_batch(pairs)) == want
        for bad in ([(0, 1, 1, 1)], [(50, 1, 1, 1), (50, 2, 2, 2)], [(1 << 30, 0, 1, 1)], [(1 << 30, 1, 257, 1)],
                    [(1 << 30, 1, 1, 1025)], [(1 << 30, 1, 1, -2)], [(k + 1, 1, 1, 1) for k in range(9)]):
            with pytest.raises(xted.XtedError) as e:
                c.set_tune_table(bad)
            assert e.value.code == xted.XTED_EINVAL
        assert list(c.distance_batch(pairs)) == want
        c.set_tune_table([])
        assert list(c.distance_batch(pairs)) == want


def test_brute_force_small(ctx):
    rng = random.Random(3)
    pairs = [(_rand_tree(rng, rng.randint(0, 9), rng.randint(1, 3), rng.randrange(3)),
              _rand_tree(rng, rng.randint(0, 9), rng.randint(1, 3), rng.randrange(3))) for _ in range(300)]
    got = ctx.distance_batch(pairs)
    for (a, b), d in zip(pairs, got):
        assert d == brute.distance(a, b)
    brute.clear_cache()


def test_batch_equals_singles_and_order(ctx):
    rng = random.Random(8)
    pairs = [(_rand_tree(rng, rng.randint(1, 150), 4, rng.randrange(3)),
              _rand_tree(rng, rng.randint(1, 150), 4, rng.randrange(3))) for _ in range(40)]
    batch = ctx.distance_batch(pairs)
    singles = [ctx.distance(a, b) for a, b in pairs]
    assert list(batch) == singles
    perm = list(range(len(pairs)))
    rng.shuffle(perm)
    again = ctx.distance_batch([pairs[i] for i in perm])
    assert [int(again[k]) for k in range(len(perm))] == [singles[i] for i in perm]


def test_empty_and_tiny(ctx):
    e = trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))
    one = trees.from_adjacency([7], [[]])
    other = trees.from_adjacency([8], [[]])
    t = gen.tree("deep", 33, 5)
    assert ctx.distance(e, e) == 0
    assert ctx.distance(e, t) == 33
    assert ctx.distance(t, e) == 33
    assert ctx.distance(one, one) == 0
    assert ctx.distance(one, other) == 1
    assert ctx.distance(one, t) == oracle.distance(one, t)


def test_standard_ted_mirror_interface():
    # the reference's own calling convention: string labels + adjacency lists
    x_node = ["a", "b", "c", "d", "e"]
    x_adj = [[1, 2], [], [3, 4], [], []]
    y_node = ["a", "c", "d", "x"]
    y_adj = [[1, 3], [2], [], []]
    a = trees.from_adjacency(trees.Interner()(x_node), x_adj)
    d = xted.standard_ted(x_node, x_adj, y_node, y_adj, 8, 1)
    intern = trees.Interner()
    assert d == oracle.distance(trees.from_adjacency(intern(x_node), x_adj),
                                trees.from_adjacency(intern(y_node), y_adj))
    assert x_node == ["a", "b", "c", "d", "e"]  # inputs are not cleared
    assert xted.standard_ted([], [], y_node, y_adj) == 4
    del a


def test_mixed_workload_sample(ctx):
    pairs = gen.mixed_batch(64, seed=77, hi=600)
    got = ctx.distance_batch(pairs)
    want = oracle.distance_batch(pairs, nthreads=8)
    assert np.array_equal(got, want)


def test_single_pair_1000_mixed_shapes(ctx):
    a, b = gen.single_pair_1000()
    assert ctx.distance(a, b) == oracle.distance(a, b)


def test_prepared_batch_repeatable(ctx):
    """Repeated runs of one prepared batch: the first is enqueued call by call,
    later ones replay the step's captured CUDA graph; all give the oracle's
    distances. A new prepare drops the old graph."""
    pairs = gen.mixed_batch(48, seed=5, hi=400)
    want = oracle.distance_batch(pairs, nthreads=8)
    ctx.prepare_batch(pairs)
    r1 = ctx.run_prepared()
    assert ctx.stats()["graph"] == 0
    for _ in range(3):
        r2 = ctx.run_prepared()
        assert ctx.stats()["graph"] == 1
        assert np.array_equal(r1, r2)
    assert np.array_equal(r1, want)
    other = gen.mixed_batch(20, seed=6, hi=300)
    ctx.prepare_batch(other)
    for k in range(3):
        got = ctx.run_prepared()
        assert ctx.stats()["graph"] == (0 if k == 0 else 1)
        assert np.array_equal(got, oracle.distance_batch(other, nthreads=8))


def test_large_pair_properties(ctx):
    """20,000-node pairs: size-independent properties (the oracle would take
    minutes here): identity, symmetry, bounds, and agreement of both
    decompositions on a 4,000-node pair with the oracle."""
    a, b = gen.single_pair_20000(shape="caterpillar")
    assert ctx.distance(a, a) == 0
    d_ab = ctx.distance(a, b)
    assert d_ab == ctx.distance(b, a)
    assert 0 <= d_ab <= len(a) + len(b)
    r, s = gen.tree("random", 4000, 41, "uniform", 64), gen.tree("random", 4000, 42, "uniform", 64)
    want = oracle.distance(r, s)
    for orient in (xted.ORIENT_RIGHT, xted.ORIENT_LEFT):
        with xted.Context(orientation=orient) as c:
            assert c.distance(r, s) == want


@pytest.mark.parametrize("n", [2049, 2300, 2817])
def test_generic_wide_path_edges(ctx, n):
    """Column segments just above the register paths' 2,048-column limit run on
    the generic wide path (per-thread column runs of uneven length, the last
    threads short or idle, far columns owned by other threads): caterpillars
    and random trees of these sizes against the oracle."""
    a = gen.tree("caterpillar", n, 100 + n, "uniform", 8)
    b = gen.tree("caterpillar", n - 7, 200 + n, "uniform", 8)
    r = gen.tree("random", n, 300 + n, "uniform", 8)
    pairs = [(a, b), (r, a), (b, r)]
    got = ctx.distance_batch(pairs)
    assert list(got) == [oracle.distance(x, y) for x, y in pairs]


@pytest.mark.parametrize("n", [2049, 2817])
def test_striped_wide_units_match_oracle(n):
    """Striped units (a column segment wider than 2,048 split into stripes run
    by several blocks at once, carries and far columns passed between them),
    forced on every wide unit: caterpillars and random trees against the oracle,
    and a 4,000-node random pair in both decompositions."""
    a = gen.tree("caterpillar", n, 100 + n, "uniform", 8)
    b = gen.tree("caterpillar", n - 7, 200 + n, "uniform", 8)
    r = gen.tree("random", n, 300 + n, "uniform", 8)
    pairs = [(a, b), (r, a), (b, r)]
    with xted.Context(stripe_min_cells=1) as c:
        got = c.distance_batch(pairs)
    assert list(got) == [oracle.distance(x, y) for x, y in pairs]
    if n == 2817:
        r4, s4 = gen.tree("random", 4000, 41, "uniform", 64), gen.tree("random", 4000, 42, "uniform", 64)
        want = oracle.distance(r4, s4)
        for orient in (xted.ORIENT_RIGHT, xted.ORIENT_LEFT):
            with xted.Context(orientation=orient, stripe_min_cells=1) as c:
                assert c.distance(r4, s4) == want


def test_striped_equals_one_block_on_20000_node_pairs():
    """The 20,000-node pairs with stripes (the default) and with every wide
    unit on one block give the same distances."""
    pairs = [gen.single_pair_20000(shape="random"), gen.single_pair_20000(shape="caterpillar")]
    with xted.Context(stripe_min_cells=-1) as c:
        one = c.distance_batch(pairs)
    with xted.Context() as c:
        striped = c.distance_batch(pairs)
    assert list(one) == list(striped)


@pytest.mark.parametrize("shape", ["deep", "wide"])
def test_striped_deep_and_wide_shapes(shape):
    """Forced stripes on a deep-narrow tree (many far columns cross stripe
    boundaries) and a wide-shallow one (short subtrees), as either tree of the
    pair, against the oracle."""
    a = gen.tree(shape, 2600, 7, "uniform", 8)
    b = gen.tree("random", 2500, 8, "uniform", 8)
    with xted.Context(stripe_min_cells=1) as c:
        got = c.distance_batch([(a, b), (b, a)])
    want = oracle.distance(a, b)
    assert list(got) == [want, want]
