"""The multi-GPU sharding on one GPU (needs a B200): each rank's share of a
pair list, and each rank's corpus shard, computed one after another on this
GPU through the C ABI, then assembled or merged as the ranks would do it; the
result must equal the whole batch and the single-corpus top-k. (The
collectives themselves are covered by the two-rank gloo test on CPU.)"""
import numpy as np
import pytest

import xted
from xted import gen, multi

pytestmark = pytest.mark.gpu


def test_pair_shards_assemble_to_the_whole_batch():
    pairs = gen.mixed_batch(300, seed=23, hi=900)
    with xted.Context() as ctx:
        whole = ctx.distance_batch(pairs)
        cells = multi.estimate_cells(pairs)
        assert cells.sum() == ctx.stats()["cells"]  # the estimate is the planner's own count
        for world in (2, 3):
            out = np.full(len(pairs), -1, np.int32)
            for part in multi.shard_pairs(cells, world):
                out[part] = ctx.distance_batch([pairs[int(p)] for p in part])
            assert np.array_equal(out, whole)


def test_corpus_shards_merge_to_the_global_topk():
    corpus = gen.corpus(120, seed=24, lo=20, hi=300)
    queries = gen.corpus(4, seed=25, lo=20, hi=300)
    k = 9
    with xted.Context() as ctx:
        ctx.corpus_load(corpus)
        want = [ctx.query_wait(ctx.query_submit(q, k))[:2] for q in queries]
    parts = [[] for _ in queries]
    for lo, hi in multi.shard_corpus(corpus, 3):
        with xted.Context() as ctx:
            ctx.corpus_load(corpus[lo:hi])
            for qi, q in enumerate(queries):
                ids, ds = ctx.query_wait(ctx.query_submit(q, k))[:2]
                parts[qi].append((np.where(ids >= 0, ids + lo, -1), ds))
    for qi in range(len(queries)):
        ids, ds = multi.topk_merge(parts[qi], k)
        assert ids.tolist() == want[qi][0].tolist() and ds.tolist() == want[qi][1].tolist()
