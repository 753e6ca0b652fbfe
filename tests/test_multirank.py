"""The benchmark's multi-rank path on CPU: two gloo ranks run the rank logic
of bench.py (process group set-up, per-rank workload shards, max-over-ranks
timing, whole-job aggregation), as torchrun would launch it on two GPUs."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "XTED_BENCH_BACKEND": "gloo"})
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "x-ted_b200"))
    try:
        import bench
        w, r, _ = bench.dist_setup(None)
        pairs, cfg = bench.make_workload("batched256", r)
        first = (pairs[0][0].labels[:8].tolist(), len(pairs))
        # rank 1 is the slow one: 2 s against 1 s; cells 10 and 20
        value, gcups, tmax = bench.aggregate(256, 3, 1000.0 * (r + 1), 10 * (r + 1), w)
        bench.barrier(w)
        import torch.distributed as dist
        dist.destroy_process_group()
        q.put((r, w, cfg["seed"], first, value, gcups, tmax))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


@pytest.mark.timeout(180)
def test_two_gloo_ranks_shard_and_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=150) for _ in procs]
    for p in procs:
        p.join(timeout=30)
    assert all(len(o) == 7 for o in out), out
    out.sort()
    (r0, w0, s0, f0, v0, g0, t0), (r1, w1, s1, f1, v1, g1, t1) = out
    assert (w0, w1) == (2, 2)
    assert s0 != s1 and f0 != f1          # each rank holds its own batch (weak scaling)
    assert t0 == t1 == 2000.0             # time is the slowest rank's
    assert v0 == v1 == pytest.approx(256 * 2 * 3 / 2.0)
    assert g0 == g1 == pytest.approx(30 * 3 / 2.0 / 1e9)


def _shard_main(rank, world, port, q):
    """Two gloo ranks run the library's sharded paths with the oracle standing
    in for each rank's GPU (no GPU here): a pair list split by estimated cells
    and gathered, and a corpus split in contiguous shards with the top-k merge."""
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "x-ted_b200"))
    try:
        import datetime

        import torch.distributed as dist

        import oracle
        from xted import gen, multi
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        pairs = gen.mixed_batch(40, seed=17, lo=5, hi=120)
        seen = []

        def compute(ps):
            seen.append(len(ps))
            return oracle.distance_batch(ps)

        got = multi.distance_batch_sharded(pairs, compute)
        corpus = gen.corpus(30, seed=18, lo=1, hi=80)
        queries = gen.corpus(3, seed=19, lo=1, hi=80)
        shard = {}

        def load(trees_):
            shard["trees"] = trees_

        def local_topk(qt, k):
            d = [oracle.distance(qt, t) for t in shard["trees"]]
            order = sorted(range(len(d)), key=lambda i: (d[i], i))[:k]
            return order, [d[i] for i in order]

        sc = multi.ShardedCorpus(corpus, load, local_topk)
        answers = [tuple(x.tolist() for x in sc.query(qt, 7)) for qt in queries]
        dist.destroy_process_group()
        q.put((rank, got.tolist(), seen, sc.lo, sc.hi, answers))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


@pytest.mark.timeout(240)
def test_two_gloo_ranks_shard_pairs_and_corpus():
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "x-ted_b200"))
    import oracle
    from xted import gen
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=200) for _ in procs], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=30)
    assert all(len(o) == 6 for o in out), out
    pairs = gen.mixed_batch(40, seed=17, lo=5, hi=120)
    want = oracle.distance_batch(pairs).tolist()
    assert out[0][1] == want and out[1][1] == want           # every rank holds every distance
    assert sum(out[0][2]) + sum(out[1][2]) == 40 and min(out[0][2][0], out[1][2][0]) > 0
    assert out[0][3] == 0 and out[0][4] == out[1][3] and out[1][4] == 30  # contiguous corpus shards
    corpus = gen.corpus(30, seed=18, lo=1, hi=80)
    for qi, qt in enumerate(gen.corpus(3, seed=19, lo=1, hi=80)):
        d = [oracle.distance(qt, t) for t in corpus]
        order = sorted(range(30), key=lambda i: (d[i], i))[:7]
        assert out[0][5][qi] == (order, [d[i] for i in order]) == out[1][5][qi]
