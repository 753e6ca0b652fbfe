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
