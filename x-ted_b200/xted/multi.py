"""Several GPUs, one process per GPU: sharding of the batch and serving paths.

Tree pairs are independent, and so are the corpus trees a serving query is
compared with, so the work splits across ranks with no exchange on the data
path. A pair list is partitioned by estimated DP cells (the keyroot-table
cells of each pair, from ``xted_pair_cells`` on the host) so every rank gets
about the same work; each rank computes its shard on its own GPU and the
distances are gathered once at the end. A corpus is split into contiguous
shards by the same estimate; a query runs on every shard, each rank returns
its exact local top-k with global corpus ids, and the merge of those k-lists
is the exact global top-k (ties by lower corpus index, as one GPU answers).

The reference has no multi-GPU code; this follows the partitioning its
independent pairs allow. The collectives are torch.distributed's (NCCL on
GPUs, gloo for CPU tests): one reduction of the distance vector for a batch,
one all-gather of k (id, distance) pairs per query.
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .trees import Tree


def estimate_cells(pairs: Sequence[Tuple[Tree, Tree]], orientation: int = _lib.ORIENT_AUTO) -> np.ndarray:
    """DP cells each pair will take under `orientation` (host-side; no GPU).
    Pairs with an empty tree cost one cell."""
    from .api import pair_cells
    out = np.ones(len(pairs), np.int64)
    for p, (a, b) in enumerate(pairs):
        if a.n and b.n:
            out[p] = max(1, pair_cells(a, b, orientation)[2])
    return out


def shard_pairs(cells: np.ndarray, world: int) -> List[np.ndarray]:
    """Longest-processing-time split: pairs by decreasing cells, each to the
    least-loaded rank so far (ties to the lower rank). Returns each rank's pair
    indices in increasing order; every index appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.argsort(-np.asarray(cells, np.int64), kind="stable")
    heap = [(0, r) for r in range(world)]
    parts: List[list] = [[] for _ in range(world)]
    for p in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(p))
        heapq.heappush(heap, (load + int(cells[p]), r))
    return [np.array(sorted(x), np.int64) for x in parts]


def _dist():
    import torch.distributed as dist
    return dist


def _device_for(group):
    import torch
    dist = _dist()
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")


def distance_batch_sharded(pairs: Sequence[Tuple[Tree, Tree]], compute: Callable, group=None,
                           cells: Optional[np.ndarray] = None) -> np.ndarray:
    """Distances of every pair of `pairs`, the work split across the ranks of
    `group` by estimated cells. `compute(list of pairs) -> int32 array` runs
    this rank's shard (normally ``Context.distance_batch`` on this rank's
    GPU). Every rank must call this with the same pair list; every rank gets
    the whole result (one MAX all-reduce of the distance vector, which holds
    -1 where another rank owns the pair)."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    if cells is None:
        cells = estimate_cells(pairs)
    mine = shard_pairs(cells, world)[rank]
    out = np.full(len(pairs), -1, np.int32)
    if mine.size:
        got = np.asarray(compute([pairs[int(p)] for p in mine]), np.int32)
        out[mine] = got
    t = torch.from_numpy(out.astype(np.int64)).to(_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return t.cpu().numpy().astype(np.int32)


def topk_merge(parts: Sequence[Tuple[Sequence[int], Sequence[int]]], k: int) -> Tuple[np.ndarray, np.ndarray]:
    """Exact top-k of the union of per-shard top-k lists (ids are global
    corpus indices, -1 entries are padding): ascending distance, ties by lower
    id; padded with -1 when fewer than k exist."""
    cand = [(int(d), int(i)) for ids, dists in parts for i, d in zip(ids, dists) if int(i) >= 0]
    cand.sort()
    cand = cand[:k]
    ids = np.full(k, -1, np.int32)
    ds = np.full(k, -1, np.int32)
    for n, (d, i) in enumerate(cand):
        ids[n], ds[n] = i, d
    return ids, ds


def shard_corpus(corpus: Sequence[Tree], world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) ranges of the corpus with about equal total DP work
    per rank (a query's cells against a tree grow with the tree's keyroot
    subtree sizes, taken here as its node count squared)."""
    w = np.array([max(1, t.n) ** 2 for t in corpus], np.float64)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        bounds.append(int(np.searchsorted(cum, total * r / world, side="left")))
    bounds.append(len(corpus))
    for r in range(1, len(bounds)):
        bounds[r] = max(bounds[r], bounds[r - 1])
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


class ShardedCorpus:
    """One rank's share of a corpus spread over the ranks of `group`.

    `load(shard)` makes the rank's trees resident (normally
    ``Context.corpus_load``); `local_topk(query, k) -> (ids, dists)` answers a
    query on the rank's shard with shard-local ids (normally
    ``Context.query_wait(Context.query_submit(query, k))[:2]``). ``query``
    returns the exact global top-k on every rank."""

    def __init__(self, corpus: Sequence[Tree], load: Callable, local_topk: Callable, group=None):
        dist = _dist()
        self.group = group
        self.world, self.rank = dist.get_world_size(group), dist.get_rank(group)
        self.ranges = shard_corpus(corpus, self.world)
        self.lo, self.hi = self.ranges[self.rank]
        self._local_topk = local_topk
        load(list(corpus[self.lo:self.hi]))

    def query(self, q: Tree, k: int) -> Tuple[np.ndarray, np.ndarray]:
        dist = _dist()
        if self.hi > self.lo:
            ids, ds = self._local_topk(q, k)
            ids = np.where(np.asarray(ids) >= 0, np.asarray(ids) + self.lo, -1)
            part = (ids.tolist(), np.asarray(ds).tolist())
        else:
            part = ([], [])
        parts: list = [None] * self.world
        dist.all_gather_object(parts, part, group=self.group)
        return topk_merge(parts, k)
