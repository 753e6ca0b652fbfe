"""Seeded synthetic workloads without the CUDA library.

The same trees as ``xted_gen_tree`` of the C ABI (``csrc/gen.cpp``): the same
xoshiro256** stream seeded through splitmix64, the same shape rules and the
same label draws, in plain Python. It exists so that a process which must not
load ``lib/libxted.so`` (the benchmark's reference arm, which times the
reference X-TED_CPU alone) can still build the exact pairs of a workload.
A CPU test requires it to match the C generator array for array on every
shape and label kind.

It is slow (a Python loop per node), so it is meant for samples of a
workload: ``mixed_specs`` draws the sizes, shapes and tree seeds of a whole
mixed batch cheaply, and ``mixed_pairs`` builds only the pairs asked for.
"""
from __future__ import annotations

import math
from collections import deque
from typing import List, Sequence, Tuple

import numpy as np

from .trees import Tree

SHAPES = {"random": 0, "wide": 1, "deep": 2, "caterpillar": 3}
LABELS = {"uniform": 0, "zipf": 1}
_M64 = (1 << 64) - 1


def mix(*xs: int) -> int:
    """Seed mixing of the workload generators (FNV-style, 64-bit)."""
    h = 0x243F6A8885A308D3
    for x in xs:
        h = (h ^ (x & _M64)) * 0x100000001B3 & _M64
        h ^= h >> 29
    return h


class _Rng:
    """xoshiro256** seeded by four splitmix64 outputs (csrc/gen.cpp: Rng)."""

    def __init__(self, seed: int):
        s = []
        seed &= _M64
        for _ in range(4):
            seed = (seed + 0x9E3779B97F4A7C15) & _M64
            z = seed
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
            s.append(z ^ (z >> 31))
        self.s = s

    def next(self) -> int:
        s0, s1, s2, s3 = self.s
        x = (s1 * 5) & _M64
        r = ((((x << 7) | (x >> 57)) & _M64) * 9) & _M64
        t = (s1 << 17) & _M64
        s2 ^= s0
        s3 ^= s1
        s1 ^= s2
        s0 ^= s3
        s2 ^= t
        s3 = ((s3 << 45) | (s3 >> 19)) & _M64
        self.s = [s0, s1, s2, s3]
        return r

    def below(self, k: int) -> int:
        return (self.next() * k) >> 64

    def unit(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def _to_tree(ch: List[List[int]], labels: List[int]) -> Tree:
    n = len(ch)
    order, stack = [], [0]
    while stack:
        v = stack.pop()
        order.append(v)
        stack.extend(reversed(ch[v]))
    newid = [0] * n
    for k, v in enumerate(order):
        newid[v] = k
    off = np.zeros(n + 1, np.int32)
    idx: List[int] = []
    for k, v in enumerate(order):
        idx.extend(newid[c] for c in ch[v])
        off[k + 1] = len(idx)
    return Tree(np.asarray(labels, np.int32), off, np.asarray(idx, np.int32))


def tree(shape: str, n: int, seed: int, labels: str = "uniform", alphabet: int = 26) -> Tree:
    """One tree, identical to xted.gen.tree (the C generator) for the same arguments."""
    if n <= 0:
        return Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))
    g = _Rng(seed)
    sh = SHAPES[shape]
    ch: List[List[int]] = [[] for _ in range(n)]
    if sh == 0:
        for i in range(1, n):
            ch[g.below(i)].append(i)
    elif sh == 1:
        depth = [0] * n
        q = deque([0])
        cnt = 1
        while cnt < n and q:
            v = q.popleft()
            if depth[v] >= 4:
                continue
            f = 40
            if v != 0:
                f = 1
                while g.unit() >= 0.25:
                    f += 1
            k = 0
            while k < f and cnt < n:
                ch[v].append(cnt)
                depth[cnt] = depth[v] + 1
                q.append(cnt)
                cnt += 1
                k += 1
        if cnt < n:
            cand = [v for v in range(cnt) if depth[v] < 4]
            while cnt < n:
                v = cand[g.below(len(cand))]
                ch[v].append(cnt)
                depth[cnt] = depth[v] + 1
                cnt += 1
    elif sh == 2:
        spine = min(100, max(1, (n + 1) // 2))
        for i in range(1, spine):
            ch[i - 1].append(i)
        q = deque(range(spine))
        cnt = spine
        while cnt < n and q:
            v = q.popleft()
            f = 1 + g.below(3)
            extra = f - len(ch[v])
            k = 0
            while k < extra and cnt < n:
                pos = g.below(len(ch[v]) + 1)
                ch[v].insert(pos, cnt)
                q.append(cnt)
                cnt += 1
                k += 1
            if not q and cnt < n:
                q.append(cnt - 1)
    else:
        spine = (n + 9) // 10
        cnt = spine
        for s in range(spine):
            k = 0
            while k < 9 and cnt < n:
                ch[s].append(cnt)
                cnt += 1
                k += 1
            if s + 1 < spine:
                ch[s].append(s + 1)
        while cnt < n:
            ch[spine - 1].append(cnt)
            cnt += 1
    if LABELS[labels] == 0:
        lab = [g.below(alphabet) for _ in range(n)]
    else:
        cdf, s = [], 0.0
        for r in range(alphabet):
            s += 1.0 / math.pow(float(r + 1), 1.1)
            cdf.append(s)
        lab = []
        for _ in range(n):
            u = g.unit() * s
            lo, hi = 0, alphabet - 1
            while lo < hi:
                mid = (lo + hi) // 2
                if cdf[mid] < u:
                    lo = mid + 1
                else:
                    hi = mid
            lab.append(lo)
    return _to_tree(ch, lab)


TreeSpec = Tuple[str, int, int]  # (shape, nodes, seed)


def mixed_specs(npairs: int, seed: int, lo: int = 50, hi: int = 2000) -> List[Tuple[TreeSpec, TreeSpec]]:
    """Shape, size and seed of both trees of every pair of a mixed batch:
    sizes log-uniform in [lo, hi], shapes uniform over the four kinds, every
    tree drawn independently (the draws of xted.gen.mixed_batch)."""
    rng = np.random.default_rng(mix(seed, 99) % (2**63))
    names = list(SHAPES)
    out = []
    for p in range(npairs):
        ts = []
        for s in range(2):
            n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
            shape = names[int(rng.integers(0, 4))]
            ts.append((shape, n, mix(seed, p, s)))
        out.append((ts[0], ts[1]))
    return out


def mixed_pairs(npairs: int, seed: int, which: Sequence[int], lo: int = 50, hi: int = 2000,
                alphabet: int = 1000) -> List[Tuple[Tree, Tree]]:
    """Pairs `which` of xted.gen.mixed_batch(npairs, seed, lo, hi, alphabet),
    built without the CUDA library."""
    specs = mixed_specs(npairs, seed, lo, hi)
    return [tuple(tree(sh, n, sd, "zipf", alphabet) for sh, n, sd in specs[p]) for p in which]
