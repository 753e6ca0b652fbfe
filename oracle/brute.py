"""TEST INFRASTRUCTURE ONLY -- brute-force ordered tree edit distance.

An independent checker for small trees (at most 12 nodes each). It is the
textbook recursive definition of the edit distance between ordered forests
(unit costs: delete 1, insert 1, rename 0 if labels are equal else 1), memoised
on sub-forests; it uses no keyroots and no Zhang-Shasha tables, so agreement
with the reference restatement is evidence for both.

For forests F, G with rightmost roots v, w:
  d(F, G) = min( d(F - v, G) + 1,
                 d(F, G - w) + 1,
                 d(F - T(v), G - T(w)) + d(kids(v), kids(w)) + [lab v != lab w] )
where F - v replaces v by its children and F - T(v) removes v's subtree.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np


def _to_nested(t):
    """Preorder CSR -> nested tuple (label, (child, ...))."""
    n = len(t.labels)
    if n == 0:
        return ()

    def build(v):
        kids = tuple(build(int(c)) for c in t.idx[t.off[v]:t.off[v + 1]])
        return (int(t.labels[v]), kids)

    return (build(0),)


def _size(forest) -> int:
    return sum(1 + _size(k) for _, k in forest)


@lru_cache(maxsize=None)
def _fd(F, G) -> int:
    if not F:
        return _size(G)
    if not G:
        return _size(F)
    (lv, kv), (lw, kw) = F[-1], G[-1]
    d_del = _fd(F[:-1] + kv, G) + 1
    d_ins = _fd(F, G[:-1] + kw) + 1
    d_ren = _fd(F[:-1], G[:-1]) + _fd(kv, kw) + (0 if lv == lw else 1)
    return min(d_del, d_ins, d_ren)


def distance(a, b) -> int:
    if len(a.labels) > 12 or len(b.labels) > 12:
        raise ValueError("brute force is limited to trees of at most 12 nodes")
    return _fd(_to_nested(a), _to_nested(b))


def clear_cache():
    _fd.cache_clear()


__all__ = ["distance", "clear_cache", "np"]
