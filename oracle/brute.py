"""TEST INFRASTRUCTURE ONLY -- brute-force ordered tree edit distance.

An independent checker for small trees (at most 12 nodes each). It is the
textbook recursive definition of the edit distance between ordered forests
(costs: delete cd, insert ci, rename cr if labels differ else 0; the
reference's unit costs are cd = ci = cr = 1), memoised on sub-forests; it uses no keyroots and no Zhang-Shasha tables, so agreement
with the reference restatement is evidence for both.

For forests F, G with rightmost roots v, w:
  d(F, G) = min( d(F - v, G) + cd,
                 d(F, G - w) + ci,
                 d(F - T(v), G - T(w)) + d(kids(v), kids(w)) + cr [lab v != lab w] )
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
def _fd(F, G, cd=1, ci=1, cr=1) -> int:
    if not F:
        return _size(G) * ci
    if not G:
        return _size(F) * cd
    (lv, kv), (lw, kw) = F[-1], G[-1]
    d_del = _fd(F[:-1] + kv, G, cd, ci, cr) + cd
    d_ins = _fd(F, G[:-1] + kw, cd, ci, cr) + ci
    d_ren = _fd(F[:-1], G[:-1], cd, ci, cr) + _fd(kv, kw, cd, ci, cr) + (0 if lv == lw else cr)
    return min(d_del, d_ins, d_ren)


def distance(a, b, costs=None) -> int:
    """costs = (delete, insert, rename); None is unit cost."""
    if len(a.labels) > 12 or len(b.labels) > 12:
        raise ValueError("brute force is limited to trees of at most 12 nodes")
    cd, ci, cr = costs if costs is not None else (1, 1, 1)
    return _fd(_to_nested(a), _to_nested(b), int(cd), int(ci), int(cr))


def clear_cache():
    _fd.cache_clear()


__all__ = ["distance", "clear_cache", "np"]
