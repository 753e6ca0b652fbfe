"""Host-side interface of the tree-edit-distance path.

``standard_ted`` mirrors the reference entry point
``int standard_ted(vector<string>& x_node, vector<vector<int>>& x_adj,
vector<string>& y_node, vector<vector<int>>& y_adj, int num_threads,
int parallel_version)`` (X-TED_CPU/TED.cpp:177, X-TED_GPU/TED.cu:116):
same arguments, same meaning, same empty-tree rules. Two differences are
deliberate: the label lists are not cleared (the reference clears them,
X-TED_CPU/TED.cpp:160-161), and malformed input raises ``XtedError``
(XTED_EINVAL) instead of being undefined behaviour. ``num_threads`` and
``parallel_version`` are accepted and ignored, as X-TED_GPU ignores them.

``Context`` wraps one ``xted_ctx`` (one device, one stream).
"""
from __future__ import annotations

import ctypes
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .trees import Interner, Tree, from_adjacency

_CTX: Optional["Context"] = None


class Context:
    def __init__(self, device: int = 0, orientation: int = _lib.ORIENT_AUTO,
                 narrow_width: Optional[int] = None, run_rows: Optional[int] = None,
                 ctas_per_sm: int = 0, wait_timeout_s: float = 20.0, mem_limit: int = 0,
                 wide_rows: int = 0, half_width: int = 0, tuned: Optional[bool] = None,
                 stripe_min_cells: int = 0, costs: Optional[Tuple[int, int, int]] = None):
        """`costs` = (delete, insert, rename) edit costs, integers >= 0; None is
        the reference's unit cost (1, 1, 1). Delete applies to nodes of the
        first tree of a pair, insert to nodes of the second."""
        L = _lib.lib()
        o = _lib.COpts()
        L.xted_opts_default(ctypes.byref(o))
        o.device = device
        o.orientation = orientation
        if narrow_width is not None:
            o.narrow_width = narrow_width
        if run_rows is not None:
            o.run_rows = run_rows
        o.ctas_per_sm = ctas_per_sm
        o.wide_rows = wide_rows
        o.half_width = half_width
        # the autotuned per-size table applies unless the granularity is given explicitly
        if tuned is None:
            tuned = narrow_width is None and run_rows is None and half_width == 0
        o.tuned = 1 if tuned else 0
        o.wait_timeout_s = wait_timeout_s
        o.mem_limit = mem_limit
        o.stripe_min_cells = stripe_min_cells
        if costs is not None:
            o.cost_del, o.cost_ins, o.cost_ren = (int(x) for x in costs)
        self.opts = o
        h = ctypes.c_void_p()
        _lib.check(L.xted_create(ctypes.byref(h), ctypes.byref(o)), "xted_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().xted_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def distance(self, a: Tree, b: Tree) -> int:
        keep: list = []
        ca, cb = _lib.ctree(a, keep), _lib.ctree(b, keep)
        out = ctypes.c_int32(0)
        _lib.check(_lib.lib().xted_distance(self._h, ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(out)),
                   "xted_distance")
        return int(out.value)

    @staticmethod
    def _views(pairs):
        """C tree arrays for a pair list (numpy-backed xted_tree arrays)."""
        A = _lib.tree_array([a for a, _ in pairs])
        B = _lib.tree_array([b for _, b in pairs])
        return _lib.tree_ptr(A), _lib.tree_ptr(B), (A, B)

    def distance_batch(self, pairs: Sequence[Tuple[Tree, Tree]]) -> np.ndarray:
        n = len(pairs)
        A, B, keep = self._views(pairs)
        out = np.zeros(max(n, 1), np.int32)
        _lib.check(_lib.lib().xted_distance_batch(self._h, A, B, n, out.ctypes.data_as(_lib._i32p)),
                   "xted_distance_batch")
        return out[:n]

    def distance_matrix(self, trees_: Sequence[Tree], pair_budget: int = 0) -> np.ndarray:
        """All-pairs TED matrix (symmetric, zero diagonal) through the batch path."""
        n = len(trees_)
        arr = _lib.tree_array(list(trees_))
        out = np.zeros((max(n, 1), max(n, 1)), np.int32)
        _lib.check(_lib.lib().xted_distance_matrix(self._h, _lib.tree_ptr(arr), n, int(pair_budget),
                                                   out.ctypes.data_as(_lib._i32p)), "xted_distance_matrix")
        return out[:n, :n]

    def prepare_batch(self, pairs: Sequence[Tuple[Tree, Tree]]) -> None:
        """Plan and upload a batch once (inputs resident on the device)."""
        A, B, keep = self._views(pairs)
        self._prepared_n = len(pairs)
        _lib.check(_lib.lib().xted_prepare_batch(self._h, A, B, len(pairs)), "xted_prepare_batch")

    def run_prepared(self) -> np.ndarray:
        out = np.zeros(max(self._prepared_n, 1), np.int32)
        _lib.check(_lib.lib().xted_run_prepared(self._h, out.ctypes.data_as(_lib._i32p)), "xted_run_prepared")
        return out[:self._prepared_n]

    def set_tune_table(self, rows: Sequence[Tuple[int, int, int, int]]) -> None:
        """Plans later batches and corpora with this size-bucket table instead
        of the compiled one (xted_set_tune_table): rows of (max_n, run_rows,
        narrow_width, half_width), max_n strictly increasing; an empty list
        restores the compiled table. Needs the context's `tuned` option."""
        arr = np.ascontiguousarray(np.asarray(list(rows), np.int32).reshape(-1, 4))
        _lib.check(_lib.lib().xted_set_tune_table(self._h, arr.ctypes.data_as(_lib._i32p), int(arr.shape[0])),
                   "xted_set_tune_table")

    def test_fault(self, kind: int = _lib.XTED_FAULT_HOLD_PAIR) -> None:
        """Arms one host-side fault for the next batch call or posted serving
        query (xted_test_fault): with XTED_FAULT_HOLD_PAIR one pair's first
        level is never made ready, so the call fails with XTED_ETIMEOUT after
        the context's bounded wait. For failure-handling tests."""
        _lib.check(_lib.lib().xted_test_fault(self._h, int(kind)), "xted_test_fault")

    def stats(self) -> dict:
        s = _lib.CStats()
        _lib.check(_lib.lib().xted_last_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    # ---- serving: a resident corpus and exact top-k queries ----

    def corpus_load(self, corpus: Sequence[Tree]) -> None:
        """Makes `corpus` the resident corpus (ids are list positions)."""
        keep: list = []
        arr = (_lib.CTree * max(len(corpus), 1))()
        for i, t in enumerate(corpus):
            arr[i] = _lib.ctree(t, keep)
        _lib.check(_lib.lib().xted_corpus_load(self._h, arr, len(corpus)), "xted_corpus_load")

    def query_submit(self, q: Tree, k: int = 10) -> int:
        """Queues a top-k query; returns its ticket at once."""
        keep: list = []
        cq = _lib.ctree(q, keep)
        t = ctypes.c_uint64(0)
        _lib.check(_lib.lib().xted_query_submit(self._h, ctypes.byref(cq), int(k), ctypes.byref(t)),
                   "xted_query_submit")
        self._k = getattr(self, "_k", {})
        self._k[t.value] = int(k)
        return int(t.value)

    def query_poll(self, ticket: int):
        """None while running; else (ids, dists, queue_ms, total_ms)."""
        k = self._k.get(ticket, 1)
        ids = np.zeros(k, np.int32)
        dists = np.zeros(k, np.int32)
        done = ctypes.c_int32(0)
        qm, tm = ctypes.c_double(0), ctypes.c_double(0)
        rc = _lib.lib().xted_query_poll_timed(self._h, ctypes.c_uint64(ticket), ids.ctypes.data_as(_lib._i32p),
                                              dists.ctypes.data_as(_lib._i32p), ctypes.byref(done),
                                              ctypes.byref(qm), ctypes.byref(tm))
        if rc != 0:
            self._k.pop(ticket, None)
            _lib.check(rc, "xted_query_poll")
        if not done.value:
            return None
        self._k.pop(ticket, None)
        return ids, dists, qm.value, tm.value

    def query_wait(self, ticket: int, poll_s: float = 0.0002, timeout_s: float = 600.0):
        """Polls until the query is done; returns (ids, dists, queue_ms, total_ms)."""
        import time
        t_end = time.monotonic() + timeout_s
        while True:
            r = self.query_poll(ticket)
            if r is not None:
                return r
            if time.monotonic() > t_end:
                raise TimeoutError(f"query {ticket} not done after {timeout_s} s")
            time.sleep(poll_s)

    def serve_drain(self) -> None:
        _lib.check(_lib.lib().xted_serve_drain(self._h), "xted_serve_drain")

    def serve_stats(self) -> dict:
        out = np.zeros(8, np.int64)
        _lib.check(_lib.lib().xted_serve_stats(self._h, out.ctypes.data_as(_lib._i64p), 8), "xted_serve_stats")
        return {"launches": int(out[0]), "queries": int(out[1]), "pairs": int(out[2]), "cells": int(out[3]),
                "pairs_pruned": int(out[4]), "second_rounds": int(out[5]), "bound_us": int(out[6]),
                "plan_us": int(out[7])}

    def serve_options(self, prune: int = 2, first_round: int = 0) -> None:
        """Exact top-k pruning: 0 off, 1 label bound, 2 preorder-sequence bound
        (default); see xted_serve_options."""
        _lib.check(_lib.lib().xted_serve_options(self._h, int(prune), int(first_round)), "xted_serve_options")


def default_context() -> Context:
    global _CTX
    if _CTX is None:
        _CTX = Context()
    return _CTX


def pair_cells(a: Tree, b: Tree, orientation: int = _lib.ORIENT_AUTO) -> Tuple[int, int, int]:
    keep: list = []
    ca, cb = _lib.ctree(a, keep), _lib.ctree(b, keep)
    out = (ctypes.c_int64 * 3)()
    _lib.check(_lib.lib().xted_pair_cells(ctypes.byref(ca), ctypes.byref(cb), orientation, out))
    return int(out[0]), int(out[1]), int(out[2])


def distance_noalloc(a: Tree, b: Tree, device: int = 0) -> int:
    """One pair through xted_distance_noalloc: computed in the library's fixed
    device arena, with no device allocation and no context. For callers that
    must not allocate device memory (memory held by another allocator's pool,
    or after an allocation failed). Calls that overlap on the GPU race on the
    shared arena; raises XtedError(XTED_ETOOBIG) for pairs that do not fit."""
    keep: list = []
    ta, tb = _lib.ctree(a, keep), _lib.ctree(b, keep)
    out = ctypes.c_int32(0)
    _lib.check(_lib.lib().xted_distance_noalloc(ctypes.byref(ta), ctypes.byref(tb), int(device),
                                                ctypes.byref(out)), "xted_distance_noalloc")
    return int(out.value)


def validate(t: Tree) -> bool:
    keep: list = []
    c = _lib.ctree(t, keep)
    return _lib.lib().xted_validate(ctypes.byref(c)) == _lib.XTED_OK


def standard_ted(x_node: Sequence[str], x_adj: Sequence[Sequence[int]], y_node: Sequence[str],
                 y_adj: Sequence[Sequence[int]], num_threads: int = 0, parallel_version: int = 0,
                 ctx: Optional[Context] = None) -> int:
    """The reference's entry point (X-TED_CPU/TED.cpp:177-190) on the GPU."""
    m, n = len(x_adj), len(y_adj)
    if m == 0:  # X-TED_CPU/TED.cpp:181-186
        return n
    if n == 0:
        return m
    intern = Interner()
    a = from_adjacency(intern(x_node), x_adj)
    b = from_adjacency(intern(y_node), y_adj)
    return (ctx or default_context()).distance(a, b)
