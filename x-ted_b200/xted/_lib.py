"""ctypes binding of lib/libxted.so (the C ABI declared in include/xted.h).

The shared library is the product: there is no Python or CPU fallback. If the
library is missing, loading raises; if no sm_100 device is present, creating a
context returns XTED_ENODEV and raises XtedError.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libxted.so")

XTED_OK = 0
XTED_EINVAL = -1
XTED_ENOMEM = -2
XTED_ETIMEOUT = -3
XTED_ECUDA = -4
XTED_ENODEV = -5
XTED_ENOTFOUND = -6
XTED_EAGAIN = -7
XTED_ETOOBIG = -8
XTED_NOALLOC_ARENA_BYTES = 16 << 20
XTED_MAX_NODES = 65535
XTED_SERVE_MAX_QUERY = 8192
XTED_FAULT_NONE, XTED_FAULT_HOLD_PAIR = 0, 1
XTED_COST_BOUND = 1 << 17

ORIENT_AUTO, ORIENT_RIGHT, ORIENT_LEFT = 0, 1, 2

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


class CTree(ctypes.Structure):
    _fields_ = [("labels", _i32p), ("child_off", _i32p), ("child_idx", _i32p), ("n", ctypes.c_int32)]


class COpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("orientation", ctypes.c_int32),
                ("narrow_width", ctypes.c_int32), ("run_rows", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("wide_rows", ctypes.c_int32), ("half_width", ctypes.c_int32), ("tuned", ctypes.c_int32),
                ("wait_timeout_s", ctypes.c_double), ("mem_limit", ctypes.c_int64),
                ("stripe_min_cells", ctypes.c_int64), ("cost_del", ctypes.c_int32), ("cost_ins", ctypes.c_int32),
                ("cost_ren", ctypes.c_int32), ("pad_", ctypes.c_int32)]


class CStats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_int64), ("cells", ctypes.c_int64), ("cells_right", ctypes.c_int64),
                ("tasks", ctypes.c_int64), ("units", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64), ("host_plan_ms", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("levels_max", ctypes.c_int32), ("grid", ctypes.c_int32), ("dp_ms", ctypes.c_double),
                ("graph", ctypes.c_int32), ("pad", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class XtedError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = lib().xted_strerror(code).decode()
        super().__init__(f"{what}: {msg} ({code})" if what else f"{msg} ({code})")


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built (run __graft_entry__.build() or make -C x-ted_b200)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        sig = {
            "xted_opts_default": (None, [P(COpts)]),
            "xted_strerror": (ctypes.c_char_p, [ctypes.c_int]),
            "xted_create": (ctypes.c_int, [P(ctypes.c_void_p), P(COpts)]),
            "xted_destroy": (ctypes.c_int, [ctypes.c_void_p]),
            "xted_distance": (ctypes.c_int, [ctypes.c_void_p, P(CTree), P(CTree), _i32p]),
            "xted_distance_batch": (ctypes.c_int, [ctypes.c_void_p, P(CTree), P(CTree), ctypes.c_int32,
                                                   _i32p]),
            "xted_last_stats": (ctypes.c_int, [ctypes.c_void_p, P(CStats)]),
            "xted_distance_matrix": (ctypes.c_int, [ctypes.c_void_p, P(CTree), ctypes.c_int32, ctypes.c_int64,
                                                    _i32p]),
            "xted_prepare_batch": (ctypes.c_int, [ctypes.c_void_p, P(CTree), P(CTree), ctypes.c_int32]),
            "xted_run_prepared": (ctypes.c_int, [ctypes.c_void_p, _i32p]),
            "xted_pair_cells": (ctypes.c_int, [P(CTree), P(CTree), ctypes.c_int32, _i64p]),
            "xted_validate": (ctypes.c_int, [P(CTree)]),
            "xted_gen_tree": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32,
                                             ctypes.c_int32, _i32p, _i32p, _i32p]),
            "xted_corpus_load": (ctypes.c_int, [ctypes.c_void_p, P(CTree), ctypes.c_int32]),
            "xted_query_submit": (ctypes.c_int, [ctypes.c_void_p, P(CTree), ctypes.c_int32,
                                                 P(ctypes.c_uint64)]),
            "xted_query_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _i32p, _i32p, _i32p]),
            "xted_serve_drain": (ctypes.c_int, [ctypes.c_void_p]),
            "xted_distance_noalloc": (ctypes.c_int, [P(CTree), P(CTree), ctypes.c_int32, _i32p]),
            "xted_query_poll_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _i32p, _i32p, _i32p,
                                                     P(ctypes.c_double), P(ctypes.c_double)]),
            "xted_serve_stats": (ctypes.c_int, [ctypes.c_void_p, _i64p, ctypes.c_int32]),
            "xted_serve_options": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
            "xted_parse_adjacency": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                    _i32p, _i32p, _i32p, _i32p]),
            "xted_parse_bracket": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int32, _i32p, _i32p,
                                                  _i64p, _i32p, _i32p, _i64p]),
            "xted_test_fault": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
            "xted_set_tune_table": (ctypes.c_int, [ctypes.c_void_p, _i32p, ctypes.c_int32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(code: int, what: str = "") -> None:
    if code != XTED_OK:
        raise XtedError(code, what)


# numpy view of an xted_tree array: building the C array in one vectorised
# assignment costs about a microsecond per tree, where filling ctypes
# structures one by one costs tens.
TREE_DTYPE = np.dtype([("labels", np.uintp), ("child_off", np.uintp), ("child_idx", np.uintp),
                       ("n", np.int32), ("_pad", np.int32)])
assert TREE_DTYPE.itemsize == ctypes.sizeof(CTree)


def tree_record(t) -> tuple:
    """(labels, child_off, child_idx pointers, n) of a Tree, cached on the tree
    object together with the contiguous int32 arrays the pointers refer to."""
    cv = getattr(t, "_xted_cv", None)
    if cv is not None and cv[0] is t.labels and cv[1] is t.off and cv[2] is t.idx:
        return cv[4]
    lab = np.ascontiguousarray(t.labels, dtype=np.int32)
    off = np.ascontiguousarray(t.off, dtype=np.int32)
    idx = np.ascontiguousarray(t.idx, dtype=np.int32)
    hold = (lab if lab.size else np.zeros(1, np.int32), off if off.size else np.zeros(1, np.int32),
            idx if idx.size else np.zeros(1, np.int32))
    rec = (hold[0].ctypes.data, hold[1].ctypes.data, hold[2].ctypes.data, int(len(t.labels)), 0)
    try:
        t._xted_cv = (t.labels, t.off, t.idx, hold, rec)
    except AttributeError:  # objects that take no attributes: no caching
        pass
    return rec


def tree_array(trees_) -> np.ndarray:
    """Contiguous xted_tree array of `trees_` (each tree keeps its buffers alive)."""
    arr = np.empty(max(len(trees_), 1), TREE_DTYPE)
    if len(trees_):
        arr[:len(trees_)] = [tree_record(t) for t in trees_]
    return arr


def tree_ptr(arr: np.ndarray):
    return arr.ctypes.data_as(ctypes.POINTER(CTree))


def ctree(t, keep: list) -> CTree:
    """xted_tree view of a Tree (keeps the int32 arrays alive in `keep`)."""
    lab = np.ascontiguousarray(t.labels, dtype=np.int32)
    off = np.ascontiguousarray(t.off, dtype=np.int32)
    idx = np.ascontiguousarray(t.idx, dtype=np.int32)
    if idx.size == 0:
        idx = np.zeros(1, np.int32)
    if off.size == 0:
        off = np.zeros(1, np.int32)
    if lab.size == 0:
        lab = np.zeros(1, np.int32)
    keep.extend((lab, off, idx))
    return CTree(lab.ctypes.data_as(_i32p), off.ctypes.data_as(_i32p), idx.ctypes.data_as(_i32p),
                 int(len(t.labels)))
