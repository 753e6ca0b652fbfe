"""TEST INFRASTRUCTURE ONLY -- the oracle for the tree-edit-distance path.

Three checkers, none of which is part of the product:

* ``distance`` / ``distance_batch``: ``liboracle.so``, a plain-C restatement of
  the reference X-TED_CPU algorithm (``oracle/xted_oracle.c``; every function
  there cites the reference file:line it follows).
* ``ref_distance`` / ``ref_distance_str``: ``_ref/libxted_ref.so``, the
  reference X-TED_CPU sources themselves (X-TED_CPU/TED.cpp,
  parallel_computing.cpp, dataset_preprocess.cpp) compiled by
  ``oracle/Makefile``, called through their own ``standard_ted``
  (X-TED_CPU/TED.cpp:177).
* ``brute.distance``: an independent memoised forest-edit-distance recursion
  for trees of at most 12 nodes (no keyroots, no Zhang-Shasha).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package.

A tree argument is any object with int32 numpy arrays ``labels`` (n),
``off`` (n+1) and ``idx`` (n-1): preorder CSR child lists.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


def _p32(a):
    return a.ctypes.data_as(_i32p)


def _p64(a):
    return a.ctypes.data_as(_i64p)


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle)")
        lib = ctypes.CDLL(path)
        lib.xo_distance.restype = ctypes.c_int
        lib.xo_distance.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, ctypes.c_int, _i32p, _i32p, _i32p]
        lib.xo_distance_cost.restype = ctypes.c_int
        lib.xo_distance_cost.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, ctypes.c_int, _i32p, _i32p, _i32p,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.xo_tree_stats.restype = None
        lib.xo_tree_stats.argtypes = [ctypes.c_int, _i32p, _i32p, _i64p]
        lib.xo_distance_batch.restype = ctypes.c_int
        lib.xo_distance_batch.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, _i64p, _i64p, _i64p,
                                          _i64p, _i64p, _i64p, ctypes.c_int, _i32p]
        _LIB = lib
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libxted_ref.so"))


def _ref():
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libxted_ref.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/_ref/libxted_ref.so is not built (make -C oracle ref)")
        lib = ctypes.CDLL(path)
        for name in ("xr_standard_ted_int",):
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, ctypes.c_int, _i32p, _i32p, _i32p,
                          ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        f = lib.xr_standard_ted_str
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), _i32p, _i32p, ctypes.c_int,
                      ctypes.POINTER(ctypes.c_char_p), _i32p, _i32p, ctypes.c_int,
                      ctypes.POINTER(ctypes.c_double)]
        _REF = lib
    return _REF


def _arrs(t):
    lab = np.ascontiguousarray(t.labels, dtype=np.int32)
    off = np.ascontiguousarray(t.off, dtype=np.int32)
    idx = np.ascontiguousarray(t.idx, dtype=np.int32)
    if idx.size == 0:
        idx = np.zeros(1, dtype=np.int32)
    return lab, off, idx


def distance(a, b, costs=None) -> int:
    """TED by the C restatement of X-TED_CPU: unit cost (the reference's), or
    with costs = (delete, insert, rename)."""
    la, ao, ai = _arrs(a)
    lb, bo, bi = _arrs(b)
    cd, ci, cr = costs if costs is not None else (1, 1, 1)
    d = _lib().xo_distance_cost(len(a.labels), _p32(la), _p32(ao), _p32(ai),
                                len(b.labels), _p32(lb), _p32(bo), _p32(bi), int(cd), int(ci), int(cr))
    if d < 0:
        raise MemoryError("oracle allocation failed")
    return int(d)


def distance_batch(pairs, nthreads: int = 1) -> np.ndarray:
    """Distances of a list of (a, b) pairs, pairs spread over nthreads threads."""
    chunks, offs = [], []
    pos = 0

    def put(arr):
        nonlocal pos
        arr = np.ascontiguousarray(arr, dtype=np.int32)
        chunks.append(arr if arr.size else np.zeros(1, np.int32))
        o = pos
        pos += max(arr.size, 1)
        return o

    m = np.zeros(len(pairs), np.int32)
    n = np.zeros(len(pairs), np.int32)
    o6 = np.zeros((6, len(pairs)), np.int64)
    for p, (a, b) in enumerate(pairs):
        m[p], n[p] = len(a.labels), len(b.labels)
        o6[0, p], o6[1, p], o6[2, p] = put(a.labels), put(a.off), put(a.idx)
        o6[3, p], o6[4, p], o6[5, p] = put(b.labels), put(b.off), put(b.idx)
    flat = np.concatenate(chunks) if chunks else np.zeros(1, np.int32)
    out = np.zeros(len(pairs), np.int32)
    rows = [np.ascontiguousarray(o6[k]) for k in range(6)]
    _lib().xo_distance_batch(len(pairs), _p32(m), _p32(n), _p32(flat), *[_p64(r) for r in rows],
                             int(nthreads), _p32(out))
    return out


def tree_stats(t):
    """(K, max keyroot depth, sum of keyroot subtree sizes) per X-TED_CPU."""
    la, ao, ai = _arrs(t)
    out = np.zeros(4, np.int64)
    _lib().xo_tree_stats(len(t.labels), _p32(ao), _p32(ai), _p64(out))
    return int(out[0]), int(out[1]), int(out[2])


def ref_distance(a, b, num_threads: int = 1):
    """(distance, level-loop ms) from the reference X-TED_CPU standard_ted."""
    la, ao, ai = _arrs(a)
    lb, bo, bi = _arrs(b)
    ms = ctypes.c_double(-1.0)
    d = _ref().xr_standard_ted_int(len(a.labels), _p32(la), _p32(ao), _p32(ai),
                                   len(b.labels), _p32(lb), _p32(bo), _p32(bi),
                                   int(num_threads), ctypes.byref(ms))
    return int(d), float(ms.value)


def ref_distance_str(a_labels, a, b_labels, b, num_threads: int = 1):
    """Like ref_distance but with the original label strings."""
    _, ao, ai = _arrs(a)
    _, bo, bi = _arrs(b)
    ca = (ctypes.c_char_p * max(len(a_labels), 1))(*[s.encode() for s in a_labels])
    cb = (ctypes.c_char_p * max(len(b_labels), 1))(*[s.encode() for s in b_labels])
    ms = ctypes.c_double(-1.0)
    d = _ref().xr_standard_ted_str(len(a_labels), ca, _p32(ao), _p32(ai), len(b_labels), cb,
                                   _p32(bo), _p32(bi), int(num_threads), ctypes.byref(ms))
    return int(d), float(ms.value)
