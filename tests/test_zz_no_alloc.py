"""xted_distance_noalloc: the allocation-free single-pair entry point.

Collected last on purpose (file name), so it runs both after every other test
in one process and alone in a fresh one. Each GPU test calls the entry point
through the C ABI twice in a row and compares it with xted_distance.
"""
import ctypes

import numpy as np
import pytest

import xted
from xted import _lib, gen, trees

PAIRS = [
    ("random", 120, "random", 90),
    ("deep", 200, "caterpillar", 150),
    ("wide", 300, "random", 64),
    ("caterpillar", 40, "deep", 260),
    ("random", 1, "random", 50),
    ("random", 700, "random", 700),
]


def _pairs():
    out = []
    for k, (sa, na, sb, nb) in enumerate(PAIRS):
        a = gen.tree(sa, na, 1000 + k, "zipf", 16)
        b = gen.tree(sb, nb, 2000 + k, "zipf", 16)
        out.append((a, b))
    return out


def _noalloc(a, b, device=0):
    keep = []
    ta, tb = _lib.ctree(a, keep), _lib.ctree(b, keep)
    out = ctypes.c_int32(-1)
    rc = _lib.lib().xted_distance_noalloc(ctypes.byref(ta), ctypes.byref(tb), device, ctypes.byref(out))
    return rc, out.value


def test_rejects_pairs_beyond_the_arena():
    # checked before any device call, so this runs without a GPU too
    big = gen.tree("random", 3000, 5)
    rc, _ = _noalloc(big, big)
    assert rc == xted.XTED_ETOOBIG
    assert "arena" in _lib.lib().xted_strerror(rc).decode()


@pytest.mark.gpu
def test_noalloc_matches_batched_entry_twice_in_a_row():
    pairs = _pairs()
    with xted.Context(device=0) as ctx:
        want = [ctx.distance(a, b) for a, b in pairs]
    for _ in range(2):
        got = []
        for k, (a, b) in enumerate(pairs):
            rc, d = _noalloc(a, b)
            assert rc == 0, (k, rc)
            got.append(d)
        assert got == want


@pytest.mark.gpu
def test_noalloc_later_calls_take_no_device_memory_and_keep_the_device():
    """After the first (warm-up) call, which loads the module and commits the
    arena, further calls leave the device's free memory unchanged; every call
    restores the caller's current device."""
    import torch
    torch.cuda.init()
    a, b = _pairs()[1]
    assert _noalloc(a, b)[0] == 0  # warm-up: module load and arena commit happen here (or earlier)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for a, b in _pairs():
        assert _noalloc(a, b)[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert torch.cuda.current_device() == 0


@pytest.mark.gpu
def test_noalloc_edge_cases():
    t = gen.tree("random", 30, 9)
    empty = trees.Tree(np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32))
    assert _noalloc(t, empty) == (0, 30)
    assert _noalloc(empty, t) == (0, 30)
    assert _noalloc(empty, empty) == (0, 0)
    assert _noalloc(t, t) == (0, 0)
    # children out of preorder: rejected by the device-side validation
    bad = trees.Tree(np.array([0, 1, 2], np.int32), np.array([0, 2, 2, 2], np.int32), np.array([2, 1], np.int32))
    assert _noalloc(bad, t)[0] == xted.XTED_EINVAL
    assert _noalloc(t, bad)[0] == xted.XTED_EINVAL
    # and the arena is still usable afterwards
    a, b = _pairs()[0]
    with xted.Context(device=0) as ctx:
        assert _noalloc(a, b) == (0, ctx.distance(a, b))
