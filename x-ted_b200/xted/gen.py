"""Seeded synthetic workloads (through ``xted_gen_tree`` of the C ABI).

The reference ships no benchmark generator; its full datasets are not
available offline, so seeded synthetic trees with the benchmark's shapes,
sizes and label distributions stand in for them.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import _lib
from .synth import LABELS, SHAPES, mix as _mix, mixed_specs
from .trees import Tree


def tree(shape: str, n: int, seed: int, labels: str = "uniform", alphabet: int = 26) -> Tree:
    lab = np.zeros(max(n, 1), np.int32)
    off = np.zeros(n + 1, np.int32)
    idx = np.zeros(max(n - 1, 1), np.int32)
    _lib.check(_lib.lib().xted_gen_tree(SHAPES[shape], n, seed & (2**64 - 1), LABELS[labels], alphabet,
                                        lab.ctypes.data_as(_lib._i32p), off.ctypes.data_as(_lib._i32p),
                                        idx.ctypes.data_as(_lib._i32p)), "xted_gen_tree")
    return Tree(lab[:n].copy(), off, idx[:max(n - 1, 0)].copy())


def single_pair_100(seed: int = 1) -> Tuple[Tree, Tree]:
    """Two 100-node random recursive trees, labels uniform over 26 ids."""
    return (tree("random", 100, _mix(seed, 1), "uniform", 26),
            tree("random", 100, _mix(seed, 2), "uniform", 26))


def single_pair_1000(seed: int = 2) -> Tuple[Tree, Tree]:
    """Wide-shallow vs deep-narrow, 1000 nodes each, Zipf(1.1) over 10,000 ids."""
    return (tree("wide", 1000, _mix(seed, 1), "zipf", 10000),
            tree("deep", 1000, _mix(seed, 2), "zipf", 10000))


def single_pair_20000(seed: int = 3, shape: str = "random") -> Tuple[Tree, Tree]:
    """20,000 vs 20,000 nodes (random recursive or caterpillar), 64 uniform labels."""
    return (tree(shape, 20000, _mix(seed, 1), "uniform", 64),
            tree(shape, 20000, _mix(seed, 2), "uniform", 64))


def mixed_batch(npairs: int = 4096, seed: int = 4, lo: int = 50, hi: int = 2000,
                alphabet: int = 1000) -> List[Tuple[Tree, Tree]]:
    """Pairs with log-uniform sizes in [lo, hi], shapes uniform over the four
    kinds, labels Zipf(1.1) over `alphabet` ids, every tree drawn independently."""
    return [tuple(tree(sh, n, sd, "zipf", alphabet) for sh, n, sd in spec)
            for spec in mixed_specs(npairs, seed, lo, hi)]


def corpus(ntrees: int = 1000, seed: int = 5, lo: int = 100, hi: int = 1000,
           alphabet: int = 1000) -> List[Tree]:
    """Serving corpus / query trees: sizes uniform in [lo, hi], mixed shapes."""
    rng = np.random.default_rng(_mix(seed, 7) % (2**63))
    names = list(SHAPES)
    return [tree(names[int(rng.integers(0, 4))], int(rng.integers(lo, hi + 1)), _mix(seed, k), "zipf",
                 alphabet) for k in range(ntrees)]
