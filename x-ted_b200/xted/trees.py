"""Ordered labelled trees in the form the C-ABI takes: preorder CSR.

A tree of n nodes is numbered in preorder (root 0). ``off`` (n+1) and ``idx``
(n-1) list the children of node v, in order, as ``idx[off[v]:off[v+1]]``;
``labels`` holds an int32 id per node. This is the reference's input
(X-TED_CPU/TED.cpp:177: ``vector<string>`` labels plus a preorder
``vector<vector<int>>`` adjacency) with string labels interned to ids, which is
exact because the reference only ever compares labels for equality
(X-TED_CPU/TED.cpp:153-159).

Also here: the reference's text-format parsers (``node_process`` and
``pre_process``, X-TED_CPU/dataset_preprocess.cpp:3-81) so that files in the
reference's dataset format load identically.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Iterable, List, Sequence

import numpy as np


@dataclass
class Tree:
    labels: np.ndarray  # int32 [n]
    off: np.ndarray     # int32 [n+1]
    idx: np.ndarray     # int32 [max(n-1, 0)]

    @property
    def n(self) -> int:
        return int(self.labels.shape[0])

    def __len__(self) -> int:
        return self.n

    def adjacency(self) -> List[List[int]]:
        return [self.idx[self.off[v]:self.off[v + 1]].tolist() for v in range(self.n)]

    def parent(self) -> np.ndarray:
        p = np.full(self.n, -1, np.int32)
        for v in range(self.n):
            p[self.idx[self.off[v]:self.off[v + 1]]] = v
        return p


def from_adjacency(labels: Sequence[int], adj: Sequence[Sequence[int]]) -> Tree:
    n = len(adj)
    if len(labels) != n:
        raise ValueError(f"{len(labels)} labels for {n} adjacency rows")
    off = np.zeros(n + 1, np.int32)
    for v, ch in enumerate(adj):
        off[v + 1] = off[v] + len(ch)
    idx = np.fromiter((c for ch in adj for c in ch), dtype=np.int32, count=int(off[-1]))
    return Tree(np.asarray(labels, dtype=np.int32).reshape(n), off, idx)


def from_parent(labels: Sequence[int], parent: Sequence[int]) -> Tree:
    """Preorder parent array (parent[0] == -1) -> Tree. Siblings are ordered by
    their preorder index, which is their left-to-right order."""
    parent = np.asarray(parent, dtype=np.int64)
    n = parent.shape[0]
    adj: List[List[int]] = [[] for _ in range(n)]
    for v in range(1, n):
        adj[int(parent[v])].append(v)
    return from_adjacency(labels, adj)


def is_preorder(t: Tree) -> bool:
    """True when the CSR lists a single tree rooted at 0 whose numbering is a
    preorder traversal with children in increasing order (the reference assumes
    this and never checks it, README.md:31-44)."""
    n = t.n
    if n == 0:
        return True
    if t.off.shape[0] != n + 1 or t.off[0] != 0 or t.off[-1] != n - 1:
        return False
    expect = 1
    stack = [0]
    # iterative preorder walk: the k-th visited node must be k
    order = []
    while stack:
        v = stack.pop()
        order.append(v)
        ch = t.idx[t.off[v]:t.off[v + 1]]
        for c in ch[::-1]:
            if c < 0 or c >= n:
                return False
            stack.append(int(c))
        if len(order) > n:
            return False
    del expect
    return order == list(range(n))


def mirror(t: Tree) -> Tree:
    """Reverse every child list and renumber in preorder (TED is invariant
    under mirroring both trees)."""
    n = t.n
    if n == 0:
        return t
    order = []
    stack = [0]
    while stack:
        v = stack.pop()
        order.append(v)
        stack.extend(int(c) for c in t.idx[t.off[v]:t.off[v + 1]])  # reversed visit
    new = np.empty(n, np.int64)
    new[np.asarray(order)] = np.arange(n)
    adj: List[List[int]] = [[] for _ in range(n)]
    for v in range(n):
        adj[int(new[v])] = [int(new[c]) for c in t.idx[t.off[v]:t.off[v + 1]][::-1]]
    labels = np.empty(n, np.int32)
    labels[new] = t.labels
    return from_adjacency(labels, adj)


# ---------------------------------------------------------------------------
# The reference's dataset text format (X-TED_CPU/dataset_preprocess.cpp).
# ---------------------------------------------------------------------------

def node_process(line: str) -> List[str]:
    """Space-separated labels; a token is emitted only when a space follows it
    (X-TED_CPU/dataset_preprocess.cpp:68-81)."""
    out, part = [], []
    for ch in line:
        if ch != " ":
            part.append(ch)
        else:
            out.append("".join(part))
            part = []
    return out


def _to_vector(s: str) -> List[int]:
    # X-TED_CPU/dataset_preprocess.cpp:7-34: strip the brackets, split on ','
    s = s[1:-1]
    if not s:
        return []
    vals, word = [], ""
    for i, ch in enumerate(s):
        if ch != " " and ch != ",":
            word += ch
            if i == len(s) - 1:
                vals.append(int(word))
                word = ""
        elif ch == ",":
            vals.append(int(word))
            word = ""
    return vals


def pre_process(line: str) -> List[List[int]]:
    """``[[1, 2], [], ...]`` -> adjacency (X-TED_CPU/dataset_preprocess.cpp:36-66)."""
    s = line[1:-1]
    parts = []
    i = 0
    while i < len(s):
        if s[i] == "[":
            k = s.index("]", i)
            parts.append(s[i:k + 1])
        i += 1
    return [_to_vector(p) for p in parts]


def read_lines(path: str) -> List[str]:
    """Lines as std::getline returns them (newline stripped, nothing else)."""
    with open(path, "rb") as f:
        data = f.read().decode("utf-8", errors="surrogateescape")
    lines = data.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    return lines


class Interner:
    """Maps label strings to dense int32 ids (equality-preserving)."""

    def __init__(self) -> None:
        self.ids: Dict[str, int] = {}

    def __call__(self, labels: Iterable[str]) -> np.ndarray:
        out = []
        for s in labels:
            v = self.ids.get(s)
            if v is None:
                v = len(self.ids)
                self.ids[s] = v
            out.append(v)
        return np.asarray(out, dtype=np.int32)


def load_pair(labels_path: str, adj_path: str, i: int = 0, j: int = 1):
    """Trees i and j of a reference dataset file pair, labels interned jointly.
    Returns (tree_i, tree_j, strings_i, strings_j)."""
    nodes, adjs = read_lines(labels_path), read_lines(adj_path)
    si, sj = node_process(nodes[i]), node_process(nodes[j])
    ai, aj = pre_process(adjs[i]), pre_process(adjs[j])
    intern = Interner()
    ti = from_adjacency(intern(si), ai)
    tj = from_adjacency(intern(sj), aj)
    return ti, tj, si, sj


# ---- large corpora: the library's C parsers ----

def parse_adjacency(line: str):
    """``[[1, 2], [], ...]`` -> (child_off, child_idx) int32 arrays, read by the
    library's parser (the grammar of ``pre_process``, at C speed)."""
    import ctypes

    from . import _lib
    raw = line.encode("utf-8", errors="surrogateescape")
    cap_n = raw.count(b"[") + 1
    cap_e = raw.count(b",") + 2
    off = np.zeros(cap_n + 1, np.int32)
    idx = np.zeros(max(cap_e, 1), np.int32)
    n, e = ctypes.c_int32(0), ctypes.c_int32(0)
    _lib.check(_lib.lib().xted_parse_adjacency(raw, len(raw), cap_n, cap_e, off.ctypes.data_as(_lib._i32p),
                                               idx.ctypes.data_as(_lib._i32p), ctypes.byref(n), ctypes.byref(e)),
               "xted_parse_adjacency")
    return off[:n.value + 1].copy(), idx[:e.value].copy()


def _unescape(label: str) -> str:
    out, i = [], 0
    while i < len(label):
        if label[i] == "\\" and i + 1 < len(label):
            out.append(label[i + 1])
            i += 2
        else:
            out.append(label[i])
            i += 1
    return "".join(out)


def parse_bracket(text: str, intern: "Interner | None" = None):
    """One tree in bracket notation, ``{a{b}{c{d}}}`` -> (Tree, label strings).
    Labels are interned with ``intern`` (a fresh Interner if None)."""
    import ctypes

    from . import _lib
    raw = text.encode("utf-8", errors="surrogateescape")
    cap = raw.count(b"{") + 1
    off = np.zeros(cap + 1, np.int32)
    idx = np.zeros(cap, np.int32)
    at = np.zeros(cap, np.int64)
    ln = np.zeros(cap, np.int32)
    n, end = ctypes.c_int32(0), ctypes.c_int64(0)
    _lib.check(_lib.lib().xted_parse_bracket(raw, len(raw), cap, off.ctypes.data_as(_lib._i32p),
                                             idx.ctypes.data_as(_lib._i32p), at.ctypes.data_as(_lib._i64p),
                                             ln.ctypes.data_as(_lib._i32p), ctypes.byref(n), ctypes.byref(end)),
               "xted_parse_bracket")
    k = n.value
    strings = [_unescape(raw[int(a):int(a) + int(b)].decode("utf-8", errors="surrogateescape"))
               for a, b in zip(at[:k], ln[:k])]
    intern = intern if intern is not None else Interner()
    return Tree(intern(strings), off[:k + 1].copy(), idx[:max(k - 1, 0)].copy()), strings


def to_bracket(strings: Sequence[str], t: Tree) -> str:
    """Bracket notation of a tree (labels escaped)."""
    def esc(x: str) -> str:
        return x.replace("\\", "\\\\").replace("{", "\\{").replace("}", "\\}")
    out = []
    stack = [(0, False)]
    while stack:
        v, closing = stack.pop()
        if closing:
            out.append("}")
            continue
        out.append("{" + esc(strings[v]))
        stack.append((v, True))
        for c in reversed(t.idx[t.off[v]:t.off[v + 1]].tolist()):
            stack.append((c, False))
    return "".join(out)


def load_dataset(labels_path: str, adj_path: str, intern: "Interner | None" = None):
    """Every tree of a reference dataset file pair (one tree per line), labels
    interned jointly. Returns (trees, label strings per tree)."""
    intern = intern if intern is not None else Interner()
    nodes, adjs = read_lines(labels_path), read_lines(adj_path)
    out_t, out_s = [], []
    for lab_line, adj_line in zip(nodes, adjs):
        strings = lab_line.split(" ")[:-1]  # node_process's rule: a token ends at each space
        off, idx = parse_adjacency(adj_line)
        if len(off) - 1 != len(strings):
            raise ValueError(f"{len(strings)} labels for {len(off) - 1} adjacency rows")
        out_t.append(Tree(intern(strings), off, idx))
        out_s.append(strings)
    return out_t, out_s


def load_bracket(path: str, intern: "Interner | None" = None):
    """Every tree of a bracket-notation file (one tree per line)."""
    intern = intern if intern is not None else Interner()
    out_t, out_s = [], []
    for line in read_lines(path):
        if line.strip():
            t, strings = parse_bracket(line, intern)
            out_t.append(t)
            out_s.append(strings)
    return out_t, out_s
