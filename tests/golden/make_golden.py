"""Regenerate the golden fixtures from the reference X-TED_CPU.

Run in a container that holds the reference tree (read at /root/reference)
after ``make -C oracle all ref``:

    python tests/golden/make_golden.py datasets    # -> datasets.json.gz
    python tests/golden/make_golden.py synthetic   # -> synthetic.json.gz
    python tests/golden/make_golden.py bracket     # -> bracket.json.gz
    python tests/golden/make_golden.py configs     # -> configs.json.gz

datasets: tree pair (0, 1) of every file of the reference's sampled datasets
  (Sampled_Dataset/*, Sampled_Dataset_Extra_Large_Trees/*), which is the pair the
  reference CLI computes (X-TED_CPU/TED_test.cpp:31). Labels are interned to
  int ids per pair; the expected distance is the reference's own
  ``standard_ted`` on the ORIGINAL label strings, cross-checked for the small
  files against the ``The distance = d`` line of the reference CLI built from
  the same sources.

synthetic: seeded trees from the product generator (all four shapes, sizes
  1..400, both label alphabets), expected distances from the reference
  ``standard_ted`` on decimal-string labels.

configs: the benchmark workloads themselves, regenerated from their seeds by
  the product generator (xted.gen): the 1,000-node wide-shallow vs deep-narrow
  pair, both 20,000-node pairs (random recursive and caterpillar), every pair
  of the 4,096-pair mixed batch (seed 4), and the first 8 queries of the
  serving pool (seed 6) against the whole 1,000-tree serving corpus (seed 5).
  Expected distances from the reference ``standard_ted`` (all 8 threads for a
  single pair; one thread per pair, one spawned worker per core, for the
  batches). Trees are stored as a short SHA-256 of their CSR arrays, so a
  change of the generator fails loudly instead of silently changing the
  workload.

Every tree of datasets/synthetic is stored as {"labels": [...], "parent": [...]}
in preorder.
"""
from __future__ import annotations

import glob
import gzip
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "x-ted_b200"))

import oracle  # noqa: E402
from xted import trees  # noqa: E402

REF = "/root/reference"


def _tree_json(t):
    return {"labels": t.labels.tolist(), "parent": t.parent().tolist()}


def _cli_distance(lab_path, adj_path):
    exe = os.path.join(REPO, "oracle", "_ref", "X-TED_CPU")
    out = subprocess.run([exe, "8", lab_path, adj_path], capture_output=True, text=True,
                         check=True).stdout
    ds = [int(l.split("=")[1]) for l in out.splitlines() if l.startswith("The distance =")]
    assert len(set(ds)) == 1, ds
    return ds[0]


def datasets():
    files = sorted(glob.glob(os.path.join(REF, "Sampled_Dataset", "*", "*_nodes*.txt")))
    files += sorted(glob.glob(os.path.join(REF, "Sampled_Dataset_Extra_Large_Trees", "*", "*",
                                           "*_nodes_*.txt")))
    cases = []
    for lab in files:
        base = os.path.basename(lab)
        if "_adj" in base or "synthetic_tree" in base:
            continue
        adj = lab.replace("_nodes_", "_nodes_adj_") if "_nodes_" in base else \
            lab.replace("_nodes.txt", "_nodes_adj.txt")
        a, b, sa, sb = trees.load_pair(lab, adj, 0, 1)
        assert trees.is_preorder(a) and trees.is_preorder(b), lab
        d, _ = oracle.ref_distance_str(sa, a, sb, b, num_threads=8)
        small = max(a.n, b.n) <= 1200
        if small:
            assert _cli_distance(lab, adj) == d, lab
        name = os.path.relpath(lab, REF)
        cases.append({"name": name, "a": _tree_json(a), "b": _tree_json(b), "distance": d,
                      "cli_checked": small})
        print(f"{name}: m={a.n} n={b.n} d={d}", flush=True)
    with gzip.open(os.path.join(HERE, "datasets.json.gz"), "wt") as f:
        json.dump({"source": "reference X-TED_CPU standard_ted, tree pair (0,1)", "cases": cases}, f)


def synthetic():
    from xted import gen  # product generator (needs the built library)
    cases = []
    seed = 20261203
    shapes = ["random", "wide", "deep", "caterpillar"]
    sizes = [1, 2, 3, 5, 8, 13, 21, 34, 55, 100, 150, 250, 400]
    k = 0
    for si, sa in enumerate(shapes):
        for sb in shapes:
            for na in sizes:
                nb = sizes[(sizes.index(na) * 7 + si + 3) % len(sizes)]
                alpha = 4 if k % 3 == 0 else (26 if k % 3 == 1 else 1000)
                a = gen.tree(sa, na, seed + 2 * k, labels="uniform", alphabet=alpha)
                b = gen.tree(sb, nb, seed + 2 * k + 1, labels="uniform", alphabet=alpha)
                d, _ = oracle.ref_distance(a, b, num_threads=4)
                cases.append({"name": f"{sa}{na}-{sb}{nb}-a{alpha}", "a": _tree_json(a),
                              "b": _tree_json(b), "distance": d})
                k += 1
    # the plain single-pair workload: two 100-node random recursive trees, 26 labels
    a = gen.tree("random", 100, 1, labels="uniform", alphabet=26)
    b = gen.tree("random", 100, 2, labels="uniform", alphabet=26)
    d, _ = oracle.ref_distance(a, b, num_threads=4)
    cases.append({"name": "single-pair-100x100-seed1-2", "a": _tree_json(a), "b": _tree_json(b),
                  "distance": d})
    with gzip.open(os.path.join(HERE, "synthetic.json.gz"), "wt") as f:
        json.dump({"source": "reference X-TED_CPU standard_ted on generator trees", "cases": cases},
                  f)
    print(f"{len(cases)} synthetic cases")


def bracket():
    """The reference's bracket-notation files (read by none of its code) for
    1,000 and 2,000 nodes, with the trees its label/adjacency files hold for
    the same datasets (lines 0 and 1, parsed by the reference's own rules) and
    the reference distance of the pair."""
    cases = []
    for n in (1000, 2000):
        d = os.path.join(REF, "Sampled_Dataset_Extra_Large_Trees", "synthetic", f"{n}_nodes")
        with open(os.path.join(d, f"synthetic_tree_{n}.txt"), "rb") as f:
            text = f.read().decode("utf-8", errors="surrogateescape")
        lab, adj = (os.path.join(d, f"synthetic_nodes_{n}.txt"), os.path.join(d, f"synthetic_nodes_adj_{n}.txt"))
        nodes, adjs = trees.read_lines(lab), trees.read_lines(adj)
        expect = []
        for k in (0, 1):
            strings = trees.node_process(nodes[k])
            t = trees.from_adjacency(list(range(len(strings))), trees.pre_process(adjs[k]))
            expect.append({"labels": strings, "parent": t.parent().tolist()})
        a, b, sa, sb = trees.load_pair(lab, adj, 0, 1)
        dist, _ = oracle.ref_distance_str(sa, a, sb, b, num_threads=8)
        cases.append({"name": os.path.relpath(os.path.join(d, f"synthetic_tree_{n}.txt"), REF), "text": text,
                      "trees": expect, "distance": dist})
        print(f"bracket {n}: d={dist}", flush=True)
    with gzip.open(os.path.join(HERE, "bracket.json.gz"), "wt") as f:
        json.dump({"source": "reference bracket files; expected trees from its label/adjacency files; distance "
                             "from its standard_ted", "cases": cases}, f)


def tree_hash(t):
    """First 16 hex digits of the SHA-256 of a tree's labels | off | idx (int32)."""
    import hashlib

    import numpy as np
    h = hashlib.sha256()
    for arr in (t.labels, t.off, t.idx):
        h.update(np.ascontiguousarray(arr, dtype=np.int32).tobytes())
    return h.hexdigest()[:16]


def _ref_pair(pair):
    a, b = pair
    return oracle.ref_distance(a, b, num_threads=1)


def _ref_parallel(pairs):
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        return [d for d, _ in pool.map(_ref_pair, pairs, chunksize=1)]


def configs():
    import time

    from xted import gen
    out = {"source": "reference X-TED_CPU standard_ted on the benchmark workloads (xted.gen seeds)"}
    singles = []
    for name, pair in (("single1000", gen.single_pair_1000()),
                       ("single20000_caterpillar", gen.single_pair_20000(shape="caterpillar")),
                       ("single20000_random", gen.single_pair_20000(shape="random"))):
        a, b = pair
        t0 = time.perf_counter()
        d, level_ms = oracle.ref_distance(a, b, num_threads=8)
        wall = time.perf_counter() - t0
        singles.append({"name": name, "a": tree_hash(a), "b": tree_hash(b), "m": a.n, "n": b.n, "distance": d,
                        "ref_level_ms_8_threads": round(level_ms, 1), "ref_wall_s_8_threads": round(wall, 2)})
        print(f"{name}: d={d} ({wall:.1f} s)", flush=True)
    out["singles"] = singles
    pairs = gen.mixed_batch(4096, seed=4)
    t0 = time.perf_counter()
    dist = _ref_parallel(pairs)
    print(f"batch4096: {len(dist)} pairs ({time.perf_counter() - t0:.1f} s)", flush=True)
    out["batch4096"] = {"seed": 4, "npairs": 4096, "hashes": [[tree_hash(a), tree_hash(b)] for a, b in pairs],
                        "distances": dist}
    corpus = gen.corpus(1000, seed=5)
    queries = gen.corpus(64, seed=6)[:8]
    t0 = time.perf_counter()
    flat = _ref_parallel([(q, t) for q in queries for t in corpus])
    print(f"serve: {len(flat)} pairs ({time.perf_counter() - t0:.1f} s)", flush=True)
    out["serve"] = {"corpus_seed": 5, "ntrees": 1000, "query_seed": 6, "nqueries": len(queries),
                    "corpus_hashes": [tree_hash(t) for t in corpus], "query_hashes": [tree_hash(q) for q in queries],
                    "distances": [flat[k * len(corpus):(k + 1) * len(corpus)] for k in range(len(queries))]}
    with gzip.open(os.path.join(HERE, "configs.json.gz"), "wt") as f:
        json.dump(out, f)


if __name__ == "__main__":
    what = sys.argv[1:] or ["datasets", "synthetic", "bracket", "configs"]
    for w in what:
        {"datasets": datasets, "synthetic": synthetic, "bracket": bracket, "configs": configs}[w]()
