"""Autotuner of the batch planner's granularity, per tree-size bucket.

For each size bucket it builds a seeded batch of pairs whose trees all fall in
the bucket (the four shapes of the mixed workload, Zipf(1.1) labels), runs the
persistent DP with every candidate granularity (row-run length, widest narrow
chunk, widest half-block chunk) and keeps the fastest. The result is written as
``x-ted_b200/csrc/tune_table.h``, which the library compiles in: a context plans
each tree with the row of its size bucket unless the caller sets the
granularity explicitly.

A bucket's best row is tuned on a batch large enough to fill the GPU, which
favours coarse tasks; a smaller batch is bound by its last levels, where coarse
tasks leave blocks idle. So before the header is written each changed row is
tried on mixed batches of several sizes (``MIXED_SIZES``, through
``Context.set_tune_table``, no rebuild) against the table already in the
header, and kept only if the batches are faster in total and none of them is
slower by more than ``--tolerance``.

    python -m xted.autotune            # needs an sm_100 GPU; rebuild afterwards
    python -m xted.autotune --quick    # fewer candidates, for a smoke run
"""
from __future__ import annotations

import argparse
import itertools
import json
import math
import os
import sys
import time

import numpy as np

from . import gen
from .api import Context

BUCKETS = [  # (max_n, tree sizes drawn log-uniformly from [lo, hi), pairs in the batch)
    (128, 50, 128, 8192),
    (256, 128, 256, 4096),
    (512, 256, 512, 2048),
    (1024, 512, 1024, 1024),
    (2048, 1024, 2048, 384),
    (1 << 30, 2048, 4096, 96),
]
MIXED_SIZES = (1024, 2048, 4096)  # pairs of gen.mixed_batch(n, seed=4) the guard times
RUN_ROWS = [16, 32, 64, 128]
NARROW = [128, 256]
HALF = [-1, 384, 512, 768, 1024]

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "csrc", "tune_table.h")


def bucket_pairs(lo: int, hi: int, npairs: int, seed: int):
    rng = np.random.default_rng(seed)
    shapes = list(gen.SHAPES)
    out = []
    for p in range(npairs):
        ts = []
        for s in range(2):
            n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi - 1)))))
            ts.append(gen.tree(shapes[int(rng.integers(0, 4))], n, seed * 100003 + 2 * p + s, "zipf", 1000))
        out.append(tuple(ts))
    return out


def time_config(pairs, run_rows, narrow, half, reps=2, device=0):
    with Context(device=device, run_rows=run_rows, narrow_width=narrow, half_width=half, tuned=False) as c:
        c.prepare_batch(pairs)
        c.run_prepared()
        best = math.inf
        for _ in range(reps):
            c.run_prepared()
            best = min(best, c.stats()["dp_ms"])
    return best


def read_header(path=HEADER):
    """The (max_n, run_rows, narrow_width, half_width) rows of a tune_table.h."""
    rows = []
    for line in open(path):
        t = line.strip()
        if t.startswith("{") and t.endswith("},"):
            f = [x.strip() for x in t[1:-2].split(",")]
            rows.append((1 << 30 if f[0] == "1 << 30" else int(f[0]), int(f[1]), int(f[2]), int(f[3])))
    return rows


def accept(base, cand, tol=0.01):
    """A table is better when the batches are faster in total and none is slower by more than tol."""
    return sum(cand) < sum(base) and all(c <= b * (1 + tol) for b, c in zip(base, cand))


def guarded_merge(current, proposed, time_fn, tol=0.01):
    """Adopts the proposed rows into the current table one bucket at a time, each
    only if accept() holds on time_fn(table) (a list of batch times); returns the
    table, its times and the indices of the rows taken from the proposal."""
    if [r[0] for r in current] != [r[0] for r in proposed]:
        raise ValueError("the two tables have different size buckets")
    table = [tuple(r) for r in current]
    base = time_fn(table)
    taken = []
    for k, row in enumerate(proposed):
        if tuple(row) == table[k]:
            continue
        trial = table[:k] + [tuple(row)] + table[k + 1:]
        t = time_fn(trial)
        if accept(base, t, tol):
            table, base = trial, t
            taken.append(k)
    return table, base, taken


def mixed_timer(sizes=MIXED_SIZES, reps=2, device=0):
    """time_fn for guarded_merge: best DP time of each mixed batch under a table."""
    batches = [gen.mixed_batch(n, seed=4) for n in sizes]

    def time_fn(rows):
        out = []
        with Context(device=device) as c:
            c.set_tune_table(rows)
            for pairs in batches:
                c.prepare_batch(pairs)
                c.run_prepared()
                best = math.inf
                for _ in range(reps):
                    c.run_prepared()
                    best = min(best, c.stats()["dp_ms"])
                out.append(best)
        return out
    return time_fn


def write_header(rows, notes, path=HEADER):
    lines = [
        "// tune_table.h -- granularity per tree-size bucket, written by",
        "// x-ted_b200/xted/autotune.py (do not edit by hand; rerun the tuner).",
        "//",
        "// Row k applies to trees with fewer than max_n nodes (the last row to all",
        "// larger ones): the row-run length of the tree as a row tree, and the widest",
        "// narrow (one warp) and half-block chunks of the tree as a column tree.",
    ]
    lines += ["// " + n for n in notes]
    lines += ["#pragma once", "", '#include "xted_internal.h"', "", "static const XTuneRow kTuneTable[] = {"]
    for max_n, rr, nw, hw in rows:
        lines.append(f"    {{{'1 << 30' if max_n >= (1 << 30) else max_n}, {rr}, {nw}, {hw}}},")
    lines += ["};", "static const int kTuneRows = (int)(sizeof(kTuneTable) / sizeof(kTuneTable[0]));", ""]
    with open(path, "w") as f:
        f.write("\n".join(lines))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--quick", action="store_true", help="default-adjacent candidates only")
    ap.add_argument("--out", default=HEADER)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--tolerance", type=float, default=0.01,
                    help="largest slowdown of one mixed batch a changed row may cause")
    ap.add_argument("--no-guard", action="store_true", help="write the per-bucket bests unchecked")
    args = ap.parse_args(argv)
    cands = list(itertools.product(RUN_ROWS, NARROW, HALF))
    if args.quick:
        cands = [(32, 256, 512), (64, 256, 512), (64, 256, -1), (128, 256, 512)]
    rows, notes = [], []
    t_all = time.time()
    for k, (max_n, lo, hi, npairs) in enumerate(BUCKETS):
        pairs = bucket_pairs(lo, hi, npairs, seed=17 + k)
        res = []
        for rr, nw, hw in cands:
            ms = time_config(pairs, rr, nw, hw, device=args.device)
            res.append((ms, rr, nw, hw))
            print(json.dumps({"bucket": [lo, hi], "run_rows": rr, "narrow_width": nw, "half_width": hw,
                              "dp_ms": round(ms, 3)}), flush=True)
        res.sort()
        best = res[0]
        default = next((r for r in res if r[1:] == (64, 256, 512)), None)
        rows.append((max_n, best[1], best[2], best[3]))
        notes.append(f"sizes [{lo}, {hi}), {npairs} pairs: best {best[0]:.2f} ms (run_rows {best[1]}, narrow "
                     f"{best[2]}, half {best[3]})" + (f", untuned default {default[0]:.2f} ms" if default else ""))
    if not args.no_guard:
        current = read_header(args.out if os.path.exists(args.out) else HEADER)
        timer, seen = mixed_timer(device=args.device), []

        def timed(table):
            t = timer(table)
            seen.append(t)
            print(json.dumps({"mixed_pairs": list(MIXED_SIZES), "table": table, "dp_ms": t}), flush=True)
            return t
        rows, times, taken = guarded_merge(current, rows, timed, args.tolerance)
        notes.append(f"mixed batches of {list(MIXED_SIZES)} pairs: {[round(t, 2) for t in seen[0]]} ms with the "
                     f"previous table, {[round(t, 2) for t in times]} ms with this one; rows taken from this "
                     f"run: {taken} (the others kept)")
    notes.append(f"{len(cands)} candidates per bucket, {time.time() - t_all:.0f} s on "
                 f"{os.environ.get('XTED_TUNE_GPU', 'a B200')}")
    write_header(rows, notes, args.out)
    print("wrote", args.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
