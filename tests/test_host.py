"""Host-side logic and the C ABI surface (CPU only; no device calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
import xted
from xted import gen, trees

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_node_process_matches_reference_rule():
    # X-TED_CPU/dataset_preprocess.cpp:68-81: a token is emitted only at a space
    assert trees.node_process("a b c ") == ["a", "b", "c"]
    assert trees.node_process("a b c") == ["a", "b"]
    assert trees.node_process("a  b ") == ["a", "", "b"]


def test_pre_process_matches_reference_format():
    assert trees.pre_process("[[1, 2], [], [3, 4], [], []]") == [[1, 2], [], [3, 4], [], []]
    assert trees.pre_process("[[]]") == [[]]
    assert trees.pre_process("[[1], [2], []]") == [[1], [2], []]


def test_from_parent_roundtrip():
    t = gen.tree("random", 300, 9)
    u = trees.from_parent(t.labels, t.parent())
    assert np.array_equal(t.off, u.off) and np.array_equal(t.idx, u.idx)


@pytest.mark.parametrize("shape", ["random", "wide", "deep", "caterpillar"])
def test_generator_valid_and_deterministic(shape):
    for n in (1, 2, 17, 500):
        t = gen.tree(shape, n, 77, "zipf", 1000)
        assert len(t) == n
        assert trees.is_preorder(t)
        assert xted.validate(t)
        u = gen.tree(shape, n, 77, "zipf", 1000)
        assert np.array_equal(t.labels, u.labels) and np.array_equal(t.idx, u.idx)
        assert t.labels.min() >= 0 and t.labels.max() < 1000


def _depths(t):
    d = np.zeros(len(t), np.int64)
    for v in range(len(t)):
        for c in t.idx[t.off[v]:t.off[v + 1]]:
            d[c] = d[v] + 1
    return d


def test_generator_shapes():
    w = gen.tree("wide", 1000, 1)
    assert _depths(w).max() <= 4 and w.off[1] - w.off[0] == 40
    d = gen.tree("deep", 1000, 1)
    assert _depths(d).max() >= 99
    c = gen.tree("caterpillar", 1000, 1)
    # spine child is the last child of every spine node
    assert c.off[1] - c.off[0] == 10 and c.idx[c.off[1] - 1] == 10
    assert _depths(c).max() == 100


def test_validate_rejects_malformed():
    ok = trees.from_adjacency([0, 1, 2], [[1, 2], [], []])
    assert xted.validate(ok)
    bad_order = trees.Tree(np.array([0, 1, 2], np.int32), np.array([0, 2, 2, 2], np.int32),
                           np.array([2, 1], np.int32))  # children out of preorder
    assert not xted.validate(bad_order)
    bad_range = trees.Tree(np.array([0, 1], np.int32), np.array([0, 1, 1], np.int32), np.array([5], np.int32))
    assert not xted.validate(bad_range)
    bad_count = trees.Tree(np.array([0, 1, 2], np.int32), np.array([0, 1, 1, 1], np.int32), np.array([1], np.int32))
    assert not xted.validate(bad_count)
    not_pre = trees.from_adjacency([0, 1, 2, 3], [[1, 3], [], [], []])  # node 2 unreachable
    assert not xted.validate(not_pre)


def test_pair_cells_match_oracle_keyroot_sums():
    for s in ("random", "wide", "deep", "caterpillar"):
        a = gen.tree(s, 400, 3)
        b = gen.tree("random", 250, 4)
        cr, cl, chosen = xted.pair_cells(a, b)
        assert cr == oracle.tree_stats(a)[2] * oracle.tree_stats(b)[2]
        assert cl == oracle.tree_stats(trees.mirror(a))[2] * oracle.tree_stats(trees.mirror(b))[2]
        assert chosen == min(cr, cl)


def _declared_functions():
    hdr = open(os.path.join(REPO, "include", "xted.h")).read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(xted_\w+)\s*\(", hdr, re.M)))


def test_library_exports_every_declared_symbol():
    names = _declared_functions()
    assert "xted_distance" in names and "xted_query_poll" in names
    L = ctypes.CDLL(xted.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_context_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(xted.XtedError) as e:
        xted.Context()
    assert e.value.code == xted.XTED_ENODEV


def test_planner_emulation_matches_oracle(tmp_path):
    """Runs the batch planner's functions (plan_core.h, the code of the device
    planning kernels) sequentially with a CPU emulation of the unit execution
    (tests/cpp/plan_emu.cpp) and checks distances and plan invariants; every
    fourth single-segment unit is also computed in column stripes of 2-16
    columns (the multi-block decomposition) and must write the same table."""
    obj = tmp_path / "xo.o"
    exe = tmp_path / "plan_emu"
    subprocess.run(["gcc", "-O2", "-c", os.path.join(REPO, "oracle", "xted_oracle.c"), "-o", str(obj)], check=True)
    # the second build makes runs of more than 30 rows "long" (single-unit
    # narrow tasks), which the product reaches only on trees above 4,096 nodes;
    # the third plans every whole-block unit wider than 40 columns as stripe
    # tasks (the product: wider than 2,048), checking their layout
    exe_long = tmp_path / "plan_emu_long"
    exe_st = tmp_path / "plan_emu_stripes"
    for flags, out in (([], exe), (["-DXTED_LONG_RUN_ROWS=30"], exe_long), (["-DXTED_STRIPE_MIN_WIDTH=40"], exe_st)):
        subprocess.run(["g++", "-O2", "-std=c++17", "-I/usr/local/cuda/include", *flags,
                        os.path.join(REPO, "tests", "cpp", "plan_emu.cpp"), str(obj), "-o", str(out), "-lpthread"],
                       check=True)
    for prog, window in ((exe, "8"), (exe, "2"), (exe_long, "8"), (exe_st, "8")):  # "2": forces stack reloads
        r = subprocess.run([str(prog), "100", "250", "99", window], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("ok")


def test_serving_planner_emulation_matches_oracle(tmp_path):
    """Runs the serving planner (serve_plan.h: corpus pools, per-slot query
    plans, offset fix-ups) and an interleaved execution of several queries'
    pairs with the kernels' row math (tests/cpp/serve_emu.cpp), checking
    every index against its pool and every distance against the oracle."""
    obj = tmp_path / "xo.o"
    exe = tmp_path / "serve_emu"
    subprocess.run(["gcc", "-O2", "-c", os.path.join(REPO, "oracle", "xted_oracle.c"), "-o", str(obj)], check=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I/usr/local/cuda/include",
                    os.path.join(REPO, "tests", "cpp", "serve_emu.cpp"), str(obj), "-o", str(exe), "-lpthread"],
                   check=True)
    for seed in ("7", "8", "9"):
        r = subprocess.run([str(exe), "12", "150", seed], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("ok")


def test_tune_table_well_formed():
    """The autotuned per-size table the library compiles in: sizes ascending,
    the last row open-ended, every value inside the planner's limits."""
    src = open(os.path.join(REPO, "x-ted_b200", "csrc", "tune_table.h")).read()
    rows = re.findall(r"\{\s*([0-9<\s]+),\s*(-?\d+),\s*(-?\d+),\s*(-?\d+)\s*\}", src)
    assert rows
    max_n = [eval(r[0]) for r in rows]  # noqa: S307 -- integer literals and shifts from the generated header
    assert max_n == sorted(max_n) and max_n[-1] >= 1 << 30
    for _, rr, nw, hw in rows:
        assert 1 <= int(rr) <= 4096 and 0 <= int(nw) <= 256 and int(hw) <= 1024


def test_autotune_guard_keeps_rows_that_help_every_batch():
    """The autotuner's mixed-batch guard (xted.autotune.guarded_merge) on a fake
    timer: a proposed row is taken only if the batches get faster in total and
    none slows by more than the tolerance, one bucket at a time."""
    from xted import autotune as A
    current = A.read_header()
    assert [r[0] for r in current] == [b[0] for b in A.BUCKETS]
    # the (1,024, 2,048, 4,096)-pair times each proposed row would cause, as deltas in ms
    effect = {1: (-2.0, -1.0, -3.0),   # faster everywhere: taken
              2: (+5.0, +1.0, -10.0),  # faster in total, 5% slower on 1,024 pairs (coarse tasks): refused
              4: (-0.5, +0.1, -0.5)}   # 0.1 ms slower on 2,048 pairs, inside 1%: taken
    proposed = [r if k not in effect else (r[0], r[1] * 2, r[2], r[3]) for k, r in enumerate(current)]

    def fake(rows):
        t = [100.0, 125.0, 230.0]
        for k, d in effect.items():
            if tuple(rows[k]) == tuple(proposed[k]):
                t = [a + b for a, b in zip(t, d)]
        return t
    table, times, taken = A.guarded_merge(current, proposed, fake, tol=0.01)
    assert taken == [1, 4]
    assert table[2] == current[2] and table[1] == proposed[1] and table[4] == proposed[4]
    assert times == fake(table)
    assert A.accept([1.0, 1.0], [0.9, 1.009]) and not A.accept([1.0, 1.0], [0.8, 1.02])
    with pytest.raises(ValueError):
        A.guarded_merge(current, proposed[:-1], fake)


def test_autotune_header_round_trip(tmp_path):
    """What the autotuner writes is what it (and the library build) reads back."""
    from xted import autotune as A
    rows = [(128, 16, 128, -1), (1024, 64, 256, 768), (1 << 30, 128, 128, 512)]
    path = str(tmp_path / "tune_table.h")
    A.write_header(rows, ["a note"], path)
    assert A.read_header(path) == rows
    src = open(path).read()
    assert "// a note" in src and "static const XTuneRow kTuneTable[]" in src


def _bracket_cases():
    import gzip
    import json
    with gzip.open(os.path.join(REPO, "tests", "golden", "bracket.json.gz"), "rt") as f:
        return json.load(f)["cases"]


def test_bracket_parser_against_reference_files():
    """The reference's bracket files hold the same trees as its label and
    adjacency files (fixture made from both, tests/golden/make_golden.py)."""
    for case in _bracket_cases():
        ts, ss = [], []
        for line in case["text"].split("\n"):
            if line.strip():
                t, strings = trees.parse_bracket(line)
                ts.append(t)
                ss.append(strings)
        assert len(ts) == len(case["trees"]) == 2
        for t, strings, want in zip(ts, ss, case["trees"]):
            assert strings == want["labels"]
            assert t.parent().tolist() == want["parent"]
            assert xted.validate(t)


def test_bracket_round_trip_with_escapes():
    t = gen.tree("random", 300, 12, "zipf", 40)
    strings = [("{x}" if v % 5 == 0 else "") + str(v) + ("\\" if v % 7 == 0 else "") for v in t.labels.tolist()]
    u, back = trees.parse_bracket(trees.to_bracket(strings, t))
    assert back == strings
    assert np.array_equal(u.off, t.off) and np.array_equal(u.idx, t.idx)


def test_adjacency_parser_matches_reference_rules(golden_datasets, tmp_path):
    """The C adjacency parser against pre_process (the reference's rules) on
    every golden dataset tree, and whole-file loading."""
    lab_lines, adj_lines, want = [], [], []
    for name, a, b, _ in golden_datasets[:12]:
        for t in (a, b):
            line = "[" + ", ".join("[" + ", ".join(str(c) for c in t.idx[t.off[v]:t.off[v + 1]]) + "]"
                                   for v in range(len(t))) + "]"
            off, idx = trees.parse_adjacency(line)
            assert np.array_equal(off, t.off) and np.array_equal(idx, t.idx), name
            assert trees.pre_process(line) == t.adjacency()
            lab_lines.append("".join(f"L{x} " for x in t.labels.tolist()))
            adj_lines.append(line)
            want.append(t)
    (tmp_path / "n.txt").write_text("\n".join(lab_lines) + "\n")
    (tmp_path / "a.txt").write_text("\n".join(adj_lines) + "\n")
    got, strings = trees.load_dataset(str(tmp_path / "n.txt"), str(tmp_path / "a.txt"))
    assert len(got) == len(want)
    for g, w, s in zip(got, want, strings):
        assert np.array_equal(g.off, w.off) and np.array_equal(g.idx, w.idx)
        assert s == [f"L{x}" for x in w.labels.tolist()]


def test_adjacency_parser_rejects_bad_text():
    for bad in ["[[1, 2], [3", "[[1,, 2]]", "[[a]]", "no brackets"]:
        with pytest.raises(xted.XtedError):
            trees.parse_adjacency(bad)


def test_bench_cpu_baselines_small_sample():
    """The benchmark's two CPU baselines of the reference code (its own
    sequential mode with all cores per pair, and one thread per pair on
    spawned worker processes) on a small sample: rates and labels."""
    import bench
    from xted import gen
    pairs = [(gen.tree("random", 30 + i, i, "uniform", 8), gen.tree("deep", 25 + i, 100 + i, "uniform", 8))
             for i in range(12)]
    v1, i1 = bench.cpu_reference(pairs, 5.0, 1)
    v2, i2 = bench.cpu_reference_pair_parallel(pairs, 5.0, 1)
    assert v1 > 0 and v2 > 0
    assert i1["pairs"] == 12 and i2["pairs"] == 12
    assert "in sequence" in i1["sample"] and "pair-parallel" in i2["sample"]
    assert i2["cores"] == (os.cpu_count() or 1)


def test_bench_reference_arm_builds_its_workload_without_the_cuda_library():
    """The benchmark's reference arm times the reference X-TED_CPU alone: its
    workload (the sampled pairs of the 4,096-pair batch) comes from the
    pure-Python generator and the process never maps lib/libxted.so."""
    import subprocess
    import sys
    code = ("import sys; sys.argv = ['bench.py']\n"
            "import bench\n"
            "pairs, which, cfg, stride = bench.reference_workload('batched')\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(len(pairs), which[1], stride, 'libxted.so' in maps)\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=REPO, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["128", "32", "32", "False"]


def test_cpp_wrapper_compiles_and_converts():
    """include/xted.hpp (the reference-signature C++ wrapper) compiled by
    tests/cpp/Makefile; its string interning and adjacency-to-CSR conversion
    checked on the host (tests/cpp/hpp_check.cpp)."""
    import subprocess
    subprocess.run(["make", "-C", os.path.join(REPO, "tests", "cpp")], check=True, capture_output=True)
    r = subprocess.run([os.path.join(REPO, "tests", "cpp", "_build", "hpp_check")], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_shard_pairs_balances_and_covers():
    """Pair-list sharding by estimated cells (longest first, to the least
    loaded rank): every pair on exactly one rank, loads within one pair's
    cells of each other; the exact top-k merge of per-shard lists; contiguous
    corpus shards."""
    import numpy as np
    from xted import multi
    rng = np.random.default_rng(3)
    cells = rng.integers(1, 10 ** 6, 1000)
    for world in (1, 2, 3, 8):
        parts = multi.shard_pairs(cells, world)
        allp = np.sort(np.concatenate(parts))
        assert np.array_equal(allp, np.arange(1000))
        loads = [int(cells[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(cells.max())
    ids, ds = multi.topk_merge([([4, 9, -1], [2, 5, -1]), ([1, 7], [2, 3])], 3)
    assert ids.tolist() == [1, 4, 7] and ds.tolist() == [2, 2, 3]
    ids, ds = multi.topk_merge([([0], [1])], 3)
    assert ids.tolist() == [0, -1, -1] and ds.tolist() == [1, -1, -1]
    from xted import gen
    corpus = gen.corpus(50, seed=2, lo=1, hi=300)
    ranges = multi.shard_corpus(corpus, 4)
    assert ranges[0][0] == 0 and ranges[-1][1] == 50
    assert all(ranges[r][1] == ranges[r + 1][0] for r in range(3))
