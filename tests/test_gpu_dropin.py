"""The reference's own caller on this library (needs a B200).

tests/cpp/_build/X-TED_CPU_on_xted is the reference's harness
(X-TED_CPU/main.cpp, TED_test.cpp and its parsers dataset_preprocess.cpp,
compiled unmodified) linked against include/xted.hpp through
tests/cpp/dropin_standard_ted.cpp instead of the reference's TED.cpp and
parallel_computing.cpp (built by `make -C tests/cpp dropin` where the
reference tree is). It reads the reference's label and adjacency text files,
computes tree pair (0, 1) 20 times through the reference's call site
(X-TED_CPU/TED_test.cpp:43) and prints "The distance = d" each time; every
line must equal the reference's own distance from the golden fixture.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(REPO, "tests", "cpp", "_build", "X-TED_CPU_on_xted")


def _write_pair(tmp_path, a, b, tag):
    """Tree pair (a, b) as lines 0 and 1 of the reference's two text formats:
    labels as space-terminated tokens, adjacency as [[c, ...], [], ...]."""
    lab = tmp_path / f"{tag}_nodes.txt"
    adj = tmp_path / f"{tag}_nodes_adj.txt"
    with open(lab, "w") as f:
        for t in (a, b):
            f.write("".join(f"L{int(x)} " for x in t.labels) + "\n")
    with open(adj, "w") as f:
        for t in (a, b):
            rows = ("[" + ", ".join(str(int(c)) for c in t.idx[t.off[v]:t.off[v + 1]]) + "]" for v in range(t.n))
            f.write("[" + ", ".join(rows) + "]\n")
    return str(lab), str(adj)


def test_reference_harness_runs_on_xted(golden_datasets, tmp_path):
    assert os.path.exists(EXE), f"{EXE} is not built (make -C tests/cpp dropin, with the reference tree present)"
    cases = [c for c in golden_datasets if max(c[1].n, c[2].n) <= 1000][::6][:6]
    assert cases
    for k, (name, a, b, want) in enumerate(cases):
        lab, adj = _write_pair(tmp_path, a, b, f"c{k}")
        r = subprocess.run([EXE, "8", lab, adj], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (name, r.stderr[-2000:])
        got = [int(l.split("=")[1]) for l in r.stdout.splitlines() if l.startswith("The distance =")]
        assert got == [want] * 20, (name, got[:3], want)
