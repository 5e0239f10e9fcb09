"""The drop-in hybrid_* command line drivers on the reference README's example
files (README.md:50,53 invocations, :57-96 files), with the reference's
synthesized weights (u+v)%128+1.  Values after the two snapshots were worked
by hand (see tests/test_oracle.py::test_readme_known_answers)."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "c-gpustreamgraph_b200", "bin")
FIX = os.path.join(REPO, "tests", "golden", "readme")


def run(app, tmp_path, *extra):
    out = tmp_path / f"{app}.out"
    cmd = [os.path.join(BIN, app), "-graphfile", os.path.join(FIX, "input.txt"),
           "-format", "market_big", "-hybrid", "0", "-SEGMENT", "512", "-weight_num", "1",
           "-weight", "1", "-update_size", os.path.join(FIX, "stream_size.txt"),
           "-updatefile", os.path.join(FIX, "update.txt"), "-cache", "0", "-output", str(out),
           *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "batch number 1" in r.stdout and "Overall: Test passed" in r.stdout
    return out.read_text().split("\n"), r.stdout


def values(lines):
    vals = {}
    for ln in lines:
        if not ln.strip():
            continue
        p = ln.split()
        vals[int(p[0])] = None if p[1] == "INF" else int(p[1])
    return [vals[i] for i in sorted(vals)]


def test_cli_sssp_bfs_cc(tmp_path):
    lines, _ = run("hybrid_sssp", tmp_path, "-source_node", "0")
    assert values(lines) == [0, None, None, 4, 5]
    lines, _ = run("hybrid_bfs", tmp_path, "-source_node", "0")
    assert values(lines) == [0, None, None, 1, 1]
    lines, _ = run("hybrid_cc", tmp_path)
    assert values(lines) == [0, 1, 2, 0, 0]


def test_cli_pagerank(tmp_path):
    lines, stdout = run("hybrid_pr", tmp_path, "-error", "0.000001")
    got = np.array([float(ln.split()[1]) for ln in lines if ln.strip()])
    src = np.array([0, 0, 1, 2], np.uint32)
    dst = np.array([3, 4, 4, 3], np.uint32)
    row, col, _ = O.csr_file_order(5, src, dst)
    assert np.max(np.abs(got - O.pagerank(5, row, col))) <= 1e-6
    assert "v 0 data" in stdout


def test_cli_rejects_unknown_flags(tmp_path):
    r = subprocess.run([os.path.join(BIN, "hybrid_sssp"), "-graphfile", "x", "-nope", "1"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "unknown command line flag" in r.stderr
