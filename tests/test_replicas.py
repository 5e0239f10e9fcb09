"""Multi-GPU is replicas only (one independent engine per rank, no
collective on the data path): the bench's rank plumbing is checked here on
CPU with gloo, world size 2 -- the max/sum reductions that turn per-rank
timings into the whole-job line, the barrier, and that only rank 0 prints
(the reference arm runs on rank 0 alone, the others exit 0)."""
import json
import os
import re
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, {repo!r})
import bench
R = bench.Ranks()
assert R.world == 2 and R.pg
mine = [1.5, 4.0][R.rank]
R.barrier()
out = {{"rank": R.rank, "max": R.max(mine), "sum": R.sum(mine)}}
R.barrier()
R.close()
print(json.dumps(out), flush=True)
"""


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run(args, timeout=240):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_port()}"] + args
    return subprocess.run(cmd, cwd=REPO, env=env, capture_output=True, text=True, timeout=timeout)


def test_rank_reductions_gloo(tmp_path):
    w = tmp_path / "worker.py"
    w.write_text(WORKER.format(repo=REPO))
    p = _run([str(w)])
    assert p.returncode == 0, p.stderr[-2000:]
    # the two ranks' lines can interleave on the shared stdout
    lines = [json.loads(x) for x in re.findall(r"\{[^{}]*\}", p.stdout)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    for x in lines:
        assert x["max"] == 4.0 and x["sum"] == 5.5


@pytest.mark.parametrize("workload", ["ppr", "served"])
def test_reference_arm_prints_once_under_torchrun(workload):
    p = _run(["bench.py", "--impl", "reference", "--workload", workload, "--gpus", "2",
              "--steps", "1", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and "unavailable" in lines[0]
