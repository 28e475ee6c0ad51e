"""bench.py's multi-process plumbing on CPU: two gloo ranks on 127.0.0.1.

The replicas-only N > 1 path has one collective, the max over ranks of the
step times; the reference arm works on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO

CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import torch
import bench

class Args:
    impl = sys.argv[2]

rank, local, world, pg = bench.dist_setup(Args())
assert world == 2 and pg is not None
out = bench.max_over_ranks(pg, [1.0 + rank, 10.0 - rank, 0.5], torch.device("cpu"))
ref = bench.run_reference(Args(), rank, world) if rank == 1 else "skipped"
print(json.dumps({"rank": rank, "out": out, "backend": str(pg.get_backend()), "ref": ref}))
pg.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("impl", ("ours", "reference"))
def test_two_gloo_ranks(impl):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("CPU test (with a GPU the ours arm would pick NCCL)")
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, str(REPO), impl], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for r in outs:
        assert r["backend"] == "gloo"
        assert r["out"] == [2.0, 10.0, 0.5]  # each value's maximum, on every rank
    assert outs[1]["ref"] is None  # the reference arm: rank 0 alone works


def test_single_rank_needs_no_group():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench.max_over_ranks(None, [3, 4.5], None) == [3.0, 4.5]
