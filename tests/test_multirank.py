"""CPU (gloo, world size 2) tests of bench.py's multi-rank host logic: every
rank runs its own replica, the timed region is the max over ranks, and the
reference arm prints one line from rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

WORKER = r'''
import datetime, os, sys
sys.path.insert(0, %r)
import torch.distributed as dist
import bench
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
v = bench.max_over_ranks(1.5 + r, dist, device="cpu")
w = bench.max_over_ranks(-float(r), dist, device="cpu")
with open(os.path.join(os.environ["OUT_DIR"], "rank%%d.txt" %% r), "w") as f:
    f.write("%%r %%r" %% (v, w))
dist.destroy_process_group()
''' % ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_torchrun(tmp_path, script, args=(), nproc=2, env=None):
    f = tmp_path / "worker.py"
    f.write_text(script)
    e = dict(os.environ)
    e.update(env or {})
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(nproc),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), str(f)] + list(args)
    return subprocess.run(["timeout", "-k", "10", "120"] + cmd, capture_output=True, text=True, env=e)


def test_max_over_ranks_gloo(tmp_path):
    r = run_torchrun(tmp_path, WORKER, env={"OUT_DIR": str(tmp_path)})
    assert r.returncode == 0, r.stderr[-2000:]
    vals = {}
    for rank in (0, 1):
        v, w = (tmp_path / ("rank%d.txt" % rank)).read_text().split()
        vals[rank] = (float(v), float(w))
    assert vals == {0: (2.5, 0.0), 1: (2.5, 0.0)}


def test_reference_arm_prints_once_under_two_ranks(tmp_path):
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference not compiled here")
    r = subprocess.run(["timeout", "-k", "10", "300", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
                        os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3", "--ref-n", "16"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
