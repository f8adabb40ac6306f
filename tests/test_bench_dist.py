"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1
set up the process group, agree on the slowest rank's time (max over
ranks), and compute the weak-scaling whole-job value; the reference arm's
non-zero ranks exit without joining any collective."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_setup(None, backend="gloo", timeout_s=30)
t = [3.0, 5.0][rank]                      # per-rank milliseconds
bench.barrier(ws)
m = bench.allreduce_max(ws, t)
v = bench.weak_value(ws, 1e9, m)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "ws": ws, "max": m, "value": v}}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, ws, port):
    e = dict(os.environ)
    e.update(WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
             MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    return e


def test_two_gloo_ranks_take_max_and_weak_value():
    port = _free_port()
    code = CHILD.format(root=ROOT)
    procs = [subprocess.Popen([sys.executable, "-c", code], env=_env(r, 2, port),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["ws"] == 2 and o["max"] == 5.0
        assert o["value"] == pytest.approx(2 * 1e9 / 5e-3)


def test_reference_arm_other_ranks_exit_without_work():
    port = _free_port()
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "3", "--warmup", "3"],
                       env=_env(1, 2, port), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    old = {k: os.environ.pop(k, None) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        assert bench.dist_env() == (1, 0, 0)
        assert bench.allreduce_max(1, 7.5) == 7.5
        assert bench.weak_value(1, 2e9, 4.0) == pytest.approx(5e11)
    finally:
        for k, v in old.items():
            if v is not None:
                os.environ[k] = v
