"""bench.py's multi-rank plumbing on CPU: two gloo ranks (launched like
torchrun: RANK / WORLD_SIZE / MASTER_* in the environment) agree on the
max-over-ranks step time and the whole-job value; the reference arm's
non-zero ranks exit without work or output."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

RANK_CODE = r"""
import datetime, json, os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
world, rank, _ = bench.dist_setup()
dist.init_process_group("gloo", init_method="env://", world_size=world, rank=rank,
                        timeout=datetime.timedelta(seconds=60))
ms = [1.5, 4.25][rank]
m = bench.max_over_ranks(ms, world, "cpu")
print(json.dumps({{"rank": rank, "ms_max": m, "value": bench.whole_job_tflops(6e9, world, m)}}))
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_single_rank_is_its_own_max():
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.whole_job_tflops(2e12, 1, 1000.0) == 2.0


def test_two_gloo_ranks_share_the_max_and_the_whole_job_value():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_CODE.format(root=ROOT)],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    want = 6e9 * 2 / (4.25e-3) / 1e12
    for o in outs:
        assert o["ms_max"] == 4.25
        assert abs(o["value"] - want) < 1e-9 * want


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
