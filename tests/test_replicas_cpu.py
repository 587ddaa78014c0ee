"""The multi-process plumbing of `bench.py --gpus N` (one independent
replica of the workload per rank, no data-path collective): two gloo ranks
on the CPU meet at the barrier, agree on the slowest rank's time, and form
the whole-job rate from it; the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

CHILD = r"""
import json, os, sys
sys.path.insert(0, os.environ["ROOT"])
import torch.distributed as dist
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%s" % os.environ["PORT"], rank=rank,
                        world_size=world)
bench.rank_barrier(world)
ms = 10.0 + 5.0 * rank                        # each rank's own step time
mx = bench.max_over_ranks_on(ms, world, "cpu")
rate = bench.job_rate(2.0e9, world, mx)
class A: steps = 1; warmup = 3
if rank != 0:
    bench.run_reference(A, rank, world)           # must return without work or output
bench.rank_barrier(world)
dist.destroy_process_group()
print(json.dumps({"rank": rank, "max_ms": mx, "rate": rate}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_the_slowest_rank():
    port = str(_free_port())
    procs = []
    for r in range(2):
        env = dict(os.environ, ROOT=ROOT, RANK=str(r), WORLD_SIZE="2", PORT=port, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["max_ms"] == 15.0                     # the slower rank's time on both
        assert abs(o["rate"] - 2 * 2.0e9 / 15e-3 / 1e9) < 1e-9
    assert [o["rank"] for o in outs] == [0, 1]
