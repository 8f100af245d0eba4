"""The N > 1 host path of bench.py on CPU: two gloo ranks.

bench.py runs one process per GPU (torchrun), times its own replica, takes
the maximum step time over ranks (an all-reduce) and reports the whole job's
solves per second; the reference arm runs on rank 0 alone.  The ranks see no
GPU and use gloo, which bench.py selects when CUDA is absent.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    w, r, local, pg = bench.dist_setup(None)
    ms = 10.0 + 5.0 * r  # rank 1 is the slower replica
    ms_max = bench.max_over_ranks(ms, pg, None)
    out.put((r, w, pg.get_backend(), ms_max, bench.whole_job_value(w, 4, ms_max)))
    pg.barrier()
    pg.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for r, w, backend, ms_max, value in res:
        assert w == 2 and backend == "gloo"
        assert ms_max == 15.0
        assert value == 2 * 4 / 0.015  # both ranks' solves over the slower rank's time


def test_reference_arm_runs_on_rank_zero_only():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--workload", "nodal", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    p = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
