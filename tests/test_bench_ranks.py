"""The multi-process logic of bench.py on CPU: two gloo ranks (world size 2,
one process each) time different amounts, every rank gets the maximum, the
whole-job rate counts both replicas' work against that maximum, and the
reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)  # rank 1 is the slow one
        out[rank] = (ms, bench.job_tflops(world, 2.0 * 8192 ** 3, 10, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_with_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 15.0  # both ranks report the slowest time
    per_replica = 2.0 * 8192 ** 3 * 10 / 15e-3 / 1e12
    assert out[0][1] == pytest.approx(2 * per_replica)  # both replicas' work, max time


def test_reference_arm_does_no_work_off_rank_zero():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reference_arm(None, 1) is None  # returns before reading any argument


def test_gpus_flag_without_a_launcher_starts_that_many_ranks():
    """`python bench.py --gpus 2` with no RANK in the environment must run two
    ranks (it relaunches itself under torch.distributed.run), never one replica
    under a two-GPU label.  Checked on the reference arm, which needs no GPU:
    rank 0 prints one line whose n_gpus is the launched world size."""
    import json
    import subprocess

    sys.path.insert(0, ROOT)
    import bench

    cmd = bench.launcher_command(["--gpus", "2"], 2, 12345)
    assert "--nproc-per-node=2" in cmd and "127.0.0.1" in cmd and cmd[-2:] == ["--gpus", "2"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    env["OMP_NUM_THREADS"] = "2"
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                          "--impl", "reference", "--n", "192", "--steps", "1", "--warmup", "0",
                          "--cpu-seconds", "0.05"], capture_output=True, text=True, env=env,
                         timeout=240, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
