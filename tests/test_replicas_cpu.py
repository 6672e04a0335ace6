"""CPU: the N>1 path of bench.py (independent replicas, one process per GPU)
with the gloo backend at world size 2: the barrier, the max over ranks of the
device time and the whole-job rate; and the reference arm, which runs on
rank 0 only."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rep = bench.Replicas(dist, "cpu")
        rep.barrier()
        # rank r processed 1000 units in (r+1) s: the job rate is all units
        # over the slowest rank's time
        rate = rep.job_rate(1000.0, float(rank + 1))
        q.put((rank, rep.world, rep.max(float(10 * rank + 3)), rate))
        rep.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_gloo_world2():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, world, mx, rate in res:
        assert world == 2
        assert mx == 13.0                       # max over ranks of 3 and 13
        assert rate == pytest.approx(2000.0 / 2.0)


def test_single_process_replicas_are_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    rep = bench.Replicas(None)
    assert rep.world == 1 and rep.max(4.5) == 4.5 and rep.job_rate(100.0, 2.0) == 50.0


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
