"""The multi-rank (replica) logic of bench.py on CPU: gloo, world size 2.

Each rank advances its own jet; the timed region's device time is the max over ranks
and the whole-job throughput counts every rank's points. The reference arm runs on
rank 0 only.
"""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms_local = 10.0 + 5.0 * rank  # the slower rank must decide the time
    ms = bench.reduce_max(ms_local, world, "cpu")
    out[rank] = (ms, bench.replica_throughput(1000, 4, world, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_throughput_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    # 2 ranks x 1000 points x 4 steps in 15 ms
    assert abs(res[0][1] - 2 * 1000 * 4 / 0.015) < 1e-6


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


@pytest.mark.parametrize("world", [1])
def test_single_rank_needs_no_process_group(world):
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.5, world, "cpu") == 3.5
