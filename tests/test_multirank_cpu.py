"""The N>1 path of bench.py on CPU: two gloo ranks, each with its own replica
timing, agree on the slowest rank's time and on the whole-job value; the
reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms_local = 2.0 + rank                    # rank 1 is the slow one
    ms = bench.max_over_ranks(ms_local, world)
    value = bench.aggregate_value(1000.0, ms, world)
    out[rank] = (ms, value)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms, value = res[0]
    assert ms == 3.0
    assert value == pytest.approx(1000.0 * 2 / 3.0e-3)


def test_reference_arm_only_rank0_prints(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
