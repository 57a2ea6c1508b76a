"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1), the timing
reduction (max over ranks), the whole-job value of replicas, and the reference arm's
non-zero ranks exiting without work."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = 100.0 + 50.0 * rank                  # rank 1 is the slow one
    m = bench.reduce_max(local_ms, dist, "cpu")
    value = bench.replica_value(world, 5, 2e9, m)
    dist.barrier()
    out[rank] = (m, value)
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, port = 2, free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 150.0
    # 2 replicas x 5 steps x 2 GB over 150 ms
    assert res[0][1] == pytest.approx(2 * 5 * 2e9 / 0.150 / 1e9)


def test_single_process_reduction_is_identity():
    import bench
    assert bench.reduce_max(3.5, None, "cpu") == 3.5


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch, capsys):
    import sys

    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse_args()) == 0
    assert capsys.readouterr().out == ""
