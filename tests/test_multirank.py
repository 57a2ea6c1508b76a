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


# ---- the batched QAOA path over several ranks: partition and gather --------------------

def test_shard_instances_partition_and_balance():
    import numpy as np
    from orkan_b200.batch import shard_instances
    rng = np.random.default_rng(3)
    ns = rng.integers(16, 25, 4096)
    for world in (1, 2, 3, 4, 8):
        parts = shard_instances(ns, world)
        assert len(parts) == world
        allidx = np.concatenate(parts)
        assert sorted(allidx.tolist()) == list(range(len(ns)))          # every instance exactly once
        assert all(np.all(np.diff(p) > 0) for p in parts)             # ascending
        load = [int(sum(1 << int(ns[i]) for i in p)) for p in parts]
        assert max(load) - min(load) <= 1 << int(ns.max())            # within one largest instance
        assert [p.tolist() for p in shard_instances(ns, world)] == [p.tolist() for p in parts]
    assert shard_instances(ns, 1)[0].tolist() == list(range(len(ns)))
    # fewer instances than ranks: the extra ranks get none
    parts = shard_instances([5, 7], 4)
    assert [len(p) for p in parts] == [1, 1, 0, 0] and parts[0].tolist() == [1]


def _batch_rank(rank, world, port, out):
    """One rank of a sharded batch with the oracle as the per-instance evaluator."""
    import datetime

    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from oracle import restate as R
    from orkan_b200.batch import gather_means, random_regular_graph, shard_instances
    rng = np.random.default_rng(11)
    ns = rng.integers(4, 9, 24)
    edges = [random_regular_graph(int(n), 3, rng) for n in ns]
    g, b = rng.uniform(0, np.pi, (24, 2)), rng.uniform(0, np.pi / 2, (24, 2))
    idx = shard_instances(ns, world)[rank]
    local = [R.qaoa_mean(int(ns[i]), R.maxcut_cost(int(ns[i]), edges[i]), g[i], b[i]) for i in idx]
    out[rank] = (gather_means(len(ns), idx, local, dist, "cpu").tolist(), len(idx))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_gathers_every_mean_in_order():
    import numpy as np

    from oracle import restate as R
    from orkan_b200.batch import random_regular_graph
    world, port = 2, free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_batch_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    rng = np.random.default_rng(11)
    ns = rng.integers(4, 9, 24)
    edges = [random_regular_graph(int(n), 3, rng) for n in ns]
    g, b = rng.uniform(0, np.pi, (24, 2)), rng.uniform(0, np.pi / 2, (24, 2))
    want = [R.qaoa_mean(int(n), R.maxcut_cost(int(n), e), g[i], b[i]) for i, (n, e) in enumerate(zip(ns, edges))]
    assert res[0][0] == res[1][0] == want                  # bit for bit: x + 0.0 == x
    assert res[0][1] > 0 and res[1][1] > 0 and res[0][1] + res[1][1] == 24
