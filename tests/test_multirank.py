"""world_size-2 gloo tests of the benchmark's multi-rank logic (replicas only: no data-path
collective; each rank integrates its own system, the job's time is the slowest rank)."""
import importlib.util
import os

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = _bench()
    t = b.max_over_ranks(10.0 + 5.0 * rank, dist, torch, device="cpu")
    seed = b.replica_seed(2024, rank)
    ref = b.run_reference(type("A", (), {"n": 64, "seed": 1, "dt": 1 / 64, "eta": 0.03,
                                         "steps": 1, "prec": "mixed"})(), rank, world)
    q.put((rank, t, seed, ref is None))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_time_reduction_and_seeds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] == 15.0          # both ranks see the max
    assert out[0][2] != out[1][2]                   # independent replicas
    assert out[0][3] is False and out[1][3] is True  # reference arm runs on rank 0 only


def test_aggregate_value():
    b = _bench()
    assert b.aggregate_value(10, 4, 2000.0) == pytest.approx(20.0)


def _shard_worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    import hhs
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = _bench()
    sizes = b.cluster_sizes(7, count=12, lo=8, hi=64)
    mine = hhs.batch_shard(sizes, world, rank)
    vals = []
    for k in mine:  # one FP64 HOLD step of each local cluster on the CPU oracle
        s = hhs.plummer(int(sizes[k]), 100 + int(k))
        oracle.hold_step(s, 1 / 64, True, 0.03)
        vals.append(float(np.sum(s["vx"] * s["m"]) + s["x"][0]))
    got = b.gather_by_index(mine, vals, len(sizes), dist)
    q.put((rank, list(map(int, mine)), got.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_batched_sharding_two_ranks_matches_one_process():
    """Clusters sharded over 2 gloo ranks by hhs_batch_partition: every cluster runs on
    exactly one rank and the gathered per-cluster results equal one process doing all."""
    import numpy as np
    import hhs
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    b = _bench()
    sizes = b.cluster_sizes(7, count=12, lo=8, hi=64)
    assert sorted(out[0][1] + out[1][1]) == list(range(len(sizes)))
    expect = []
    for k in range(len(sizes)):
        s = hhs.plummer(int(sizes[k]), 100 + k)
        oracle.hold_step(s, 1 / 64, True, 0.03)
        expect.append(float(np.sum(s["vx"] * s["m"]) + s["x"][0]))
    assert out[0][2] == out[1][2] == expect


def test_batch_partition_balances_pair_work():
    import numpy as np
    import hhs
    b = _bench()
    sizes = b.cluster_sizes(2024)
    for world in (1, 2, 4, 8):
        rank_of, load = hhs.batch_partition(sizes, world)
        assert set(rank_of.tolist()) <= set(range(world))
        assert np.isclose(load.sum(), float(np.sum(sizes.astype(np.float64) ** 2)))
        for r in range(world):
            assert load[r] == float(np.sum(sizes[rank_of == r].astype(np.float64) ** 2))
        # LPT bound: no rank exceeds the mean by more than the largest single job
        assert load.max() <= load.mean() + float(sizes.max()) ** 2
    with pytest.raises(hhs.HHSError):
        hhs.batch_partition([4, -1], 2)
    with pytest.raises(hhs.HHSError):
        hhs.batch_partition([4, 1], 0)
