"""The multi-GPU HOLD step (hhs_hold_step_dist) on one B200.

Ranks are emulated by host threads or processes that share the device, each with its
own replica, context and stream. Their kernels never wait for one another: every
cross-rank wait is a host barrier between launches (stream synchronise, then a
threading or gloo barrier). A sharded launch stores each result into every replica,
so after each step all replicas are equal. The shared launches run the engine's tiled
phases (symmetric pair-rate timestep, bulk-copied kick tiles), so FP64 replicas equal one
hhs_hold_step_host run bit for bit, and mixed ones equal a one-rank run of the same
schedule and stay within the mixed tolerance of the host step."""
import datetime
import hashlib
import os
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m", "ts", "id")


def _digest(out):
    h = hashlib.sha256()
    for k in FIELDS:
        h.update(np.ascontiguousarray(out[k]).tobytes())
    return h.hexdigest()


def _host_reference(hhs, s0, n, steps, prec, dt=1 / 64, eps=0.0):
    sy, ctx = hhs.ParticleSystem(n), hhs.Context(n, eps=eps)
    sy.upload(s0)
    for _ in range(steps):
        hhs.hold_step_host(ctx, sy, n, dt, True, prec)
    out = sy.download(n)
    ctx.destroy()
    sy.free()
    return out


def _run_threads(hhs, torch, s0, n, world, steps, prec, min_pairs, dt=1 / 64, eps=0.0,
                 subtree_engine=False):
    systems = [hhs.ParticleSystem(n) for _ in range(world)]
    ctxs = [hhs.Context(n, eps=eps) for _ in range(world)]
    streams = [torch.cuda.Stream() for _ in range(world)]
    for sy in systems:
        sy.upload(s0)
    torch.cuda.synchronize()
    bar = threading.Barrier(world, timeout=120)
    calls = [0] * world

    def barrier_of(r):
        def fn(_stream):
            streams[r].synchronize()
            calls[r] += 1
            bar.wait()
            return True
        return fn

    dists = [hhs.Dist(r, world, systems, barrier_of(r), min_pairs, subtree_engine)
             for r in range(world)]
    errors = [None] * world

    def work(r):
        try:
            for _ in range(steps):
                dists[r].step(ctxs[r], systems[r], n, dt, True, prec, streams[r].cuda_stream)
            streams[r].synchronize()
        except Exception as e:  # noqa: BLE001 -- reported below
            errors[r] = e
            bar.abort()

    threads = [threading.Thread(target=work, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert errors == [None] * world, errors
    outs = [sy.download(n) for sy in systems]
    for d in dists:
        d.destroy()
    for c in ctxs:
        c.destroy()
    return outs, calls


@pytest.mark.parametrize("world,prec,min_pairs,eps", [(2, 0, 0, 0.0), (3, 0, 0, 0.0),
                                                      (2, 1, 0, 0.0), (4, 1, 0, 0.0),
                                                      (2, 0, 1 << 16, 0.0), (3, 1, 1 << 14, 0.0),
                                                      (2, 0, 0, 0.02), (3, 1, 0, 0.02)])
def test_sharded_step_replicas_equal_the_one_gpu_host_step(hhs, cuda, world, prec, min_pairs,
                                                           eps):
    n, steps = 2048, 3
    s0 = hhs.plummer(n, 41)
    outs, calls = _run_threads(hhs, cuda, s0, n, world, steps, prec, min_pairs, eps=eps)
    assert len(set(calls)) == 1 and calls[0] > 0  # every rank took the same barriers
    host = _host_reference(hhs, s0, n, steps, prec, eps=eps)
    ref = host if prec == 0 else _run_threads(hhs, cuda, s0, n, 1, steps, prec, min_pairs,
                                                eps=eps)[0][0]
    for out in outs:
        for k in FIELDS:
            assert np.array_equal(out[k], ref[k]), k
    if prec != 0:
        dx = max(np.abs(outs[0][k] - host[k]).max() for k in ("x", "y", "z"))
        assert dx < 1e-6, dx


def test_fp64_sharded_step_equals_the_oracle(hhs, cuda, oracle):
    n = 1024
    s0 = hhs.plummer(n, 42)
    outs, _ = _run_threads(hhs, cuda, s0, n, 2, 2, 0, 0)
    s = {k: v.copy() for k, v in s0.items()}
    for _ in range(2):
        oracle.hold_step(s, 1 / 64, True, 0.03)
    for out in outs:
        for k in FIELDS:
            assert np.array_equal(out[k], s[k]), k


def test_a_failed_barrier_ends_the_step_with_a_peer_error(hhs, cuda):
    n = 512
    s0 = hhs.plummer(n, 43)
    mine, other = hhs.ParticleSystem(n), hhs.ParticleSystem(n)
    mine.upload(s0)
    other.upload(s0)
    ctx = hhs.Context(n)
    d = hhs.Dist(0, 2, [mine, other], lambda _s: False, 0)
    with pytest.raises(hhs.HHSError) as e:
        d.step(ctx, mine, n, 1 / 64, True, 0)
    assert e.value.status == 8  # HHS_ERR_PEER, before any store into the peer
    assert np.array_equal(other.download(n)["vx"], s0["vx"])
    d.destroy()
    hhs.hold_step_host(ctx, mine, n, 1 / 64, True, 0)  # the context still works
    ctx.check()
    with pytest.raises(hhs.HHSError):
        hhs.Dist(0, 2, [mine, None], lambda _s: True)  # a missing peer replica
    with pytest.raises(hhs.HHSError):
        hhs.Dist(0, 9, [mine] * 9, lambda _s: True)  # more ranks than one node
    ctx.destroy()


def _ipc_worker(rank, world, port, q, n, steps, prec, min_pairs=0, engine=False):
    import torch
    import torch.distributed as tdist
    import hhs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world,
                             timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    s0 = hhs.plummer(n, 44)
    sy, ctx = hhs.ParticleSystem(n), hhs.Context(n)
    sy.upload(s0)
    dh = hhs.DistHold(ctx, sy, min_pairs=min_pairs, timeout=60.0, subtree_engine=engine)
    for _ in range(steps):
        dh.step(n, 1 / 64, True, prec)
    torch.cuda.synchronize()
    mine = sy.download(n)
    got = _digest(mine)
    dh.close()
    tdist.barrier()  # no rank frees its system while a peer still maps it
    ref = one = None
    dx = 0.0
    if rank == 0:
        host = _host_reference(hhs, s0, n, steps, prec)
        ref = _digest(host)
        dx = float(max(np.max(np.abs(mine[k] - host[k])) for k in ("x", "y", "z")))
        if engine or prec != 0:  # the same schedule on one rank, in this process
            one = _digest(_run_threads(hhs, torch, s0, n, 1, steps, prec, min_pairs,
                                       subtree_engine=engine)[0][0])
    q.put((rank, got, ref, one, dx))
    tdist.barrier()
    tdist.destroy_process_group()


@pytest.mark.parametrize("prec,min_pairs,engine", [(0, 0, False), (1, 0, False),
                                                    (0, 1 << 18, True), (1, 1 << 18, True)])
def test_two_processes_share_one_system_through_cuda_ipc(cuda, prec, min_pairs, engine):
    """Two processes on one GPU, each mapping the other's system with CUDA IPC and a gloo
    peer barrier between launches: both replicas end equal to the one-GPU host step.
    With the subtree engine (subtrees below min_pairs as engine launches from their
    level; the two processes' launches are time-sliced, never concurrent), FP64 still
    equals the host step; mixed equals a one-rank run of the same schedule and stays
    within the mixed tolerance of the host step."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 33500 + os.getpid() % 1000 + prec + (2 if engine else 0)
    procs = [ctx.Process(target=_ipc_worker,
                         args=(r, 2, port, q, 1536, 2, prec, min_pairs, engine))
             for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1]
    if prec == 0:
        assert out[0][1] == out[0][2]
    else:
        assert out[0][1] == out[0][3]
        assert out[0][4] < 1e-6
    if engine:
        assert out[0][1] == out[0][3]


def _nccl_worker(port, q, n, steps):
    import torch
    import torch.distributed as tdist
    import hhs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    tdist.init_process_group("nccl", rank=0, world_size=1,
                             timeout=datetime.timedelta(seconds=60),
                             device_id=torch.device("cuda", 0))
    s0 = hhs.plummer(n, 45)
    sy, ctx = hhs.ParticleSystem(n), hhs.Context(n)
    sy.upload(s0)
    dh = hhs.DistHold(ctx, sy, min_pairs=0)
    stream = torch.cuda.Stream()
    for _ in range(steps):
        dh.step(n, 1 / 64, True, 1, stream.cuda_stream)
    stream.synchronize()
    got = _digest(sy.download(n))
    dh.close()
    # mixed precision: the same sharded schedule on one rank without NCCL
    ref = _digest(_run_threads(hhs, torch, s0, n, 1, steps, 1, 0)[0][0])
    q.put((got, ref, dh.barrier.nccl))
    tdist.destroy_process_group()


def test_nccl_peer_barrier_on_one_rank(cuda):
    """The stream-ordered NCCL barrier (a one-value all-reduce on the library's stream),
    on a one-rank group: every launch goes through the sharded path."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_worker, args=(34500 + os.getpid() % 1000, q, 1024, 2))
    p.start()
    got, ref, nccl = q.get(timeout=600)
    p.join(timeout=120)
    assert p.exitcode == 0
    assert nccl and got == ref
