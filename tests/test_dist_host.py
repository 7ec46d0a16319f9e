"""CPU tests of the multi-GPU HOLD step's host logic (hhs_hold_step_dist): the sink shards
of a split level, their assembly over world_size-2 gloo ranks, and the peer barrier's
failure report. No GPU: the library is loaded for its host-only shard arithmetic and
the per-sink physics is the oracle's."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp


def _cost(nf, ns, lo, hi):
    """Pair terms of sinks [lo, hi): fast sinks (index < nf) cost ns, slow ones ns + nf."""
    f = max(0, min(hi, nf) - lo)
    s = (hi - lo) - f
    return f * ns + s * (ns + nf)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7, 8])
def test_shards_cover_the_sinks_in_order_with_balanced_cost(hhs, world):
    rng = np.random.default_rng(world)
    cases = [(0, 0), (0, 1), (1, 0), (5, 0), (0, 5), (3, 10), (10, 3), (1, 262143),
             (131072, 131072), (0, 16384), (2, 2)]
    cases += [tuple(int(v) for v in rng.integers(0, 5000, 2)) for _ in range(20)]
    for nf, ns in cases:
        n = nf + ns
        bounds = [hhs.dist_shard(nf, ns, r, world) for r in range(world)]
        assert bounds[0][0] == 0 and bounds[-1][1] == n
        for r in range(world - 1):
            assert bounds[r][1] == bounds[r + 1][0]
        for lo, hi in bounds:
            assert 0 <= lo <= hi <= n
        total = _cost(nf, ns, 0, n)
        if total == 0:
            continue
        heaviest = ns + nf if ns > 0 else ns  # one slow sink
        for lo, hi in bounds:
            assert abs(_cost(nf, ns, lo, hi) - total / world) <= heaviest + 1e-9, (nf, ns, lo, hi)


def test_shard_rejects_bad_arguments(hhs):
    for args in [(-1, 4, 0, 2), (4, -1, 0, 2), (4, 4, 2, 2), (4, 4, -1, 2), (4, 4, 0, 0),
                 (2 ** 31 - 1, 1, 0, 2)]:
        with pytest.raises(hhs.HHSError) as e:
            hhs.dist_shard(*args)
        assert e.value.status == 1


def _level_kick(oracle, s, fast, slow, sinks, dt):
    """New velocities of the given sinks of one split level (sink index space: the fast
    list, then the slow list), as the kick of a level applies them."""
    nf = len(fast)
    take = lambda idx: {k: np.ascontiguousarray(s[k][idx]) for k in ("x", "y", "z", "vx", "vy",
                                                                       "vz", "m")}
    src_slow, src_fast = take(slow), take(fast)
    out = []
    for k in sinks:
        g = fast[k] if k < nf else slow[k - nf]
        one = take(np.array([g]))
        oracle.kick(one, src_slow, dt)
        if k >= nf and nf > 0:
            oracle.kick(one, src_fast, dt)
        out.append((one["vx"][0], one["vy"][0], one["vz"][0]))
    return np.array(out).reshape(-1, 3)


def _level(hhs, n):
    s = hhs.plummer(n, 21)
    ts = np.abs(s["x"]) + 0.1
    fast = np.flatnonzero(ts <= np.quantile(ts, 0.3)).astype(np.int32)
    slow = np.flatnonzero(ts > np.quantile(ts, 0.3)).astype(np.int32)
    return s, fast, slow


def _kick_worker(rank, world, port, q):
    import torch.distributed as dist
    import hhs
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s, fast, slow = _level(hhs, 300)
    lo, hi = hhs.dist_shard(len(fast), len(slow), rank, world)
    mine = _level_kick(oracle, s, fast, slow, range(lo, hi), 1 / 64)
    parts = [None] * world
    dist.all_gather_object(parts, (lo, hi, mine))
    q.put((rank, np.concatenate([p[2] for p in sorted(parts, key=lambda p: p[0])])))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_level_kick_over_two_gloo_ranks_equals_one_rank(hhs, oracle):
    """Each gloo rank kicks its shard of a split level's sinks; the all-gathered result
    is bit-identical to one rank kicking every sink (per sink, a shard does the same
    operations in the same order)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + os.getpid() % 1000
    procs = [ctx.Process(target=_kick_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    s, fast, slow = _level(hhs, 300)
    full = _level_kick(oracle, s, fast, slow, range(len(fast) + len(slow)), 1 / 64)
    assert np.array_equal(out[0][1], full) and np.array_equal(out[1][1], full)


def _barrier_worker(rank, world, port, q, absent):
    import datetime
    import time
    import torch.distributed as dist
    import hhs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    b = hhs.PeerBarrier(timeout=3.0)
    first = b(None)  # every rank arrives
    if absent and rank == 1:
        time.sleep(8.0)  # alive, but misses the next barrier
        q.put((rank, first, None, ""))
        return
    second = b(None)
    q.put((rank, first, second, str(b.failure or "")))
    if not absent:
        dist.destroy_process_group()


@pytest.mark.parametrize("absent", [False, True])
def test_peer_barrier_reports_a_rank_that_does_not_arrive(absent):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 32500 + os.getpid() % 1000 + (7 if absent else 0)
    procs = [ctx.Process(target=_barrier_worker, args=(r, 2, port, q, absent)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
    assert out[0][1] is True and out[1][1] is True
    if absent:
        assert out[0][2] is False and "1" in out[0][3]
    else:
        assert out[0][2] is True and out[1][2] is True


def _fake_system(hhs, n, base):
    """A particle-system struct whose arrays are never touched: hhs_dist_create only
    records the peer addresses."""
    import ctypes
    c = hhs.CParticleSystem()
    c.n = n
    for k, name in enumerate(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "ts", "m")):
        setattr(c, name, ctypes.cast(ctypes.c_void_p(base + 8 * n * k), ctypes.POINTER(ctypes.c_double)))
    c._base = ctypes.c_void_p(base)
    return c


def test_dist_create_validates_ranks_replicas_and_barrier(hhs):
    ok = lambda _s: True
    reps = [_fake_system(hhs, 1000, 1 << 40), _fake_system(hhs, 1000, 1 << 41),
            _fake_system(hhs, 1000, 1 << 42)]
    d = hhs.Dist(1, 3, reps, ok, 0)  # host-only: no device call
    d.destroy()
    d = hhs.Dist(0, 1, [None], ok)   # one rank needs no replicas
    d.destroy()
    bad = [
        lambda: hhs.Dist(3, 3, reps, ok),                       # rank out of range
        lambda: hhs.Dist(0, 9, reps * 3, ok),                   # more ranks than one node
        lambda: hhs.Dist(0, 3, [reps[0], None, reps[2]], ok),   # a missing replica
        lambda: hhs.Dist(0, 2, [reps[0], _fake_system(hhs, 0, 1 << 43)], ok),  # empty peer
        lambda: hhs.Dist(0, 3, [reps[0], reps[1], _fake_system(hhs, 999, 1 << 43)], ok),
        lambda: hhs.Dist(0, 2, reps[:2], ok, -1),               # negative threshold
    ]
    for make in bad:
        with pytest.raises(hhs.HHSError) as e:
            make()
        assert e.value.status == 1


def test_dist_callback_errors_become_a_failed_barrier(hhs):
    """A barrier callable that raises is reported to the library as a failed barrier
    (the callback never lets a Python exception cross into C), and the exception is kept."""
    seen = []

    def boom(stream):
        seen.append(stream)
        raise RuntimeError("peer lost")
    d = hhs.Dist(0, 1, [None], boom, 0)
    assert d._cb(None, None) == 1 and isinstance(d.failure, RuntimeError) and seen == [None]
    good = hhs.Dist(0, 1, [None], lambda _s: True, 0)
    assert good._cb(None, None) == 0
    d.destroy()
    good.destroy()


def _agree_worker(rank, world, port, q, differ):
    import torch.distributed as dist
    import hhs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    reps = [_fake_system(hhs, 4096, 1 << (40 + r)) for r in range(world)]
    d = hhs.Dist(rank, world, reps, lambda _s: True, 0)
    d.set_agreement(hhs.group_minmax())
    tuning = {"small_n": 64, "units_per_cta": 16, "ctas_per_sm": 2, "warp_n": 32,
              "cluster_size": 4, "mid_n": 640, "packed": 0, "mid_dist_n": 96,
              "overlap": 1}
    if differ and rank == 1:
        tuning["cluster_size"] = 8  # this rank's engine would sum in another order
    h = hhs.config_hash(tuning, 284, hhs.PREC_MIXED, 4096, 1 / 64, 0.03)
    q.put((rank, d.check(h)))
    d.destroy()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("differ", [False, True])
def test_ranks_with_different_engine_tuning_are_rejected(hhs, differ):
    """The mixed-precision sums' order follows each rank's engine launch shape and tuning;
    two gloo ranks compare their configuration hashes before a step, and a mismatch ends
    the step on every rank with HHS_ERR_INVALID_ARG instead of letting replicas drift."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 33500 + os.getpid() % 1000 + (7 if differ else 0)
    procs = [ctx.Process(target=_agree_worker, args=(r, 2, port, q, differ)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [s for _, s in out] == ([1, 1] if differ else [0, 0])


def test_config_hash_covers_every_field(hhs):
    base = {"small_n": 64, "units_per_cta": 16, "ctas_per_sm": 2, "warp_n": 32,
            "cluster_size": 4, "mid_n": 640, "packed": 0, "mid_dist_n": 96,
              "overlap": 1}
    h0 = hhs.config_hash(base, 284, hhs.PREC_MIXED, 4096, 1 / 64, 0.03)
    assert h0 == hhs.config_hash(dict(base), 284, hhs.PREC_MIXED, 4096, 1 / 64, 0.03)
    seen = {h0}
    for k in base:
        t = dict(base)
        t[k] += 1
        seen.add(hhs.config_hash(t, 284, hhs.PREC_MIXED, 4096, 1 / 64, 0.03))
    for args in ((296, hhs.PREC_MIXED, 4096, 1 / 64, 0.03), (284, hhs.PREC_FP64, 4096, 1 / 64, 0.03),
                 (284, hhs.PREC_MIXED, 4097, 1 / 64, 0.03), (284, hhs.PREC_MIXED, 4096, 1 / 32, 0.03),
                 (284, hhs.PREC_MIXED, 4096, 1 / 64, 0.02)):
        seen.add(hhs.config_hash(base, *args))
    seen.add(hhs.config_hash(base, 284, hhs.PREC_MIXED, 4096, 1 / 64, 0.03, eps=1e-3))
    assert len(seen) == 1 + len(base) + 6
