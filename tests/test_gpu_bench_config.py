"""Parity at the configurations the benchmark reports, with the library's default tuning
(hhs.Context as created: thread-block clusters of 4, subtree solver up to 640 particles,
pair work spread over the cluster above 96 members).

* Plummer N=16384, equal masses, eta=0.03, dt=2^-6, seed 2024 (the headline workload):
  one mixed-precision step against the FP64 oracle -- position and energy bounds, and the
  node-by-node hierarchy (level, n, n_fast of every hold_step call) -- and one FP64 step
  of the same default schedule bit for bit against the oracle.
* Plummer N=65536, Salpeter masses on [0.1, 100], eta=0.02 (the deep-hierarchy
  workload): one mixed step against one FP64 step of the device schedule (which equals
  the oracle bit for bit), with the split agreement counted per level.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m", "ts")
TRACE_CAP = 1 << 16


def _traced_step(hhs, torch, ctx, d, n, dt, prec):
    nodes = torch.zeros((TRACE_CAP, 4), dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.set_trace(nodes.data_ptr(), TRACE_CAP, count.data_ptr())
    hhs.hold_step(ctx, d, n, 0.0, dt, True, prec)
    ctx.check()
    ctx.set_trace(None, 0, None)
    k = int(count.item())
    assert k <= TRACE_CAP
    return nodes[:k].cpu().numpy()


def _per_level(trace):
    """{level: (nodes, sum of n, sum of n_fast)}"""
    out = {}
    for lvl in np.unique(trace[:, 0]):
        t = trace[trace[:, 0] == lvl]
        out[int(lvl)] = (len(t), int(t[:, 1].sum()), int(t[:, 2].sum()))
    return out


def _split_agreement(a, b):
    """Per level: nodes whose (n, n_fast) agree between two traces walked in call order,
    over the nodes of trace a."""
    agree = {}
    m = min(len(a), len(b))
    same = np.all(a[:m, :3] == b[:m, :3], axis=1)
    for lvl in np.unique(a[:, 0]):
        sel = a[:m, 0] == lvl
        agree[int(lvl)] = (int(same[sel].sum()), int((a[:, 0] == lvl).sum()))
    return agree


def _assert_close_hierarchy(a, b):
    """Per level, node count and summed fast counts agree to within what a handful of
    timesteps lying within the mixed tolerance of a pivot can change."""
    assert abs(len(a) - len(b)) <= 1, (a, b)
    for lvl in set(a) & set(b):
        (na, sa, fa), (nb, sb, fb) = a[lvl], b[lvl]
        assert abs(na - nb) <= max(2, nb // 100), (lvl, a[lvl], b[lvl])
        assert abs(fa - fb) <= max(8, fb // 1000), (lvl, a[lvl], b[lvl])


def test_default_tuning_headline_mixed_step_against_oracle(cuda, hhs, oracle):
    torch = cuda
    n, dt, eta = 16384, 2.0 ** -6, 0.03
    s = hhs.plummer(n, 2024)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=eta)  # default tuning, as the benchmark runs it
    d = hhs.ParticleSystem(n)
    d.upload(s)
    e0 = hhs.energy_host(s)
    trace = _traced_step(hhs, torch, ctx, d, n, dt, hhs.PREC_MIXED)
    out = d.download()
    tr, otrace = oracle.hold_step(ref, dt, True, eta, capacity=TRACE_CAP)
    dx = max(np.abs(out[k] - ref[k]).max() for k in ("x", "y", "z"))
    de = (hhs.energy_host(out) - hhs.energy_host(ref)) / e0
    agree = _split_agreement(trace, otrace)
    print(f"\nN=16384 mixed vs oracle: max|dx|={dx:.3e} dE/E diff={de:.3e} "
          f"nodes {len(trace)} vs {len(otrace)}; per-level agreement {agree}")
    assert dx <= 1e-7, dx
    assert abs(de) <= 1e-9, de
    # the hierarchy: per level the same nodes and fast counts as the oracle's, up to a
    # timestep that falls within the mixed tolerance of a level's pivot
    _assert_close_hierarchy(_per_level(trace), _per_level(otrace))


def test_default_tuning_headline_fp64_step_bit_exact(cuda, hhs, oracle):
    torch = cuda
    n, dt, eta = 16384, 2.0 ** -6, 0.03
    s = hhs.plummer(n, 2024)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=eta)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    trace = _traced_step(hhs, torch, ctx, d, n, dt, hhs.PREC_FP64)
    out = d.download()
    tr, otrace = oracle.hold_step(ref, dt, True, eta, capacity=TRACE_CAP)
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    assert np.array_equal(trace, otrace)
    assert ctx.simtime() == pytest.approx(tr.leaf_time, rel=1e-15)


def test_deep_hierarchy_mixed_step_against_fp64_schedule(cuda, hhs):
    torch = cuda
    n, dt, eta = 65536, 2.0 ** -6, 0.02
    s = hhs.plummer(n, 2024, hhs.MASS_SALPETER)
    e0 = hhs.energy_host(s)
    res = {}
    for name, prec in (("mixed", hhs.PREC_MIXED), ("fp64", hhs.PREC_FP64)):
        ctx = hhs.Context(n, 64, eta=eta)
        d = hhs.ParticleSystem(n)
        d.upload(s)
        res[name] = (_traced_step(hhs, torch, ctx, d, n, dt, prec), d.download())
    (tm, om), (tf, of) = res["mixed"], res["fp64"]
    dx = max(np.abs(om[k] - of[k]).max() for k in ("x", "y", "z"))
    de = (hhs.energy_host(om) - hhs.energy_host(of)) / e0
    agree = _split_agreement(tm, tf)
    lm, lf = _per_level(tm), _per_level(tf)
    print(f"\nN=65536 Salpeter mixed vs FP64: max|dx|={dx:.3e} dE/E diff={de:.3e} "
          f"nodes {len(tm)} vs {len(tf)} levels {max(lf)}\nper-level agreement {agree}")
    assert max(lf) >= 10                      # a deep hierarchy
    _assert_close_hierarchy(lm, lf)
    assert dx <= 1e-6, dx
    assert abs(de) <= 1e-8, de


class _DevArray:
    """A device pointer seen as an FP64 array (CUDA array interface), for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3}


def _sum_of_magnitudes(s, eps, src=None, rows=None, block=512):
    """Per particle, the sum over its sources of |m_j (x_j - x_i) / (d^2 + eps^2)^(3/2)|:
    every other particle, or only those in `src` for the particles in `rows`."""
    x, y, z, m = s["x"], s["y"], s["z"], s["m"]
    out = np.empty(len(x))
    for b in range(0, len(x), block):
        dx = x[None, :] - x[b:b + block, None]
        dy = y[None, :] - y[b:b + block, None]
        dz = z[None, :] - z[b:b + block, None]
        d2 = dx * dx + dy * dy + dz * dz
        with np.errstate(divide="ignore", invalid="ignore"):
            t = m[None, :] * np.sqrt(d2) / (d2 + eps * eps) ** 1.5
        t[d2 == 0.0] = 0.0
        if rows is not None:
            t[rows[b:b + block][:, None] & ~src[None, :]] = 0.0
        out[b:b + block] = t.sum(1)
    return out


@pytest.mark.parametrize("n,eps", [(4096, 0.0), (16384, 0.0), (24576, 0.0), (3000, 0.01)])
def test_engine_mixed_kick_accelerations_against_oracle(cuda, hhs, oracle, n, eps):
    """The kick phase of the device step in mixed precision (bulk-copied slow tiles, each
    fast-slow pair -- and, for slow sets of 2048 or more, each slow-slow pair -- evaluated
    once for both particles, FP32 pair terms with a Newton-corrected 1/d^3, compensated row
    sums and tree-ordered column sums) on a split node -- fast set every third particle --
    against the FP64 direct sums of the oracle over the same sets. The sizes cover one and
    two fast sinks per thread (fast sets below / from 8192), slow chunks of one and two
    row passes, and (n=3000) the one-directional slow units of small slow sets."""
    torch = cuda
    s = hhs.plummer(n, 77 + n)
    ctx = hhs.Context(n, 64, eta=0.03, eps=eps)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    assert hhs.lib().hhs_engine_kick_accelerations(ctx.h, d.ref, n, None) == 0
    ctx.check()
    a = np.stack([torch.as_tensor(_DevArray(ctypes.cast(getattr(d.c, k), ctypes.c_void_p).value,
                                            n), device="cuda").cpu().numpy()
                  for k in ("ax", "ay", "az")])
    fast = np.arange(n) % 3 == 0
    take = lambda m: {k: np.ascontiguousarray(v[m]) for k, v in s.items()}
    acc = np.zeros((3, n))
    acc[:, fast] = oracle.kick(take(fast), take(~fast), 1.0, eps=eps)  # fast: slow sources
    acc[:, ~fast] = oracle.kick(take(~fast), s, 1.0, eps=eps)          # slow: everyone
    amag = np.sqrt((acc ** 2).sum(0))
    dev = np.sqrt(((a - acc) ** 2).sum(0))
    err = dev / amag
    smag = _sum_of_magnitudes(s, eps, src=~fast, rows=fast)
    err_s = dev / smag
    print(f"\nengine kick n={n} eps={eps}: |da|/|a| max {err.max():.3e} median "
          f"{np.median(err):.3e}; |da|/sum|a_ij| max {err_s.max():.3e}")
    # the summation error bound: relative to the sum of the pair terms' magnitudes (a
    # particle whose pulls nearly cancel has a small |a| but the same absolute error)
    assert err_s.max() < 5e-7, err_s.max()
    # relative to |a| itself where the pulls do not cancel much (|a| at least a quarter of
    # the sum of magnitudes)
    weak = amag >= 0.25 * smag
    assert err[weak].max() < 1e-6 and np.median(err) < 1e-7, (err[weak].max(), np.median(err))


@pytest.mark.parametrize("n,eta", [(3000, 0.03), (16384, 0.03), (20000, 0.02)])
def test_engine_mixed_timesteps_against_oracle(cuda, hhs, oracle, n, eta):
    """The timestep phase of the device step in mixed precision (members packed in column
    pairs, column tiles bulk-copied, one rate per unordered pair in f32x2 arithmetic
    feeding both particles' maxima, tiles unmasked away from the diagonal) over a whole
    node, against the FP64 timesteps of the oracle: the largest relative difference stays
    at the FP32 rounding of the pair expression (rsqrtf without a Newton step), far inside
    the width of a timestep level. Each lane of the packed arithmetic runs the scalar
    expression's operations in its order, and a maximum does not depend on the order of
    its terms, so the result also equals the plain one-thread-per-sink mixed kernel
    (hhs_timesteps) bit for bit."""
    s = hhs.plummer(n, 900 + n)
    ref = oracle.timesteps(s, eta)
    ctx = hhs.Context(n, 64, eta=eta)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    assert hhs.lib().hhs_engine_timestep_rates(ctx.h, d.ref, n, None) == 0
    ctx.check()
    ts = d.download()["ts"]
    rel = np.abs(ts - ref) / ref
    print(f"\nengine timesteps n={n}: max rel {rel.max():.3e} median {np.median(rel):.3e}")
    assert rel.max() < 2e-6, rel.max()
    plain = hhs.ParticleSystem(n)
    plain.upload(s)
    hhs.timesteps(ctx, plain, n, hhs.PREC_MIXED)
    assert np.array_equal(plain.download()["ts"], ts)
    # a second call on the same context: the rate words were left at zero
    d.upload(s)
    assert hhs.lib().hhs_engine_timestep_rates(ctx.h, d.ref, n, None) == 0
    ctx.check()
    assert np.array_equal(d.download()["ts"], ts)
