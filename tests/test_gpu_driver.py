"""GPU tests of the softened kick and of the driver around the HOLD step: the FP64
energy diagnostic, binary snapshots (checkpoint / resume) and hold(), the integration
loop declared at src/hold.cuh:20-35 of the reference."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m", "ts")
EPS = 0.01


def _copy(s):
    return {k: v.copy() for k, v in s.items()}


# ------------------------------------------------------------------------------ softening
@pytest.mark.parametrize("schedule,n,small_n,mid_n", [("host", 300, 0, 0), ("engine", 300, 0, 0),
                                                      ("engine", 2048, 256, 0),
                                                      ("engine", 300, 100000, 0),
                                                      ("engine", 2048, 64, 640)])
def test_softened_hold_fp64_bit_exact(cuda, hhs, oracle, schedule, n, small_n, mid_n):
    """With eps > 0 every kick uses d2 + eps^2; both schedules stay bit-exact."""
    s = hhs.plummer(n, 90 + n)
    ref = _copy(s)
    ctx = hhs.Context(n, 64, eta=0.03, eps=EPS)
    ctx.set_tuning(small_n, mid_n=mid_n)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    dt = 1.0 / 64
    for _ in range(2):
        if schedule == "host":
            hhs.hold_step_host(ctx, d, n, dt, True, hhs.PREC_FP64)
        else:
            hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_FP64)
        oracle.hold_step(ref, dt, True, 0.03, eps=EPS)
    ctx.check()
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    # and softening changes the answer (the parameter is not ignored)
    plain = _copy(s)
    for _ in range(2):
        oracle.hold_step(plain, dt, True, 0.03)
    assert not np.array_equal(plain["vx"], ref["vx"])


@pytest.mark.parametrize("small_n", [0, 256])
def test_softened_hold_mixed_close(cuda, hhs, oracle, small_n):
    n = 4096
    s = hhs.plummer(n, 93)
    ref = _copy(s)
    ctx = hhs.Context(n, 64, eta=0.03, eps=EPS)
    ctx.set_tuning(small_n)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    hhs.hold_step(ctx, d, n, 0.0, 1.0 / 64, True, hhs.PREC_MIXED)
    ctx.check()
    out = d.download()
    oracle.hold_step(ref, 1.0 / 64, True, 0.03, eps=EPS)
    dx = max(np.abs(out[k] - ref[k]).max() for k in ("x", "y", "z"))
    assert dx < 1e-7, dx


def test_softened_batched_fp64_bit_exact(cuda, hhs, oracle):
    sizes = [64, 500, 1500, 7, 260]
    parts = [hhs.plummer(nk, 400 + k) for k, nk in enumerate(sizes)]
    packed = {f: np.concatenate([p[f] for p in parts]) for f in FIELDS}
    packed["id"] = np.arange(sum(sizes), dtype=np.int32)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    n = int(offsets[-1])
    d = hhs.ParticleSystem(n)
    d.upload(packed)
    b = hhs.Batch(offsets, 64, eta=0.03, eps=EPS)
    b.set_tuning(1024, 64, 8)
    b.step(d, 1.0 / 64, True, hhs.PREC_FP64)
    b.check()
    out = d.download()
    for k, p in enumerate(parts):
        oracle.hold_step(p, 1.0 / 64, True, 0.03, eps=EPS)
        sl = slice(offsets[k], offsets[k + 1])
        for f in FIELDS:
            assert np.array_equal(out[f][sl], p[f]), (k, f)


# ------------------------------------------------------------------------------ energy
def _energy_numpy(s, eps):
    x = np.stack([s["x"], s["y"], s["z"]], 1)
    d = x[:, None, :] - x[None, :, :]
    r = np.sqrt((d * d).sum(-1) + eps * eps)
    np.fill_diagonal(r, np.inf)
    pot = -0.5 * np.sum(s["m"][:, None] * s["m"][None, :] / r)
    kin = 0.5 * np.sum(s["m"] * (s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2))
    return kin, pot


@pytest.mark.parametrize("n", [2, 257, 3000])
def test_device_energy_matches_oracle(cuda, hhs, oracle, n):
    s = hhs.plummer(n, 70 + n)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    k, p = hhs.energy(d, n)
    _, (ko, po) = oracle.energy(s)
    assert k == pytest.approx(ko, rel=1e-13, abs=1e-300)
    assert p == pytest.approx(po, rel=1e-13)
    ks, ps = hhs.energy(d, n, eps=0.05)
    kn, pn = _energy_numpy(s, 0.05)
    assert ks == pytest.approx(kn, rel=1e-12)
    assert ps == pytest.approx(pn, rel=1e-12)
    assert ps > p  # softening makes the potential shallower


def test_device_energy_rejects_bad_arguments(cuda, hhs):
    d = hhs.ParticleSystem(8)
    d.upload(hhs.plummer(8, 1))
    with pytest.raises(hhs.HHSError):
        hhs.energy(d, 9)
    with pytest.raises(hhs.HHSError):
        hhs.energy(d, 0)


# ------------------------------------------------------------------------------ snapshots
def test_snapshot_roundtrip_is_bitwise(cuda, hhs, tmp_path):
    n = 1000
    s = hhs.plummer(n, 5)
    s["id"] = np.arange(n, dtype=np.int32)[::-1].copy()
    d = hhs.ParticleSystem(n)
    d.upload(s)
    path = str(tmp_path / "snap.hhs")
    hhs.snapshot_write(d, n, 0.625, path, eta=0.03, eps=0.0, dt=1.0 / 64, step=40)
    assert os.path.getsize(path) == 80 + n * (8 * 8 + 4)
    e = hhs.ParticleSystem(n + 10)
    n2, t, step = hhs.snapshot_read(e, path)
    assert (n2, t, step) == (n, 0.625, 40)
    out = e.download(n)
    for k in FIELDS + ("id",):
        assert np.array_equal(out[k], s[k]), k
    small = hhs.ParticleSystem(n - 1)
    with pytest.raises(hhs.HHSError):
        hhs.snapshot_read(small, path)
    bad = tmp_path / "bad.hhs"
    bad.write_bytes(b"not a snapshot" * 10)
    with pytest.raises(hhs.HHSError):
        hhs.snapshot_read(e, str(bad))


# ------------------------------------------------------------------------------ hold()
def test_hold_driver_equals_steps_and_resumes(cuda, hhs, oracle, tmp_path):
    """hold(0, 4 dt) with a diagnostic every 2 steps: the state equals four single FP64
    steps of the oracle bit for bit, the log holds the energies at 0, 2dt and 4dt, and
    resuming from the step-2 snapshot reproduces the step-4 state."""
    n, dt = 600, 1.0 / 64
    s = hhs.plummer(n, 17)
    ref = _copy(s)
    ctx = hhs.Context(n, 64, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    prefix = str(tmp_path / "run")
    log = hhs.hold(ctx, d, n, 0.0, 4 * dt, dt, hhs.PREC_FP64, snapshot_every=2, prefix=prefix)
    ctx.check()
    out = d.download()
    energies = []
    for step in range(5):
        if step % 2 == 0:
            _, (k, p) = oracle.energy(ref)
            energies.append(k + p)
        if step < 4:
            oracle.hold_step(ref, dt, True, 0.03)
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    assert [t for t, _ in log] == [0.0, 2 * dt, 4 * dt]
    for (_, e), eo in zip(log, energies):
        assert e == pytest.approx(eo, rel=1e-12)
    assert abs((log[-1][1] - log[0][1]) / log[0][1]) < 1e-6
    for step in (0, 2, 4):
        assert os.path.exists(f"{prefix}_{step:06d}.hhs")
    # resume from the step-2 checkpoint
    r = hhs.ParticleSystem(n)
    n2, t, step = hhs.snapshot_read(r, f"{prefix}_000002.hhs")
    assert (n2, step) == (n, 2) and t == 2 * dt
    ctx2 = hhs.Context(n, 64, eta=0.03)
    hhs.hold(ctx2, r, n, t, 4 * dt, dt, hhs.PREC_FP64)
    ctx2.check()
    out2 = r.download()
    for k in FIELDS:
        assert np.array_equal(out2[k], out[k]), k


def test_hold_driver_rejects_bad_ranges(cuda, hhs):
    n = 16
    ctx = hhs.Context(n, 8)
    d = hhs.ParticleSystem(n)
    d.upload(hhs.plummer(n, 2))
    with pytest.raises(hhs.HHSError):
        hhs.hold(ctx, d, n, 1.0, 0.5, 0.1)
    with pytest.raises(hhs.HHSError):
        hhs.hold(ctx, d, n, 0.0, 1.0, 0.0)
