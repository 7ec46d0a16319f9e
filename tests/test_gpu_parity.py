"""GPU parity tests: the CUDA path through the C ABI against the FP64 oracle, the golden
fixtures from the reference's own test inputs, and the reference's own GPU kernels
(compiled under oracle/_ref) where they were built."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, REF_GPU

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m", "ts")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


def _scan_gpu(hhs, torch, a_dev, n, offset=0):
    out = torch.empty(n + offset, dtype=torch.int32, device="cuda")
    ws_bytes = hhs.scan_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    src = a_dev[offset:offset + n]
    dst = out[offset:offset + n]
    hhs.scan_exclusive_i32(_ptr(src), _ptr(dst), n, _ptr(ws), ws_bytes,
                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert hhs.scan_workspace_status(_ptr(ws), ctypes.c_void_p(
        torch.cuda.current_stream().cuda_stream)) == 0
    return dst


def _ref_gpu():
    if not os.path.exists(REF_GPU):
        return None
    L = ctypes.CDLL(REF_GPU)
    vp, d, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    L.ref_scan_predicate.argtypes = [vp, vp, i, i]
    L.ref_timesteps.argtypes = [vp, vp, vp, vp, d, i]
    L.ref_kick_slow.argtypes = [vp, vp, vp, vp, d, d, i]
    L.ref_kick_sf.argtypes = [vp, vp, vp, vp, vp, d, d, i, i]
    L.ref_drift.argtypes = [vp, vp, d, d, i]
    return L


def ref_scan_small_sizes(n, bs, unroll=4):
    """Sizes passed to scan_predicate_small by the reference's host recursion
    (src/split.cuh:438-565, 588-599) for an n-element scan with block size bs."""
    e = bs * unroll
    calls = []

    def large(m):
        rem = m % e
        large_ev(m - rem)
        if rem:
            calls.append(rem)

    def large_ev(m):
        nb = (m + e - 1) // e
        if nb > e:
            large(nb)
        else:
            calls.append(nb)

    if n > e:
        large(n)
    else:
        calls.append(n)
    return calls


def ref_scan_in_bounds(n, bs):
    """scan_predicate_small(m) writes indices up to max(v, 4) + v - 1 of a 2v-int dynamic
    shared buffer (v = next power of two >= m, src/split.cuh:150-159,445-457), past its
    end for m < 3. Such sizes are never run."""
    return all(m >= 3 for m in ref_scan_small_sizes(n, bs))


# ------------------------------------------------------------------------------ scan
def test_ref_scan_size_filter():
    assert ref_scan_small_sizes(1023, 128) == [1, 511]
    assert not ref_scan_in_bounds(1023, 128)
    assert ref_scan_in_bounds(1023, 256) and ref_scan_in_bounds(2048, 128)


def test_scan_matches_golden_reference_test_inputs(cuda, hhs):
    torch = cuda
    from make_golden import PROGRAMS, reference_test_inputs
    cases = json.load(open(os.path.join(GOLDEN, "scan_reference_tests.json")))["cases"]
    ref = _ref_gpu()
    k = 0
    for prog, sizes in PROGRAMS.items():
        for total in reference_test_inputs(sizes):
            c = cases[k]
            k += 1
            pred = torch.from_numpy((total <= np.float32(5.0)).astype(np.int32)).cuda()
            out = _scan_gpu(hhs, torch, pred, len(total)).cpu().numpy()
            assert _digest(out) == c["sha256_exclusive_scan"], (prog, c["n"])
            if ref is not None:
                for bs in (128, 256):
                    if not ref_scan_in_bounds(len(total), bs):
                        continue
                    rout = torch.empty_like(pred)
                    assert ref.ref_scan_predicate(_ptr(pred), _ptr(rout), len(total), bs) == 0
                    assert np.array_equal(rout.cpu().numpy(), out), (prog, c["n"], bs)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 127, 4095, 4096, 4097, 8191, 65536 + 3,
                               (1 << 20) + 7, (1 << 22) + 5, (1 << 23) + 4099,
                               (1 << 24), (1 << 25) + 4099, (1 << 26) + 3])
@pytest.mark.parametrize("offset", [0, 1])
def test_scan_random_values_sizes_alignment(cuda, hhs, oracle, n, offset):
    torch = cuda
    rng = np.random.default_rng(n + offset)
    a = rng.integers(-1000, 1000, n + offset).astype(np.int32)
    dev = torch.from_numpy(a).cuda()
    out = _scan_gpu(hhs, torch, dev, n, offset).cpu().numpy()
    assert np.array_equal(out, oracle.scan_exclusive(a[offset:]))


_SUPER_CHUNK_CHECK = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import hhs
n = 3 * (1 << 22) + 4099
for offset in (0, 1):
    a = np.random.default_rng(offset).integers(-1000, 1000, n + offset).astype(np.int32)
    dev = torch.from_numpy(a).cuda()
    out = torch.empty_like(dev)
    wb = hhs.scan_workspace_size(n)
    ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        hhs.scan_exclusive_i32(ctypes.c_void_p(dev[offset:].data_ptr()),
                               ctypes.c_void_p(out[offset:].data_ptr()), n,
                               ctypes.c_void_p(ws.data_ptr()), wb, None)
        torch.cuda.synchronize()
        ref = np.concatenate([[0], np.cumsum(a[offset:], dtype=np.int64)[:-1]]).astype(np.int32)
        assert np.array_equal(out[offset:].cpu().numpy(), ref), offset
print("ok")
"""


@pytest.mark.parametrize("variant", ["11", "12", "13"])
def test_large_scan_forms_carry_the_running_total(cuda, variant):
    """The large-input scan in the wave form (launch-shape variants): waves of 2^22, 2^23
    or 2^24 values (three, two or one wave, the running total carried from wave to wave,
    the last wave ragged); aligned and unaligned, twice in a row on one workspace."""
    import subprocess
    import sys
    from conftest import PKG
    r = subprocess.run([sys.executable, "-c", _SUPER_CHUNK_CHECK, PKG], capture_output=True,
                       text=True, timeout=600, env={**os.environ, "HHS_SCAN_VARIANT": variant})
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]


_STREAM_CHECK = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import hhs
def P(t):
    return ctypes.c_void_p(t.data_ptr())
rng = np.random.default_rng(23)
# ragged tails (n mod 4 != 0), fewer values than one chunk, more chunks than resident CTAs
sizes = [1, 3, 4, 5, 4099, 16384, 65536 + 6, (1 << 22) + 7, 148 * 3 * 16384 + 4097,
         (1 << 24) + 2]
wb = hhs.scan_workspace_size(max(sizes))
ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
for n in sizes:
    a = rng.integers(-1000, 1000, n).astype(np.int32)
    ref = np.zeros(n, np.int64)
    ref[1:] = np.cumsum(a, dtype=np.int64)[:-1]
    ref = ref.astype(np.int32)
    dev = torch.from_numpy(a).cuda()
    out = torch.full_like(dev, -7)
    for _ in range(2):
        hhs.scan_exclusive_i32(P(dev), P(out), n, P(ws), wb, None)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref), ("scan", n)
    flags = np.where(rng.random(n) < 0.3, rng.integers(1, 9, n), 0).astype(np.int32)
    sel = np.flatnonzero(flags).astype(np.int32)
    fs = np.zeros(n, np.int64)
    fs[1:] = np.cumsum(flags != 0)[:-1]
    fdev = torch.from_numpy(flags).cuda()
    for scan_out in (True, False):
        idx = torch.full_like(fdev, -1)
        cnt = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        sc = torch.full_like(fdev, -7)
        hhs.compact_flags_i32(P(fdev), P(sc) if scan_out else None, P(idx), P(cnt), n, P(ws),
                              wb, None)
        torch.cuda.synchronize()
        k = int(cnt.item())
        assert k == len(sel), ("count", n, k)
        assert np.array_equal(idx.cpu().numpy()[:k], sel), ("indices", n)
        if scan_out:
            assert np.array_equal(sc.cpu().numpy(), fs.astype(np.int32)), ("flag scan", n)
print("ok")
"""


@pytest.mark.parametrize("variant", ["20", "21", "22", "23", "24"])
def test_streamed_scan_shapes_match_numpy(cuda, variant):
    """The streamed single-pass scan (persistent CTAs, bulk-copied chunks) in each launch
    shape: exclusive scan and stream compaction (with and without the scan output) at ragged
    sizes from 1 to 2^24 + 2, including inputs shorter than one chunk and inputs with more
    chunks than resident CTAs; twice in a row on one workspace, against numpy."""
    import subprocess
    import sys
    from conftest import PKG
    r = subprocess.run([sys.executable, "-c", _STREAM_CHECK, PKG], capture_output=True,
                       text=True, timeout=600, env={**os.environ, "HHS_SCAN_VARIANT": variant})
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]


def test_wave_barrier_wait_gives_up_and_reports_timeout(cuda, hhs, oracle):
    """Failure detection without a GPU fault: every grid barrier of the wave-form scan
    waits for one CTA more than the launch has; the bounded waits give up after 20 ms,
    the call returns HHS_ERR_TIMEOUT, and the same workspace then serves a correct
    compaction in the wave form."""
    torch = cuda
    n = (1 << 24) + 11
    ws_bytes = hhs.scan_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    flags = np.random.default_rng(8).integers(0, 2, n).astype(np.int32)
    dev = torch.from_numpy(flags).cuda()
    out = torch.empty_like(dev)
    assert hhs.scan_selftest_wave_barrier(_ptr(dev), _ptr(out), n, _ptr(ws), ws_bytes, 20000,
                                          st) == 4
    idx = torch.full_like(dev, -1)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    hhs.compact_flags_i32(_ptr(dev), _ptr(out), _ptr(idx), _ptr(cnt), n, _ptr(ws), ws_bytes, st)
    assert hhs.scan_workspace_status(_ptr(ws), st) == 0
    k = int(cnt.item())
    assert k == int(flags.sum())
    assert np.array_equal(out.cpu().numpy(), oracle.scan_exclusive(flags))
    assert np.array_equal(idx.cpu().numpy()[:k], np.flatnonzero(flags).astype(np.int32))


def test_scan_lookback_wait_gives_up_and_reports_timeout(cuda, hhs, oracle):
    """Failure detection without a GPU fault: with the first tile left out, every look-back
    waits for a predecessor that never publishes; the bounded waits give up, the call
    returns HHS_ERR_TIMEOUT, and the context stays usable for a correct scan after it."""
    torch = cuda
    n = 1 << 16
    ws_bytes = hhs.scan_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    a = np.random.default_rng(5).integers(0, 2, n).astype(np.int32)
    dev = torch.from_numpy(a).cuda()
    out = torch.empty_like(dev)
    status = hhs.scan_selftest_stalled_predecessor(_ptr(dev), _ptr(out), n, _ptr(ws), ws_bytes,
                                                   2048, st)
    assert hhs.STATUS[status] == "HHS_ERR_TIMEOUT"
    hhs.scan_exclusive_i32(_ptr(dev), _ptr(out), n, _ptr(ws), ws_bytes, st)
    assert hhs.scan_workspace_status(_ptr(ws), st) == 0
    assert np.array_equal(out.cpu().numpy(), oracle.scan_exclusive(a))
    assert hhs.scan_selftest_stalled_predecessor(_ptr(dev), _ptr(out), 100, _ptr(ws), ws_bytes,
                                                 2048, st) != 0  # fewer than two tiles


def test_scan_repeated_calls_reuse_workspace(cuda, hhs, oracle):
    torch = cuda
    n = 300001
    ws_bytes = hhs.scan_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for seed in range(3):
        a = np.random.default_rng(seed).integers(0, 2, n).astype(np.int32)
        dev = torch.from_numpy(a).cuda()
        out = torch.empty_like(dev)
        hhs.scan_exclusive_i32(_ptr(dev), _ptr(out), n, _ptr(ws), ws_bytes, st)
        assert np.array_equal(out.cpu().numpy(), oracle.scan_exclusive(a))


@pytest.mark.parametrize("log2n", [26, 28])
def test_scan_full_size_properties(cuda, hhs, log2n):
    """2^26 and 2^28 Bernoulli flags: checked through size-independent properties on the
    device (differences reproduce the input, first is 0, last + input = total)."""
    torch = cuda
    n = 1 << log2n
    g = torch.Generator(device="cuda").manual_seed(log2n)
    flags = (torch.rand(n, device="cuda", generator=g) < 0.1).to(torch.int32)
    out = _scan_gpu(hhs, torch, flags, n)
    assert int(out[0]) == 0
    assert torch.equal(out[1:] - out[:-1], flags[:-1])
    assert int(out[-1]) + int(flags[-1]) == int(flags.sum())
    del out, flags
    torch.cuda.empty_cache()


# ------------------------------------------------------------------------------ split
def _device_partition(torch):
    return torch.zeros(2, dtype=torch.int32, device="cuda")


@pytest.mark.parametrize("n,frac", [(2, 0.5), (3, 0.0), (64, 1.0), (1000, 0.3), (4097, 0.05),
                                    (20000, 0.6), (20000, "one")])
def test_split_matches_oracle(cuda, hhs, oracle, n, frac):
    torch = cuda
    rng = np.random.default_rng(n)
    s = {k: rng.standard_normal(n) for k in FIELDS}
    s["ts"] = rng.random(n)
    s["id"] = rng.permutation(n).astype(np.int32)
    if frac == "one":
        pivot = float(np.sort(s["ts"])[0])  # exactly one fast particle -> fold
    else:
        pivot = float(np.quantile(s["ts"], frac)) if frac > 0 else -1.0
    ctx = hhs.Context(n, 4)
    tot, slow, fast = hhs.ParticleSystem(n), hhs.ParticleSystem(n), hhs.ParticleSystem(n)
    tot.upload(s)
    part = _device_partition(torch)
    pred = torch.empty(n, dtype=torch.int32, device="cuda")
    scan = torch.empty(n, dtype=torch.int32, device="cuda")
    hhs.split(ctx, tot, slow, fast, pivot, n, _ptr(part), _ptr(pred), _ptr(scan))
    torch.cuda.synchronize()
    ctx.check()
    n_slow, n_fast = part.cpu().numpy().tolist()
    order, nf = oracle.split(s["ts"], pivot)
    assert (n_fast, n_slow) == (nf, n - nf)
    p_ref = (s["ts"] <= pivot).astype(np.int32)
    assert np.array_equal(pred.cpu().numpy(), p_ref)
    assert np.array_equal(scan.cpu().numpy(), oracle.scan_exclusive(p_ref))
    F = fast.download(nf) if nf else None
    Ls = slow.download(n - nf)
    for k in FIELDS:
        assert np.array_equal(Ls[k], s[k][order[nf:]]), k
        if nf:
            assert np.array_equal(F[k], s[k][order[:nf]]), k
    assert np.array_equal(Ls["id"], s["id"][order[nf:]])
    # parent_id: update_system scatters both halves back onto an empty parent
    back = hhs.ParticleSystem(n)
    hhs.update_system(back, slow, n - nf)
    if nf:
        hhs.update_system(back, fast, nf)
    b = back.download()
    for k in FIELDS:
        assert np.array_equal(b[k], s[k]), k


# ------------------------------------------------------------------------------ physics
def _plummer(hhs, n, seed, spectrum=0):
    return hhs.plummer(n, seed, spectrum)


@pytest.mark.parametrize("n", [2, 3, 129, 1000])
def test_timesteps_fp64_bit_exact(cuda, hhs, oracle, n):
    s = _plummer(hhs, max(n, 2), 3)
    ctx = hhs.Context(n, 4, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    hhs.timesteps(ctx, d, n, hhs.PREC_FP64)
    out = d.download()
    assert np.array_equal(out["ts"], oracle.timesteps(s, 0.03))


@pytest.mark.parametrize("n", [2, 1000, 5000])
def test_timesteps_mixed_close(cuda, hhs, oracle, n):
    s = _plummer(hhs, n, 4)
    ctx = hhs.Context(n, 4, eta=0.02)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    hhs.timesteps(ctx, d, n, hhs.PREC_MIXED)
    out = d.download()["ts"]
    ref = oracle.timesteps(s, 0.02)
    rel = np.abs(out - ref) / ref
    assert rel.max() < 2e-6, rel.max()


@pytest.mark.parametrize("n", [1, 7, 1000])
def test_kick_slow_and_sf_fp64_bit_exact(cuda, hhs, oracle, n):
    s = _plummer(hhs, max(n, 2), 5)
    s = {k: v[:n].copy() for k, v in s.items()}
    d = hhs.ParticleSystem(n)
    d.upload(s)
    hhs.kick_slow(d, 0.01, 0.5, n, hhs.PREC_FP64)
    out = d.download()
    ref = {k: v.copy() for k, v in s.items()}
    oracle.kick(ref, s, 0.5 * 0.01)
    for k in ("vx", "vy", "vz", "x"):
        assert np.array_equal(out[k], ref[k]), k
    # kick_sf: sinks in one system, sources in another
    src = _plummer(hhs, 333, 6)
    so = hhs.ParticleSystem(333)
    so.upload(src)
    hhs.kick_sf(so, d, 1.0, 0.02, n, 333, hhs.PREC_FP64)
    out2 = d.download()
    oracle.kick(ref, src, 0.02 * 1.0)
    for k in ("vx", "vy", "vz"):
        assert np.array_equal(out2[k], ref[k]), k


def test_kick_mixed_close(cuda, hhs, oracle):
    n = 4000
    s = _plummer(hhs, n, 8)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    hhs.kick_slow(d, 1.0, 1.0, n, hhs.PREC_MIXED)
    out = d.download()
    ref = {k: v.copy() for k, v in s.items()}
    acc = oracle.kick(ref, s, 1.0)
    amag = np.sqrt((acc ** 2).sum(0))
    for c, k in enumerate(("vx", "vy", "vz")):
        err = np.abs((out[k] - s[k]) - acc[c]) / amag
        assert err.max() < 1e-6, (k, err.max())


def test_drift_update_and_aos_roundtrip(cuda, hhs):
    n = 777
    s = _plummer(hhs, n, 9)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    hhs.drift(d, 0.125, 0.5, n)
    out = d.download()
    for a, v in (("x", "vx"), ("y", "vy"), ("z", "vz")):
        assert np.array_equal(out[a], s[a] + s[v] * (0.125 * 0.5))
    # AoS (vec3) upload / download
    L = hhs.lib()
    pos3 = np.ascontiguousarray(np.stack([s["x"], s["y"], s["z"]], 1))
    vel3 = np.ascontiguousarray(np.stack([s["vx"], s["vy"], s["vz"]], 1))
    dp = ctypes.POINTER(ctypes.c_double)
    assert L.hhs_particle_system_upload_aos(d.ref, n, pos3.ctypes.data_as(dp),
                                            vel3.ctypes.data_as(dp), None, None, None,
                                            None) == 0
    back = d.download()
    assert np.array_equal(back["x"], s["x"]) and np.array_equal(back["vz"], s["vz"])
    p2, v2 = np.zeros_like(pos3), np.zeros_like(vel3)
    assert L.hhs_particle_system_download_aos(d.ref, n, p2.ctypes.data_as(dp),
                                              v2.ctypes.data_as(dp), None, None, None,
                                              None) == 0
    assert np.array_equal(p2, pos3) and np.array_equal(v2, vel3)


# ------------------------------------------------------------------------------ HOLD
@pytest.mark.parametrize("n,steps,spectrum", [(64, 3, 0), (300, 3, 0), (1024, 2, 1)])
def test_hold_step_host_fp64_bit_exact(cuda, hhs, oracle, n, steps, spectrum):
    s = _plummer(hhs, n, 10 + n, spectrum)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    dt = 1.0 / 64
    leaf = 0.0
    for _ in range(steps):
        hhs.hold_step_host(ctx, d, n, dt, True, hhs.PREC_FP64)
        tr, _ = oracle.hold_step(ref, dt, True, 0.03)
        leaf += tr.leaf_time
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    assert ctx.simtime() == pytest.approx(leaf, rel=1e-15)


def test_hold_step_mixed_close(cuda, hhs, oracle):
    n = 1024
    s = _plummer(hhs, n, 77)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    dt = 1.0 / 64
    e0 = hhs.energy_host(s)
    hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_MIXED)
    ctx.check()
    out = d.download()
    oracle.hold_step(ref, dt, True, 0.03)
    dx = max(np.abs(out[k] - ref[k]).max() for k in ("x", "y", "z"))
    assert dx < 1e-8, dx
    # energy: mixed and FP64 steps agree far below the integrator's own error
    e1, e_ref = hhs.energy_host(out), hhs.energy_host(ref)
    assert abs((e1 - e_ref) / e0) < 1e-9, (e1 - e_ref) / e0
    assert abs((e1 - e0) / e0) < 1e-6


# ------------------------------------------------------------------------------ reference
@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference GPU shims not built")
def test_reference_gpu_kernels_pin_the_oracle(cuda, hhs, oracle):
    """The reference's own timestep / kick / drift kernels (compiled with -fmad=false)
    agree bit for bit with the oracle (kick: up to the reference's repulsive sign)."""
    torch = cuda
    ref = _ref_gpu()
    n = 512  # a multiple of 256: the timestep kernel's tail-tile read stays out of play
    s = _plummer(hhs, n, 12)
    pos = torch.from_numpy(np.stack([s["x"], s["y"], s["z"]], 1).copy()).cuda()
    vel = torch.from_numpy(np.stack([s["vx"], s["vy"], s["vz"]], 1).copy()).cuda()
    acc = torch.zeros_like(pos)
    m = torch.from_numpy(s["m"].copy()).cuda()
    ts = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert ref.ref_timesteps(_ptr(pos), _ptr(vel), _ptr(m), _ptr(ts), 0.03, n) == 0
    assert np.array_equal(ts.cpu().numpy(), oracle.timesteps(s, 0.03))
    assert ref.ref_kick_slow(_ptr(pos), _ptr(vel), _ptr(acc), _ptr(m), 0.01, 1.0, n) == 0
    o = {k: v.copy() for k, v in s.items()}
    a = oracle.kick(o, s, -0.01)  # repulsive reference sign == attractive with -dt
    assert np.array_equal(acc.cpu().numpy(), -a.T)
    v = vel.cpu().numpy()
    assert np.array_equal(v[:, 0], o["vx"]) and np.array_equal(v[:, 2], o["vz"])
    assert ref.ref_drift(_ptr(pos), _ptr(vel), 0.5, 0.5, n) == 0
    p = pos.cpu().numpy()
    assert np.array_equal(p[:, 1], s["y"] + v[:, 1] * (0.5 * 0.5))


# ------------------------------------------------------------------------------ engine
@pytest.mark.parametrize("n,small_n,spectrum", [(64, 0, 0), (300, 0, 0), (300, 64, 0),
                                                (300, 100000, 0), (2048, 256, 1),
                                                (5000, 512, 0)])
def test_hold_step_engine_fp64_bit_exact(cuda, hhs, oracle, n, small_n, spectrum):
    """The persistent device schedule in FP64 reproduces the oracle bit for bit, with every
    node on the grid (small_n = 0), every node in one CTA (huge small_n) or mixed."""
    s = _plummer(hhs, n, 20 + n, spectrum)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    ctx.set_tuning(small_n, cluster_size=1, mid_n=0)  # grid, block and tiny paths only
    d = hhs.ParticleSystem(n)
    d.upload(s)
    dt = 1.0 / 64
    leaf, nodes, kp, tp = 0.0, 0, 0.0, 0.0
    for _ in range(2):
        hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_FP64)
        tr, _ = oracle.hold_step(ref, dt, True, 0.03)
        leaf += tr.leaf_time
        nodes += tr.count
        kp += tr.kick_pairs
        tp += tr.ts_pairs
    ctx.check()
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    st = ctx.stats()
    assert st["nodes"] == nodes and st["kick_pairs"] == kp and st["ts_pairs"] == tp
    assert ctx.simtime() == pytest.approx(leaf, rel=1e-15)


@pytest.mark.parametrize("n,small_n,packed", [(1024, 0, 0), (4096, 256, 0), (16384, 512, 0),
                                              (1024, 0, 1), (5000, 64, 1)])
def test_hold_step_engine_mixed_close(cuda, hhs, oracle, n, small_n, packed):
    s = _plummer(hhs, n, 30 + n)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    ctx.set_tuning(small_n, packed=packed, cluster_size=1, mid_n=0)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    e0 = hhs.energy_host(s)
    dt = 1.0 / 64
    hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_MIXED)
    ctx.check()
    out = d.download()
    oracle.hold_step(ref, dt, True, 0.03)
    dx = max(np.abs(out[k] - ref[k]).max() for k in ("x", "y", "z"))
    assert dx < 1e-7, dx
    e1, e_ref = hhs.energy_host(out), hhs.energy_host(ref)
    assert abs((e1 - e_ref) / e0) < 1e-9, (e1 - e_ref) / e0


# ------------------------------------------------------------------------------ C++ API
def test_reference_style_cpp_caller(cuda, hhs):
    """tests/cpp/test_compat.cpp uses the reference's template API through include/hhs.hpp;
    its result equals the same FP64 steps driven through the C ABI from Python."""
    import subprocess
    from conftest import ROOT
    exe = os.path.join(ROOT, "tests", "cpp", "_build", "test_compat")
    if not os.path.exists(exe):
        pytest.skip("compat test binary not built")
    n, steps = 1024, 2
    out = subprocess.run([exe, str(n), str(steps)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "[FAIL]" not in out.stdout, out.stdout
    res = json.loads(out.stdout.strip().splitlines()[-1])
    s = hhs.plummer(n, 99)
    ctx = hhs.Context(n, 64, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    for _ in range(steps):
        hhs.hold_step(ctx, d, n, 0.0, 1.0 / 64, True, hhs.PREC_FP64)
    o = d.download()
    h = 1469598103934665603
    pos = np.stack([o["x"], o["y"], o["z"]], 1).tobytes()
    vel = np.stack([o["vx"], o["vy"], o["vz"]], 1).tobytes()
    for blob in (pos, vel, o["ts"].tobytes()):
        for b in blob:
            h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    assert res["fnv"] == f"{h:016x}"
    assert res["x0"] == o["x"][0]
    assert res["simtime"] == pytest.approx(ctx.simtime(), rel=1e-15)


def test_autotune_restores_state_and_keeps_results(cuda, hhs, oracle):
    n = 1500
    s = _plummer(hhs, n, 41)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    t = ctx.autotune(d, n, 1.0 / 64, hhs.PREC_FP64)
    assert t["ms_per_step"] > 0 and t["ctas_per_sm"] in (1, 2)
    after = d.download()
    for k in FIELDS:
        assert np.array_equal(after[k], s[k]), k
    assert ctx.simtime() == 0.0 and ctx.stats()["nodes"] == 0
    table = ctx.autotune_results()
    assert len(table) >= 8 and all(r["ms_per_step"] > 0 for r in table)
    assert t["ms_per_step"] == min(r["ms_per_step"] for r in table)
    hhs.hold_step(ctx, d, n, 0.0, 1.0 / 64, True, hhs.PREC_FP64)
    ctx.check()
    oracle.hold_step(ref, 1.0 / 64, True, 0.03)
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k


def test_batch_autotune_restores_state_and_keeps_results(cuda, hhs, oracle):
    """The batched autotuner leaves the systems, leaf times and counters as it found
    them, keeps the fastest candidate, and the next step still equals the oracle."""
    sizes = [64, 100, 33, 500, 1500, 2100, 7, 260]
    parts, packed, offsets = _packed(hhs, sizes, 310)
    n = int(offsets[-1])
    d = hhs.ParticleSystem(n)
    d.upload(packed)
    b = hhs.Batch(offsets, 64, eta=0.03)
    best, table = b.autotune(d, 1.0 / 64, hhs.PREC_FP64)
    assert len(table) == 12 and best["ms_per_step"] == min(t["ms_per_step"] for t in table)
    after = d.download()
    for f in FIELDS:
        assert np.array_equal(after[f], packed[f]), f
    assert np.all(b.simtime() == 0.0)
    b.step(d, 1.0 / 64, True, hhs.PREC_FP64)
    b.check()
    out = d.download()
    for k, p in enumerate(parts):
        oracle.hold_step(p, 1.0 / 64, True, 0.03)
        sl = slice(offsets[k], offsets[k + 1])
        for f in FIELDS:
            assert np.array_equal(out[f][sl], p[f]), (k, f)


@pytest.mark.parametrize("n,p", [(1, 1.0), (5, 0.5), (4097, 0.01), (100003, 0.5),
                                 ((1 << 20) + 5, 0.1), ((1 << 22) + 7, 0.3), (1 << 23, 0.01),
                                 ((1 << 25) + 13, 0.2)])
def test_compact_flags_matches_oracle(cuda, hhs, oracle, n, p):
    torch = cuda
    rng = np.random.default_rng(n)
    flags = (rng.random(n) < p).astype(np.int32) * rng.integers(1, 5, n).astype(np.int32)
    dev = torch.from_numpy(flags).cuda()
    scan = torch.empty_like(dev)
    idx = torch.full_like(dev, -1)
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws_bytes = hhs.scan_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    hhs.compact_flags_i32(_ptr(dev), _ptr(scan), _ptr(idx), _ptr(cnt), n, _ptr(ws), ws_bytes,
                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    pred = (flags != 0).astype(np.int32)
    k = int(cnt.item())
    assert k == pred.sum()
    assert np.array_equal(scan.cpu().numpy(), oracle.scan_exclusive(pred))
    order, _ = oracle.split(np.where(pred == 1, 0.0, 1.0), 0.5)
    if k != 1:
        assert np.array_equal(idx.cpu().numpy()[:k], order[:k])
    else:
        assert idx.cpu().numpy()[0] == np.nonzero(pred)[0][0]


@pytest.mark.parametrize("warp_n,small_n", [(32, 0), (0, 0), (32, 256), (16, 100000)])
def test_engine_warp_solver_fp64_bit_exact(cuda, hhs, oracle, warp_n, small_n):
    n = 700
    s = _plummer(hhs, n, 55)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    ctx.set_tuning(small_n=small_n, warp_n=warp_n, cluster_size=1, mid_n=0)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    nodes = 0
    for _ in range(2):
        hhs.hold_step(ctx, d, n, 0.0, 1.0 / 64, True, hhs.PREC_FP64)
        tr, _ = oracle.hold_step(ref, 1.0 / 64, True, 0.03)
        nodes += tr.count
    ctx.check()
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    assert ctx.stats()["nodes"] == nodes


def _packed(hhs, sizes, seed0):
    parts = [hhs.plummer(nk, seed0 + k) for k, nk in enumerate(sizes)]
    packed = {f: np.concatenate([p[f] for p in parts]) for f in FIELDS}
    packed["id"] = np.arange(sum(sizes), dtype=np.int32)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    return parts, packed, offsets


@pytest.mark.parametrize("sizes,big_n,prec,mid_n", [
    ([64, 100, 33, 2, 500, 1500, 3000, 7, 260], 1024, 0, 640),
    ([64, 100, 33, 2, 500, 1500, 3000, 7, 260], 1024, 0, 0),
    ([300] * 12 + [2000] * 3, 128, 0, 640),
    ([300] * 12 + [2000] * 3, 128, 0, 0),
    ([64, 100, 33, 2, 500, 1500, 3000, 7, 260], 1024, 1, 640)])
def test_hold_batched_matches_per_system_oracle(cuda, hhs, oracle, sizes, big_n, prec, mid_n):
    """Independent systems in one launch: large ones on a thread-block cluster, small ones
    on one CTA, with (mid_n = 640) or without the shared-memory subtree solver."""
    parts, packed, offsets = _packed(hhs, sizes, 300)
    n = int(offsets[-1])
    d = hhs.ParticleSystem(n)
    d.upload(packed)
    b = hhs.Batch(offsets, 64, eta=0.03)
    b.set_tuning(big_n, 64, 8)
    b.set_mid(mid_n, 96)
    dt = 1.0 / 64
    leaf = np.zeros(len(sizes))
    for _ in range(2):
        b.step(d, dt, True, prec)
        for k, p in enumerate(parts):
            tr, _ = oracle.hold_step(p, dt, True, 0.03)
            leaf[k] += tr.leaf_time
    b.check()
    out = d.download()
    for k, p in enumerate(parts):
        sl = slice(offsets[k], offsets[k + 1])
        for f in FIELDS:
            if prec == 0:
                assert np.array_equal(out[f][sl], p[f]), (k, f)
            elif f in ("x", "y", "z"):
                assert np.max(np.abs(out[f][sl] - p[f])) < 1e-7, (k, f)
    assert np.allclose(b.simtime(), leaf, rtol=1e-15, atol=0)


def test_hold_integrate_graph_matches_steps(cuda, hhs, oracle):
    n = 800
    s = _plummer(hhs, n, 61)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    for _ in range(2):  # capture, then replay
        hhs.hold_integrate(ctx, d, n, 1.0 / 64, 2, hhs.PREC_FP64)
    ctx.check()
    for _ in range(4):
        oracle.hold_step(ref, 1.0 / 64, True, 0.03)
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k


# ------------------------------------------------------------------------------ cluster solver
@pytest.mark.parametrize("n,cs,mid_n,dist_n,spectrum", [
    (2, 1, 640, 96, 0), (24, 8, 640, 96, 0), (33, 2, 640, 0, 0),
    (300, 1, 640, 96, 0), (300, 2, 640, 16, 0), (300, 8, 640, 16, 0), (640, 4, 640, 0, 1),
    (2048, 8, 640, 96, 0), (2048, 8, 256, 32, 1), (5000, 4, 640, 64, 0)])
def test_hold_step_cluster_solver_fp64_bit_exact(cuda, hhs, oracle, n, cs, mid_n, dist_n,
                                                 spectrum):
    """Subtrees of at most mid_n particles solved from shared memory on one thread-block
    cluster (cs CTAs; pair work spread over the cluster above dist_n members, nodes of up
    to 32 members on one warp) reproduce the oracle bit for bit, with its work counters."""
    s = _plummer(hhs, n, 40 + n, spectrum)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03)
    ctx.set_tuning(64, cluster_size=cs, mid_n=mid_n, mid_dist_n=dist_n)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    dt = 1.0 / 64
    leaf, nodes, kp, tp = 0.0, 0, 0.0, 0.0
    for _ in range(2):
        hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_FP64)
        tr, _ = oracle.hold_step(ref, dt, True, 0.03)
        leaf += tr.leaf_time
        nodes += tr.count
        kp += tr.kick_pairs
        tp += tr.ts_pairs
    ctx.check()
    out = d.download()
    for k in FIELDS:
        assert np.array_equal(out[k], ref[k]), k
    st = ctx.stats()
    assert st["nodes"] == nodes and st["kick_pairs"] == kp and st["ts_pairs"] == tp
    assert ctx.simtime() == pytest.approx(leaf, rel=1e-15)


@pytest.mark.parametrize("cs,dist_n", [(1, 96), (8, 32), (8, 96)])
def test_hold_step_cluster_solver_mixed_close(cuda, hhs, oracle, cs, dist_n):
    n = 4096
    s = _plummer(hhs, n, 44)
    ref = {k: v.copy() for k, v in s.items()}
    ctx = hhs.Context(n, 64, eta=0.03, eps=0.001)
    ctx.set_tuning(64, cluster_size=cs, mid_n=640, mid_dist_n=dist_n)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    e0 = hhs.energy_host(s)
    hhs.hold_step(ctx, d, n, 0.0, 1.0 / 64, True, hhs.PREC_MIXED)
    ctx.check()
    out = d.download()
    oracle.hold_step(ref, 1.0 / 64, True, 0.03, eps=0.001)
    dx = max(np.abs(out[k] - ref[k]).max() for k in ("x", "y", "z"))
    assert dx < 1e-7, dx
    assert abs((hhs.energy_host(out) - hhs.energy_host(ref)) / e0) < 1e-8


# ------------------------------------------------------------------------------ CPU-order split
@pytest.mark.parametrize("n", [1, 2, 3, 100, 4097, 65536, 1 << 22])
def test_split_cpu_order_matches_oracle(cuda, hhs, oracle, n):
    """hhs_split_cpu_order leaves the permutation of the HHS CPU integrators' in-place
    partition (cpu_split), bit for bit, with ties at the pivot and all-fast / all-slow."""
    torch = cuda
    rng = np.random.default_rng(n)
    ws_bytes = hhs.split_cpu_order_workspace_size(n)
    ws = torch.empty(ws_bytes + 256, dtype=torch.uint8, device="cuda")
    base = (ws.data_ptr() + 255) & ~255
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for kind, pivot in (("rand", 0.3), ("rand", 0.5), ("ties", 2.0), ("rand", -1.0), ("rand", 2.0)):
        ts = rng.random(n) if kind == "rand" else rng.integers(0, 5, n).astype(np.float64)
        d_ts = torch.from_numpy(ts).cuda()
        order = torch.empty(n, dtype=torch.int32, device="cuda")
        counts = torch.zeros(2, dtype=torch.int32, device="cuda")
        hhs.split_cpu_order(_ptr(d_ts), n, pivot, _ptr(order), _ptr(counts),
                            ctypes.c_void_p(base), ws_bytes, st)
        ref, nf = oracle.split_cpu_order(ts, pivot)
        c = counts.cpu().numpy()
        assert c[1] == nf and c[0] == n - nf
        assert np.array_equal(order.cpu().numpy(), ref), (kind, pivot)
