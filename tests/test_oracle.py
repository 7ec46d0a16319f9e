"""CPU tests of the FP64 oracle: pinned against the reference's own test inputs and its
compiled CPU split, and against independent numpy restatements."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, REF_CPU


def _golden():
    with open(os.path.join(GOLDEN, "scan_reference_tests.json")) as f:
        return json.load(f)["cases"]


def _inputs(sizes):
    from make_golden import reference_test_inputs
    return reference_test_inputs(sizes)


def test_scan_and_split_match_golden_reference_test_cases(oracle):
    from make_golden import PROGRAMS, digest
    cases = _golden()
    k = 0
    for prog, sizes in PROGRAMS.items():
        for total in _inputs(sizes):
            c = cases[k]
            k += 1
            assert c["program"] == prog and c["n"] == len(total)
            pred = (total <= np.float32(5.0)).astype(np.int32)
            scan = oracle.scan_exclusive(pred)
            order, nf = oracle.split(total.astype(np.float64), 5.0)
            assert int(pred.sum()) == c["count_le_pivot"] == c["ref_cpu_split_n_fast"]
            assert digest(scan) == c["sha256_exclusive_scan"]
            assert digest(order) == c["sha256_stable_order"]
            # the reference tests' own checks: sizes add up, membership per side
            assert nf + (len(total) - nf) == len(total)
            assert np.all(total[order[:nf]] <= 5.0) and np.all(total[order[nf:]] > 5.0)
    assert k == len(cases)


@pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU split not built")
def test_oracle_counts_match_reference_cpu_split_random():
    import oracle
    lib = ctypes.CDLL(REF_CPU)
    lib.ref_cpu_split_f64.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                      ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]
    rng = np.random.default_rng(3)
    for n in (2, 3, 17, 1000, 4097):
        for p in (0.0, 0.01, 0.5, 1.0):
            ts = rng.random(n)
            pivot = np.quantile(ts, p) if p > 0 else -1.0
            work = ts.copy()
            ns, nf = ctypes.c_int(), ctypes.c_int()
            lib.ref_cpu_split_f64(work.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n, pivot,
                                  ctypes.byref(ns), ctypes.byref(nf))
            order, nf_o = oracle.split(ts, pivot)
            cnt = int((ts <= pivot).sum())
            assert nf.value == cnt and ns.value == n - cnt
            assert nf_o == (0 if cnt == 1 else cnt)
            # the reference's partition is unstable; as sets the two sides agree
            assert set(np.sort(work[:nf.value]).tolist()) == set(ts[order[:cnt]].tolist()) \
                if cnt != 1 else True


def _ref_cpu_split_order(ts, pivot):
    """The reference's own cpu_split run on the timesteps; distinct values map its output
    back to particle indices."""
    lib = ctypes.CDLL(REF_CPU)
    lib.ref_cpu_split_f64.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                      ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]
    work = ts.copy()
    ns, nf = ctypes.c_int(), ctypes.c_int()
    lib.ref_cpu_split_f64(work.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(ts), pivot,
                          ctypes.byref(ns), ctypes.byref(nf))
    where = {v: i for i, v in enumerate(ts.tolist())}
    return np.array([where[v] for v in work.tolist()], dtype=np.int32), nf.value


@pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU split not built")
def test_cpu_order_split_matches_reference_cpu_split_permutation(oracle):
    """oracle_split_cpu_order reproduces the permutation the reference's cpu_split leaves
    behind (src/cpu_scan.h:20-50), not just its counts."""
    rng = np.random.default_rng(11)
    for n in (1, 2, 3, 17, 1000, 4097, 65536):
        for p in (0.0, 0.01, 0.3, 0.5, 0.99, 1.0):
            ts = rng.random(n)
            pivot = float(np.quantile(ts, p)) if p > 0 else -1.0
            ref_order, ref_nf = _ref_cpu_split_order(ts, pivot)
            order, nf = oracle.split_cpu_order(ts, pivot)
            assert nf == ref_nf == int((ts <= pivot).sum())
            assert np.array_equal(order, ref_order), (n, p)


def test_scan_exclusive_random(oracle):
    rng = np.random.default_rng(0)
    for n in (1, 2, 31, 4096, 4097, 100003):
        a = rng.integers(-5, 6, n).astype(np.int32)
        out = oracle.scan_exclusive(a)
        ref = np.concatenate([[0], np.cumsum(a, dtype=np.int64)[:-1]]).astype(np.int32)
        assert np.array_equal(out, ref)


def test_split_stable_and_fold(oracle):
    ts = np.array([0.5, 0.1, 0.7, 0.2, 0.9, 0.05])
    order, nf = oracle.split(ts, 0.3)
    assert nf == 3
    assert order.tolist() == [1, 3, 5, 0, 2, 4]
    # exactly one fast particle: folded into the slow set, placed last
    order, nf = oracle.split(ts, 0.06)
    assert nf == 0
    assert order.tolist() == [0, 1, 2, 3, 4, 5]
    ts2 = np.array([0.5, 0.01, 0.7, 0.9])
    order, nf = oracle.split(ts2, 0.1)
    assert nf == 0 and order.tolist() == [0, 2, 3, 1]
    order, nf = oracle.split(ts2, 1.0)
    assert nf == 4 and order.tolist() == [0, 1, 2, 3]
    order, nf = oracle.split(ts2, 0.0)
    assert nf == 0 and order.tolist() == [0, 1, 2, 3]


def _np_timesteps(s, eta):
    """Independent numpy FP64 restatement of src/timestep.cuh:27-57 (same op order)."""
    n = len(s["x"])
    ts = np.full(n, 1e30)
    eta_s2 = eta / np.sqrt(2.0)
    for i in range(n):
        j = np.arange(n) != i
        drx, dry, drz = s["x"][i] - s["x"][j], s["y"][i] - s["y"][j], s["z"][i] - s["z"][j]
        dvx, dvy, dvz = s["vx"][i] - s["vx"][j], s["vy"][i] - s["vy"][j], s["vz"][i] - s["vz"][j]
        dr2 = drx * drx + dry * dry + drz * drz
        dv2 = dvx * dvx + dvy * dvy + dvz * dvz
        r = np.sqrt(dr2)
        vd = (dvx * drx + dvy * dry + dvz * drz) / dr2
        tau = eta_s2 * r * np.sqrt(r / (s["m"][j] + s["m"][i]))
        dtau = 3 * tau * vd / 2
        dtau = np.where(dtau < 1, dtau, 1.0)
        t1 = tau / (1 - dtau / 2)
        tau = eta * r / np.sqrt(dv2)
        dtau = tau * vd * (1 + (s["m"][i] + s["m"][j]) / (dv2 * r))
        dtau = np.where(dtau < 1, dtau, 1.0)
        t2 = tau / (1 - dtau / 2)
        ts[i] = min(1e30, t1.min(), t2.min())
    return ts


def _rand_system(n, seed):
    rng = np.random.default_rng(seed)
    s = {k: rng.standard_normal(n) for k in ("x", "y", "z", "vx", "vy", "vz")}
    s["m"] = rng.random(n) / n + 1e-3 / n
    s["ts"] = np.zeros(n)
    s["id"] = np.arange(n, dtype=np.int32)
    return s


def test_timesteps_match_numpy_and_are_symmetric(oracle):
    s = _rand_system(200, 1)
    ts = oracle.timesteps(s, 0.03)
    assert np.array_equal(ts, _np_timesteps(s, 0.03))
    # the pair timestep is exactly symmetric: a 2-body system gives equal timesteps
    two = {k: v[:2].copy() for k, v in s.items()}
    t2 = oracle.timesteps(two, 0.03)
    assert t2[0] == t2[1]


def test_kick_matches_numpy(oracle):
    s = _rand_system(300, 2)
    sink = {k: v.copy() for k, v in s.items()}
    acc = oracle.kick(sink, s, 0.25)
    for i in (0, 17, 299):
        dx, dy, dz = s["x"] - s["x"][i], s["y"] - s["y"][i], s["z"] - s["z"][i]
        d2 = dx * dx + dy * dy + dz * dz
        ok = d2 != 0
        inv = 1.0 / (d2[ok] * np.sqrt(d2[ok]))
        a = np.array([np.sum(dx[ok] * s["m"][ok] * inv), np.sum(dy[ok] * s["m"][ok] * inv),
                      np.sum(dz[ok] * s["m"][ok] * inv)])
        assert np.allclose(acc[:, i], a, rtol=1e-12, atol=0)
        # attractive: acceleration points towards the centre of mass on average
    assert np.allclose(sink["vx"], s["vx"] + acc[0] * 0.25, rtol=0, atol=0)


def test_softened_kick_matches_numpy_and_eps0_is_plain(oracle):
    s = _rand_system(200, 3)
    plain = {k: v.copy() for k, v in s.items()}
    zero = {k: v.copy() for k, v in s.items()}
    a0 = oracle.kick(plain, s, 0.1)
    lib = oracle.lib()
    ax, ay, az = np.zeros(200), np.zeros(200), np.zeros(200)
    d = oracle._d
    lib.oracle_kick(200, d(zero["x"]), d(zero["y"]), d(zero["z"]), d(zero["vx"]), d(zero["vy"]),
                    d(zero["vz"]), d(ax), d(ay), d(az), 200, d(s["x"]), d(s["y"]), d(s["z"]),
                    d(s["m"]), 0.1)
    assert np.array_equal(a0[0], ax) and np.array_equal(zero["vz"], plain["vz"])
    eps = 0.3
    soft = {k: v.copy() for k, v in s.items()}
    a = oracle.kick(soft, s, 0.1, eps=eps)
    for i in (0, 99, 199):
        dx, dy, dz = s["x"] - s["x"][i], s["y"] - s["y"][i], s["z"] - s["z"][i]
        d2 = dx * dx + dy * dy + dz * dz + eps * eps
        w = s["m"] / (d2 * np.sqrt(d2))
        assert np.allclose(a[:, i], [np.sum(dx * w), np.sum(dy * w), np.sum(dz * w)],
                           rtol=1e-12, atol=0)


def test_hold_step_conserves_energy_and_tracks_leaf_time(oracle, hhs):
    s = hhs.plummer(512, 11)
    e0, _ = oracle.energy(s)
    assert abs(e0 + 0.25) < 1e-12
    dt = 1.0 / 64
    for step in range(4):
        tr, nodes = oracle.hold_step(s, dt, True, 0.03, capacity=100000)
        assert abs(tr.leaf_time - dt) < 1e-15 * (step + 1) or tr.leaf_time > 0
        assert nodes[0, 0] == 0 and nodes[0, 1] == 512 and nodes[0, 3] == 1
        assert tr.max_level >= 2
    e1, _ = oracle.energy(s)
    assert abs((e1 - e0) / e0) < 1e-6
    assert sorted(s["id"].tolist()) == list(range(512))


def test_hold_step_leaf_dt_sum(oracle, hhs):
    # every root-to-leaf path covers dt exactly once per leaf visit: the leaf sum equals
    # dt summed over leaves, which for a tree of halving dts is a multiple of dt/2^L
    s = hhs.plummer(128, 5)
    tr, nodes = oracle.hold_step(s, 1.0 / 32, True, 0.03, capacity=100000)
    leaves = nodes[nodes[:, 2] == 0]
    assert tr.leaf_time == pytest.approx(np.sum((1.0 / 32) / 2.0 ** leaves[:, 0]), rel=1e-15)


def test_oracle_plummer_equals_product_generator_bit_for_bit(oracle, hhs):
    """The benchmark's CPU-baseline leg builds its inputs with the oracle's generator (so
    that process never maps the product library); both arms must integrate the same
    arrays."""
    for n, seed, mass in ((2, 1, 0), (1024, 2024, 0), (16384, 2024, 0), (4096, 5, 1),
                          (3000, 9, 2)):
        a, b = oracle.plummer(n, seed, mass), hhs.plummer(n, seed, mass)
        for k in ("x", "y", "z", "vx", "vy", "vz", "m", "ts", "id"):
            assert np.array_equal(a[k], b[k]), (n, seed, mass, k)
    with pytest.raises(ValueError):
        oracle.plummer(1, 3)
