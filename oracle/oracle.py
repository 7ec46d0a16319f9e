"""ctypes loader for the CPU FP64 oracle (hhs_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Only the tests, the smoke
check and the benchmark's CPU-baseline leg import this module. See hhs_oracle.h for
the reference lines each function restates.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_hhs.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class Node(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int32), ("n", ctypes.c_int32),
                ("n_fast", ctypes.c_int32), ("calc_ts", ctypes.c_int32)]


class Trace(ctypes.Structure):
    _fields_ = [("nodes", ctypes.POINTER(Node)), ("capacity", ctypes.c_int64),
                ("count", ctypes.c_int64), ("max_level", ctypes.c_int32),
                ("leaf_time", ctypes.c_double), ("kick_pairs", ctypes.c_double),
                ("ts_pairs", ctypes.c_double)]


def build(force=False):
    """Compile the oracle with gcc (no fused multiply-add, OpenMP)."""
    src = os.path.join(HERE, "hhs_oracle.c")
    if not force and os.path.exists(LIB_PATH) and \
            os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
                           "-fPIC", "-shared", "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_timesteps.argtypes = [ctypes.c_int] + [_dp] * 7 + [ctypes.c_double, _dp]
        L.oracle_scan_exclusive_i32.argtypes = [ctypes.c_int64, _ip, _ip]
        L.oracle_split.argtypes = [ctypes.c_int, _dp, ctypes.c_double, _ip]
        L.oracle_split.restype = ctypes.c_int
        L.oracle_split_cpu_order.argtypes = [ctypes.c_int, _dp, ctypes.c_double, _ip]
        L.oracle_split_cpu_order.restype = ctypes.c_int
        L.oracle_kick.argtypes = [ctypes.c_int] + [_dp] * 9 + [ctypes.c_int] + [_dp] * 4 + \
            [ctypes.c_double]
        L.oracle_kick_soft.argtypes = [ctypes.c_int] + [_dp] * 9 + [ctypes.c_int] + \
            [_dp] * 4 + [ctypes.c_double, ctypes.c_double]
        L.oracle_hold_step_soft.argtypes = [ctypes.c_int] + [_dp] * 8 + [
            _ip, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
            ctypes.POINTER(Trace)]
        L.oracle_drift.argtypes = [ctypes.c_int] + [_dp] * 6 + [ctypes.c_double]
        L.oracle_hold_step.argtypes = [ctypes.c_int] + [_dp] * 8 + [_ip, ctypes.c_double,
                                                                     ctypes.c_int, ctypes.c_double,
                                                                     ctypes.POINTER(Trace)]
        L.oracle_energy.argtypes = [ctypes.c_int] + [_dp] * 7 + [_dp]
        L.oracle_threads.restype = ctypes.c_int
        L.oracle_plummer.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int] + [_dp] * 7
        L.oracle_plummer.restype = ctypes.c_int
        _lib = L
    return _lib


def _d(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _i(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def timesteps(s, eta):
    ts = np.empty_like(s["x"])
    lib().oracle_timesteps(len(ts), _d(s["x"]), _d(s["y"]), _d(s["z"]), _d(s["vx"]),
                           _d(s["vy"]), _d(s["vz"]), _d(s["m"]), eta, _d(ts))
    return ts


def scan_exclusive(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    out = np.empty_like(a)
    lib().oracle_scan_exclusive_i32(len(a), _i(a), _i(out))
    return out


def split(ts, pivot):
    """Returns (order, n_fast): order[:n_fast] fast, order[n_fast:] slow (parent indices)."""
    ts = np.ascontiguousarray(ts, dtype=np.float64)
    order = np.empty(len(ts), dtype=np.int32)
    nf = lib().oracle_split(len(ts), _d(ts), pivot, _i(order))
    return order, nf


def split_cpu_order(ts, pivot):
    """Permutation of cpu_split (fast first, unstable order) and n_fast."""
    ts = np.ascontiguousarray(ts, dtype=np.float64)
    order = np.empty(len(ts), dtype=np.int32)
    nf = lib().oracle_split_cpu_order(len(ts), _d(ts), pivot, _i(order))
    return order, nf


def kick(sink, src, dtfac, eps=0.0):
    """Updates sink['vx'..'vz'] in place; returns acc (3, n_sink)."""
    n = len(sink["x"])
    acc = np.zeros((3, n))
    ax, ay, az = acc[0], acc[1], acc[2]
    lib().oracle_kick_soft(n, _d(sink["x"]), _d(sink["y"]), _d(sink["z"]), _d(sink["vx"]),
                           _d(sink["vy"]), _d(sink["vz"]), _d(ax), _d(ay), _d(az),
                           len(src["x"]), _d(src["x"]), _d(src["y"]), _d(src["z"]),
                           _d(src["m"]), dtfac, eps * eps)
    return acc


def drift(s, dtfac):
    lib().oracle_drift(len(s["x"]), _d(s["x"]), _d(s["y"]), _d(s["z"]), _d(s["vx"]),
                       _d(s["vy"]), _d(s["vz"]), dtfac)


def hold_step(s, dt, calc_ts, eta, capacity=0, eps=0.0):
    """One recursive HOLD step in place on dict-of-arrays s. Returns (trace, nodes)."""
    nodes = (Node * capacity)() if capacity > 0 else None
    tr = Trace(nodes if nodes is not None else None, capacity, 0, 0, 0.0, 0.0, 0.0)
    lib().oracle_hold_step_soft(len(s["x"]), _d(s["x"]), _d(s["y"]), _d(s["z"]),
                                _d(s["vx"]), _d(s["vy"]), _d(s["vz"]), _d(s["m"]),
                                _d(s["ts"]), _i(s["id"]), dt, int(calc_ts), eta, eps * eps,
                                ctypes.byref(tr))
    out = None
    if nodes is not None:
        k = min(tr.count, capacity)
        out = np.array([(nodes[i].level, nodes[i].n, nodes[i].n_fast, nodes[i].calc_ts)
                        for i in range(k)], dtype=np.int32).reshape(-1, 4)
    return tr, out


def energy(s):
    out = np.zeros(2)
    lib().oracle_energy(len(s["x"]), _d(s["x"]), _d(s["y"]), _d(s["z"]), _d(s["vx"]),
                        _d(s["vy"]), _d(s["vz"]), _d(s["m"]), _d(out))
    return out[0] + out[1], out


def plummer(n, seed, mass_spectrum=0):
    """Seeded Plummer sphere in Henon units (dict of float64 arrays plus ts and id), the
    same arrays as the product generator gives for the same seed."""
    s = {k: np.empty(n) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    rc = lib().oracle_plummer(n, seed, mass_spectrum,
                              *[_d(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")])
    if rc != 0:
        raise ValueError(f"oracle_plummer: bad arguments (n={n}, mass={mass_spectrum})")
    s["ts"] = np.zeros(n)
    s["id"] = np.arange(n, dtype=np.int32)
    return s


def threads():
    return lib().oracle_threads()
