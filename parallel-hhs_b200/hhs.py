"""Python host binding of libhhs_b200.so (the C ABI declared in include/hhs.h).

Mirrors the reference's host-side operator interface (src/hold.cuh, src/timestep.cuh,
src/split.cuh, src/kick.cuh, src/drift.cuh, src/update_system.cuh): a device
ParticleSystem, a Context (the reference's nbodysystem_globals plus a per-level arena)
and the timesteps / split / kick_slow / kick_sf / drift / update_system / hold_step
entry points. Errors raise HHSError carrying the library status instead of exiting.

The CUDA library is required: importing this module fails loudly if it is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhhs_b200.so")

PREC_FP64 = 0
PREC_MIXED = 1
MASS_EQUAL, MASS_SALPETER, MASS_TWO_COMPONENT = 0, 1, 2

STATUS = {0: "HHS_OK", 1: "HHS_ERR_INVALID_ARG", 2: "HHS_ERR_CUDA", 3: "HHS_ERR_OOM",
          4: "HHS_ERR_TIMEOUT", 5: "HHS_ERR_DEVICE_FAULT_FLAG", 6: "HHS_ERR_DEPTH",
          7: "HHS_ERR_CAPACITY", 8: "HHS_ERR_PEER"}


class HHSError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)}")


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p


class Partition(ctypes.Structure):
    _fields_ = [("n_slow", ctypes.c_int32), ("n_fast", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [("eta", ctypes.c_double), ("eps", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_uint64), ("max_level", ctypes.c_int32),
                ("_pad", ctypes.c_int32), ("kick_pairs", ctypes.c_double),
                ("ts_pairs", ctypes.c_double)]


class Profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_uint64 * 8), ("ms", ctypes.c_double * 8),
                ("pairs", ctypes.c_double * 8)]


# kind 7: stages inside the cluster subtree solver, by slot (56 load, 57 timesteps, 58 split,
# 59 kick, 60 warp subtrees, 61 write-back) in the per-level table
PROFILE_KINDS = ("timesteps", "kick", "split", "update", "engine", "subtree", "cluster_node",
                 "subtree_stages")


class BatchTuning(ctypes.Structure):
    _fields_ = [("big_n", ctypes.c_int32), ("small_n", ctypes.c_int32),
                ("units_per_cta", ctypes.c_int32), ("mid_n", ctypes.c_int32),
                ("mid_dist_n", ctypes.c_int32), ("ms_per_step", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("small_n", ctypes.c_int32), ("units_per_cta", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("warp_n", ctypes.c_int32),
                ("cluster_size", ctypes.c_int32), ("mid_n", ctypes.c_int32),
                ("packed", ctypes.c_int32), ("mid_dist_n", ctypes.c_int32),
                ("overlap", ctypes.c_int32), ("ms_per_step", ctypes.c_double)]


class RunLog(ctypes.Structure):
    _fields_ = [("time", _dp), ("energy", _dp), ("capacity", ctypes.c_int32),
                ("n_entries", ctypes.c_int32)]


class CParticleSystem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32)] + \
        [(k, _dp) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "ts", "m")] + \
        [("id", _ip), ("parent_id", _ip), ("_base", _vp)]


# hhs_barrier_fn: int32_t (*)(void* user, void* stream)
BARRIER_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p)
# hhs_minmax_fn: int32_t (*)(void* user, uint64_t value, uint64_t* out_min, uint64_t* out_max)
MINMAX_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64,
                             ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64))

# every symbol of include/hhs.h, with its ctypes signature (restype, argtypes)
SIGNATURES = {
    "hhs_particle_system_alloc": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_int32]),
    "hhs_particle_system_free": (ctypes.c_int, [ctypes.POINTER(CParticleSystem)]),
    "hhs_particle_system_upload": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_int32]
                                   + [_dp] * 8 + [_ip, _vp]),
    "hhs_particle_system_download": (ctypes.c_int, [ctypes.POINTER(CParticleSystem),
                                                    ctypes.c_int32] + [_dp] * 8 + [_ip, _vp]),
    "hhs_particle_system_upload_aos": (ctypes.c_int, [ctypes.POINTER(CParticleSystem),
                                                      ctypes.c_int32] + [_dp] * 4 + [_ip, _vp]),
    "hhs_particle_system_download_aos": (ctypes.c_int, [ctypes.POINTER(CParticleSystem),
                                                        ctypes.c_int32] + [_dp] * 4 + [_ip, _vp]),
    "hhs_workspace_size": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    "hhs_ctx_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, Params,
                                      ctypes.POINTER(_vp)]),
    "hhs_ctx_destroy": (ctypes.c_int, [_vp]),
    "hhs_ctx_set_params": (ctypes.c_int, [_vp, Params]),
    "hhs_ctx_get_simtime": (ctypes.c_int, [_vp, _dp, _vp]),
    "hhs_ctx_flush_simtime": (ctypes.c_int, [_vp, _vp]),
    "hhs_ctx_check": (ctypes.c_int, [_vp, _vp]),
    "hhs_ctx_clear_errors": (ctypes.c_int, [_vp, _vp]),
    "hhs_timesteps": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_int32,
                                     ctypes.c_int, _vp]),
    "hhs_split": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem),
                                 ctypes.POINTER(CParticleSystem), ctypes.POINTER(CParticleSystem),
                                 _vp, _vp, ctypes.c_double, ctypes.c_int32, _vp, _vp]),
    "hhs_kick_slow": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int32, ctypes.c_int, _vp]),
    "hhs_kick_sf": (ctypes.c_int, [ctypes.POINTER(CParticleSystem),
                                   ctypes.POINTER(CParticleSystem), ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.c_int, _vp]),
    "hhs_drift": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int32, _vp]),
    "hhs_update_system": (ctypes.c_int, [ctypes.POINTER(CParticleSystem),
                                         ctypes.POINTER(CParticleSystem), ctypes.c_int32, _vp]),
    "hhs_hold_step": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.POINTER(CParticleSystem),
                                     ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int32, ctypes.c_int, _vp]),
    "hhs_hold_integrate": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_int32,
                                          ctypes.c_double, ctypes.c_int32, ctypes.c_int, _vp]),
    "hhs_hold_step_host": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_int32,
                                          ctypes.c_double, ctypes.c_int32, ctypes.c_int, _vp]),
    "hhs_dist_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int32, ctypes.c_int32,
                                       ctypes.POINTER(CParticleSystem), BARRIER_FN, _vp,
                                       ctypes.c_int64]),
    "hhs_dist_destroy": (ctypes.c_int, [_vp]),
    "hhs_dist_set_subtree_engine": (ctypes.c_int, [_vp, ctypes.c_int32]),
    "hhs_dist_set_agreement": (ctypes.c_int, [_vp, MINMAX_FN, _vp]),
    "hhs_dist_config_hash": (ctypes.c_int, [ctypes.POINTER(Tuning), ctypes.c_int32, ctypes.c_int,
                                            ctypes.c_int32, ctypes.c_double, Params,
                                            ctypes.POINTER(ctypes.c_uint64)]),
    "hhs_dist_check": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "hhs_dist_shard": (ctypes.c_int, [ctypes.c_int32] * 4 + [_ip, _ip]),
    "hhs_hold_step_dist": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(CParticleSystem),
                                          ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                          ctypes.c_int, _vp]),
    "hhs_ipc_handle": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), _vp]),
    "hhs_ipc_open": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.POINTER(CParticleSystem)]),
    "hhs_ipc_close": (ctypes.c_int, [ctypes.POINTER(CParticleSystem)]),
    "hhs_scan_workspace_size": (ctypes.c_size_t, [ctypes.c_int64]),
    "hhs_scan_exclusive_i32": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_size_t,
                                              _vp]),
    "hhs_split_cpu_order_workspace_size": (ctypes.c_size_t, [ctypes.c_int64]),
    "hhs_split_cpu_order": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_double, _vp, _vp, _vp,
                                           ctypes.c_size_t, _vp]),
    "hhs_scan_workspace_status": (ctypes.c_int, [_vp, _vp]),
    "hhs_scan_selftest_stalled_predecessor": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp,
                                                              ctypes.c_size_t, ctypes.c_uint32,
                                                              _vp]),
    "hhs_scan_selftest_wave_barrier": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp,
                                                       ctypes.c_size_t, ctypes.c_uint32, _vp]),
    "hhs_scan_exclusive_i32_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp]),
    "hhs_scan_noalloc_status": (ctypes.c_int, [_vp]),
    "hhs_ctx_set_trace": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp]),
    "hhs_ctx_autotune_results": (ctypes.c_int, [_vp, _vp, ctypes.c_int32,
                                                ctypes.POINTER(ctypes.c_int32)]),
    "hhs_batch_autotune": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_double,
                                          ctypes.c_int, ctypes.POINTER(BatchTuning), _vp,
                                          ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), _vp]),
    "hhs_engine_kick_accelerations": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
    "hhs_engine_timestep_rates": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
    "hhs_scan_noalloc_selftest_stalled_predecessor": (ctypes.c_int, [_vp, _vp, ctypes.c_int64,
                                                                     ctypes.c_uint32, _vp]),
    "hhs_compact_flags_i32": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64, _vp,
                                             ctypes.c_size_t, _vp]),
    "hhs_ic_plummer": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32]
                       + [_dp] * 7),
    "hhs_host_potential_energy": (ctypes.c_double, [ctypes.c_int32] + [_dp] * 4),
    "hhs_host_kinetic_energy": (ctypes.c_double, [ctypes.c_int32] + [_dp] * 4),
    "hhs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "hhs_ctx_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats), _vp]),
    "hhs_ctx_reset_stats": (ctypes.c_int, [_vp, _vp]),
    "hhs_ctx_set_profiling": (ctypes.c_int, [_vp, ctypes.c_int32]),
    "hhs_ctx_get_profile": (ctypes.c_int, [_vp, ctypes.POINTER(Profile)]),
    "hhs_ctx_get_level_profile": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_uint64)]),
    "hhs_kernel_launch_count": (ctypes.c_uint64, []),
    "hhs_measure_fma_peaks": (ctypes.c_int, [_dp, _dp, _vp]),
    "hhs_measure_fma2_peak": (ctypes.c_int, [_dp, _vp]),
    "hhs_batch_create": (ctypes.c_int, [ctypes.c_int32, _ip, ctypes.c_int32, Params,
                                        ctypes.POINTER(_vp)]),
    "hhs_batch_destroy": (ctypes.c_int, [_vp]),
    "hhs_batch_set_tuning": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "hhs_hold_batched": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_double,
                                        ctypes.c_int32, ctypes.c_int, _vp]),
    "hhs_batch_get_simtime": (ctypes.c_int, [_vp, _dp, _vp]),
    "hhs_batch_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats), _vp]),
    "hhs_batch_reset_stats": (ctypes.c_int, [_vp, _vp]),
    "hhs_batch_check": (ctypes.c_int, [_vp, _vp]),
    "hhs_batch_set_mid": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "hhs_batch_partition": (ctypes.c_int, [ctypes.c_int32, _ip, ctypes.c_int32, _ip, _dp]),
    "hhs_energy": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_int32, ctypes.c_double,
                                  _dp, _dp, _vp]),
    "hhs_snapshot_write": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_int32,
                                          ctypes.c_double, ctypes.POINTER(Params), ctypes.c_double,
                                          ctypes.c_int32, ctypes.c_char_p, _vp]),
    "hhs_snapshot_read": (ctypes.c_int, [ctypes.POINTER(CParticleSystem), ctypes.c_char_p, _ip,
                                         _dp, _ip, _vp]),
    "hhs_hold": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_int32,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                ctypes.c_int32, ctypes.c_char_p, ctypes.POINTER(RunLog), _vp]),
    "hhs_ctx_set_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(Tuning)]),
    "hhs_ctx_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(Tuning)]),
    "hhs_ctx_get_launch": (ctypes.c_int, [_vp, _ip, _ip]),
    "hhs_ctx_autotune": (ctypes.c_int, [_vp, ctypes.POINTER(CParticleSystem), ctypes.c_int32,
                                        ctypes.c_double, ctypes.c_int, ctypes.POINTER(Tuning),
                                        _vp]),
}

_lib = None


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status, what):
    if status != 0:
        raise HHSError(status, what)


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _i(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m", "ts")


def plummer(n, seed, mass_spectrum=MASS_EQUAL):
    """Seeded Plummer sphere in Henon units (host arrays, dict of float64)."""
    s = {k: np.empty(n) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    _check(lib().hhs_ic_plummer(n, seed, mass_spectrum,
                                *[_d(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")]),
           "hhs_ic_plummer")
    s["ts"] = np.zeros(n)
    s["id"] = np.arange(n, dtype=np.int32)
    return s


def energy_host(s):
    n = len(s["x"])
    k = lib().hhs_host_kinetic_energy(n, _d(s["vx"]), _d(s["vy"]), _d(s["vz"]), _d(s["m"]))
    p = lib().hhs_host_potential_energy(n, _d(s["x"]), _d(s["y"]), _d(s["z"]), _d(s["m"]))
    return k + p


class ParticleSystem:
    """particle_system<double> on the device (src/particle_system.cuh:20-54), SoA."""

    def __init__(self, n):
        self.c = CParticleSystem()
        _check(lib().hhs_particle_system_alloc(ctypes.byref(self.c), n), "alloc")
        self.n = n

    @property
    def ref(self):
        return ctypes.byref(self.c)

    def upload(self, s, n=None, stream=None):
        n = len(s["x"]) if n is None else n
        _check(lib().hhs_particle_system_upload(self.ref, n, *[_d(s.get(k)) for k in FIELDS],
                                                _i(s.get("id")), stream), "upload")

    def download(self, n=None, stream=None, fields=FIELDS + ("id",)):
        n = self.n if n is None else n
        out = {k: np.empty(n) for k in FIELDS if k in fields}
        if "id" in fields:
            out["id"] = np.empty(n, dtype=np.int32)
        _check(lib().hhs_particle_system_download(self.ref, n, *[_d(out.get(k)) for k in FIELDS],
                                                  _i(out.get("id")), stream), "download")
        return out

    def free(self):
        if self.c._base:
            _check(lib().hhs_particle_system_free(self.ref), "free")

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """nbodysystem_globals<double> plus the per-level arena (src/particle_system.cuh:65-104)."""

    def __init__(self, n_max, max_levels=64, eta=0.03, eps=0.0):
        self.h = _vp()
        _check(lib().hhs_ctx_create(n_max, max_levels, Params(eta, eps), ctypes.byref(self.h)),
               "hhs_ctx_create")

    def check(self, stream=None):
        _check(lib().hhs_ctx_check(self.h, stream), "hhs_ctx_check")

    def simtime(self, stream=None):
        t = ctypes.c_double(0)
        _check(lib().hhs_ctx_get_simtime(self.h, ctypes.byref(t), stream), "simtime")
        return t.value

    def flush_simtime(self, stream=None):
        _check(lib().hhs_ctx_flush_simtime(self.h, stream), "flush_simtime")

    def stats(self, stream=None):
        st = Stats()
        _check(lib().hhs_ctx_get_stats(self.h, ctypes.byref(st), stream), "stats")
        return {"nodes": st.nodes, "max_level": st.max_level, "kick_pairs": st.kick_pairs,
                "ts_pairs": st.ts_pairs}

    def reset_stats(self, stream=None):
        _check(lib().hhs_ctx_reset_stats(self.h, stream), "reset_stats")

    def set_trace(self, nodes_ptr, capacity, count_ptr):
        """Records every node of hhs_hold_step into device buffers (4 int32 per node and a
        uint64 count); set_trace(None, 0, None) switches it off."""
        _check(lib().hhs_ctx_set_trace(self.h, nodes_ptr, capacity, count_ptr), "set_trace")

    def set_tuning(self, small_n=None, units_per_cta=None, ctas_per_sm=None, warp_n=None,
                   cluster_size=None, mid_n=None, packed=None, mid_dist_n=None, overlap=None):
        t = Tuning()
        _check(lib().hhs_ctx_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        if small_n is not None:
            t.small_n = small_n
        if units_per_cta is not None:
            t.units_per_cta = units_per_cta
        if ctas_per_sm is not None:
            t.ctas_per_sm = ctas_per_sm
        if warp_n is not None:
            t.warp_n = warp_n
        if cluster_size is not None:
            t.cluster_size = cluster_size
        if mid_n is not None:
            t.mid_n = mid_n
        if packed is not None:
            t.packed = int(packed)
        if mid_dist_n is not None:
            t.mid_dist_n = mid_dist_n
        if overlap is not None:
            t.overlap = int(overlap)
        _check(lib().hhs_ctx_set_tuning(self.h, ctypes.byref(t)), "set_tuning")

    def tuning(self):
        t = Tuning()
        _check(lib().hhs_ctx_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        return {"small_n": t.small_n, "units_per_cta": t.units_per_cta,
                "ctas_per_sm": t.ctas_per_sm, "warp_n": t.warp_n,
                "cluster_size": t.cluster_size, "mid_n": t.mid_n, "packed": t.packed,
                "mid_dist_n": t.mid_dist_n, "overlap": t.overlap}

    def launch(self):
        """(grid CTAs for FP64, grid CTAs for mixed, dynamic shared memory bytes per CTA)."""
        g = np.zeros(2, dtype=np.int32)
        sm = ctypes.c_int32()
        _check(lib().hhs_ctx_get_launch(self.h, _i(g), ctypes.byref(sm)), "get_launch")
        return int(g[0]), int(g[1]), sm.value

    def autotune(self, sys, n, dt, prec=1, stream=None):
        t = Tuning()
        _check(lib().hhs_ctx_autotune(self.h, sys.ref, n, dt, prec, ctypes.byref(t), stream),
               "autotune")
        return {"small_n": t.small_n, "units_per_cta": t.units_per_cta,
                "ctas_per_sm": t.ctas_per_sm, "warp_n": t.warp_n,
                "cluster_size": t.cluster_size, "mid_n": t.mid_n, "packed": t.packed,
                "mid_dist_n": t.mid_dist_n, "overlap": t.overlap, "ms_per_step": t.ms_per_step}

    def autotune_results(self):
        """Every candidate the last autotune timed, as tuning dicts with ms_per_step."""
        cnt = ctypes.c_int32()
        _check(lib().hhs_ctx_autotune_results(self.h, None, 0, ctypes.byref(cnt)), "results")
        arr = (Tuning * max(1, cnt.value))()
        _check(lib().hhs_ctx_autotune_results(self.h, arr, cnt.value, ctypes.byref(cnt)),
               "results")
        return [{k: getattr(t, k) for k, _ in Tuning._fields_} for t in arr[:cnt.value]]

    def set_profiling(self, on):
        _check(lib().hhs_ctx_set_profiling(self.h, int(on)), "set_profiling")

    def profile(self):
        p = Profile()
        _check(lib().hhs_ctx_get_profile(self.h, ctypes.byref(p)), "profile")
        return {PROFILE_KINDS[k]: {"launches": p.launches[k], "ms": p.ms[k], "pairs": p.pairs[k]}
                for k in range(8) if p.launches[k]}

    def level_profile(self):
        ms = np.zeros(8 * 64)
        cnt = np.zeros(8 * 64, dtype=np.uint64)
        _check(lib().hhs_ctx_get_level_profile(self.h, _d(ms),
                                               cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))),
               "level_profile")
        return ms.reshape(8, 64), cnt.reshape(8, 64)

    def destroy(self):
        if self.h:
            _check(lib().hhs_ctx_destroy(self.h), "hhs_ctx_destroy")
            self.h = _vp()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def batch_partition(sizes, n_ranks):
    """Rank of each independent system, balancing the per-rank sum of N^2
    (hhs_batch_partition); returns (rank_of, load)."""
    sz = np.ascontiguousarray(sizes, dtype=np.int32)
    rank_of = np.zeros(len(sz), dtype=np.int32)
    load = np.zeros(n_ranks)
    _check(lib().hhs_batch_partition(len(sz), _i(sz), n_ranks, _i(rank_of), _d(load)),
           "hhs_batch_partition")
    return rank_of, load


def batch_shard(sizes, n_ranks, rank):
    """Indices (ascending) of the systems this rank integrates."""
    rank_of, _ = batch_partition(sizes, n_ranks)
    return np.nonzero(rank_of == rank)[0]


class Batch:
    """Many independent systems in one particle system (hhs_batch)."""

    def __init__(self, offsets, max_levels=64, eta=0.03, eps=0.0):
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        self.n_sys = len(off) - 1
        self.offsets = off
        self.h = _vp()
        _check(lib().hhs_batch_create(self.n_sys, _i(off), max_levels, Params(eta, eps),
                                      ctypes.byref(self.h)), "hhs_batch_create")

    def set_tuning(self, big_n=1024, small_n=64, units_per_cta=8):
        _check(lib().hhs_batch_set_tuning(self.h, big_n, small_n, units_per_cta), "batch tuning")

    def set_mid(self, mid_n=640, mid_dist_n=96):
        _check(lib().hhs_batch_set_mid(self.h, mid_n, mid_dist_n), "batch set_mid")

    def step(self, sys, dt, calc_timestep=True, prec=PREC_MIXED, stream=None):
        _check(lib().hhs_hold_batched(self.h, sys.ref, dt, int(calc_timestep), prec, stream),
               "hhs_hold_batched")

    def autotune(self, sys, dt, prec=PREC_MIXED, stream=None):
        """hhs_batch_autotune: (best tuning dict, [every candidate timed])."""
        best = BatchTuning()
        table = (BatchTuning * 64)()
        cnt = ctypes.c_int32()
        _check(lib().hhs_batch_autotune(self.h, sys.ref, dt, prec, ctypes.byref(best), table, 64,
                                        ctypes.byref(cnt), stream), "hhs_batch_autotune")
        as_dict = lambda t: {k: getattr(t, k) for k, _ in BatchTuning._fields_}
        return as_dict(best), [as_dict(t) for t in table[:cnt.value]]

    def check(self, stream=None):
        _check(lib().hhs_batch_check(self.h, stream), "hhs_batch_check")

    def simtime(self, stream=None):
        out = np.zeros(self.n_sys)
        _check(lib().hhs_batch_get_simtime(self.h, _d(out), stream), "batch simtime")
        return out

    def stats(self, stream=None):
        st = Stats()
        _check(lib().hhs_batch_get_stats(self.h, ctypes.byref(st), stream), "batch stats")
        return {"nodes": st.nodes, "max_level": st.max_level, "kick_pairs": st.kick_pairs,
                "ts_pairs": st.ts_pairs}

    def reset_stats(self, stream=None):
        _check(lib().hhs_batch_reset_stats(self.h, stream), "batch reset_stats")

    def destroy(self):
        if self.h:
            _check(lib().hhs_batch_destroy(self.h), "hhs_batch_destroy")
            self.h = _vp()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def timesteps(ctx, sys, n, prec=PREC_FP64, stream=None):
    _check(lib().hhs_timesteps(ctx.h, sys.ref, n, prec, stream), "hhs_timesteps")


def split(ctx, total, slow, fast, pivot, n, part_ptr, pred_ptr=None, scan_ptr=None, stream=None):
    _check(lib().hhs_split(ctx.h, total.ref, slow.ref, fast.ref, pred_ptr, scan_ptr, pivot, n,
                           part_ptr, stream), "hhs_split")


def kick_slow(sys, dt, fac, n, prec=PREC_FP64, stream=None):
    _check(lib().hhs_kick_slow(sys.ref, dt, fac, n, prec, stream), "hhs_kick_slow")


def kick_sf(so_sys, si_sys, dt, fac, n_sink, m_src, prec=PREC_FP64, stream=None):
    _check(lib().hhs_kick_sf(so_sys.ref, si_sys.ref, dt, fac, n_sink, m_src, prec, stream),
           "hhs_kick_sf")


def drift(sys, dt, fac, n, stream=None):
    _check(lib().hhs_drift(sys.ref, dt, fac, n, stream), "hhs_drift")


def update_system(prev, cur, n, stream=None):
    _check(lib().hhs_update_system(prev.ref, cur.ref, n, stream), "hhs_update_system")


def hold_step(ctx, sys, n, stime, dt, calc_timestep=True, prec=PREC_MIXED, clevel=0,
              stream=None):
    """hold_step<double,BS>(clevel, globals, sys, N, stime, stime+dt, dt, calc_timestep)."""
    _check(lib().hhs_hold_step(ctx.h, clevel, sys.ref, n, stime, stime + dt, dt,
                               int(calc_timestep), prec, stream), "hhs_hold_step")


def hold_integrate(ctx, sys, n, dt, steps, prec=PREC_MIXED, stream=None):
    """`steps` top-level steps as one replayed CUDA graph (hhs_hold_integrate)."""
    _check(lib().hhs_hold_integrate(ctx.h, sys.ref, n, dt, steps, prec, stream),
           "hhs_hold_integrate")


def energy(sys, n, eps=0.0, stream=None):
    """FP64 (kinetic, potential) of the first n particles, computed on the device."""
    k, p = ctypes.c_double(), ctypes.c_double()
    _check(lib().hhs_energy(sys.ref, n, eps, ctypes.byref(k), ctypes.byref(p), stream),
           "hhs_energy")
    return k.value, p.value


def snapshot_write(sys, n, time, path, eta=0.03, eps=0.0, dt=0.0, step=0, stream=None):
    prm = Params(eta, eps)
    _check(lib().hhs_snapshot_write(sys.ref, n, time, ctypes.byref(prm), dt, step,
                                    path.encode(), stream), "hhs_snapshot_write")


def snapshot_read(sys, path, stream=None):
    n, t, st = ctypes.c_int32(), ctypes.c_double(), ctypes.c_int32()
    _check(lib().hhs_snapshot_read(sys.ref, path.encode(), ctypes.byref(n), ctypes.byref(t),
                                   ctypes.byref(st), stream), "hhs_snapshot_read")
    return n.value, t.value, st.value


def hold(ctx, sys, n, stime, etime, dt, prec=PREC_MIXED, snapshot_every=0, prefix=None,
         max_log=1024, stream=None):
    """hold(): integrate stime..etime; returns [(time, energy)] diagnostics."""
    t = np.zeros(max_log)
    e = np.zeros(max_log)
    log = RunLog(_d(t), _d(e), max_log, 0)
    _check(lib().hhs_hold(ctx.h, sys.ref, n, stime, etime, dt, prec, snapshot_every,
                          prefix.encode() if prefix else None, ctypes.byref(log), stream),
           "hhs_hold")
    return list(zip(t[:log.n_entries].tolist(), e[:log.n_entries].tolist()))


def hold_step_host(ctx, sys, n, dt, calc_timestep=True, prec=PREC_FP64, stream=None):
    _check(lib().hhs_hold_step_host(ctx.h, sys.ref, n, dt, int(calc_timestep), prec, stream),
           "hhs_hold_step_host")


def launch_count():
    return lib().hhs_kernel_launch_count()


def measure_fma_peaks(stream=None):
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(lib().hhs_measure_fma_peaks(ctypes.byref(a), ctypes.byref(b), stream), "fma_peaks")
    return a.value, b.value


def measure_fma2_peak(stream=None):
    a = ctypes.c_double()
    _check(lib().hhs_measure_fma2_peak(ctypes.byref(a), stream), "fma2_peak")
    return a.value


def scan_workspace_size(n):
    return lib().hhs_scan_workspace_size(n)


def scan_exclusive_i32(d_in, d_out, n, d_ws, ws_bytes, stream=None):
    _check(lib().hhs_scan_exclusive_i32(d_in, d_out, n, d_ws, ws_bytes, stream),
           "hhs_scan_exclusive_i32")


def compact_flags_i32(d_flags, d_scan, d_idx, d_count, n, d_ws, ws_bytes, stream=None):
    _check(lib().hhs_compact_flags_i32(d_flags, d_scan, d_idx, d_count, n, d_ws, ws_bytes,
                                       stream), "hhs_compact_flags_i32")


def scan_selftest_stalled_predecessor(d_in, d_out, n, d_ws, ws_bytes, max_polls, stream=None):
    """Status of a scan whose first tile never publishes (HHS_ERR_TIMEOUT expected)."""
    return lib().hhs_scan_selftest_stalled_predecessor(d_in, d_out, n, d_ws, ws_bytes,
                                                       max_polls, stream)


def scan_selftest_wave_barrier(d_in, d_out, n, d_ws, ws_bytes, timeout_us, stream=None):
    """Makes every grid barrier of the wave-form scan wait for a CTA that does not exist;
    returns the status (HHS_ERR_TIMEOUT = 4 when the bounded waits gave up)."""
    return lib().hhs_scan_selftest_wave_barrier(d_in, d_out, n, d_ws, ws_bytes, timeout_us,
                                                stream)


def split_cpu_order(d_ts, n, pivot, d_order, d_counts, d_ws, ws_bytes, stream=None):
    _check(lib().hhs_split_cpu_order(d_ts, n, pivot, d_order, d_counts, d_ws, ws_bytes, stream),
           "hhs_split_cpu_order")


def split_cpu_order_workspace_size(n):
    return lib().hhs_split_cpu_order_workspace_size(n)


def scan_workspace_status(d_ws, stream=None):
    return lib().hhs_scan_workspace_status(d_ws, stream)


# ---------------------------------------------------------------- one system, several GPUs
IPC_HANDLE_BYTES = 64


def dist_shard(n_fast, n_slow, rank, world):
    """Sink range [lo, hi) of `rank` for a launch whose first n_fast sinks cost n_slow pair
    terms and whose other n_slow sinks cost n_slow + n_fast (hhs_dist_shard)."""
    lo, hi = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().hhs_dist_shard(n_fast, n_slow, rank, world, ctypes.byref(lo), ctypes.byref(hi)),
           "hhs_dist_shard")
    return lo.value, hi.value


def ipc_handle(sys):
    """64-byte CUDA IPC handle of a ParticleSystem's device allocation."""
    buf = ctypes.create_string_buffer(IPC_HANDLE_BYTES)
    _check(lib().hhs_ipc_handle(sys.ref, buf), "hhs_ipc_handle")
    return buf.raw


class PeerView:
    """Another process's system of capacity n mapped into this one (hhs_ipc_open)."""

    def __init__(self, handle, n):
        self.c = CParticleSystem()
        buf = ctypes.create_string_buffer(bytes(handle), IPC_HANDLE_BYTES)
        _check(lib().hhs_ipc_open(buf, n, ctypes.byref(self.c)), "hhs_ipc_open")
        self.n = n

    def close(self):
        if self.c._base:
            _check(lib().hhs_ipc_close(ctypes.byref(self.c)), "hhs_ipc_close")


class Dist:
    """hhs_dist: this rank's side of one system replicated on `world` GPUs.

    replicas[r] is rank r's system as this process addresses it (a ParticleSystem in the
    same process, a PeerView of another process, or a CParticleSystem); replicas[rank] is
    not used. barrier(stream) returns True once every rank's work enqueued on its stream
    before the call is complete before any later work (False: a peer failed or did not
    arrive). Launches of at least min_pairs pair terms are split across the ranks; with
    subtree_engine, subtrees below that run as one engine launch on every rank."""

    def __init__(self, rank, world, replicas, barrier, min_pairs=1 << 24, subtree_engine=True):
        arr = (CParticleSystem * world)()
        for r, p in enumerate(replicas):
            if r != rank and p is not None:
                arr[r] = p if isinstance(p, CParticleSystem) else p.c
        self.barrier = barrier
        self.failure = None

        def _cb(_user, stream):
            try:
                return 0 if barrier(stream) else 1
            except Exception as e:  # a callback must not raise into the library
                self.failure = e
                return 1
        self._cb = BARRIER_FN(_cb)
        self.h = _vp()
        _check(lib().hhs_dist_create(ctypes.byref(self.h), rank, world, arr, self._cb, None,
                                     int(min_pairs)), "hhs_dist_create")
        _check(lib().hhs_dist_set_subtree_engine(self.h, int(bool(subtree_engine))),
               "hhs_dist_set_subtree_engine")
        self.rank, self.world = rank, world
        self._agree = None

    def set_agreement(self, minmax):
        """minmax(value) -> (min, max) of an unsigned 64-bit value over all ranks; with it
        every step first checks that all ranks run the same configuration."""
        def _cb(_user, value, out_min, out_max):
            try:
                lo, hi = minmax(int(value))
                out_min[0], out_max[0] = lo, hi
                return 0
            except Exception as e:
                self.failure = e
                return 1
        self._agree = MINMAX_FN(_cb)
        _check(lib().hhs_dist_set_agreement(self.h, self._agree, None), "hhs_dist_set_agreement")

    def check(self, config_hash):
        """hhs_dist_check: the status code (0 when every rank passed the same hash)."""
        return lib().hhs_dist_check(self.h, ctypes.c_uint64(config_hash))

    def step(self, ctx, sys, n, dt, calc_timestep=True, prec=PREC_MIXED, stream=None):
        """One top-level HOLD step of this rank's replica (hhs_hold_step_dist)."""
        _check(lib().hhs_hold_step_dist(ctx.h, self.h, sys.ref, n, dt, int(bool(calc_timestep)),
                                        prec, stream), "hhs_hold_step_dist")

    def destroy(self):
        if self.h:
            lib().hhs_dist_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def config_hash(tuning, grid_ctas, prec, n, dt, eta, eps=0.0):
    """hhs_dist_config_hash of a tuning dict (as Context.tuning() returns)."""
    t = Tuning()
    for k, v in tuning.items():
        if hasattr(t, k):
            setattr(t, k, v)
    out = ctypes.c_uint64()
    _check(lib().hhs_dist_config_hash(ctypes.byref(t), grid_ctas, prec, n, dt, Params(eta, eps),
                                      ctypes.byref(out)), "hhs_dist_config_hash")
    return out.value


def group_minmax(group=None):
    """A minmax callback over a torch.distributed group (two all-reduces of the value's
    two 32-bit halves, packed so min/max order is the 64-bit order)."""
    def minmax(value):
        import torch
        import torch.distributed as tdist
        dev = "cuda" if tdist.get_backend(group) == "nccl" else "cpu"
        out = []
        for op in (tdist.ReduceOp.MIN, tdist.ReduceOp.MAX):
            # int64 holds values below 2^63; shift the unsigned range into it
            t = torch.tensor([value - (1 << 63)], dtype=torch.int64, device=dev)
            tdist.all_reduce(t, op=op, group=group)
            out.append(int(t.item()) + (1 << 63))
        return out[0], out[1]
    return minmax


class PeerBarrier:
    """The barrier of a Dist over a torch.distributed process group.

    NCCL group: a one-element all-reduce enqueued on the library's stream, so the host
    does not wait; a rank that is gone ends that collective when the group's timeout
    runs out. Other backends (gloo): synchronise the stream, then a monitored barrier,
    which reports the rank that did not arrive within `timeout` seconds."""

    def __init__(self, group=None, timeout=30.0):
        import torch
        import torch.distributed as tdist
        self.group, self.timeout = group, timeout
        self.nccl = tdist.get_backend(group) == "nccl"
        self.token = torch.zeros(1, dtype=torch.int32, device="cuda") if self.nccl else None
        self.failure = None

    def __call__(self, stream):
        import datetime
        import torch
        import torch.distributed as tdist
        try:
            if self.nccl:
                st = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
                with torch.cuda.stream(st):
                    tdist.all_reduce(self.token, group=self.group)
            else:
                if torch.cuda.is_available():
                    if stream:
                        torch.cuda.ExternalStream(stream).synchronize()
                    else:
                        torch.cuda.synchronize()
                tdist.monitored_barrier(group=self.group,
                                        timeout=datetime.timedelta(seconds=self.timeout))
            return True
        except Exception as e:
            self.failure = e
            return False


class DistHold:
    """One system integrated on every rank of a torch.distributed group, one GPU each.

    Every rank uploads the same initial state into its own ParticleSystem; the handles
    of all ranks' systems are exchanged over the group and mapped with CUDA IPC, and each
    step() is hhs_hold_step_dist on this rank's replica: the O(n^2) timestep and kick
    launches of at least min_pairs pair terms are split by sink and their kernels write
    every result into all replicas over NVLink. The replicas stay bit-identical to
    each other and to hhs_hold_step_host on one GPU."""

    def __init__(self, ctx, sys, group=None, min_pairs=1 << 24, timeout=30.0, barrier=None,
                 subtree_engine=True):
        import torch.distributed as tdist
        self.rank = tdist.get_rank(group)
        self.world = tdist.get_world_size(group)
        handles = [None] * self.world
        tdist.all_gather_object(handles, (ipc_handle(sys), sys.n), group=group)
        self.views = {}
        replicas = []
        for r, (h, n) in enumerate(handles):
            if r == self.rank:
                replicas.append(None)
                continue
            self.views[r] = PeerView(h, n)
            replicas.append(self.views[r])
        self.barrier = barrier if barrier is not None else PeerBarrier(group, timeout)
        self.dist = Dist(self.rank, self.world, replicas, self.barrier, min_pairs,
                         subtree_engine)
        self.dist.set_agreement(group_minmax(group))
        self.ctx, self.sys = ctx, sys

    def step(self, n, dt, calc_timestep=True, prec=PREC_MIXED, stream=None):
        self.dist.step(self.ctx, self.sys, n, dt, calc_timestep, prec, stream)

    def close(self):
        """Unmaps the peers. Call on every rank after the last step (whose closing
        barrier has ordered every peer store)."""
        self.dist.destroy()
        for v in self.views.values():
            v.close()
        self.views = {}
