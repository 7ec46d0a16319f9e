"""CPU tests of the C ABI library: it loads, exports every symbol include/hhs.h declares,
and its host-only parts work without a GPU."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "hhs.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hhs_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(hhs):
    lib = hhs.lib()
    names = _declared_symbols()
    assert len(names) >= 29
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding declares a signature for each of them
    assert set(names) <= set(hhs.SIGNATURES)


def test_status_strings(hhs):
    for code, name in hhs.STATUS.items():
        assert hhs.lib().hhs_status_string(code).decode() == name


def test_invalid_arguments_return_status_without_device(hhs):
    L = hhs.lib()
    sys_ = hhs.CParticleSystem()
    assert L.hhs_particle_system_alloc(ctypes.byref(sys_), 0) == 1
    h = ctypes.c_void_p()
    assert L.hhs_ctx_create(0, 64, hhs.Params(0.03, 0.0), ctypes.byref(h)) == 1
    assert L.hhs_ctx_create(16, 64, hhs.Params(-1.0, 0.0), ctypes.byref(h)) == 1
    assert L.hhs_scan_exclusive_i32(None, None, 0, None, 0, None) == 0
    assert L.hhs_scan_exclusive_i32(None, None, -1, None, 0, None) == 1
    assert L.hhs_hold_step(None, 0, None, 16, 0.0, 1.0, 1.0, 1, 1, None) == 1
    assert L.hhs_workspace_size(0, 4) == 0
    assert L.hhs_workspace_size(1024, 64) > 2 * 64 * 1024 * 4
    assert L.hhs_scan_workspace_size(1 << 20) >= 256 + 8 * ((1 << 20) // 2048)


def test_plummer_ic_deterministic_henon_units(hhs):
    a = hhs.plummer(2048, 42)
    b = hhs.plummer(2048, 42)
    c = hhs.plummer(2048, 43)
    for k in ("x", "vx", "m"):
        assert np.array_equal(a[k], b[k])
    assert not np.array_equal(a["x"], c["x"])
    assert abs(hhs.energy_host(a) + 0.25) < 1e-13
    assert abs(np.sum(a["m"]) - 1.0) < 1e-14
    com = [np.sum(a["m"] * a[k]) for k in ("x", "y", "z", "vx", "vy", "vz")]
    assert np.max(np.abs(com)) < 1e-14
    r = np.sqrt(a["x"] ** 2 + a["y"] ** 2 + a["z"] ** 2)
    # Plummer half-mass radius in Henon units is ~0.77 (a = 3*pi/16, r_h = 1.305 a)
    assert 0.6 < np.median(r) < 0.95


def test_mass_spectra(hhs):
    s = hhs.plummer(20000, 1, hhs.MASS_SALPETER)
    m = s["m"] / s["m"].min()
    assert abs(np.sum(s["m"]) - 1.0) < 1e-12
    assert m.max() / m.min() > 100  # spans most of [0.1, 100]
    t = hhs.plummer(20000, 2, hhs.MASS_TWO_COMPONENT)
    u = np.unique(np.round(t["m"] / t["m"].min(), 9))
    assert u.tolist() == [1.0, 10.0]
    frac = np.mean(t["m"] > t["m"].min() * 5)
    assert 0.09 < frac < 0.11
    assert abs(hhs.energy_host(t) + 0.25) < 1e-12
