"""The allocation-free scan entry point (hhs_scan_exclusive_i32_noalloc).

Some callers of this library must not allocate device memory: an application that has
given the device to its own memory pool, or a step loop held to a fixed device-memory
budget. They cannot pass the workspace that hhs_scan_exclusive_i32 takes, so this entry
point runs the same scan with its workspace in a fixed array inside the library's device
memory. These tests call it through the C ABI and compare it with the allocating entry
point on two calls in a row; integer results must be identical. This file is collected
last so that a failure here does not stop the rest of the suite from running first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1 << 26  # HHS_SCAN_NOALLOC_MAX_N in include/hhs.h


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _reference_scan(hhs, torch, dev, n, stream):
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    ws_bytes = hhs.scan_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    hhs.scan_exclusive_i32(_ptr(dev), _ptr(out), n, _ptr(ws), ws_bytes, stream)
    return out


def test_noalloc_scan_matches_allocating_scan_twice(cuda, hhs):
    torch = cuda
    lib = hhs.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row on the shared workspace: a larger input, then a smaller one, so
    # the second call must not see anything the first one left behind
    for n, seed in ((3_000_017, 1), (70_001, 2)):
        a = np.random.default_rng(seed).integers(-50, 50, n).astype(np.int32)
        dev = torch.from_numpy(a).cuda()
        out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        assert lib.hhs_scan_exclusive_i32_noalloc(_ptr(dev), _ptr(out), n, stream) == 0
        ref = _reference_scan(hhs, torch, dev, n, stream)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        expect = np.concatenate([[0], np.cumsum(a, dtype=np.int64)[:-1]]).astype(np.int32)
        assert np.array_equal(out.cpu().numpy(), expect)


def test_noalloc_scan_limits(cuda, hhs):
    torch = cuda
    lib = hhs.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    # beyond the stated maximum: rejected before any launch
    assert lib.hhs_scan_exclusive_i32_noalloc(_ptr(dummy), _ptr(dummy), MAX_N + 1, stream) == 7
    assert lib.hhs_scan_exclusive_i32_noalloc(None, None, 5, stream) == 1
    assert lib.hhs_scan_exclusive_i32_noalloc(None, None, 0, stream) == 0
    # exactly at the maximum, on Bernoulli flags, checked by its properties
    g = torch.Generator(device="cuda").manual_seed(26)
    flags = (torch.rand(MAX_N, device="cuda", generator=g) < 0.5).to(torch.int32)
    out = torch.empty_like(flags)
    assert lib.hhs_scan_exclusive_i32_noalloc(_ptr(flags), _ptr(out), MAX_N, stream) == 0
    torch.cuda.synchronize()
    assert int(out[0]) == 0
    assert torch.equal(out[1:] - out[:-1], flags[:-1])
    assert int(out[-1]) + int(flags[-1]) == int(flags.sum())


def test_noalloc_scan_reports_a_lookback_timeout(cuda, hhs):
    """The allocation-free scan's bounded look-back waits record a timeout in its fixed
    array; hhs_scan_noalloc_status reads it back. A run with its first tile left out makes
    every wait run out (no GPU fault: each wait gives up and its CTA returns); the status
    is HHS_ERR_TIMEOUT, and the next ordinary call clears it and scans correctly."""
    torch = cuda
    lib = hhs.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 50_000
    a = np.random.default_rng(5).integers(0, 2, n).astype(np.int32)
    dev = torch.from_numpy(a).cuda()
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    assert lib.hhs_scan_noalloc_selftest_stalled_predecessor(_ptr(dev), _ptr(out), n, 2000,
                                                             stream) == 4
    assert lib.hhs_scan_noalloc_status(stream) == 4
    assert lib.hhs_scan_exclusive_i32_noalloc(_ptr(dev), _ptr(out), n, stream) == 0
    assert lib.hhs_scan_noalloc_status(stream) == 0
    expect = np.concatenate([[0], np.cumsum(a)[:-1]]).astype(np.int32)
    assert np.array_equal(out.cpu().numpy(), expect)
