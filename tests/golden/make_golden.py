"""Generates tests/golden/*.json (committed fixtures; this script is how they were made).

scan_reference_tests.json -- the inputs of the reference's own split/scan tests
  (tests/test_scan.cu:23-28, tests/test_scan_multi_block.cu:27-32,192-217,
  tests/test_scan_unrolled.cu:30-34,192-215): glibc rand() from its default seed, one
  fresh process per test program, total[i] = 10.0f * ((float)rand()/(float)RAND_MAX),
  pivot 5.0f, predicate total <= pivot. For every case it records the count of
  predicate-true elements as computed by the reference's CPU split (src/cpu_scan.h,
  compiled by oracle/build_oracle.py into oracle/_ref) and by the oracle, plus SHA-256
  digests of the oracle's exact exclusive scan and stable partition order (int32 LE).

Run from the repository root after oracle/build_oracle.py:  python tests/golden/make_golden.py
"""
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

PROGRAMS = {
    "test_scan.cu": [1024],
    "test_scan_multi_block.cu": [512, 512, 1023, 2048, 2151, 524288, 588021, 1048576, 2097152],
    "test_scan_unrolled.cu": [512, 4090, 2048, 2151, 524288, 588021, 1048576, 2097152],
}


def reference_test_inputs(sizes):
    """Yields the float32 arrays a reference test program draws, in order."""
    libc = ctypes.CDLL("libc.so.6")
    libc.rand.restype = ctypes.c_int
    libc.srand(1)  # the glibc default state of a fresh process
    rand_max = np.float32(2147483647)
    for n in sizes:
        raw = np.fromiter((libc.rand() for _ in range(n)), dtype=np.int64, count=n)
        r = raw.astype(np.float32) / rand_max
        yield (np.float32(10.0) * r).astype(np.float32)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i4").tobytes()).hexdigest()


def main():
    import oracle
    ref_cpu = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so"))
    ref_cpu.ref_cpu_split_f32.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                          ctypes.c_float, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]
    cases = []
    for prog, sizes in PROGRAMS.items():
        for idx, total in enumerate(reference_test_inputs(sizes)):
            n = len(total)
            pred = (total <= np.float32(5.0)).astype(np.int32)
            scan = oracle.scan_exclusive(pred)
            order, nf = oracle.split(total.astype(np.float64), 5.0)
            work = total.copy()
            ns_ref, nf_ref = ctypes.c_int(), ctypes.c_int()
            ref_cpu.ref_cpu_split_f32(work.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n,
                                      5.0, ctypes.byref(ns_ref), ctypes.byref(nf_ref))
            count = int(pred.sum())
            assert nf_ref.value == count, (prog, n, nf_ref.value, count)
            assert nf == (0 if count == 1 else count)
            cases.append({"program": prog, "case": idx, "n": n, "pivot": 5.0,
                          "count_le_pivot": count, "ref_cpu_split_n_fast": nf_ref.value,
                          "ref_cpu_split_n_slow": ns_ref.value,
                          "sha256_exclusive_scan": digest(scan),
                          "sha256_stable_order": digest(order),
                          "first8_scan": scan[:8].tolist(), "last_scan": int(scan[-1])})
            print(prog, idx, n, count)
    with open(os.path.join(HERE, "scan_reference_tests.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
