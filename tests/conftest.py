import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "parallel-hhs_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_GPU = os.path.join(ORACLE, "_ref", "libref_gpu_nofma.so")
REF_CPU = os.path.join(ORACLE, "_ref", "libref_cpu.so")
for p in (PKG, ORACLE, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def hhs():
    import hhs as m
    m.lib()
    return m


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.build()
    return o
