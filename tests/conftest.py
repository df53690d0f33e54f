"""Shared fixtures.  `-m gpu` tests need a CUDA device and the built library;
everything else runs on the CPU (oracle, host logic, ABI symbol checks)."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgpulsm.so")
    config.addinivalue_line("markers", "slow: full-size configuration")


def package():
    return importlib.import_module("gpu-lsm-tree_b200")


@pytest.fixture(scope="session")
def gl():
    return package()


@pytest.fixture(scope="session")
def workloads():
    return importlib.import_module("gpu-lsm-tree_b200.workloads")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def to_dev(a, device="cuda:0"):
    """numpy u32/u64 array -> torch CUDA tensor with the same bit pattern."""
    import torch

    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        t = torch.from_numpy(a.view(np.int32))
    elif a.dtype == np.uint64:
        t = torch.from_numpy(a.view(np.int64))
    elif a.dtype == np.uint8:
        t = torch.from_numpy(a)
    else:
        raise TypeError(a.dtype)
    return t.to(device)


def to_host(t, dtype=np.uint32):
    a = t.detach().cpu().numpy()
    return a.view(dtype)


def empty_u32(n, device="cuda:0"):
    import torch

    return torch.empty(max(n, 1), dtype=torch.int32, device=device)
