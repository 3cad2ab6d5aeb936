"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
CPU.  The native libraries are built in-tree before the session (a no-op when
they are up to date)."""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import flite3d_b200.build as b
    b.build_prepro()
    b.build_oracle()
    try:
        b.build_gpu()
    except Exception as e:  # nvcc may be absent on a CPU-only host
        print("GPU library not rebuilt:", e)
    yield


def oracle_backend():
    from flite3d_b200.solver import Backend
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    return Backend(lib, "oracle_")


@pytest.fixture(scope="session")
def oracle():
    return oracle_backend()


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from flite3d_b200.solver import Backend
    from flite3d_b200 import _abi
    return Backend(_abi.gpu_lib(), "flite_")
