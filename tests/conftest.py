"""Shared pytest configuration.

Markers: ``gpu`` -- needs a CUDA device (B200, sm_100a); everything else runs
on the CPU.  The CPU oracle (``oracle/``) and the engine libraries are built
on demand when missing (``make``; nvcc cross-compiles without a GPU).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


GPU = _gpu_available()


def pytest_collection_modifyitems(config, items):
    if GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def mpb():
    import mpc_cuda_b200 as M

    if not (os.path.exists(M.LIB_PATH) and os.path.exists(M.HOST_LIB_PATH)):
        M.build()
    return M


def to_dev(arr: np.ndarray):
    import torch

    a = np.ascontiguousarray(arr, dtype=np.uint8).reshape(-1)
    if a.size % 16:
        a = np.concatenate([a, np.zeros(16 - a.size % 16, np.uint8)])
    return torch.from_numpy(a.copy()).cuda()


def to_host(t) -> np.ndarray:
    return t.cpu().numpy()
