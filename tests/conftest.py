import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("marl-ochre_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device and the built libmarl_cuda.so")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def marl():
    import marl_cuda

    marl_cuda.load()
    return marl_cuda


def deterministic_field(dims) -> np.ndarray:
    """init_deterministic_field (crates/marl-field/src/field.rs:257-268)."""
    X, Y, Z = dims
    z, y, x, s = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), np.arange(12), indexing="ij")
    return (((x * 13 + y * 17 + z * 19 + s * 23) % 541).astype(np.float32) * np.float32(0.001)).astype(np.float32)


def wave_field(dims) -> np.ndarray:
    """init_field of crates/marl-gpu/tests/gpu_diffusion.rs:7-23."""
    X, Y, Z = dims
    z, y, x, s = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), np.arange(12), indexing="ij")
    wave = ((x * 17 + y * 31 + z * 43 + s * 59) % 997).astype(np.float32) / np.float32(997.0)
    boost = np.where((s == 7) & (x > X // 3) & (x < X // 3 + 16), np.float32(2.0), np.float32(0.0))
    return (wave * (s.astype(np.float32) + np.float32(1.0)) * np.float32(0.02) + boost).astype(np.float32)


def occupancy_patterns(dims) -> dict:
    """The four occupancy patterns of crates/marl-gpu/tests/gpu_diffusion.rs:25-54."""
    X, Y, Z = dims
    empty = np.zeros((Z, Y, X), np.uint8)
    center = empty.copy()
    center[Z // 2, Y // 2, X // 2] = 1
    boundary = empty.copy()
    boundary[1, Y // 2, X // 2] = 1
    cluster = empty.copy()
    cluster[Z // 2 - 1:Z // 2 + 2, Y // 2 - 1:Y // 2 + 2, X // 2 - 1:X // 2 + 2] = 1
    return {"empty": empty, "center": center, "boundary_adjacent": boundary, "dense_cluster": cluster}
