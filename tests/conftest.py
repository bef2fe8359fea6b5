import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rel_err(a, b):
    """Normwise relative error max|a-b| / max|b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def seeded_field(shape, seed, kind="tg", lengths=(2 * np.pi,) * 3, noise=1e-3):
    """Taylor-Green field plus seeded Gaussian noise (Fortran-ordered)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x = np.arange(nx) * lengths[0] / nx
    y = np.arange(ny) * lengths[1] / ny
    z = np.arange(nz) * lengths[2] / nz
    X, Y, Z = np.meshgrid(2 * np.pi * x / lengths[0], 2 * np.pi * y / lengths[1],
                          2 * np.pi * z / lengths[2], indexing="ij")
    if kind == "tg":
        u = np.sin(X) * np.cos(Y) * np.cos(Z)
    else:
        u = rng.standard_normal(shape)
    u = u + noise * rng.standard_normal(shape)
    return np.asfortranarray(u)
