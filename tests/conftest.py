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


def band_limited_field(n, seed, kmax_frac=0.25, slope=-5.0 / 3.0):
    """Periodic n^3 field of Fourier modes 0 < |k| <= kmax_frac * n with
    amplitude |k|**slope and seeded random phases, scaled to max|u| = 1
    (Fortran-ordered, FP64)."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n, 1.0 / n)
    kr = np.fft.rfftfreq(n, 1.0 / n)
    K = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2)
    amp = np.zeros_like(K)
    band = (K > 0) & (K <= kmax_frac * n)
    amp[band] = K[band] ** slope
    spec = amp * np.exp(2j * np.pi * rng.random(K.shape))
    u = np.fft.irfftn(spec, s=(n, n, n), axes=(0, 1, 2))
    u /= np.abs(u).max()
    return np.asfortranarray(u)
