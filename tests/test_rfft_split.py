"""The half-length method the library's x transforms use for the Poisson
solve (k_rfft_x / k_irfft_x in x3div_b200/csrc/poisson.cu), restated in numpy
and checked against numpy's own real transforms on the CPU: a real line of n
= 2M points is the complex line z[m] = f[2m] + i f[2m+1]; with Z = DFT_M(z),
A = Z[k], B = conj(Z[M - k]) (indices mod M),
    F[k] = (A + B) / 2 - i e^{-2 pi i k / n} (A - B) / 2,   k = 0 .. M,
and back, from a Hermitian half spectrum G,
    Z[k] = (G[k] + conj(G[M - k])) + i e^{+2 pi i k / n} (G[k] - conj(G[M - k])),
k < M, whose unnormalised inverse DFT_M is f[2m] + i f[2m+1] for the
unnormalised c2r transform f of G.  The kernels compute the pairs (k, M - k)
together, one thread a pair; the pair loop below follows them."""
import numpy as np
import pytest

# every x length the library transforms itself: n / 2 = 2^p 3^q from 8 to 1024
LENGTHS = [16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048]


def split(z_hat, n):
    """F[0 .. M] from Z = DFT_M(z), pair by pair as k_rfft_x does."""
    m = n // 2
    wx = np.exp(-2j * np.pi * np.arange(m + 1) / n)
    out = np.empty(m + 1, dtype=complex)
    for p in range(m // 2 + 1):
        q = (m - p) % m
        zp, zq = z_hat[p], z_hat[q]
        e = 0.5 * (zp + np.conj(zq))
        d = 0.5 * (zp - np.conj(zq))
        out[p] = e - 1j * wx[p] * d
        if m - p != p:
            out[m - p] = np.conj(e) - 1j * wx[m - p] * (-np.conj(d))
    return out


def merge(g, n):
    """Z[0 .. M-1] from G[0 .. M], pair by pair as k_irfft_x does."""
    m = n // 2
    wx = np.exp(-2j * np.pi * np.arange(m + 1) / n)
    out = np.empty(m, dtype=complex)
    for p in range(m // 2 + 1):
        q = m - p
        e = g[p] + np.conj(g[q])
        d = g[p] - np.conj(g[q])
        out[p] = e + 1j * np.conj(wx[p]) * d
        if q != p and q < m:
            out[q] = np.conj(e) + 1j * np.conj(wx[q]) * (-np.conj(d))
    return out


@pytest.mark.parametrize("n", LENGTHS)
def test_split_is_the_real_transform(n):
    f = np.random.default_rng(n).standard_normal(n)
    z = f[0::2] + 1j * f[1::2]
    got = split(np.fft.fft(z), n)
    ref = np.fft.rfft(f)
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("n", LENGTHS)
def test_merge_is_the_unnormalised_c2r_transform(n):
    rng = np.random.default_rng(n + 1)
    g = np.fft.rfft(rng.standard_normal(n))  # a Hermitian half spectrum
    zi = np.fft.ifft(merge(g, n)) * (n // 2)  # unnormalised inverse DFT_M
    got = np.empty(n)
    got[0::2], got[1::2] = zi.real, zi.imag
    ref = np.fft.irfft(g, n) * n
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
