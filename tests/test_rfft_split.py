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


# --- the split fused into the last Stockham stage (k_rfft_x) and the merge
# into the first inverse stage (k_irfft_x), for lengths whose last radix R is
# 2, 3 or 4: one thread takes butterflies a = i and b = M/R - i (a = 0 with b =
# M/(2R)), whose outputs hold each other's partners M - k.

def radix_seq(n, reverse=False):
    r, m = [], n
    while m % 8 == 0 and m > 1:
        r.append(8)
        m //= 8
    for f in (4, 2):
        while m % f == 0:
            r.append(f)
            m //= f
    while m % 3 == 0:
        r.append(3)
        m //= 3
    return r[::-1] if reverse else r


def stockham_stage(x, r, ns, inverse):
    """One Stockham stage of radix r over sub-transforms of ns, as zft_stage."""
    n, s = len(x), (1 if inverse else -1)
    y = np.empty_like(x)
    for j in range(n // r):
        jm = j % ns
        v = np.array([x[j + q * (n // r)] * np.exp(s * 2j * np.pi * q * jm / (ns * r)) for q in range(r)])
        out = np.fft.ifft(v) * r if inverse else np.fft.fft(v)
        for q in range(r):
            y[(j // ns) * ns * r + jm + q * ns] = out[q]
    return y


def paired_items(nsl):
    return [(i, nsl - i if i else nsl // 2) for i in range(nsl // 2)]


PAIRED = [n for n in LENGTHS if radix_seq(n // 2)[-1] <= 4 and (n // 2 // radix_seq(n // 2)[-1]) % 2 == 0]


@pytest.mark.parametrize("n", PAIRED)
def test_paired_last_stage_is_the_real_transform(n):
    m = n // 2
    seq = radix_seq(m)
    r, nsl = seq[-1], m // seq[-1]
    f = np.random.default_rng(n + 2).standard_normal(n)
    x, ns = f[0::2] + 1j * f[1::2], 1
    for rr in seq[:-1]:
        x = stockham_stage(x, rr, ns, False)
        ns *= rr
    wx = np.exp(-2j * np.pi * np.arange(m + 1) / n)
    out = np.full(m + 1, np.nan, dtype=complex)

    def butterfly(j):
        return np.fft.fft([x[j + q * nsl] * np.exp(-2j * np.pi * q * j / m) for q in range(r)])

    for i, (a, b) in enumerate(paired_items(nsl)):
        ya, yb = butterfly(a), butterfly(b)
        for q in range(r):
            pa = yb[r - 1 - q] if i else ya[(r - q) % r]
            pb = ya[r - 1 - q] if i else yb[r - 1 - q]
            for j, y, p in ((a, ya, pa), (b, yb, pb)):
                k = j + q * nsl
                out[k] = 0.5 * (y[q] + np.conj(p)) - 0.5j * wx[k] * (y[q] - np.conj(p))
        if i == 0:
            out[m] = 0.5 * (ya[0] + np.conj(ya[0])) - 0.5j * wx[m] * (ya[0] - np.conj(ya[0]))
    ref = np.fft.rfft(f)
    assert np.abs(out - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("n", PAIRED)
def test_paired_first_inverse_stage_is_the_c2r_transform(n):
    m = n // 2
    seq = radix_seq(m, reverse=True)
    r, nsl = seq[0], m // seq[0]
    g = np.fft.rfft(np.random.default_rng(n + 3).standard_normal(n))
    wx = np.exp(-2j * np.pi * np.arange(m + 1) / n)
    x = np.full(m, np.nan, dtype=complex)

    def merge(k, kp):
        return (g[k] + np.conj(g[kp])) + 1j * np.conj(wx[k]) * (g[k] - np.conj(g[kp]))

    for i, (a, b) in enumerate(paired_items(nsl)):
        for j in (a, b):
            z = []
            for q in range(r):
                k = j + q * nsl
                if j == 0:
                    kp = m if q == 0 else ((r - q) % r) * nsl
                else:
                    kp = (nsl - j) + (r - 1 - q) * nsl
                assert k + kp == m or (k + kp) % m == 0
                z.append(merge(k, kp))
            out = np.fft.ifft(z) * r  # sub-transforms of size 1: no twiddles
            x[j * r: j * r + r] = out
    ns = r
    for rr in seq[1:]:
        x = stockham_stage(x, rr, ns, True)
        ns *= rr
    got = np.empty(n)
    got[0::2], got[1::2] = x.real, x.imag
    ref = np.fft.irfft(g, n) * n
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
