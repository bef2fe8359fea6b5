"""Pins of the CPU oracle against the reference's own known answers (no GPU).

The reference ships no golden vectors and cannot be compiled here (Fortran +
MPI + 2decomp&FFT; no gfortran).  Its own known-answer formulas are:
  * the modified wavenumber of the staggered derivative and the transfer
    function of the interpolation, src/poisson.f90:522-533 and :631-650;
  * the analytic derivatives of the vel field, src/mom.f90:88-113 etc.
Every periodic compact operator is circulant, so a Fourier mode must come out
scaled by exactly those factors (to round-off).  The first derivative is
pinned by its own transfer function (Lele's 6th-order scheme the reference
implements), and the second derivative -- absent from the reference -- by
its analytic transfer function only.
"""
import numpy as np
import pytest

from conftest import rel_err

X, Y, Z = 0, 1, 2
KINDS = ["der", "der2", "dervp", "derpv", "intvp", "intpv"]


def transfer(kind, w, c):
    """Fourier factor of each operator for a mode of phase w = k*d, written
    with the reference's scalars (c = oracle.lhs output)."""
    al, a, b, cc, dd = c["alfa"], c["a"], c["b"], c["c"], c["d"]
    den = 1.0 + 2.0 * al * np.cos(w)
    if kind == "der":
        return (2 * a * np.sin(w) + 2 * b * np.sin(2 * w)) / den
    if kind == "der2":
        return (2 * a * (np.cos(w) - 1) + 2 * b * (np.cos(2 * w) - 1)) / den
    if kind in ("dervp", "derpv"):
        # waves(): wp = acix6*2*dx*sin(w/2) + bcix6*2*dx*sin(1.5w), / (1 + 2 alcaix6 cos w); xkx = wp/dx
        return (2 * a * np.sin(w / 2) + 2 * b * np.sin(1.5 * w)) / den
    # waves() :640-648: (2 aicix6 cos(w/2) + 2 (bicix6 cos 1.5w + cicix6 cos 2.5w + dicix6 cos 3.5w)) / (1 + 2 ailcaix6 cos w)
    return (2 * a * np.cos(w / 2) + 2 * (b * np.cos(1.5 * w) + cc * np.cos(2.5 * w) + dd * np.cos(3.5 * w))) / den


def mode_case(kind, n, m, L):
    """Input and expected output along one line for mode m."""
    d = L / n
    k = 2 * np.pi * m / L
    i = np.arange(n)
    xv = i * d            # velocity grid
    xp = (i + 0.5) * d    # pressure grid (staggered by half a cell)
    src_x = xp if kind in ("derpv", "intpv") else xv
    dst_x = xp if kind in ("dervp", "intvp") else xv
    u = np.sin(k * src_x)
    return u, dst_x, k * d, k


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("direction", [X, Y, Z])
@pytest.mark.parametrize("n", [8, 9, 16, 17, 64])
def test_fourier_modes(oracle, kind, direction, n):
    L = 2 * np.pi if n != 17 else 1.0
    c = oracle.lhs(kind, n, L / n)
    modes = sorted({1, 2, max(1, n // 4), max(1, n // 2 - 1)})
    other = [5, 4]
    for m in modes:
        u1, dst_x, w, k = mode_case(kind, n, m, L)
        T = transfer(kind, w, c)
        if kind in ("der", "dervp", "derpv"):
            expect1 = T * np.cos(k * dst_x)
        else:
            expect1 = T * np.sin(k * dst_x)
        # embed the line in a 3-D field, varying along the other axes too
        shape = [other[0], other[1]]
        shape.insert(direction, n)
        g = 1.0 + 0.25 * np.arange(other[0] * other[1]).reshape(other)
        u = np.moveaxis(u1[:, None, None] * g[None], 0, direction)
        exp = np.moveaxis(expect1[:, None, None] * g[None], 0, direction)
        out = oracle.apply(kind, direction, np.asfortranarray(u), L / n)
        assert rel_err(out, exp) < 1e-12, (kind, direction, n, m)


def circulant(n, taps):
    A = np.zeros((n, n))
    for off, v in taps.items():
        for i in range(n):
            A[i, (i + off) % n] += v
    return A


STENCIL_TAPS = {
    "der": lambda c: {1: c["a"], -1: -c["a"], 2: c["b"], -2: -c["b"]},
    "der2": lambda c: {1: c["a"], 0: -2 * c["a"] - 2 * c["b"], -1: c["a"], 2: c["b"], -2: c["b"]},
    "dervp": lambda c: {1: c["a"], 0: -c["a"], 2: c["b"], -1: -c["b"]},
    "derpv": lambda c: {0: c["a"], -1: -c["a"], 1: c["b"], -2: -c["b"]},
    "intvp": lambda c: {1: c["a"], 0: c["a"], 2: c["b"], -1: c["b"], 3: c["c"], -2: c["c"], 4: c["d"], -3: c["d"]},
    "intpv": lambda c: {0: c["a"], -1: c["a"], 1: c["b"], -2: c["b"], 2: c["c"], -3: c["c"], 3: c["d"], -4: c["d"]},
}


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [8, 13, 32])
def test_dense_cyclic_solve(oracle, kind, n):
    """The Thomas + Sherman-Morrison pipeline (prepare, thomas1d periodic
    vector, ?thomas_0) solves exactly the cyclic tridiagonal system with unit
    diagonal and alfa off-diagonals and corners."""
    d = 0.37
    c = oracle.lhs(kind, n, d)
    A = circulant(n, {0: 1.0, 1: c["alfa"], -1: c["alfa"]})
    S = circulant(n, STENCIL_TAPS[kind](c))
    rng = np.random.default_rng(7 + n)
    u = np.asfortranarray(rng.standard_normal((n, 3, 2)))
    out = oracle.apply(kind, X, u, d)
    ref = np.linalg.solve(A, S @ u.reshape(n, -1)).reshape(u.shape)
    assert rel_err(out, ref) < 1e-12


@pytest.mark.parametrize("which", [0, 1, 2])
def test_reference_test_mode_rms(oracle, which):
    """test_du/dv/dw (src/mom.f90) on the reference vel field: the RMS error
    printed by the reference equals |k' - k| * rms(ccc) exactly."""
    n = 32
    u, v, w = oracle.vel(n, n, n)
    d = 1.0 / n
    field = (u, v, w)[which]
    out = oracle.apply("der", which, field, d)
    rms = oracle.test_rms(which, out)
    c = oracle.lhs("der", n, d)
    k = 2 * np.pi
    kp = transfer("der", k * d, c)
    amp = 2.0 if which == 2 else 1.0
    predicted = amp * abs(kp - k) / np.sqrt(8.0)
    assert rms > 0
    assert abs(rms - predicted) / predicted < 1e-6


def test_poisson_projection_removes_divergence(oracle):
    """divergence -> poisson_000 -> gradp -> cor_vel leaves a field whose
    staggered divergence is round-off (the modified wavenumbers of waves()
    match the staggered operators exactly)."""
    from conftest import seeded_field
    n = (16, 12, 20)
    L = (2 * np.pi, 1.5, 3.0)
    u = seeded_field(n, 1, lengths=L, noise=1e-2)
    v = seeded_field(n, 2, kind="rand", lengths=L, noise=0)
    w = seeded_field(n, 3, kind="rand", lengths=L, noise=0)
    dx, dy, dz = (l / m for l, m in zip(L, n))
    div0 = oracle.divergence(u, v, w, dx, dy, dz)
    p = oracle.poisson(div0, *L)
    px, py, pz = oracle.gradp(p, dx, dy, dz)
    oracle.cor_vel(u, v, w, px, py, pz)
    div1 = oracle.divergence(u, v, w, dx, dy, dz)
    assert np.abs(div1).max() < 1e-12 * np.abs(div0).max()


def test_poisson_against_dense_spectral(oracle):
    """poisson_000's per-mode algebra (phase shifts that cancel, division by
    -K) equals -fft(rhs)/K with K from the 1-D tables."""
    from conftest import seeded_field
    nx, ny, nz = 12, 10, 8
    L = (1.0, 2.0, 3.0)
    rhs = seeded_field((nx, ny, nz), 5, kind="rand", lengths=L, noise=0)
    out = oracle.poisson(rhs, *L)
    t = oracle.poisson_tables(nx, ny, nz, *L)
    K = (t["k2x"][:, None, None] * (t["ty"][None, :, None] * t["tz"][None, None, :]) ** 2
         + t["k2y"][None, :, None] * (t["tx"][:, None, None] * t["tz"][None, None, :]) ** 2
         + t["k2z"][None, None, :] * (t["tx"][:, None, None] * t["ty"][None, :, None]) ** 2)
    R = np.fft.fftn(rhs)
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(K < 1e-16, 0.0, -R / K)
    ref = np.real(np.fft.ifftn(P))
    assert rel_err(out, ref) < 1e-12


def test_euler_step_runs_and_projects(oracle):
    from conftest import seeded_field
    n = (16, 16, 16)
    u = seeded_field(n, 11)
    v = seeded_field(n, 12)
    w = seeded_field(n, 13)
    du, div_before, p = oracle.euler_step(u, v, w, 1e-3, lengths=(2 * np.pi,) * 3)
    d = 2 * np.pi / 16
    div_after = oracle.divergence(u, v, w, d, d, d)
    assert np.isfinite(u).all()
    assert np.abs(div_after).max() < 1e-11 * max(np.abs(div_before).max(), 1e-30)


# ---- non-periodic first derivatives (der?_ij) --------------------------------

def _line_field(values, direction, other=(3, 2)):
    """A Fortran-ordered field whose lines along direction all carry values."""
    n = len(values)
    shape = list(other)
    shape.insert(direction, n)
    view = [1, 1, 1]
    view[direction] = n
    return np.asfortranarray(np.broadcast_to(np.asarray(values).reshape(view), shape))


def _first_line(f, direction):
    sl = [0, 0, 0]
    sl[direction] = slice(None)
    return f[tuple(sl)]


@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("npaire", [0, 1])
def test_der_np_dirichlet_exact_on_cubics(oracle, direction, npaire):
    """Dirichlet ends (ncl = 2) use third-order one-sided compact closures
    (first_deriv_exp_, src/x3d_operator_1d.f90:375-390) and the interior is
    sixth order, so a cubic's derivative is exact to round-off everywhere."""
    n = 40
    h = 1.0 / (n - 1)
    x = np.arange(n) * h
    u = _line_field(x ** 3 - 0.5 * x ** 2 + 0.3 * x, direction)
    d = oracle.der_np(direction, u, h, 2, 2, npaire)
    assert np.abs(d - _line_field(3 * x ** 2 - x + 0.3, direction)).max() < 1e-12


@pytest.mark.parametrize("npaire", [0, 1])
def test_der_np_free_slip_mirrored_modes(oracle, npaire):
    """Free-slip ends (ncl = 1) mirror the field: even (npaire = 1, cos) or
    odd (npaire = 0, sin) about each wall; the derivative of such a mode
    keeps the interior scheme's sixth-order accuracy up to the walls."""
    errs = []
    for n in (33, 65):
        h = 1.0 / (n - 1)
        x = np.arange(n) * h
        f, df = ((np.cos(np.pi * x), -np.pi * np.sin(np.pi * x)) if npaire == 1
                 else (np.sin(np.pi * x), np.pi * np.cos(np.pi * x)))
        d = oracle.der_np(0, _line_field(f, 0), h, 1, 1, npaire)
        errs.append(np.abs(_first_line(d, 0) - df).max() / np.pi)
    assert errs[1] < 1e-10
    assert np.log2(errs[0] / errs[1]) > 5.5  # sixth order


@pytest.mark.parametrize("ncl", [(1, 2), (2, 1)])
@pytest.mark.parametrize("npaire", [0, 1])
def test_der_np_mixed_ends_converge(oracle, ncl, npaire):
    """A free-slip end and a Dirichlet end: a quarter-wave mirrored at the
    free-slip wall, small error at n = 64 and at least third-order
    convergence (the one-sided closure's order)."""
    errs = []
    for n in (33, 64):
        h = 1.0 / (n - 1)
        x = np.arange(n) * h
        y = x if ncl[0] == 1 else 1 - x  # distance from the free-slip wall
        s = 1.0 if ncl[0] == 1 else -1.0  # d/dx of y
        if npaire == 1:
            f, df = np.cos(np.pi * y / 2), -s * np.pi / 2 * np.sin(np.pi * y / 2)
        else:
            f, df = np.sin(np.pi * y / 2), s * np.pi / 2 * np.cos(np.pi * y / 2)
        d = oracle.der_np(0, _line_field(f, 0), h, ncl[0], ncl[1], npaire)
        errs.append(np.abs(_first_line(d, 0) - df).max())
    assert errs[1] < (2e-7 if npaire == 1 else 1e-5)
    assert np.log2(errs[0] / errs[1]) / np.log2(63 / 32) > 2.8


def test_der_np_factors_solve_the_matrix(oracle):
    """The LU factors of first_deriv_imp_ reproduce the banded matrix of the
    rows it assembles (checked through a dense solve of random right-hand
    sides for each boundary pair and parity)."""
    n = 17
    rng = np.random.default_rng(3)
    for ncl in [(1, 1), (1, 2), (2, 1), (2, 2)]:
        for npaire in (0, 1):
            op = oracle.lhs_np(n, 0.1, ncl[0], ncl[1], npaire)
            f, s, w = op["f"], op["s"], op["w"]
            # rebuild M from the factors: M = Lo * Up, Lo(i,i-1) = s_i, Up(i,i) = 1/w_i, Up(i,i+1) = f_i
            Lo = np.eye(n) + np.diag(s[1:], -1)
            Up = np.diag(1.0 / w) + np.diag(f[:-1], 1)
            M = Lo @ Up
            al = 1.0 / 3.0
            assert np.allclose(np.diag(M)[2:n - 2], 1.0) and np.allclose(np.diag(M, 1)[2:n - 3], al)
            r = rng.standard_normal(n)
            t = r.copy()
            for i in range(1, n):
                t[i] -= t[i - 1] * s[i]
            t[-1] *= w[-1]
            for i in range(n - 2, -1, -1):
                t[i] = (t[i] - f[i] * t[i + 1]) * w[i]
            assert np.allclose(M @ t, r, atol=1e-12)


# ---- non-periodic staggered branches (src/x3d_staggered.f90, nclx = .false.) ----

def _stag_errors(oracle, kind, npaire, fun, dfun, n, L=2.0):
    """Max error of the oracle's kind along x on an n-point velocity grid
    (walls at 0 and L, nm = n - 1 pressure points at the cell centres)."""
    d = L / (n - 1)
    xv = np.arange(n) * d
    xp = (np.arange(n - 1) + 0.5) * d
    vp = kind in ("dervp", "intvp")
    src = fun(xv if vp else xp)
    exact = (dfun if kind.startswith("der") else fun)(xp if vp else xv)
    u = np.asfortranarray(np.broadcast_to(src[:, None, None], (src.size, 9, 8)))
    out = oracle.stag_np(kind, 0, u, d, 2, 1, npaire)
    return np.abs(out[:, 4, 3] - exact)


EVEN = (lambda x: np.cos(np.pi * x / 2.0) + 0.3 * np.cos(3 * np.pi * x / 2.0),
        lambda x: -np.pi / 2.0 * np.sin(np.pi * x / 2.0) - 0.45 * np.pi * np.sin(3 * np.pi * x / 2.0))
ODD = (lambda x: np.sin(np.pi * x / 2.0) + 0.2 * np.sin(np.pi * x) + 0.5,
       lambda x: np.pi / 2.0 * np.cos(np.pi * x / 2.0) + 0.2 * np.pi * np.cos(np.pi * x))


@pytest.mark.parametrize("kind,npaire,fields", [("intvp", 1, EVEN), ("intpv", 1, EVEN), ("derpv", 1, EVEN),
                                                ("dervp", 0, ODD)])
def test_stag_np_sixth_order_on_mirrored_fields(oracle, kind, npaire, fields):
    """The npaire 1 branches extend the field evenly about the walls, the odd
    closure of derxvp (:83-101) oddly about its wall values: on fields with
    that symmetry every row, boundary rows included, is 6th-order accurate
    (error ratio 64 per grid doubling; > 40 asserted)."""
    e1 = _stag_errors(oracle, kind, npaire, *fields, 33).max()
    e2 = _stag_errors(oracle, kind, npaire, *fields, 65).max()
    assert e1 < 1e-6 and e1 / e2 > 40, (kind, e1, e2)


def test_stag_np_dervp_even_rows(oracle):
    """derxvp's npaire 1 matrix carries 1 + alfa at its end rows (:579-584)
    although the derivative of an even field is odd about the wall, so its
    boundary rows are first order; the error decays away from the walls
    (the implicit rows damp it by rho = -0.15 per point) and the interior is
    6th order."""
    e1 = _stag_errors(oracle, "dervp", 1, *EVEN, 65)
    e2 = _stag_errors(oracle, "dervp", 1, *EVEN, 129)
    assert 1.8 < e1.max() / e2.max() < 2.2  # first order at the walls
    assert e1[24:-24].max() / e2[48:-48].max() > 40  # the same interior points, 6th order


def test_stag_np_missing_branches_refused(oracle):
    u = np.asfortranarray(np.ones((20, 9, 8)))
    p = np.asfortranarray(np.ones((19, 9, 8)))
    for kind, field, npaire in (("intvp", u, 0), ("derpv", p, 0), ("intpv", p, 0)):
        with pytest.raises(ValueError):
            oracle.stag_np(kind, 0, field, 0.1, 1, 1, npaire)
    uy = np.asfortranarray(np.ones((9, 20, 8)))
    with pytest.raises(ValueError):  # deryvp: npaire 0 only (:595)
        oracle.stag_np("dervp", 1, uy, 0.1, 1, 1, 1)
    oracle.stag_np("dervp", 1, uy, 0.1, 1, 1, 0)


def test_stag_np_factors_solve_the_matrix(oracle):
    """lhs_stag_np's factors reproduce the interpol_imp_ matrices: solving
    with them inverts the tridiagonal (b, c, f) assembled from the reference
    arrays (here for intpv: cibi6, cici6, cifip6 = cifi6)."""
    n, al = 12, 0.49
    lhs = oracle.lhs_stag_np("intpv", n, 0.1, 1, 1)
    m = lhs["m"]
    f = np.full(m, al); f[0] = 2 * al; f[-1] = 0.0
    b = np.full(m, al); b[-2] = 2 * al; b[-1] = 0.0
    A = np.diag(np.ones(m)) + np.diag(f[:-1], 1) + np.diag(b[:-1], -1)
    r = np.random.default_rng(1).standard_normal(m)
    z = r.copy()
    for i in range(1, m):
        z[i] -= z[i - 1] * lhs["s"][i]
    z[-1] *= lhs["w"][-1]
    for i in range(m - 2, -1, -1):
        z[i] = (z[i] - lhs["f"][i] * z[i + 1]) * lhs["w"][i]
    assert np.abs(A @ z - r).max() < 1e-13
