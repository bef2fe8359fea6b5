"""CPU FP64 oracle for x3div's Euler-timestep hot path (test infrastructure).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
bench.py may import this module; the product path never does.  It wraps the
C restatement in ``oracle/x3d_oracle.c`` (see that file's header for how the
restatement is pinned to the reference) and adds the 3-D FFTs of the spectral
Poisson solve with numpy's pocketfft, standing in for the external
2decomp&FFT library that the reference calls at src/poisson.f90:318,325,412.

Fields are numpy float64 arrays of shape (nx, ny, nz) in Fortran order, so
``u[i, j, k]`` is the reference's ``u(i+1, j+1, k+1)`` and x is contiguous.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

DER, DER2, DERVP, DERPV, INTVP, INTPV = range(6)
X, Y, Z = range(3)
KIND_NAMES = {"der": DER, "der2": DER2, "dervp": DERVP, "derpv": DERPV,
              "intvp": INTVP, "intpv": INTPV}

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the C restatement (make) and return the .so path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        i, d, p = ctypes.c_int, ctypes.c_double, _dp
        L.orc_build_lhs.argtypes = [i, i, d, p, p, p, p, p]
        L.orc_apply.argtypes = [i, i, p, p, i, i, i, d]
        L.orc_thomas_periodic.argtypes = [i, p, i, i, i, p, p, p, p, d]
        L.orc_thomas_plain.argtypes = [i, p, i, i, i, p, p, p]
        L.orc_poisson_spectral.argtypes = [p, i, i, i, d, d, d]
        L.orc_poisson_tables.argtypes = [i, i, i, d, d, d, p, p, p, p, p, p]
        L.orc_poisson_tables_bc1.argtypes = [i, d, p, p]
        L.orc_divergence.argtypes = [p, p, p, p, i, i, i, d, d, d]
        L.orc_gradp.argtypes = [p, p, p, p, i, i, i, d, d, d]
        L.orc_cor_vel.argtypes = [p, p, p, p, p, p, ctypes.c_long]
        L.orc_intt.argtypes = [p, p, d, ctypes.c_long]
        L.orc_momentum_rhs.argtypes = [p, p, p, p, p, p, i, i, i, d, d, d]
        L.orc_vel.argtypes = [p, p, p, i, i, i, d, d, d]
        L.orc_test_rms.argtypes = [i, p, i, i, i, d, d, d]
        L.orc_test_rms.restype = d
        L.orc_rhs_scalars.argtypes = [i, d, p]
        L.orc_build_der_np.argtypes = [i, d, i, i, i, p, p, p, p]
        L.orc_apply_der_np.argtypes = [i, p, p, i, i, i, d, i, i, i]
        L.orc_build_stag_np.argtypes = [i, i, d, i, i, p, p, p, ctypes.POINTER(ctypes.c_int)]
        L.orc_rhs_scalars.argtypes = [i, d, p]
        L.orc_apply_stag_np.argtypes = [i, i, p, p, i, i, i, d, i, i, i]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1)
    return a.ctypes.data_as(_dp)


def field(shape) -> np.ndarray:
    return np.zeros(shape, dtype=np.float64, order="F")


def _kind(k):
    return KIND_NAMES[k] if isinstance(k, str) else int(k)


def lhs(kind, n: int, d: float) -> dict:
    """Periodic operator of one kind on an n-point line with spacing d:
    the x3doperator1d contents (f, s, w, periodic, alfa) plus the explicit
    RHS scalars (a, b, c, d) that the reference keeps in module globals."""
    f, s, w, per = (np.zeros(n) for _ in range(4))
    c5 = np.zeros(5)
    rc = lib().orc_build_lhs(_kind(kind), n, float(d), _p(f), _p(s), _p(w), _p(per), _p(c5))
    if rc != 0:
        raise ValueError(f"oracle: bad operator request kind={kind} n={n}")
    return dict(f=f, s=s, w=w, periodic=per, alfa=c5[0], a=c5[1], b=c5[2], c=c5[3], d=c5[4])


def lhs_np(n: int, d: float, ncl1: int, ncln: int, npaire: int) -> dict:
    """Non-periodic first derivative on an n-point line (first_deriv_exp_ /
    first_deriv_imp_): factors f, s, w of parity npaire and the closure
    scalars af1, bf1, cf1, af2, afm, afn, bfn, cfn."""
    f, s, w, cl = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(8)
    rc = lib().orc_build_der_np(int(n), float(d), int(ncl1), int(ncln), int(npaire), _p(f), _p(s), _p(w), _p(cl))
    if rc != 0:
        raise ValueError(f"oracle: bad non-periodic request n={n} ncl=({ncl1},{ncln})")
    return dict(f=f, s=s, w=w, cl=cl)


def der_np(direction: int, u: np.ndarray, d: float, ncl1: int, ncln: int, npaire: int) -> np.ndarray:
    """der?_ij: non-periodic first derivative of u along direction."""
    out = field(u.shape)
    nx, ny, nz = u.shape
    rc = lib().orc_apply_der_np(int(direction), _p(out), _p(u), nx, ny, nz, float(d), int(ncl1), int(ncln),
                                int(npaire))
    if rc != 0:
        raise ValueError("oracle: bad non-periodic request")
    return out


def rhs_scalars(kind, d: float) -> dict:
    """alfa and the explicit RHS scalars a, b, c, d of an operator kind."""
    out = np.zeros(5)
    lib().orc_rhs_scalars(_kind(kind), float(d), _p(out))
    return dict(alfa=out[0], rhs=out[1:5].copy())


def lhs_stag_np(kind, n: int, d: float, ncl1: int, ncln: int) -> dict:
    """Non-periodic staggered LHS for a direction of n velocity points
    (interpol_imp_): factors f, s, w of its m rows (n - 1 for vp kinds)."""
    f, s, w = np.zeros(n), np.zeros(n), np.zeros(n)
    m = ctypes.c_int()
    rc = lib().orc_build_stag_np(_kind(kind), int(n), float(d), int(ncl1), int(ncln), _p(f), _p(s), _p(w),
                                 ctypes.byref(m))
    if rc != 0:
        raise ValueError("oracle: bad non-periodic staggered request")
    r = m.value
    return dict(f=f[:r].copy(), s=s[:r].copy(), w=w[:r].copy(), m=r)


def stag_np(kind, direction: int, u: np.ndarray, d: float, ncl1: int, ncln: int, npaire: int) -> np.ndarray:
    """A staggered routine's non-periodic branch (src/x3d_staggered.f90,
    nclx = .false.): u on the velocity grid (vp kinds) or the pressure grid
    (pv kinds, one point fewer along direction); returns the other grid."""
    k = _kind(kind)
    u = np.asfortranarray(u, dtype=np.float64)
    vp = k in (KIND_NAMES["dervp"], KIND_NAMES["intvp"])
    shape = list(u.shape)
    vel = list(u.shape)
    if vp:
        shape[direction] -= 1
    else:
        shape[direction] += 1
        vel[direction] += 1
    out = field(tuple(shape))
    rc = lib().orc_apply_stag_np(k, int(direction), _p(out), _p(u), vel[0], vel[1], vel[2], float(d), int(ncl1),
                                 int(ncln), int(npaire))
    if rc != 0:
        raise ValueError("oracle: no non-periodic branch for this routine and parity")
    return out


def apply(kind, direction: int, u: np.ndarray, d: float) -> np.ndarray:
    """One operator application (RHS stencil + periodic Thomas)."""
    u = np.asfortranarray(u, dtype=np.float64)
    out = field(u.shape)
    nx, ny, nz = u.shape
    rc = lib().orc_apply(_kind(kind), int(direction), _p(out), _p(u), nx, ny, nz, float(d))
    if rc != 0:
        raise ValueError("oracle: bad apply request")
    return out


def thomas_periodic(direction: int, t: np.ndarray, op: dict) -> np.ndarray:
    t = np.array(t, dtype=np.float64, order="F", copy=True)
    nx, ny, nz = t.shape
    lib().orc_thomas_periodic(int(direction), _p(t), nx, ny, nz, _p(op["f"]), _p(op["s"]),
                              _p(op["w"]), _p(op["periodic"]), float(op["alfa"]))
    return t


def poisson_tables(nx, ny, nz, xlx, yly, zlz):
    arrs = [np.zeros(n) for n in (nx, nx, ny, ny, nz, nz)]
    lib().orc_poisson_tables(nx, ny, nz, xlx, yly, zlz, *[_p(a) for a in arrs])
    return dict(k2x=arrs[0], tx=arrs[1], k2y=arrs[2], ty=arrs[3], k2z=arrs[4], tz=arrs[5])


def poisson(rhs: np.ndarray, xlx: float, yly: float, zlz: float) -> np.ndarray:
    """poisson_000 (src/poisson.f90:276-419).  The transforms are the
    unnormalised r2c (sign -1) along z then c2c along y and x, and the
    unnormalised c2r inverse, i.e. 2decomp's PHYSICAL_IN_Z convention."""
    rhs = np.asfortranarray(rhs, dtype=np.float64)
    nx, ny, nz = rhs.shape
    a = rhs.transpose(2, 1, 0)  # C-order (nz, ny, nx) view of the F-order field
    cw = np.fft.rfftn(a, axes=(2, 1, 0))  # real transform along axis 0 (z) -> (nz/2+1, ny, nx)
    cw = np.ascontiguousarray(cw, dtype=np.complex128)
    lib().orc_poisson_spectral(cw.ctypes.data_as(_dp), nx, ny, nz, xlx, yly, zlz)
    out = np.fft.irfftn(cw, s=(nx, ny, nz), axes=(2, 1, 0), norm="forward")
    return np.asfortranarray(out.transpose(2, 1, 0))


def poisson_tables_bc1(m: int, length: float):
    """waves() for a non-periodic direction of m pressure points
    (src/poisson.f90:539-553): k2 and the transfer function of cosine mode
    i = 0 .. m."""
    k2, tt = np.zeros(m + 1), np.zeros(m + 1)
    lib().orc_poisson_tables_bc1(int(m), float(length), _p(k2), _p(tt))
    return k2, tt


def poisson_bc(rhs: np.ndarray, lengths, periodic) -> np.ndarray:
    """The Poisson solve with homogeneous Neumann conditions on the pressure
    along the non-periodic directions (the bc = 1 case of
    decomp_2d_poisson_init, src/poisson.f90:85-99, which x3div itself stops
    on at :104-108): rhs holds the pressure grid, m = n - 1 points along a
    non-periodic direction.  The field mirrored about both walls of every
    non-periodic direction is even, so it has only the cosine modes of
    waves()'s bc = 1 tables; solved as poisson_000 on the doubled box
    (2 m points over twice the length) and cut back to the first m points."""
    a = np.asarray(rhs, dtype=np.float64)
    ext, lens = a, list(lengths)
    for d in range(3):
        if not periodic[d]:
            ext = np.concatenate([ext, np.flip(ext, axis=d)], axis=d)
            lens[d] = 2 * lens[d]
    out = poisson(np.asfortranarray(ext), *lens)
    return np.asfortranarray(out[:a.shape[0], :a.shape[1], :a.shape[2]])


def poisson_bc_dct(rhs: np.ndarray, lengths, periodic) -> np.ndarray:
    """The same solve in the cosine/Fourier basis directly: a DCT-II along
    each non-periodic direction, an FFT along each periodic one, each mode
    divided by -K with K = k2x (ty tz)^2 + k2y (tx tz)^2 + k2z (tx ty)^2
    from waves()'s bc = 1 tables (poisson_tables_bc1) or its periodic ones,
    zero where K < 1e-16, and the inverse transforms.  An independent check
    of poisson_bc."""
    import scipy.fft as sf
    a = np.asarray(rhs, dtype=np.float64)
    n = a.shape
    c = a.astype(np.complex128)
    k2, tt = [], []
    for d in range(3):
        if periodic[d]:
            t = poisson_tables(n[d], n[d], n[d], lengths[d], lengths[d], lengths[d])
            k2.append(t["k2x"])
            tt.append(t["tx"])
            c = np.fft.fft(c, axis=d)
        else:
            kk, tr = poisson_tables_bc1(n[d], lengths[d])
            k2.append(kk[:n[d]])
            tt.append(tr[:n[d]])
            c = sf.dct(c.real, type=2, axis=d) + 1j * sf.dct(c.imag, type=2, axis=d)
    tx, ty, tz = tt[0][:, None, None], tt[1][None, :, None], tt[2][None, None, :]
    K = (k2[0][:, None, None] * (ty * tz) ** 2 + k2[1][None, :, None] * (tx * tz) ** 2
         + k2[2][None, None, :] * (tx * ty) ** 2)
    c = np.where(K < 1e-16, 0.0, c / np.where(K < 1e-16, 1.0, -K))
    for d in (2, 1, 0):
        if periodic[d]:
            c = np.fft.ifft(c, axis=d)
        else:
            c = sf.idct(c.real, type=2, axis=d) + 1j * sf.idct(c.imag, type=2, axis=d)
    return np.asfortranarray(c.real)


def divergence(ux, uy, uz, dx, dy, dz):
    nx, ny, nz = ux.shape
    pp3 = field(ux.shape)
    rc = lib().orc_divergence(_p(pp3), _p(ux), _p(uy), _p(uz), nx, ny, nz, dx, dy, dz)
    assert rc == 0
    return pp3


def gradp(pp3, dx, dy, dz):
    nx, ny, nz = pp3.shape
    px, py, pz = field(pp3.shape), field(pp3.shape), field(pp3.shape)
    rc = lib().orc_gradp(_p(px), _p(py), _p(pz), _p(pp3), nx, ny, nz, dx, dy, dz)
    assert rc == 0
    return px, py, pz


def momentum_rhs(ux, uy, uz, dx, dy, dz):
    nx, ny, nz = ux.shape
    du = [field(ux.shape) for _ in range(3)]
    rc = lib().orc_momentum_rhs(*[_p(a) for a in du], _p(ux), _p(uy), _p(uz), nx, ny, nz, dx, dy, dz)
    assert rc == 0
    return tuple(du)


def intt(var, dvar, gdt):
    lib().orc_intt(_p(var), _p(dvar), float(gdt), var.size)


def cor_vel(ux, uy, uz, px, py, pz):
    lib().orc_cor_vel(_p(ux), _p(uy), _p(uz), _p(px), _p(py), _p(pz), ux.size)


def vel(nx, ny, nz, xlx=1.0, yly=1.0, zlz=1.0):
    """Reference initial field (src/mom.f90:46-53)."""
    u, v, w = field((nx, ny, nz)), field((nx, ny, nz)), field((nx, ny, nz))
    lib().orc_vel(_p(u), _p(v), _p(w), nx, ny, nz, xlx, yly, zlz)
    return u, v, w


def test_rms(which: int, du, xlx=1.0, yly=1.0, zlz=1.0) -> float:
    nx, ny, nz = du.shape
    return lib().orc_test_rms(int(which), _p(du), nx, ny, nz, xlx, yly, zlz)


def euler_step(ux, uy, uz, dt, lengths=(1.0, 1.0, 1.0)):
    """One x3div timestep (xcompact3d.f90:80-95) at a 1x1 decomposition:
    calculate_transeq_rhs, int_time, solve_poisson, cor_vel.  Updates
    ux, uy, uz in place and returns (du, pp3 divergence before projection,
    pressure after the solve)."""
    nx, ny, nz = ux.shape
    xlx, yly, zlz = lengths
    dx, dy, dz = xlx / nx, yly / ny, zlz / nz
    du = momentum_rhs(ux, uy, uz, dx, dy, dz)
    for v, dv in zip((ux, uy, uz), du):
        intt(v, dv, dt)
    div = divergence(ux, uy, uz, dx, dy, dz)
    pp3 = poisson(div, xlx, yly, zlz)
    px, py, pz = gradp(pp3, dx, dy, dz)
    cor_vel(ux, uy, uz, px, py, pz)
    return du, div, pp3
