"""Non-periodic first derivatives (der?_ij) against the oracle.

A context created with boundary conditions (x3d_ctx_create_bc: the
reference's nclx1, nclxn, ...; 1 free slip, 2 Dirichlet) builds derx (npaire
0) and derxp (npaire 1) of a non-periodic direction from first_deriv_exp_ /
first_deriv_imp_; they run on the one-thread-per-line kernels with the
boundary closures of der?_ij.  Bars as for the periodic operators: FP64 within
1e-12 of the oracle, FP32 within 1e-5 (normwise relative).  Every other
operator of such a direction, and the Euler-step compositions, refuse with
X3D_EUNSUPPORTED.  The Poisson solve takes such a context's pressure grid
(nx - 1 points along a non-periodic direction) with Neumann conditions
there, against the oracle's poisson_bc at 1e-12.
"""
import numpy as np
import pytest

from conftest import rel_err, seeded_field

pytestmark = pytest.mark.gpu

NAMES = {0: ("derx", "derxp"), 1: ("dery", "deryp"), 2: ("derz", "derzp")}


def _call(ctx, direction, t, u, op, shape):
    nx, ny, nz = shape
    if direction == 0:
        ctx.derx(t, u, op, nx, ny, nz)
    elif direction == 1:
        ctx.dery(t, u, op, None, nx, ny, nz)
    else:
        ctx.derz(t, u, op, nx, ny, nz)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(32, 24, 16), (18, 12, 10)])
@pytest.mark.parametrize("ncl", [(1, 1), (1, 2), (2, 1), (2, 2)])
def test_nonperiodic_first_derivatives_match_oracle(oracle, torch_cuda, prec, shape, ncl):
    torch = torch_cuda
    from x3div_b200 import Context, to_device, to_host
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 1e-5
    lengths = (1.0, 2.0, 1.5)
    u = seeded_field(shape, 40 + ncl[0] * 3 + ncl[1], lengths=lengths, noise=1e-2)
    for direction in range(3):
        bc = [0] * 6
        bc[2 * direction], bc[2 * direction + 1] = ncl
        ctx = Context(*shape, lengths=lengths, precision=prec, bc=bc)
        d_u = to_device(u, dt)
        used = to_host(d_u).astype(np.float64)
        h = lengths[direction] / (shape[direction] - 1)
        t = torch.full_like(d_u, np.nan)
        for npaire, name in enumerate(NAMES[direction]):
            _call(ctx, direction, t, d_u, ctx.op(name), shape)
            ref = oracle.der_np(direction, used, h, ncl[0], ncl[1], npaire)
            err = rel_err(to_host(t), ref)
            assert err < tol, (direction, name, err)
        ctx.close()


def test_nonperiodic_context_refuses_what_needs_periodicity(torch_cuda):
    torch = torch_cuda
    from x3div_b200 import Context, X3DError
    shape = (16, 16, 16)
    ctx = Context(*shape, lengths=(1.0, 1.0, 1.0), bc=(2, 2, 0, 0, 0, 0))
    with pytest.raises(X3DError):
        ctx.op("derxx")  # no non-periodic second derivative
    ctx.op("dery")  # periodic directions keep every operator
    ctx.op("intyvp")
    u = [torch.zeros(shape[::-1], dtype=torch.float64, device="cuda") for _ in range(3)]
    pp3 = torch.zeros(shape[::-1], dtype=torch.float64, device="cuda")
    with pytest.raises(X3DError):
        ctx.divergence(pp3, *u)
    with pytest.raises(X3DError):
        ctx.euler_step(*u, *[torch.empty_like(u[0]) for _ in range(3)], pp3,
                       *[torch.empty_like(u[0]) for _ in range(3)], 1e-3)
    ctx.autotune(2)  # tunes what exists, skips the rest
    ctx.close()


def test_bad_boundary_conditions_are_rejected(torch_cuda):
    from x3div_b200 import Context, X3DError
    for bc in [(0, 1, 0, 0, 0, 0), (3, 3, 0, 0, 0, 0), (1, 1, 0, 0, -1, 0)]:
        with pytest.raises(X3DError):
            Context(16, 16, 16, bc=bc)


# ---- non-periodic staggered routines (nclx = .false. branches) -------------

STAG = {0: ("derxvp", "interxvp", "derxpv", "interxpv"),
        1: ("deryvp", "interyvp", "derypv", "interypv"),
        2: ("derzvp", "interzvp", "derzpv", "interzpv")}
KIND_OF = {"der": "dervp", "int": "intvp"}


def _kind(routine):
    base = "der" if routine.startswith("der") else "int"
    return base + routine[-2:]


def _stag_call(ctx, direction, routine, t, u, op, shape):
    """A staggered routine with the reference's argument order; shape is the
    velocity grid (nx, ny, nz) and the pressure grid has one point fewer
    along direction."""
    nx, ny, nz = shape
    nm = shape[direction] - 1
    fn = getattr(ctx, routine)
    vp = routine.endswith("vp")
    if direction == 0:
        fn(t, u, op, *((nx, nm) if vp else (nm, nx)), ny, nz)
    elif direction == 1:
        lens = (ny, nm) if vp else (nm, ny)
        if routine.startswith("der"):
            fn(t, u, op, None, nx, *lens, nz)
        else:
            fn(t, u, op, nx, *lens, nz)
    else:
        fn(t, u, op, nx, ny, *((nz, nm) if vp else (nm, nz)))


def _grid(shape, direction, pressure):
    s = list(shape)
    if pressure:
        s[direction] -= 1
    return tuple(s)


def _run_stag(oracle, torch, ctx, direction, routine, op, shape, lengths, prec, ncl, npaire):
    from x3div_b200 import to_device, to_host
    dt = torch.float64 if prec == "f64" else torch.float32
    vp = routine.endswith("vp")
    in_shape = _grid(shape, direction, not vp)
    out_shape = _grid(shape, direction, vp)
    u = seeded_field(in_shape, 60 + direction * 7 + len(routine), lengths=lengths, noise=1e-2)
    d_u = to_device(u, dt)
    used = to_host(d_u).astype(np.float64)
    t = torch.full(out_shape[::-1], float("nan"), dtype=dt, device="cuda")
    _stag_call(ctx, direction, routine, t, d_u, op, shape)
    ctx.sync()
    h = lengths[direction] / (shape[direction] - 1)
    ref = oracle.stag_np(_kind(routine), direction, used, h, ncl[0], ncl[1], npaire)
    return rel_err(to_host(t), ref)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(20, 18, 16), (12, 10, 9)])
@pytest.mark.parametrize("ncl", [(1, 1), (2, 1), (2, 2)])
def test_nonperiodic_staggered_builtins_match_oracle(oracle, torch_cuda, prec, shape, ncl):
    """The built-in staggered operators of a non-periodic direction, with the
    parities x3d_operator_1d_init binds (dervp 1, derpv 0, intvp 1, intpv 1):
    where the reference has a branch for that parity the result matches the
    oracle; where it has none (deryvp, der?pv) the call is refused."""
    torch = torch_cuda
    from x3div_b200 import Context, X3DError
    tol = 1e-12 if prec == "f64" else 1e-5
    lengths = (1.0, 2.0, 1.5)
    for direction in range(3):
        bc = [0] * 6
        bc[2 * direction], bc[2 * direction + 1] = ncl
        ctx = Context(*shape, lengths=lengths, precision=prec, bc=bc)
        for routine in STAG[direction]:
            op = ctx.op(routine.replace("inter", "int"))
            npaire = 0 if routine.startswith("der") and routine.endswith("pv") else 1
            no_branch = routine.endswith("pv") and routine.startswith("der") or routine == "deryvp"
            if no_branch:
                with pytest.raises(X3DError):
                    _run_stag(oracle, torch, ctx, direction, routine, op, shape, lengths, prec, ncl, npaire)
                continue
            err = _run_stag(oracle, torch, ctx, direction, routine, op, shape, lengths, prec, ncl, npaire)
            assert err < tol, (direction, routine, ncl, err)
        ctx.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_nonperiodic_staggered_other_parities(oracle, torch_cuda, prec):
    """The reference's other non-periodic branches, through operators
    created from the oracle's factors (x3d_op_create, no periodic vector):
    derxvp/derzvp npaire 0 (the odd closure), deryvp npaire 0 (its only
    branch) and der?pv npaire 1."""
    torch = torch_cuda
    from x3div_b200 import Context, X3DError
    tol = 1e-12 if prec == "f64" else 1e-5
    shape = (20, 18, 16)
    lengths = (1.0, 2.0, 1.5)
    ncl = (2, 1)
    for direction in range(3):
        bc = [0] * 6
        bc[2 * direction], bc[2 * direction + 1] = ncl
        ctx = Context(*shape, lengths=lengths, precision=prec, bc=bc)
        h = lengths[direction] / (shape[direction] - 1)
        cases = [(STAG[direction][0], "dervp", 0), (STAG[direction][2], "derpv", 1)]
        for routine, kind, npaire in cases:
            lhs = oracle.lhs_stag_np(kind, shape[direction], h, *ncl)
            sc = oracle.rhs_scalars(kind, h)
            op = ctx.op_create(kind, direction, lhs["m"], npaire, sc["alfa"], lhs["f"], lhs["s"], lhs["w"],
                               None, sc["rhs"])
            err = _run_stag(oracle, torch, ctx, direction, routine, op, shape, lengths, prec, ncl, npaire)
            assert err < tol, (direction, routine, npaire, err)
            op.close()
        # the other parity of deryvp has no branch
        if direction == 1:
            lhs = oracle.lhs_stag_np("dervp", shape[1], h, *ncl)
            sc = oracle.rhs_scalars("dervp", h)
            op = ctx.op_create("dervp", 1, lhs["m"], 1, sc["alfa"], lhs["f"], lhs["s"], lhs["w"], None, sc["rhs"])
            with pytest.raises(X3DError):
                _run_stag(oracle, torch, ctx, 1, "deryvp", op, shape, lengths, prec, ncl, 1)
            op.close()
        ctx.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_nonperiodic_staggered_y_stretching_metric(oracle, torch_cuda, prec):
    """deryvp (npaire 0, its only non-periodic branch) and derypv (npaire 1)
    with a stretching metric: the result is scaled by ppyi / ppy on the
    output grid (src/x3d_staggered.f90:629-635, 875-881)."""
    torch = torch_cuda
    from x3div_b200 import Context, to_device, to_host
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 1e-5
    shape = (12, 20, 10)
    nx, ny, nz = shape
    lengths = (1.0, 2.0, 1.5)
    ncl = (1, 2)
    ctx = Context(*shape, lengths=lengths, precision=prec, bc=(0, 0, *ncl, 0, 0))
    h = lengths[1] / (ny - 1)
    for kind, routine, npaire in (("dervp", "deryvp", 0), ("derpv", "derypv", 1)):
        lhs = oracle.lhs_stag_np(kind, ny, h, *ncl)
        sc = oracle.rhs_scalars(kind, h)
        op = ctx.op_create(kind, 1, lhs["m"], npaire, sc["alfa"], lhs["f"], lhs["s"], lhs["w"], None, sc["rhs"])
        vp = kind == "dervp"
        in_shape = (nx, ny if vp else ny - 1, nz)
        out_n = ny - 1 if vp else ny
        u = seeded_field(in_shape, 71, lengths=lengths, noise=1e-2)
        d_u = to_device(u, dt)
        used = to_host(d_u).astype(np.float64)
        metric = 1.0 + 0.25 * np.sin(np.arange(out_n) / out_n * 2 * np.pi)
        t = torch.full((nz, out_n, nx), float("nan"), dtype=dt, device="cuda")
        if vp:
            ctx.deryvp(t, d_u, op, metric, nx, ny, ny - 1, nz)
        else:
            ctx.derypv(t, d_u, op, metric, nx, ny - 1, ny, nz)
        ctx.sync()
        ref = oracle.stag_np(kind, 1, used, h, *ncl, npaire) * metric[None, :, None]
        assert rel_err(to_host(t), ref) < tol, (routine, prec)
        op.close()
    ctx.close()


# pressure-grid shapes: the mirrored lengths 2 (n - 1) reach the fused z
# kernel (2 * 32 = 64, 2 * 48 = 96) and the 3-D cuFFT path (2 * 20 = 40)
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape,per", [((17, 12, 10), (False, True, True)), ((12, 17, 10), (True, False, True)),
                                       ((12, 10, 33), (True, True, False)), ((17, 13, 12), (False, False, True)),
                                       ((13, 17, 21), (False, False, False)), ((16, 10, 49), (True, False, False))])
def test_nonperiodic_poisson_matches_oracle(oracle, torch_cuda, prec, shape, per):
    """x3d_poisson on a context with non-periodic directions: the bc = 1
    (Neumann) case of decomp_2d_poisson_init on the pressure grid, against
    the oracle's mirrored-box solve (itself checked against a DCT/FFT
    solve from waves()'s bc = 1 tables in tests/test_oracle_poisson_bc.py),
    FP64 in both context precisions; twice, to use the kept mirrored
    context."""
    torch = torch_cuda
    from x3div_b200 import Context, to_host
    lengths = (2 * np.pi, 1.5, 3.0)
    bc = []
    for p_ in per:
        bc += [0, 0] if p_ else [1, 2]
    ctx = Context(*shape, lengths=lengths, precision=prec, bc=tuple(bc))
    pshape = tuple(n if p_ else n - 1 for n, p_ in zip(shape, per))
    for seed in (3, 4):
        g = np.random.default_rng(seed).standard_normal(pshape)  # Fortran (x, y, z) values
        rhs = torch.from_numpy(np.ascontiguousarray(g.transpose(2, 1, 0))).cuda()
        ctx.poisson(rhs)
        ctx.sync()
        ref = oracle.poisson_bc(np.asfortranarray(g), lengths, per)
        assert rel_err(to_host(rhs), ref) < 1e-12, (shape, per, seed)
    ctx.close()
