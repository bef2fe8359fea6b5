"""Non-periodic first derivatives (der?_ij) against the oracle.

A context created with boundary conditions (x3d_ctx_create_bc: the
reference's nclx1, nclxn, ...; 1 free slip, 2 Dirichlet) builds derx (npaire
0) and derxp (npaire 1) of a non-periodic direction from first_deriv_exp_ /
first_deriv_imp_; they run on the one-thread-per-line kernels with the
boundary closures of der?_ij.  Bars as for the periodic operators: FP64 within
1e-12 of the oracle, FP32 within 1e-5 (normwise relative).  Every other
operator of such a direction, and the routines that need the Poisson solver,
refuse with X3D_EUNSUPPORTED (the reference's Poisson solver stops on
non-periodic boundaries).
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
        ctx.op("derxvp")
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
