"""x3d_divergence_noalloc, the allocation-free divergence.

Hosts that cannot allocate device memory in their time loop (an OpenACC
Fortran host that maps its whole working set up front, or a solver under a
fixed device-memory budget) call this variant: its intermediate fields live
in a fixed array inside the library.  Here it is called through the C ABI and
checked against x3d_divergence on the same inputs, twice in a row, so the
second call also shows that what the first call left in the shared array
does not leak into the result.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err, seeded_field

pytestmark = pytest.mark.gpu

LEN = (2 * np.pi, 1.5, 3.0)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_divergence_matches_divergence(torch_cuda, prec):
    torch = torch_cuda
    from x3div_b200 import Context, _capi, to_device, to_host
    L = _capi.lib()
    shape = (64, 64, 64)  # X3D_NOALLOC_MAX_POINTS points, the largest grid it takes
    ctx = Context(*shape, lengths=LEN, precision=prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 1e-5
    for call in range(2):
        u = [to_device(seeded_field(shape, 10 * call + c, lengths=LEN, noise=1e-2), dt) for c in range(3)]
        ref = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
        got = torch.full_like(ref, float("nan"))
        ctx.divergence(ref, *u)
        rc = L.x3d_divergence_noalloc(ctx.handle, got.data_ptr(), *[a.data_ptr() for a in u])
        assert rc == 0, L.x3d_ctx_last_error(ctx.handle)
        ctx.sync()
        assert rel_err(to_host(got), to_host(ref)) < tol, (prec, call)
    ctx.close()


def test_noalloc_refuses_what_it_cannot_do_without_allocating(torch_cuda):
    torch = torch_cuda
    from x3div_b200 import Context, _capi
    L = _capi.lib()
    big = Context(80, 64, 64, lengths=LEN)  # above X3D_NOALLOC_MAX_POINTS
    u = [torch.zeros(64, 64, 80, dtype=torch.float64, device="cuda") for _ in range(3)]
    p = torch.empty_like(u[0])
    assert L.x3d_divergence_noalloc(big.handle, p.data_ptr(), *[a.data_ptr() for a in u]) == _capi.X3D_EINVAL
    assert b"X3D_NOALLOC_MAX_POINTS" in L.x3d_ctx_last_error(big.handle)
    big.close()
    ctx = Context(16, 16, 16, lengths=LEN)
    host = [np.zeros((16, 16, 16), order="F") for _ in range(4)]  # host arrays would need staging
    assert L.x3d_divergence_noalloc(ctx.handle, *[a.ctypes.data for a in host]) == _capi.X3D_EINVAL
    ctx.close()
