"""x3d_divergence_noalloc, the allocation-free divergence.

Hosts that cannot allocate device memory in their time loop (an OpenACC
Fortran host that maps its whole working set up front, or a solver under a
fixed device-memory budget) call this variant: its intermediate fields live
in a fixed array inside the library.  Here it is called through the C ABI and
checked against x3d_divergence on the same inputs, twice in a row, so the
second call also shows that what the first call left in the shared array
does not leak into the result.  The context that calls it never calls
anything else, and the device's free memory is the same before and after
its calls: the context allocated no scratch.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err, seeded_field

pytestmark = pytest.mark.gpu

LEN = (2 * np.pi, 1.5, 3.0)


def _noalloc(L, ctx, p, u):
    rc = L.x3d_divergence_noalloc(ctx.handle, p.data_ptr(), *[a.data_ptr() for a in u])
    assert rc == 0, L.x3d_ctx_last_error(ctx.handle)


# 64^3 is X3D_NOALLOC_MAX_POINTS points, the largest grid it takes; 32 x 48 x 16
# checks each field's offset in the array on a smaller, non-cubic grid
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 48, 16)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_divergence_matches_divergence(torch_cuda, prec, shape):
    torch = torch_cuda
    from x3div_b200 import Context, _capi, to_device, to_host
    L = _capi.lib()
    dt = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 1e-5
    fresh = Context(*shape, lengths=LEN, precision=prec)  # only ever calls the no-alloc entry point
    check = Context(*shape, lengths=LEN, precision=prec)  # the existing entry point, for reference
    inputs = [[to_device(seeded_field(shape, 10 * call + c, lengths=LEN, noise=1e-2), dt) for c in range(3)]
              for call in range(2)]
    got = [torch.full(shape[::-1], float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    ref = [torch.empty(shape[::-1], dtype=torch.float64, device="cuda") for _ in range(2)]
    # first call of the fresh context: it may load the library's module on the
    # device (the array comes with it) if no earlier test did
    _noalloc(L, fresh, got[0], inputs[0])
    fresh.sync()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for call in range(2):
        _noalloc(L, fresh, got[call], inputs[call])
    fresh.sync()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)  # no device memory taken by the calls
    for call in range(2):
        check.divergence(ref[call], *inputs[call])
    check.sync()
    for call in range(2):
        assert rel_err(to_host(got[call]), to_host(ref[call])) < tol, (prec, shape, call)
    fresh.close()
    check.close()


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
    # FP32 rows of 18 points are 72 bytes: the fused stage kernels cannot take
    # the grid, and the unfused path would need context scratch
    odd = Context(18, 12, 10, lengths=LEN, precision="f32")
    u = [torch.zeros(10, 12, 18, dtype=torch.float32, device="cuda") for _ in range(3)]
    p = torch.empty(10, 12, 18, dtype=torch.float64, device="cuda")
    assert L.x3d_divergence_noalloc(odd.handle, p.data_ptr(), *[a.data_ptr() for a in u]) == _capi.X3D_EUNSUPPORTED
    odd.close()
