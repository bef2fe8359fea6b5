"""Device-resident host arrays (x3d_buf_register, the reference's OpenACC
data regions, src/xcompact3d.f90:43-72) and the captured Euler step
(x3d_step_capture / x3d_step_launch)."""
import numpy as np
import pytest

from conftest import seeded_field

pytestmark = pytest.mark.gpu

LEN = (2 * np.pi, 1.5, 3.0)
SHAPE = (32, 24, 16)


def _fields(prec):
    dt = np.float64 if prec == "f64" else np.float32
    return [np.asfortranarray(seeded_field(SHAPE, s, lengths=LEN, noise=1e-2).astype(dt)) for s in (3, 4, 5)]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_registered_host_arrays_run_on_their_mirrors(torch_cuda, prec):
    """Three Euler steps on registered host arrays equal three steps on
    device tensors bit for bit, and the host arrays change only at
    x3d_sync_to_host."""
    torch = torch_cuda
    from x3div_b200 import Context, to_device, to_host
    ctx = Context(*SHAPE, lengths=LEN, precision=prec)
    u0 = _fields(prec)
    host_u = [a.copy(order="F") for a in u0]
    host_du = [np.zeros_like(a, order="F") for a in u0]
    host_pg = [np.zeros_like(a, order="F") for a in u0]
    host_pp = np.zeros(SHAPE, dtype=np.float64, order="F")
    arrays = host_u + host_du + [host_pp] + host_pg
    for a in arrays:
        assert ctx.buf_register(a)
    for _ in range(3):
        ctx.euler_step(*host_u, *host_du, host_pp, *host_pg, 1e-3)
    ctx.sync()
    for a, b in zip(host_u, u0):  # still the initial values: no copies back yet
        assert np.array_equal(a, b)
    for a in arrays:
        ctx.sync_to_host(a)
    tdt = torch.float64 if prec == "f64" else torch.float32
    U = [to_device(a, tdt) for a in u0]
    du = [torch.empty_like(U[0]) for _ in range(3)]
    pg = [torch.empty_like(U[0]) for _ in range(3)]
    pp3 = torch.empty(SHAPE[::-1], dtype=torch.float64, device="cuda")
    for _ in range(3):
        ctx.euler_step(*U, *du, pp3, *pg, 1e-3)
    ctx.sync()
    for a, b in zip(host_u, U):
        assert np.array_equal(a, to_host(b))
    assert np.array_equal(host_pp, to_host(pp3))
    # sync_to_device pushes host edits to the mirror
    host_u[0][...] = 0
    ctx.sync_to_device(host_u[0])
    ctx.euler_step(*host_u, *host_du, host_pp, *host_pg, 1e-3)
    ctx.sync_to_host(host_du[0])
    for a in arrays:
        ctx.buf_unregister(a)
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_captured_step_replays_the_eager_step(torch_cuda, prec):
    torch = torch_cuda
    from x3div_b200 import Context, to_device
    tdt = torch.float64 if prec == "f64" else torch.float32
    u0 = _fields(prec)

    def state():
        U = [to_device(a, tdt) for a in u0]
        return U, [torch.empty_like(U[0]) for _ in range(3)], \
            torch.empty(SHAPE[::-1], dtype=torch.float64, device="cuda"), \
            [torch.empty_like(U[0]) for _ in range(3)]

    # torch's default stream is the legacy one, which cannot be captured
    stream = torch.cuda.Stream()
    ctx = Context(*SHAPE, lengths=LEN, precision=prec, stream=stream)
    U, du, pp3, pg = state()
    torch.cuda.synchronize()
    for _ in range(4):
        ctx.euler_step(*U, *du, pp3, *pg, 1e-3)
    ctx.sync()
    V, dv, pq, ph = state()
    torch.cuda.synchronize()
    ctx.step_capture(*V, *dv, pq, *ph, 1e-3)
    ctx.sync()
    assert all(torch.equal(a, b) for a, b in zip(V, state()[0]))  # capture runs nothing
    for _ in range(4):
        ctx.step_launch()
    ctx.sync()
    for a, b in zip(U, V):
        assert torch.equal(a, b)
    assert torch.equal(pp3, pq)
    ctx.close()


def test_capture_rejects_unregistered_host_arrays(torch_cuda):
    from x3div_b200 import Context, X3DError
    ctx = Context(*SHAPE, lengths=LEN, precision="f64")
    a = [np.zeros(SHAPE, order="F") for _ in range(9)]
    p = np.zeros(SHAPE, order="F")
    with pytest.raises(X3DError):
        ctx.step_capture(*a[:6], p, *a[6:], 1e-3)
    with pytest.raises(X3DError):
        ctx.step_launch()  # nothing captured
    with pytest.raises(X3DError):
        ctx.sync_to_host(p)  # not registered
    ctx.buf_register(p)
    with pytest.raises(X3DError):
        ctx.buf_register(p)  # overlaps
    ctx.buf_unregister(p)
    ctx.close()


def test_bounded_wait_timeout_is_reported_and_the_context_survives(oracle, torch_cuda):
    """Failure detection without a GPU fault: a bounded wait that nothing
    completes gives up after 20 ms, the host sees X3D_ETIMEOUT at the next
    sync (once), and the context keeps working."""
    torch = torch_cuda
    from x3div_b200 import Context, X3DError, to_device, to_host
    from conftest import rel_err
    ctx = Context(*SHAPE, lengths=LEN, precision="f64")
    ctx.selftest_timeout(0.02)
    with pytest.raises(X3DError) as e:
        ctx.sync()
    assert e.value.code == -5
    ctx.sync()  # reported once
    u = seeded_field(SHAPE, 9, lengths=LEN, noise=1e-2)
    d_u = to_device(u)
    t = torch.empty_like(d_u)
    ctx.derx(t, d_u, ctx.op("derx"), *SHAPE)
    ctx.sync()
    assert rel_err(to_host(t), oracle.apply("der", 0, u, LEN[0] / SHAPE[0])) < 1e-12
    with pytest.raises(X3DError):
        ctx.selftest_timeout(5.0)  # limits above 1 s are refused
    ctx.close()
