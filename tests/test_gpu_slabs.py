"""The slab code path on the B200: the library's line solves on a rank's
local extents and the y <-> z transposes through NCCL (one rank), against the
oracle on the whole box."""
import socket

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

def _kind(routine):
    if routine in ("derxx", "deryy", "derzz"):
        return "der2"
    if routine.startswith("inter"):
        return "int" + routine[-2:]
    if routine.endswith(("vp", "pv")):
        return "der" + routine[-2:]
    return "der"


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_slab_sweep_on_one_nccl_rank(oracle, torch_cuda, prec):
    torch = torch_cuda
    import torch.distributed as dist
    from x3div_b200 import Context, to_host
    from x3div_b200.slabs import SWEEP, SlabLayout, sweep
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        shape = (24, 20, 16)
        lengths = (2 * np.pi, 1.5, 3.0)
        ctx = Context(*shape, lengths=lengths, precision=prec)
        dt = torch.float64 if prec == "f64" else torch.float32
        g = np.random.default_rng(3).standard_normal(shape[::-1])
        field = torch.from_numpy(g).to(device="cuda", dtype=dt)
        used = np.asfortranarray(field.double().cpu().numpy().transpose(2, 1, 0))
        res = sweep(ctx, field, SlabLayout(shape, 0, 1))
        ctx.sync()
        tol = 1e-12 if prec == "f64" else 1e-5
        for d in range(3):
            for k, (routine, _) in enumerate(SWEEP[d]):
                ref = oracle.apply(_kind(routine), d, used, lengths[d] / shape[d])
                assert rel_err(to_host(res[d][k]), ref) < tol, (d, routine)
        ctx.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("shape", [(24, 20, 16), (30, 12, 48), (16, 18, 96), (12, 10, 40)])
def test_slab_poisson_on_one_nccl_rank(oracle, torch_cuda, shape):
    """The slab Poisson solve (torch.fft x-y transforms, the half spectrum
    transposed through NCCL, x3d_poisson_zlines on the rank's y rows) against
    the oracle's poisson_000 on the whole box."""
    torch = torch_cuda
    import torch.distributed as dist
    from x3div_b200 import Context
    from x3div_b200.slabs import SlabLayout, poisson
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        lengths = (2 * np.pi, 1.5, 3.0)
        ctx = Context(*shape, lengths=lengths, precision="f64")
        g = np.random.default_rng(8).standard_normal(shape[::-1])
        rhs = torch.from_numpy(g).cuda()
        poisson(ctx, rhs, SlabLayout(shape, 0, 1))
        torch.cuda.synchronize()
        ref = oracle.poisson(np.asfortranarray(g.transpose(2, 1, 0)), *lengths)
        assert rel_err(rhs.cpu().numpy().transpose(2, 1, 0), ref) < 1e-12, shape
        ctx.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_slab_euler_steps_on_one_nccl_rank(oracle, torch_cuda, prec):
    """Three Euler steps composed on slabs (line solves on local extents,
    NCCL transposes, the slab Poisson solve) against the oracle and against
    the library's fused single-box step."""
    torch = torch_cuda
    import torch.distributed as dist
    from x3div_b200 import Context, to_host
    from x3div_b200.slabs import SlabLayout, euler_step
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        shape = (24, 20, 16)
        lengths = (2 * np.pi, 1.5, 3.0)
        dt = torch.float64 if prec == "f64" else torch.float32
        ctx = Context(*shape, lengths=lengths, precision=prec)
        g = [np.random.default_rng(30 + c).standard_normal(shape[::-1]) * 0.1 for c in range(3)]
        U = [torch.from_numpy(a).to(device="cuda", dtype=dt) for a in g]
        V = [a.clone() for a in U]
        ref = [np.asfortranarray(a.to(torch.float64).cpu().numpy().transpose(2, 1, 0)) for a in U]
        du = [torch.empty_like(U[0]) for _ in range(3)]
        pg = [torch.empty_like(U[0]) for _ in range(3)]
        pp3 = torch.empty(shape[::-1], dtype=torch.float64, device="cuda")
        dv = [torch.empty_like(U[0]) for _ in range(3)]
        pv = [torch.empty_like(U[0]) for _ in range(3)]
        pq = torch.empty_like(pp3)
        lay = SlabLayout(shape, 0, 1)
        for _ in range(3):
            euler_step(ctx, U, du, pp3, pg, 1e-3, lay)
            ctx.euler_step(*V, *dv, pq, *pv, 1e-3)
            oracle.euler_step(*ref, 1e-3, lengths=lengths)
        torch.cuda.synchronize()
        tol = 1e-11 if prec == "f64" else 1e-4
        for a, b, r in zip(U, V, ref):
            assert rel_err(to_host(a), r) < tol
            assert rel_err(to_host(a), to_host(b).astype(np.float64)) < tol
        ctx.close()
    finally:
        dist.destroy_process_group()


# the last two z lengths have no fused transform (a factor 5; above 1024)
@pytest.mark.parametrize("shape,grid", [((24, 20, 16), (2, 2)), ((30, 12, 48), (3, 2)), ((16, 18, 96), (2, 3)),
                                        ((40, 24, 64), (1, 3)), ((12, 10, 40), (2, 2)), ((10, 12, 2048), (2, 3))])
def test_poisson_zpencil_on_every_rank_block(oracle, torch_cuda, shape, grid):
    """x3d_poisson_zpencil on each rank's Z pencil of the half spectrum of a
    p_row x p_col grid (x modes and y rows both cut into blocks), one block
    after another on this GPU, reassembled and transformed back, against the
    oracle's poisson_000 on the whole box."""
    torch = torch_cuda
    from x3div_b200 import Context, X3DError
    from x3div_b200.pencils import PencilLayout
    nx, ny, nz = shape
    lengths = (2 * np.pi, 1.5, 3.0)
    ctx = Context(*shape, lengths=lengths, precision="f64")
    g = np.random.default_rng(9).standard_normal(shape[::-1])
    spec = torch.fft.rfft2(torch.from_numpy(g).cuda(), norm="backward")  # (nz, ny, nx/2+1)
    out = torch.empty_like(spec)
    L = PencilLayout((nx // 2 + 1, ny, nz), grid[0], grid[1], 0)
    for r in range(grid[0] * grid[1]):
        (i0, i1), (j0, j1), _ = L.block("z", r)
        blk = spec[:, j0:j1, i0:i1].contiguous()
        ctx.poisson_zpencil(blk, i1 - i0, i0, j1 - j0, j0)
        out[:, j0:j1, i0:i1] = blk
    p = torch.fft.irfft2(out, s=(ny, nx), norm="forward")
    torch.cuda.synchronize()
    ref = oracle.poisson(np.asfortranarray(g.transpose(2, 1, 0)), *lengths)
    assert rel_err(p.cpu().numpy().transpose(2, 1, 0), ref) < 1e-12, (shape, grid)
    with pytest.raises(X3DError):  # x modes past nx/2 + 1
        ctx.poisson_zpencil(spec, nx // 2 + 1, 1, ny, 0)
    ctx.close()
