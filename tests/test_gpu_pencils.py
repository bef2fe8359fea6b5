"""The pencil code path on the B200: the library's line solves and fused step
parts on a rank's local extents, its block-copy kernel packing and unpacking
every rank's transposes of 2-D process grids (the exchange done by hand on
this one GPU), and the step and Poisson solve through NCCL on one rank,
against the oracle on the whole box."""
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
def test_pencil_sweep_on_one_nccl_rank(oracle, torch_cuda, prec):
    torch = torch_cuda
    import torch.distributed as dist
    from x3div_b200 import Context, to_host
    from x3div_b200.pencils import SWEEP, Pencils, sweep
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
        res = sweep(ctx, field, Pencils.create(shape, 1, 1))
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
def test_pencil_poisson_on_one_nccl_rank(oracle, torch_cuda, shape):
    """The pencil Poisson solve (torch.fft x-y transforms, the half spectrum
    transposed through NCCL, x3d_poisson_zpencil on the rank's block) against
    the oracle's poisson_000 on the whole box."""
    torch = torch_cuda
    import torch.distributed as dist
    from x3div_b200 import Context
    from x3div_b200.pencils import Pencils, poisson
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        lengths = (2 * np.pi, 1.5, 3.0)
        ctx = Context(*shape, lengths=lengths, precision="f64")
        g = np.random.default_rng(8).standard_normal(shape[::-1])
        rhs = torch.from_numpy(g).cuda()
        poisson(ctx, rhs, Pencils.create(shape, 1, 1))
        torch.cuda.synchronize()
        ref = oracle.poisson(np.asfortranarray(g.transpose(2, 1, 0)), *lengths)
        assert rel_err(rhs.cpu().numpy().transpose(2, 1, 0), ref) < 1e-12, shape
        ctx.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_pencil_euler_steps_on_one_nccl_rank(oracle, torch_cuda, prec):
    """Three Euler steps composed on pencils (the fused step parts, NCCL
    transposes, the pencil Poisson solve) against the oracle and against the
    library's fused single-box step."""
    torch = torch_cuda
    import torch.distributed as dist
    from x3div_b200 import Context, to_host
    from x3div_b200.pencils import Pencils, euler_step
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
        lay = Pencils.create(shape, 1, 1)
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


@pytest.mark.parametrize("grid,shape", [((2, 2), (24, 20, 16)), ((3, 2), (11, 9, 10)), ((2, 3), (30, 12, 48)),
                                        ((1, 4), (16, 8, 12)), ((4, 1), (9, 8, 10))])
@pytest.mark.parametrize("dtype,rest", [("f32", ()), ("f64", ()), ("f64", (2,)), ("f32", (2,))])
def test_block_copies_run_every_rank_transpose(torch_cuda, grid, shape, dtype, rest):
    """x3d_copy_blocks executes every rank's pack and unpack plan of the four
    transposes on device pencils of a global array, the exchange done by hand
    (member i's i-th send block to member i): bit-exact against the target
    pencils.  Odd extents take the 4-byte path, the rest 16-byte vectors."""
    torch = torch_cuda
    from x3div_b200 import Context
    from x3div_b200.pencils import PencilLayout, copy_boxes, plan_transpose
    p_row, p_col = grid
    dt = torch.float32 if dtype == "f32" else torch.float64
    ctx = Context(*shape, precision=dtype)
    g = torch.randn(shape[::-1] + rest, dtype=torch.float64, generator=torch.Generator().manual_seed(4)).to(dt)
    gd = g.cuda()
    lays = [PencilLayout(shape, p_row, p_col, r) for r in range(p_row * p_col)]
    r_ = int(np.prod(rest)) if rest else 1

    def part(L, pencil, a):
        (x0, x1), (y0, y1), (z0, z1) = L.block(pencil)
        return a[z0:z1, y0:y1, x0:x1].contiguous()

    n0 = ctx.launch_count()
    for kind, src, dst in (("x_to_y", "x", "y"), ("y_to_x", "y", "x"), ("y_to_z", "y", "z"), ("z_to_y", "z", "y")):
        plans = [plan_transpose(L, kind) for L in lays]
        if plans[0] is None:
            continue
        sends = []
        for L, pl in zip(lays, plans):
            t = part(L, src, gd)
            if pl.pack is None:
                sends.append(t.reshape(-1))
            else:
                buf = torch.full((sum(pl.send) * r_,), float("nan"), dtype=dt, device="cuda")
                copy_boxes(ctx, buf, t, pl.pack, r_)
                sends.append(buf)
        for L, pl in zip(lays, plans):
            chunks = []
            for m in pl.members:
                mp_ = plans[m]
                i = mp_.members.index(L.rank)
                off = sum(mp_.send[:i]) * r_
                chunks.append(sends[m][off:off + mp_.send[i] * r_])
            recv = torch.cat(chunks)
            if pl.unpack is None:
                got = recv.view(pl.out_shape + rest)
            else:
                got = torch.full(pl.out_shape + rest, float("nan"), dtype=dt, device="cuda")
                copy_boxes(ctx, got, recv, pl.unpack, r_)
            torch.cuda.synchronize()
            assert torch.equal(got.cpu(), part(L, dst, g)), (kind, L.rank)
    assert ctx.launch_count() > n0  # the copies ran as library launches
    ctx.close()


def _stage_refs(oracle, U, lengths, shape):
    """The step's stage outputs on the whole box (FP64, C order), from the
    oracle's single-operator applications: the reference for every pencil
    part."""
    d = [L / n for L, n in zip(lengths, shape)]

    def A(kind, k, a):
        f = np.asfortranarray(a.transpose(2, 1, 0))
        return np.ascontiguousarray(oracle.apply(kind, k, f, d[k]).transpose(2, 1, 0))

    u = U
    ref = {}
    ref["transeq"] = {k: [A("der", k, u[k] * u[c]) + u[k] * A("der", k, u[c]) for c in range(3)] for k in range(3)}
    ref["div0"] = [A("dervp", 0, u[0]), A("intvp", 0, u[1]), A("intvp", 0, u[2])]
    ref["div1"] = [A("dervp", 1, ref["div0"][1]) + A("intvp", 1, ref["div0"][0]), A("intvp", 1, ref["div0"][2])]
    ref["div2"] = [A("intvp", 2, ref["div1"][0]) + A("dervp", 2, ref["div1"][1])]
    p = U[3]
    ref["grad2"] = [A("intpv", 2, p), A("derpv", 2, p)]
    ref["grad1"] = [A("intpv", 1, ref["grad2"][0]), A("derpv", 1, ref["grad2"][0]), A("intpv", 1, ref["grad2"][1])]
    ref["grad0"] = [A("derpv", 0, ref["grad1"][0]), A("intpv", 0, ref["grad1"][1]), A("intpv", 0, ref["grad1"][2])]
    return ref


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("grid,shape", [((2, 3), (24, 36, 32)), ((3, 2), (48, 24, 40)), ((2, 2), (30, 16, 24))])
def test_step_parts_on_every_rank_pencil(oracle, torch_cuda, prec, grid, shape):
    """x3d_transeq_part, x3d_divergence_part and x3d_gradp_part on each
    rank's X, Y and Z pencil of a 2-D process grid (local extents below the
    box's across the lines), fed the whole-box stage inputs restricted to the
    pencil, against the whole-box stage outputs restricted the same way.
    Pencils the fused kernels refuse (an x extent of 15 across y/z lines;
    FP32 x lines of 30 points) raise X3D_EUNSUPPORTED and go through the
    pencil module's composition from single-operator routines, which must
    agree too."""
    torch = torch_cuda
    from x3div_b200 import Context, X3DError
    from x3div_b200 import pencils as P
    from x3div_b200._capi import X3D_EUNSUPPORTED
    lengths = (2 * np.pi, 1.5, 3.0)
    dt_ = torch.float64 if prec == "f64" else torch.float32
    rng = np.random.default_rng(12)
    # fields as stored in the context's precision; the reference reads those values
    U = [rng.standard_normal(shape[::-1]) * 0.1 for _ in range(3)] + [rng.standard_normal(shape[::-1])]
    U = [np.asarray(torch.from_numpy(a).to(dt_).double().numpy()) for a in U[:3]] + [U[3]]
    ref = _stage_refs(oracle, U, lengths, shape)
    # the stage inputs as the library would hold them between parts
    stored = lambda a: torch.from_numpy(a).to(dt_).double().numpy()  # noqa: E731
    ctx = Context(*shape, lengths=lengths, precision=prec)
    # FP32: the part's inputs are rounded to FP32 between stages, and an
    # interpolation alone is ~6e-6 in FP32 (as in the one-box stage tests)
    tol = 1e-12 if prec == "f64" else 1e-4
    step_dt = 1e-3
    refused = 0
    for r in range(grid[0] * grid[1]):
        L = P.PencilLayout(shape, grid[0], grid[1], r)
        for k, pencil in enumerate("xyz"):
            (x0, x1), (y0, y1), (z0, z1) = L.block(pencil)
            ext = L.extents(pencil)
            cut = lambda a: np.ascontiguousarray(a[z0:z1, y0:y1, x0:x1])  # noqa: E731
            dev = lambda a, dtype=dt_: torch.from_numpy(cut(a)).to(device="cuda", dtype=dtype)  # noqa: E731

            def run(fn, *args):
                nonlocal refused
                try:
                    fn(*args)
                except X3DError as e:
                    assert e.code == X3D_EUNSUPPORTED, e
                    refused += 1
                    return False
                return True

            # momentum terms + an addend, with int_time into fresh arrays
            u = [dev(a) for a in U[:3]]
            add = [dev(a) for a in U[:3]]
            du = [torch.empty_like(u[0]) for _ in range(3)]
            un = [torch.empty_like(u[0]) for _ in range(3)]
            if not run(ctx.transeq_part, k, du, u, add, un, step_dt, ext):
                P._transeq_part(ctx, k, du, u, add, un, step_dt, ext)
            torch.cuda.synchronize()
            for c in range(3):
                want = cut(U[c]) + cut(ref["transeq"][k][c])
                assert rel_err(du[c].double().cpu().numpy(), want) < tol, (r, pencil, c)
                assert rel_err(un[c].double().cpu().numpy(), cut(U[c]) + step_dt * want) < tol, (r, pencil, c)
            # divergence
            ins = {0: U[:3], 1: [stored(a) for a in ref["div0"]], 2: [stored(a) for a in ref["div1"]]}[k]
            out = [torch.empty(L.tensor_shape(pencil), dtype=torch.float64 if k == 2 else dt_, device="cuda")
                   for _ in range({0: 3, 1: 2, 2: 1}[k])]
            args = (k, out, [dev(a) for a in ins], ext)
            if not run(ctx.divergence_part, *args):
                P._divergence_part(ctx, *args)
            torch.cuda.synchronize()
            for o, w in zip(out, ref[f"div{k}"]):
                assert rel_err(o.double().cpu().numpy(), cut(w)) < tol, (r, pencil, "div")
            # gradp, the x part with cor_vel on a copy of u
            ins = {2: [U[3]], 1: [stored(a) for a in ref["grad2"]], 0: [stored(a) for a in ref["grad1"]]}[k]
            din = [dev(a, torch.float64) for a in ins] if k == 2 else [dev(a) for a in ins]
            out = [torch.empty(L.tensor_shape(pencil), dtype=dt_, device="cuda") for _ in range({2: 2, 1: 3, 0: 3}[k])]
            uc = [dev(a) for a in U[:3]] if k == 0 else None
            args = (k, out, din, uc, ext)
            if not run(ctx.gradp_part, *args):
                P._gradp_part(ctx, *args)
            torch.cuda.synchronize()
            for c, (o, w) in enumerate(zip(out, ref[f"grad{k}"])):
                assert rel_err(o.double().cpu().numpy(), cut(w)) < tol, (r, pencil, "grad")
                if uc is not None:
                    assert rel_err(uc[c].double().cpu().numpy(), cut(U[c]) - cut(w)) < tol, (r, pencil, "cor")
    # only the x extent of 15 (rows of 60 or 120 bytes: no 16-byte tensor
    # copies) and FP32 x lines of 30 points are refused
    assert (refused > 0) == (shape[0] == 30), refused
    ctx.close()


def test_pencil_entry_points_refuse_bad_arguments(torch_cuda):
    """x3d_copy_blocks and the step parts check their arguments before
    launching anything: element sizes, negative offsets or strides, host
    arrays, directions, and pencils whose lines along their direction are
    not whole; the context keeps working afterwards."""
    torch = torch_cuda
    from x3div_b200 import Context, X3DError
    from x3div_b200._capi import X3D_EINVAL
    ctx = Context(16, 12, 10, precision="f32")
    a = torch.zeros(10, 12, 16, device="cuda")
    b = torch.zeros_like(a)
    good = (0, 0, 16, 12, 10, 16, 192, 16, 192)
    for elem, box in ((12, good), (4, (-1,) + good[1:]), (4, good[:5] + (-16,) + good[6:])):
        with pytest.raises(X3DError) as e:
            ctx.copy_blocks(b, a, elem, [box])
        assert e.value.code == X3D_EINVAL
    host = torch.zeros(10, 12, 16)
    with pytest.raises(X3DError):
        ctx.copy_blocks(b, host, 4, [good])
    u = [torch.zeros(10, 12, 16, device="cuda") for _ in range(3)]
    du = [torch.empty_like(u[0]) for _ in range(3)]
    with pytest.raises(X3DError):
        ctx.transeq_part(3, du, u, None, None, 0.0, (16, 12, 10))  # no fourth direction
    with pytest.raises(X3DError):
        ctx.transeq_part(0, du, u, None, None, 0.0, (15, 12, 10))  # x lines cut short
    with pytest.raises(X3DError):
        ctx.divergence_part(1, du[:2], u, (16, 13, 10))  # extents outside the box
    with pytest.raises(X3DError):
        ctx.gradp_part(0, du, [host, host, host], None, (16, 12, 10))  # host arrays
    # still usable: a valid copy and a valid part
    ctx.copy_blocks(b, a, 4, [good])
    ctx.transeq_part(0, du, u, None, None, 0.0, (16, 12, 10))
    ctx.sync()
    assert torch.equal(b, a)
    ctx.close()
