"""One box over a p_row x p_col process grid (x3div_b200/pencils.py,
2decomp's 2-D pencil decomposition; 1 x P is 2decomp's slabs): the pencil
blocks, the transpose plans, the four transposes over gloo, a whole sweep,
the Poisson solve and two Euler steps, with the oracle standing in for each
rank's kernels (tests/oracle_context.py), against the oracle on the whole
box."""
import os

import numpy as np
import pytest

from oracle_context import KIND, OracleContext, free_port
from x3div_b200.pencils import (SWEEP, PencilLayout, Pencils, copy_boxes, euler_step, plan_transpose, poisson,
                                split, sweep, transpose_x_to_y, transpose_y_to_x, transpose_y_to_z,
                                transpose_z_to_y)


def test_split_matches_2decomp_blocks():
    assert [split(10, 3, r) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [split(8, 4, r) for r in range(4)] == [(0, 2), (2, 4), (4, 6), (6, 8)]
    with pytest.raises(ValueError):
        PencilLayout((8, 2, 8), 1, 3, 0)


@pytest.mark.parametrize("grid,shape", [((2, 2), (12, 10, 9)), ((3, 2), (11, 9, 10)), ((1, 4), (8, 9, 12))])
def test_blocks_tile_the_box(grid, shape):
    p_row, p_col = grid
    for pencil in "xyz":
        seen = np.zeros(shape, dtype=int)
        for r in range(p_row * p_col):
            (x0, x1), (y0, y1), (z0, z1) = PencilLayout(shape, p_row, p_col, 0).block(pencil, r)
            seen[x0:x1, y0:y1, z0:z1] += 1
        assert (seen == 1).all(), pencil
    lay = PencilLayout(shape, p_row, p_col, p_row * p_col - 1)
    assert lay.coords() == (p_row - 1, p_col - 1)
    assert lay.extents("x")[0] == shape[0] and lay.extents("y")[1] == shape[1] and lay.extents("z")[2] == shape[2]


def test_slabs_are_one_row_of_pencils():
    """1 x P: the X and Y pencils coincide (z-slabs), the Z pencil is a
    y-slab, and only the y <-> z transposes exchange anything."""
    shape = (10, 8, 11)
    for r in range(3):
        p = PencilLayout(shape, 1, 3, r)
        assert p.extents("x") == p.extents("y") == (10, 8) + (split(11, 3, r)[1] - split(11, 3, r)[0],)
        assert p.extents("z") == (10, split(8, 3, r)[1] - split(8, 3, r)[0], 11)
        assert plan_transpose(p, "x_to_y") is None and plan_transpose(p, "y_to_x") is None
        assert plan_transpose(p, "y_to_z") is not None
    with pytest.raises(ValueError):
        PencilLayout((8, 2, 8), 3, 1, 0)


@pytest.mark.parametrize("grid,shape", [((2, 2), (12, 10, 9)), ((3, 2), (11, 9, 10)), ((2, 3), (9, 11, 10)),
                                        ((1, 4), (8, 9, 12)), ((4, 1), (9, 8, 6))])
@pytest.mark.parametrize("rest", [(), (2,)])
def test_transpose_plans_move_every_point_once(grid, shape, rest):
    """Every rank's plan, executed on host tensors with the exchange done by
    hand (member i's i-th send block to member i), rebuilds each rank's
    target pencil of a global array; a complex spectrum travels as pairs."""
    import torch
    p_row, p_col = grid
    g = np.random.default_rng(2).standard_normal(shape[::-1] + rest)
    lays = [PencilLayout(shape, p_row, p_col, r) for r in range(p_row * p_col)]
    r_ = int(np.prod(rest)) if rest else 1

    def part(L, pencil):
        (x0, x1), (y0, y1), (z0, z1) = L.block(pencil)
        return torch.from_numpy(np.ascontiguousarray(g[z0:z1, y0:y1, x0:x1]))

    for kind, src, dst in (("x_to_y", "x", "y"), ("y_to_x", "y", "x"), ("y_to_z", "y", "z"), ("z_to_y", "z", "y")):
        plans = [plan_transpose(L, kind) for L in lays]
        if plans[0] is None:
            continue
        sends = []
        for L, pl in zip(lays, plans):
            t = part(L, src)
            if pl.pack is None:
                sends.append(t.reshape(-1))
            else:
                buf = torch.empty(sum(pl.send) * r_, dtype=t.dtype)
                copy_boxes(None, buf, t, pl.pack, r_)
                sends.append(buf)
        for L, pl in zip(lays, plans):
            chunks = []
            for m in pl.members:
                mp_ = plans[m]
                i = mp_.members.index(L.rank)
                off = sum(mp_.send[:i]) * r_
                chunks.append(sends[m][off:off + mp_.send[i] * r_])
            recv = torch.cat(chunks)
            assert recv.numel() == sum(pl.recv) * r_
            if pl.unpack is None:
                got = recv.view(pl.out_shape + rest)
            else:
                got = torch.empty(pl.out_shape + rest, dtype=recv.dtype)
                copy_boxes(None, got, recv, pl.unpack, r_)
            assert np.array_equal(got.numpy(), part(L, dst).numpy()), (kind, L.rank)


def _rank(rank, grid, port, shape, fused, q):
    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    p_row, p_col = grid
    dist.init_process_group("gloo", rank=rank, world_size=p_row * p_col)
    try:
        pc = Pencils.create(shape, p_row, p_col)
        L = pc.layout
        g = np.random.default_rng(5).standard_normal(shape[::-1])  # (nz, ny, nx)

        def part(a, pencil):
            (x0, x1), (y0, y1), (z0, z1) = L.block(pencil)
            return a[z0:z1, y0:y1, x0:x1]

        mine = torch.from_numpy(part(g, "x").copy())
        fy = transpose_x_to_y(mine, pc)
        fz = transpose_y_to_z(fy, pc)
        ok = np.array_equal(fy.numpy(), part(g, "y")) and np.array_equal(fz.numpy(), part(g, "z"))
        back = transpose_y_to_x(transpose_z_to_y(fz, pc), pc)
        ok = ok and np.array_equal(back.numpy(), part(g, "x"))
        # trailing dimensions travel with their point (a complex spectrum as pairs of reals)
        g2 = np.stack([g, -g], axis=-1)
        t2 = transpose_y_to_z(transpose_x_to_y(torch.from_numpy(part(g2, "x").copy()), pc), pc)
        ok = ok and np.array_equal(t2.numpy(), part(g2, "z"))
        lengths = (2 * np.pi, 1.5, 3.0)
        ctx = OracleContext(oracle, shape, lengths, fused)
        res = sweep(ctx, mine, pc)
        gf = np.asfortranarray(g.transpose(2, 1, 0))
        err = 0.0
        for d in range(3):
            for k, (routine, _) in enumerate(SWEEP[d]):
                ref = part(oracle.apply(KIND[routine], d, gf, lengths[d] / shape[d]).transpose(2, 1, 0), "x")
                err = max(err, float(np.abs(res[d][k].numpy() - ref).max()))
        p = torch.from_numpy(part(g, "x").copy())
        poisson(ctx, p, pc)
        ref = part(oracle.poisson(gf, *lengths).transpose(2, 1, 0), "x")
        err = max(err, float(np.abs(p.numpy() - ref).max() / np.abs(ref).max()))
        # two timesteps on pencils against two on the whole box
        U = [np.random.default_rng(20 + c).standard_normal(shape[::-1]) * 0.1 for c in range(3)]
        ref = [np.asfortranarray(a.transpose(2, 1, 0)) for a in U]
        mine_u = [torch.from_numpy(part(a, "x").copy()) for a in U]
        du = [torch.empty_like(mine_u[0]) for _ in range(3)]
        pg = [torch.empty_like(mine_u[0]) for _ in range(3)]
        pp3 = torch.empty_like(mine_u[0])
        for _ in range(2):
            euler_step(ctx, mine_u, du, pp3, pg, 1e-3, pc)
            oracle.euler_step(*ref, 1e-3, lengths=lengths)
        for a, r in zip(mine_u, ref):
            rr = part(r.transpose(2, 1, 0), "x")
            err = max(err, float(np.abs(a.numpy() - rr).max() / np.abs(rr).max()))
        q.put((rank, ok, err))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("grid,shape,fused", [((2, 1), (12, 10, 9), True), ((2, 2), (12, 10, 9), True),
                                              ((2, 3), (9, 11, 10), True), ((3, 2), (10, 9, 8), True),
                                              ((2, 2), (10, 9, 8), False), ((1, 2), (12, 10, 9), True),
                                              ((1, 3), (10, 8, 11), False), ((1, 4), (9, 12, 8), True)])
def test_pencil_transposes_sweep_poisson_step_on_gloo_ranks(grid, shape, fused):
    """fused=False: the step's parts composed from single-operator routines
    (the path for pencils the fused kernels refuse)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    world = grid[0] * grid[1]
    procs = [ctx.Process(target=_rank, args=(r, grid, port, shape, fused, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [r for r, _, _ in res] == list(range(world))
    for r, ok, err in res:
        assert ok, r
        assert err < 1e-12, (r, err)
