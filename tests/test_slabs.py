"""One box over several ranks (x3div_b200/slabs.py, 2decomp's 1 x P
decomposition): block splits, the y <-> z transposes over gloo, a whole
sweep, the Poisson solve and two Euler steps on slabs, with the oracle
standing in for each rank's kernels, against the oracle on the whole box."""
import os
import socket

import numpy as np
import pytest

from x3div_b200.slabs import (SWEEP, SlabLayout, euler_step, poisson, split, sweep, transpose_y_to_z,
                              transpose_z_to_y)

KIND = {"derx": "der", "dery": "der", "derz": "der", "derxx": "der2", "deryy": "der2", "derzz": "der2",
        "derxvp": "dervp", "deryvp": "dervp", "derzvp": "dervp", "derxpv": "derpv", "derypv": "derpv",
        "derzpv": "derpv", "interxvp": "intvp", "interyvp": "intvp", "interzvp": "intvp",
        "interxpv": "intpv", "interypv": "intpv", "interzpv": "intpv"}


def test_split_matches_2decomp_blocks():
    assert [split(10, 3, r) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [split(8, 4, r) for r in range(4)] == [(0, 2), (2, 4), (4, 6), (6, 8)]
    with pytest.raises(ValueError):
        SlabLayout((8, 2, 8), 0, 3)


class OracleContext:
    """A stand-in for x3div_b200.Context on CPU tensors: each routine applies
    the oracle along its direction to the given local extents (whole lines),
    so the slab code runs unchanged."""

    def __init__(self, oracle, shape, lengths):
        self.o = oracle
        self.shape = shape
        self.lengths = lengths
        self.d = [L / n for L, n in zip(lengths, shape)]

    def op(self, name):
        return name

    def poisson_zpencil(self, spec, nxh_loc, i0, ny_loc, j0):
        """The z part of the spectral solve, restated with numpy's FFT and the
        oracle's modified-wavenumber tables, on a (nz, ny_loc, nxh_loc) block
        of x modes from i0 and y rows from j0."""
        import torch
        nx, ny, nz = self.shape
        t = self.o.poisson_tables(nx, ny, nz, *self.lengths)
        c = np.fft.fft(spec.numpy(), axis=0)
        i = (i0 + np.arange(nxh_loc))[None, None, :]
        j = (j0 + np.arange(ny_loc))[None, :, None]
        k = np.arange(nz)[:, None, None]
        tyz = t["ty"][j] * t["tz"][k]
        txz = t["tx"][i] * t["tz"][k]
        txy = t["tx"][i] * t["ty"][j]
        kk = t["k2x"][i] * tyz ** 2 + t["k2y"][j] * txz ** 2 + t["k2z"][k] * txy ** 2
        f = np.where(kk < 1e-16, 0.0, -1.0 / (np.where(kk < 1e-16, 1.0, kk) * (nx * ny * nz)))
        spec.copy_(torch.from_numpy(np.fft.ifft(c * f, axis=0) * nz))

    def __getattr__(self, routine):
        if routine not in KIND:
            raise AttributeError(routine)
        direction = "xyz".index(routine.replace("inter", "").replace("der", "")[0])

        def call(t, u, op, *extents):
            import torch
            f = np.asfortranarray(u.numpy().transpose(2, 1, 0))  # the local (nx, ny_r or ny, nz_r or nz)
            r = self.o.apply(KIND[routine], direction, f, self.d[direction])
            t.copy_(torch.from_numpy(np.ascontiguousarray(r.transpose(2, 1, 0))))
        return call


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, shape, q):
    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lay = SlabLayout(shape, rank, world)
        g = np.random.default_rng(5).standard_normal(shape[::-1])  # (nz, ny, nx)
        z0, z1 = lay.zslab()
        y0, y1 = lay.yslab()
        mine = torch.from_numpy(g[z0:z1].copy())
        zp = transpose_y_to_z(mine, lay)
        ok = np.array_equal(zp.numpy(), g[:, y0:y1, :])
        back = transpose_z_to_y(zp, lay)
        ok = ok and np.array_equal(back.numpy(), g[z0:z1])
        lengths = (2 * np.pi, 1.5, 3.0)
        ctx = OracleContext(oracle, shape, lengths)
        res = sweep(ctx, mine, lay)
        gf = np.asfortranarray(g.transpose(2, 1, 0))
        err = 0.0
        for d in range(3):
            for k, (routine, _) in enumerate(SWEEP[d]):
                ref = oracle.apply(KIND[routine], d, gf, lengths[d] / shape[d]).transpose(2, 1, 0)[z0:z1]
                err = max(err, float(np.abs(res[d][k].numpy() - ref).max()))
        p = torch.from_numpy(g[z0:z1].copy())
        poisson(ctx, p, lay)
        ref = oracle.poisson(gf, *lengths).transpose(2, 1, 0)[z0:z1]
        err = max(err, float(np.abs(p.numpy() - ref).max() / np.abs(ref).max()))
        # two timesteps on slabs against two on the whole box
        U = [np.random.default_rng(20 + c).standard_normal(shape[::-1]) * 0.1 for c in range(3)]
        ref = [np.asfortranarray(a.transpose(2, 1, 0)) for a in U]
        mine_u = [torch.from_numpy(a[z0:z1].copy()) for a in U]
        du = [torch.empty_like(mine_u[0]) for _ in range(3)]
        pg = [torch.empty_like(mine_u[0]) for _ in range(3)]
        pp3 = torch.empty_like(mine_u[0])
        for _ in range(2):
            euler_step(ctx, mine_u, du, pp3, pg, 1e-3, lay)
            oracle.euler_step(*ref, 1e-3, lengths=lengths)
        for a, r in zip(mine_u, ref):
            rr = r.transpose(2, 1, 0)[z0:z1]
            err = max(err, float(np.abs(a.numpy() - rr).max() / np.abs(rr).max()))
        q.put((rank, ok, err))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,shape", [(2, (12, 10, 9)), (3, (10, 8, 11)), (4, (9, 12, 8))])
def test_slab_transposes_and_sweep_on_gloo_ranks(world, shape):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, shape, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [r for r, _, _ in res] == list(range(world))
    for r, ok, err in res:
        assert ok, r
        assert err < 1e-12, (r, err)
