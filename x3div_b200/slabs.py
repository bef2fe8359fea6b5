"""One periodic box over P ranks: 2decomp's 1 x P pencil decomposition.

With p_row = 1 and p_col = P, the X and Y pencils of 2decomp coincide: each
rank holds whole x lines and whole y lines of a block of z planes (a z-slab,
(nx, ny, nz_r) in Fortran order).  A Z pencil holds whole z lines of a block of
y rows (a y-slab, (nx, ny_r, nz)).  Lines are never split, so every line-solve
routine of the library runs unchanged on a rank's slab with its local extents
(e.g. x3d_derz(ctx, t, u, op, nx, ny_r, nz) on a y-slab, with the context and
operators made for the global box).  x3d_transpose_x_to_y and y_to_x are
local; the y <-> z transposes (x3d_transpose_y_to_z / z_to_y,
src/x3d_transpose.f90:77-130, 2decomp's transpose_y_to_z / transpose_z_to_y)
become one all-to-all each: rank r sends rank s the block of its slab that s
owns in the other layout.  Blocks follow 2decomp's distribution: the first
n mod P ranks hold one plane more.

Device tensors are C-ordered (nz, ny, nx) views of the Fortran (nx, ny, nz)
layout, as in the rest of the package.  The collectives go through
torch.distributed: NCCL over NVLink for CUDA tensors, gloo for CPU tensors.
"""
from __future__ import annotations

from dataclasses import dataclass


def split(n: int, parts: int, rank: int):
    """[start, end) of block `rank` when n points are cut into `parts` blocks,
    the first n mod parts blocks one point longer."""
    if parts < 1 or not 0 <= rank < parts:
        raise ValueError("bad block request")
    base, extra = divmod(n, parts)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


@dataclass(frozen=True)
class SlabLayout:
    """Where rank `rank` of `world` keeps its part of an (nx, ny, nz) box."""
    shape: tuple
    rank: int
    world: int

    def __post_init__(self):
        nx, ny, nz = self.shape
        if ny < self.world or nz < self.world:
            raise ValueError("need at least one y row and one z plane per rank")

    def zslab(self, r=None):
        """[z0, z1): the z planes of rank r's X/Y pencil (default: this rank)."""
        return split(self.shape[2], self.world, self.rank if r is None else r)

    def yslab(self, r=None):
        """[y0, y1): the y rows of rank r's Z pencil (default: this rank)."""
        return split(self.shape[1], self.world, self.rank if r is None else r)

    @property
    def xy_extents(self):
        """(nx, ny, nz_r): local extents of this rank's X/Y pencil."""
        z0, z1 = self.zslab()
        return self.shape[0], self.shape[1], z1 - z0

    @property
    def z_extents(self):
        """(nx, ny_r, nz): local extents of this rank's Z pencil."""
        y0, y1 = self.yslab()
        return self.shape[0], y1 - y0, self.shape[2]


def _all_to_all(recv, send, out_splits, in_splits, group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.all_to_all_single(recv, send, out_splits, in_splits, group=group)
    else:  # one rank: the exchange is a copy
        recv.copy_(send)


def transpose_y_to_z(zslab, layout: SlabLayout, group=None):
    """X/Y pencil (a (nz_r, ny, nx) tensor) -> Z pencil ((nz, ny_s, nx) on
    rank s): 2decomp's transpose_y_to_z at p_row = 1."""
    import torch
    nx, ny, nz = layout.shape
    z0, z1 = layout.zslab()
    if tuple(zslab.shape) != (z1 - z0, ny, nx):
        raise ValueError("not this rank's X/Y pencil")
    blocks = [zslab[:, y0:y1, :].reshape(-1) for y0, y1 in (layout.yslab(s) for s in range(layout.world))]
    send = torch.cat(blocks)
    y0, y1 = layout.yslab()
    out_splits = [(b - a) * (y1 - y0) * nx for a, b in (layout.zslab(r) for r in range(layout.world))]
    recv = torch.empty(sum(out_splits), dtype=zslab.dtype, device=zslab.device)
    _all_to_all(recv, send, out_splits, [b.numel() for b in blocks], group)
    out = torch.empty((nz, y1 - y0, nx), dtype=zslab.dtype, device=zslab.device)
    off = 0
    for r in range(layout.world):
        a, b = layout.zslab(r)
        n = out_splits[r]
        out[a:b] = recv[off:off + n].view(b - a, y1 - y0, nx)
        off += n
    return out


def transpose_z_to_y(yslab, layout: SlabLayout, group=None):
    """Z pencil ((nz, ny_r, nx)) -> X/Y pencil ((nz_s, ny, nx) on rank s):
    2decomp's transpose_z_to_y at p_row = 1."""
    import torch
    nx, ny, nz = layout.shape
    y0, y1 = layout.yslab()
    if tuple(yslab.shape) != (nz, y1 - y0, nx):
        raise ValueError("not this rank's Z pencil")
    blocks = [yslab[a:b].reshape(-1) for a, b in (layout.zslab(s) for s in range(layout.world))]
    send = torch.cat(blocks)
    z0, z1 = layout.zslab()
    out_splits = [(z1 - z0) * (b - a) * nx for a, b in (layout.yslab(r) for r in range(layout.world))]
    recv = torch.empty(sum(out_splits), dtype=yslab.dtype, device=yslab.device)
    _all_to_all(recv, send, out_splits, [b.numel() for b in blocks], group)
    out = torch.empty((z1 - z0, ny, nx), dtype=yslab.dtype, device=yslab.device)
    off = 0
    for r in range(layout.world):
        a, b = layout.yslab(r)
        n = out_splits[r]
        out[:, a:b, :] = recv[off:off + n].view(z1 - z0, b - a, nx)
        off += n
    return out


# The six operator families of a sweep, by direction: (routine, operator).
SWEEP = {
    0: [("derx", "derx"), ("derxx", "derxx"), ("derxvp", "derxvp"), ("derxpv", "derxpv"),
        ("interxvp", "intxvp"), ("interxpv", "intxpv")],
    1: [("dery", "dery"), ("deryy", "deryy"), ("deryvp", "deryvp"), ("derypv", "derypv"),
        ("interyvp", "intyvp"), ("interypv", "intypv")],
    2: [("derz", "derz"), ("derzz", "derzz"), ("derzvp", "derzvp"), ("derzpv", "derzpv"),
        ("interzvp", "intzvp"), ("interzpv", "intzpv")],
}


def _call(ctx, routine, t, u, op, ext):
    nx, ny, nz = ext
    fn = getattr(ctx, routine)
    if routine in ("dery",):
        fn(t, u, op, None, nx, ny, nz)
    elif routine in ("deryvp", "derypv"):
        fn(t, u, op, None, nx, ny, ny, nz)
    elif routine.endswith(("xvp", "xpv")):
        fn(t, u, op, nx, nx, ny, nz)
    elif routine.endswith(("yvp", "ypv")):
        fn(t, u, op, nx, ny, ny, nz)
    elif routine.endswith(("zvp", "zpv")):
        fn(t, u, op, nx, ny, nz, nz)
    else:
        fn(t, u, op, nx, ny, nz)


def sweep(ctx, field, layout: SlabLayout, group=None):
    """The 18 operator applications of a sweep on one field of a box that is
    spread over the ranks: x and y families on the rank's X/Y pencil, z
    families on its Z pencil (one transpose each way).  ctx is a periodic
    context made for the global box; field is the rank's X/Y pencil.  Returns
    {direction: [six outputs in X/Y-pencil layout]}."""
    import torch
    ext = layout.xy_extents
    out = {}
    for d in (0, 1):
        res = []
        for routine, opname in SWEEP[d]:
            t = torch.empty_like(field)
            _call(ctx, routine, t, field, ctx.op(opname), ext)
            res.append(t)
        out[d] = res
    zp = transpose_y_to_z(field, layout, group)
    zext = layout.z_extents
    res = []
    for routine, opname in SWEEP[2]:
        t = torch.empty_like(zp)
        _call(ctx, routine, t, zp, ctx.op(opname), zext)
        res.append(transpose_z_to_y(t, layout, group))
    out[2] = res
    return out


def poisson(ctx, rhs, layout: SlabLayout, group=None):
    """poisson_000 (src/poisson.f90:276-419) on a box spread over the ranks,
    in place on this rank's X/Y pencil of the FP64 field ((nz_r, ny, nx)).
    The 2-D x-y transforms of the rank's z planes (cuFFT through torch.fft,
    unnormalised both ways) bracket the z part, which runs on the rank's
    block of y rows after a transpose of the half spectrum
    (x3d_poisson_zlines: z transforms and the mode division)."""
    import torch
    nx, ny, nz = layout.shape
    nxh = nx // 2 + 1
    spec = torch.fft.rfft2(rhs, norm="backward")  # (nz_r, ny, nxh)
    half = SlabLayout((2 * nxh, ny, nz), layout.rank, layout.world)  # the spectrum as 2 nxh reals per row
    zs = transpose_y_to_z(torch.view_as_real(spec).reshape(spec.shape[0], ny, 2 * nxh), half, group)
    y0, y1 = layout.yslab()
    ctx.poisson_zlines(torch.view_as_complex(zs.view(nz, y1 - y0, nxh, 2)), y1 - y0, y0)
    back = transpose_z_to_y(zs, half, group)
    z0, z1 = layout.zslab()
    rhs.copy_(torch.fft.irfft2(torch.view_as_complex(back.view(z1 - z0, ny, nxh, 2)), s=(ny, nx), norm="forward"))
    return rhs


def _apply(ctx, routine, opname, u, ext):
    import torch
    t = torch.empty_like(u)
    _call(ctx, routine, t, u, ctx.op(opname), ext)
    return t


def euler_step(ctx, u, du, pp3, pg, dt, layout: SlabLayout, group=None):
    """One timestep (src/xcompact3d.f90:80-95) on a box spread over the
    ranks, from the library's line solves on local extents, elementwise
    tensor arithmetic and the slab transposes, in the reference's order:
    momentum_rhs_eq (src/transeq.f90:44-355) with the x and y parts on the
    rank's X/Y pencil and the z part on its Z pencil; int_time
    (src/time_integrators.f90:40-44); divergence (src/navier.f90:98-236)
    into the FP64 pp3; the slab Poisson solve; gradp
    (src/navier.f90:249-359) and cor_vel (:64-91).  u, du, pg: the three
    velocity, increment and pressure-gradient components as this rank's X/Y
    pencils; pp3: its FP64 X/Y pencil.  In place, like x3d_euler_step."""
    import torch
    ext, zext = layout.xy_extents, layout.z_extents
    T = lambda a: transpose_y_to_z(a, layout, group)  # noqa: E731
    Ti = lambda a: transpose_z_to_y(a, layout, group)  # noqa: E731
    ux, uy, uz = u
    uzz = T(uz)
    for c in range(3):  # calculate_transeq_rhs
        uc = u[c]
        ta = ux * uc
        td = _apply(ctx, "derx", "derx", ta, ext)
        ta = _apply(ctx, "derx", "derx", uc, ext)
        duc = td + ux * ta
        td = uc * uy
        tg = _apply(ctx, "dery", "dery", td, ext)
        td = _apply(ctx, "dery", "dery", uc, ext)
        tg = tg + uy * td
        ucz = uzz if c == 2 else T(uc)
        tdz = ucz * uzz
        tgz = _apply(ctx, "derz", "derz", tdz, zext)
        tdz = _apply(ctx, "derz", "derz", ucz, zext)
        tg = tg + Ti(tgz + uzz * tdz)
        du[c].copy_(duc + tg)
    for c in range(3):  # int_time, Euler: u = dt du + u
        u[c].copy_(dt * du[c] + u[c])
    # divergence
    pp1 = _apply(ctx, "derxvp", "derxvp", ux, ext)
    pgy1 = _apply(ctx, "interxvp", "intxvp", uy, ext)
    pgz1 = _apply(ctx, "interxvp", "intxvp", uz, ext)
    upi2 = _apply(ctx, "interyvp", "intyvp", pp1, ext)
    duydypi2 = _apply(ctx, "deryvp", "deryvp", pgy1, ext) + upi2
    upi2 = _apply(ctx, "interyvp", "intyvp", pgz1, ext)
    a, b = T(duydypi2), T(upi2)
    p3 = _apply(ctx, "interzvp", "intzvp", a, zext).double() + _apply(ctx, "derzvp", "derzvp", b, zext).double()
    pp3.copy_(Ti(p3))
    poisson(ctx, pp3, layout, group)
    # gradp + cor_vel
    p3z = T(pp3).to(ux.dtype)
    ppi3 = Ti(_apply(ctx, "interzpv", "intzpv", p3z, zext))
    pgz3 = Ti(_apply(ctx, "derzpv", "derzpv", p3z, zext))
    ppi2 = _apply(ctx, "interypv", "intypv", ppi3, ext)
    pgy2 = _apply(ctx, "derypv", "derypv", ppi3, ext)
    pgzi2 = _apply(ctx, "interypv", "intypv", pgz3, ext)
    pg[0].copy_(_apply(ctx, "derxpv", "derxpv", ppi2, ext))
    pg[1].copy_(_apply(ctx, "interxpv", "intxpv", pgy2, ext))
    pg[2].copy_(_apply(ctx, "interxpv", "intxpv", pgzi2, ext))
    for c in range(3):
        u[c].sub_(pg[c])
