"""One periodic box over p_row x p_col ranks: 2decomp's 2-D pencil
decomposition.

Rank r sits at (row, col) = (r // p_col, r % p_col) of the process grid
(2decomp's MPI_CART_CREATE over dims (p_row, p_col)).  Its three pencils
hold whole lines of one direction (2decomp's xstart/xend, ystart/yend,
zstart/zend, 0-based and half-open here):

    X pencil: all nx,  y block `row` of p_row, z block `col` of p_col
    Y pencil: x block `row` of p_row,  all ny, z block `col` of p_col
    Z pencil: x block `row` of p_row,  y block `col` of p_col,  all nz

The x <-> y transposes (2decomp's transpose_x_to_y / y_to_x, called by
src/x3d_transpose.f90:16-60 and src/navier.f90:171-190) exchange blocks among
the p_row ranks of one process-grid column, the y <-> z transposes
(transpose_y_to_z / z_to_y, src/x3d_transpose.f90:77-130) among the p_col
ranks of one row: one all-to-all each.  Lines are never split, so every
line-solve routine of the library runs unchanged on a pencil with its local
extents and a context made for the global box.  With p_row = 1 the X and Y
pencils coincide (x3div_b200.slabs).

Device tensors are C-ordered (z, y, x) views of the Fortran (x, y, z)
layout, with any trailing dimensions carried along (a complex spectrum as
(..., 2) reals).  The collectives go through torch.distributed: NCCL over
NVLink for CUDA tensors, gloo for CPU tensors.
"""
from __future__ import annotations

from dataclasses import dataclass


def split(n: int, parts: int, rank: int):
    """[start, end) of block `rank` when n points are cut into `parts` blocks,
    the first n mod parts blocks one point longer (2decomp's distribution)."""
    if parts < 1 or not 0 <= rank < parts:
        raise ValueError("bad block request")
    base, extra = divmod(n, parts)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


@dataclass(frozen=True)
class PencilLayout:
    """Where rank `rank` of a p_row x p_col grid keeps its pencils of an
    (nx, ny, nz) box."""
    shape: tuple
    p_row: int
    p_col: int
    rank: int

    def __post_init__(self):
        nx, ny, nz = self.shape
        if self.p_row < 1 or self.p_col < 1 or not 0 <= self.rank < self.p_row * self.p_col:
            raise ValueError("bad process grid")
        if min(nx, ny) < self.p_row or min(ny, nz) < self.p_col:
            raise ValueError("need at least one point per block")

    def coords(self, r=None):
        """(row, col) of rank r in the process grid (default: this rank)."""
        r = self.rank if r is None else r
        return divmod(r, self.p_col)

    def block(self, pencil, r=None):
        """((x0, x1), (y0, y1), (z0, z1)) of rank r's `pencil` ('x', 'y' or
        'z')."""
        row, col = self.coords(r)
        nx, ny, nz = self.shape
        if pencil == "x":
            return (0, nx), split(ny, self.p_row, row), split(nz, self.p_col, col)
        if pencil == "y":
            return split(nx, self.p_row, row), (0, ny), split(nz, self.p_col, col)
        if pencil == "z":
            return split(nx, self.p_row, row), split(ny, self.p_col, col), (0, nz)
        raise ValueError("pencil is 'x', 'y' or 'z'")

    def extents(self, pencil, r=None):
        """(nx_l, ny_l, nz_l): local extents of rank r's `pencil`."""
        return tuple(b - a for a, b in self.block(pencil, r))

    def tensor_shape(self, pencil, r=None):
        """The C-ordered (z, y, x) shape of rank r's `pencil`."""
        return tuple(reversed(self.extents(pencil, r)))

    def xy_members(self):
        """Ranks of this rank's process-grid column, by row: the x <-> y
        transpose group (2decomp's DECOMP_2D_COMM_COL)."""
        _, col = self.coords()
        return [r * self.p_col + col for r in range(self.p_row)]

    def yz_members(self):
        """Ranks of this rank's process-grid row, by column: the y <-> z
        transpose group (2decomp's DECOMP_2D_COMM_ROW)."""
        row, _ = self.coords()
        return [row * self.p_col + c for c in range(self.p_col)]

    def with_shape(self, shape):
        """The same process grid over another box (e.g. the half spectrum)."""
        return PencilLayout(tuple(shape), self.p_row, self.p_col, self.rank)


class Pencils:
    """A PencilLayout with the process groups its transposes use.  Build one
    with Pencils.create on every rank (the group creation is collective)."""

    def __init__(self, layout: PencilLayout, xy_group=None, yz_group=None):
        self.layout = layout
        self.xy_group = xy_group
        self.yz_group = yz_group

    @classmethod
    def create(cls, shape, p_row, p_col):
        """The decomposition of `shape` over the default process group as a
        p_row x p_col grid (1 x 1 without torch.distributed).  Every rank
        calls it, in the same order as its other group creations."""
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized()):
            if p_row * p_col != 1:
                raise ValueError("a process grid above 1 x 1 needs torch.distributed")
            return cls(PencilLayout(tuple(shape), 1, 1, 0))
        world, rank = dist.get_world_size(), dist.get_rank()
        if p_row * p_col != world:
            raise ValueError("p_row * p_col must equal the world size")
        layout = PencilLayout(tuple(shape), p_row, p_col, rank)
        row, col = layout.coords()
        xy = yz = None
        # every rank creates every group, in the same order
        if 1 < p_row < world:
            for c in range(p_col):
                g = dist.new_group([r * p_col + c for r in range(p_row)])
                if c == col:
                    xy = g
        if 1 < p_col < world:
            for r in range(p_row):
                g = dist.new_group([r * p_col + c for c in range(p_col)])
                if r == row:
                    yz = g
        return cls(layout, xy, yz)

    def with_shape(self, shape):
        """The same ranks and groups over another box."""
        return Pencils(self.layout.with_shape(shape), self.xy_group, self.yz_group)


def _exchange(send_blocks, recv_shapes, group, members, like, send_flat=None):
    """All-to-all among `members` (this rank's group, in group-rank order):
    block i of send_blocks goes to members[i]; returns the blocks received,
    block i from members[i], shaped recv_shapes[i], and the flat receive
    buffer that holds them in that order.  send_flat, when given, already
    holds the send blocks back to back (no packing copy)."""
    import torch
    if len(members) == 1:
        blk = send_blocks[0].reshape(recv_shapes[0])
        return [blk], blk.reshape(-1)
    import torch.distributed as dist
    in_splits = [b.numel() for b in send_blocks]
    if send_flat is None:
        # each block is packed once, straight into its slot of the send buffer
        send_flat = torch.empty(sum(in_splits), dtype=like.dtype, device=like.device)
        off = 0
        for b, n in zip(send_blocks, in_splits):
            send_flat[off:off + n].view(b.shape).copy_(b)
            off += n
    out_splits = [int(torch.Size(s).numel()) for s in recv_shapes]
    recv = torch.empty(sum(out_splits), dtype=like.dtype, device=like.device)
    dist.all_to_all_single(recv, send_flat, out_splits, in_splits, group=group)
    res, off = [], 0
    for s, n in zip(recv_shapes, out_splits):
        res.append(recv[off:off + n].view(s))
        off += n
    return res, recv


def _check(t, pc: Pencils, pencil):
    want = pc.layout.tensor_shape(pencil)
    if tuple(t.shape[:3]) != want:
        raise ValueError(f"not this rank's {pencil} pencil: {tuple(t.shape[:3])} != {want}")
    return tuple(t.shape[3:])


def transpose_x_to_y(t, pc: Pencils):
    """X pencil -> Y pencil (2decomp's transpose_x_to_y).  Returns its input
    when the two coincide (p_row = 1)."""
    import torch
    L = pc.layout
    rest = _check(t, pc, "x")
    if L.p_row == 1:
        return t
    members = L.xy_members()
    (xa, xb), _, (za, zb) = L.block("y")
    send = [t[:, :, a:b] for a, b in (L.block("y", m)[0] for m in members)]
    ys = [L.block("x", m)[1] for m in members]
    got, _ = _exchange(send, [(zb - za, b - a, xb - xa) + rest for a, b in ys], pc.xy_group, members, t)
    out = torch.empty(L.tensor_shape("y") + rest, dtype=t.dtype, device=t.device)
    for (a, b), blk in zip(ys, got):
        out[:, a:b] = blk
    return out


def transpose_y_to_x(t, pc: Pencils):
    """Y pencil -> X pencil (2decomp's transpose_y_to_x).  Returns its input
    when the two coincide (p_row = 1)."""
    import torch
    L = pc.layout
    rest = _check(t, pc, "y")
    if L.p_row == 1:
        return t
    members = L.xy_members()
    _, (ya, yb), (za, zb) = L.block("x")
    send = [t[:, a:b] for a, b in (L.block("x", m)[1] for m in members)]
    xs = [L.block("y", m)[0] for m in members]
    got, _ = _exchange(send, [(zb - za, yb - ya, b - a) + rest for a, b in xs], pc.xy_group, members, t)
    out = torch.empty(L.tensor_shape("x") + rest, dtype=t.dtype, device=t.device)
    for (a, b), blk in zip(xs, got):
        out[:, :, a:b] = blk
    return out


def transpose_y_to_z(t, pc: Pencils):
    """Y pencil -> Z pencil (2decomp's transpose_y_to_z).  Returns its input
    when the two coincide (p_col = 1)."""
    import torch
    L = pc.layout
    rest = _check(t, pc, "y")
    if L.p_col == 1:
        return t
    members = L.yz_members()
    (xa, xb), (ya, yb), _ = L.block("z")
    send = [t[:, a:b] for a, b in (L.block("z", m)[1] for m in members)]
    zs = [L.block("y", m)[2] for m in members]
    _, recv = _exchange(send, [(b - a, yb - ya, xb - xa) + rest for a, b in zs], pc.yz_group, members, t)
    # the members' z blocks arrive in z order: the receive buffer is the Z pencil
    return recv.view(L.tensor_shape("z") + rest)


def transpose_z_to_y(t, pc: Pencils):
    """Z pencil -> Y pencil (2decomp's transpose_z_to_y).  Returns its input
    when the two coincide (p_col = 1)."""
    import torch
    L = pc.layout
    rest = _check(t, pc, "z")
    if L.p_col == 1:
        return t
    members = L.yz_members()
    (xa, xb), _, (za, zb) = L.block("y")
    send = [t[a:b] for a, b in (L.block("y", m)[2] for m in members)]
    ys = [L.block("z", m)[1] for m in members]
    # the members' z blocks are consecutive ranges of t: t is the send buffer
    got, _ = _exchange(send, [(zb - za, b - a, xb - xa) + rest for a, b in ys], pc.yz_group, members, t,
                       send_flat=t.contiguous().view(-1))
    out = torch.empty(L.tensor_shape("y") + rest, dtype=t.dtype, device=t.device)
    for (a, b), blk in zip(ys, got):
        out[:, a:b] = blk
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
    """One library routine on local extents ext = (nx_l, ny_l, nz_l), with the
    reference's argument order (periodic staggered grids: nxm = nx)."""
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


def _apply(ctx, routine, opname, u, ext):
    import torch
    t = torch.empty_like(u)
    _call(ctx, routine, t, u, ctx.op(opname), ext)
    return t


def sweep(ctx, field, pc: Pencils):
    """The 18 operator applications of a sweep on one field of a box spread
    over a process grid: x families on the rank's X pencil, y families on
    its Y pencil, z families on its Z pencil.  ctx is a periodic context made
    for the global box; field is the rank's X pencil.  Returns {direction:
    [six outputs in X-pencil layout]}."""
    L = pc.layout
    out = {0: [_apply(ctx, r, o, field, L.extents("x")) for r, o in SWEEP[0]]}
    fy = transpose_x_to_y(field, pc)
    out[1] = [transpose_y_to_x(_apply(ctx, r, o, fy, L.extents("y")), pc) for r, o in SWEEP[1]]
    fz = transpose_y_to_z(fy, pc)
    out[2] = [transpose_y_to_x(transpose_z_to_y(_apply(ctx, r, o, fz, L.extents("z")), pc), pc)
              for r, o in SWEEP[2]]
    return out


def poisson(ctx, rhs, pc: Pencils):
    """poisson_000 (src/poisson.f90:276-419) on a box spread over a process
    grid, in place on this rank's X pencil of the FP64 field.  Unnormalised
    r2c transform along x on the X pencil, c2c along y on the Y pencil (one
    2-D transform of the rank's z planes when p_row = 1), then the z part on
    the Z pencil of the half spectrum (x3d_poisson_zpencil: z transforms and
    the mode division), and back the same way, as 2decomp's distributed FFT
    does with its transposes."""
    import torch
    L = pc.layout
    nx, ny, nz = L.shape
    nxh = nx // 2 + 1
    spc = pc.with_shape((nxh, ny, nz))  # the half spectrum, complex values as (..., 2) reals
    R, C = torch.view_as_real, torch.view_as_complex
    if L.p_row == 1:
        spec_y = torch.fft.rfft2(rhs, norm="backward")
    else:
        sx = torch.fft.rfft(rhs, dim=2, norm="backward")
        spec_y = torch.fft.fft(C(transpose_x_to_y(R(sx), spc)), dim=1, norm="backward")
    zs = transpose_y_to_z(R(spec_y), spc)
    (i0, i1), (j0, j1), _ = spc.layout.block("z")
    zc = C(zs) if zs.is_contiguous() else C(zs.contiguous())
    ctx.poisson_zpencil(zc, i1 - i0, i0, j1 - j0, j0)
    back = transpose_z_to_y(R(zc), spc)
    if L.p_row == 1:
        rhs.copy_(torch.fft.irfft2(C(back), s=(ny, nx), norm="forward"))
    else:
        by = torch.fft.ifft(C(back), dim=1, norm="forward")
        rhs.copy_(torch.fft.irfft(C(transpose_y_to_x(R(by), spc)), n=nx, dim=2, norm="forward"))
    return rhs


def euler_step(ctx, u, du, pp3, pg, dt, pc: Pencils):
    """One timestep (src/xcompact3d.f90:80-95) on a box spread over a process
    grid, from the library's line solves on local extents, elementwise tensor
    arithmetic and the pencil transposes, in the reference's order:
    momentum_rhs_eq (src/transeq.f90:44-355) with its x, y and z parts on
    the rank's X, Y and Z pencils; int_time (src/time_integrators.f90:40-44);
    divergence (src/navier.f90:98-236) into the FP64 pp3; the pencil Poisson
    solve; gradp (src/navier.f90:249-359) and cor_vel (:64-91).  u, du, pg:
    the three velocity, increment and pressure-gradient components as this
    rank's X pencils; pp3: its FP64 X pencil.  In place, like
    x3d_euler_step."""
    L = pc.layout
    ex, ey, ez = L.extents("x"), L.extents("y"), L.extents("z")
    XY = lambda a: transpose_x_to_y(a, pc)  # noqa: E731
    YX = lambda a: transpose_y_to_x(a, pc)  # noqa: E731
    YZ = lambda a: transpose_y_to_z(a, pc)  # noqa: E731
    ZY = lambda a: transpose_z_to_y(a, pc)  # noqa: E731
    ux, uy, uz = u
    uys = [XY(a) for a in u]
    uzz = YZ(uys[2])
    for c in range(3):  # calculate_transeq_rhs
        uc = u[c]
        ta = ux * uc
        td = _apply(ctx, "derx", "derx", ta, ex)
        ta = _apply(ctx, "derx", "derx", uc, ex)
        duc = td + ux * ta
        ucy, uyy = uys[c], uys[1]
        td = ucy * uyy
        tg = _apply(ctx, "dery", "dery", td, ey)
        td = _apply(ctx, "dery", "dery", ucy, ey)
        tg = tg + uyy * td
        ucz = uzz if c == 2 else YZ(ucy)
        tdz = ucz * uzz
        tgz = _apply(ctx, "derz", "derz", tdz, ez)
        tdz = _apply(ctx, "derz", "derz", ucz, ez)
        tg = tg + ZY(tgz + uzz * tdz)
        du[c].copy_(duc + YX(tg))
    for c in range(3):  # int_time, Euler: u = dt du + u
        u[c].copy_(dt * du[c] + u[c])
    # divergence
    pp1 = XY(_apply(ctx, "derxvp", "derxvp", ux, ex))
    pgy1 = XY(_apply(ctx, "interxvp", "intxvp", uy, ex))
    pgz1 = XY(_apply(ctx, "interxvp", "intxvp", uz, ex))
    upi2 = _apply(ctx, "interyvp", "intyvp", pp1, ey)
    duydypi2 = _apply(ctx, "deryvp", "deryvp", pgy1, ey) + upi2
    upi2 = _apply(ctx, "interyvp", "intyvp", pgz1, ey)
    a, b = YZ(duydypi2), YZ(upi2)
    p3 = _apply(ctx, "interzvp", "intzvp", a, ez).double() + _apply(ctx, "derzvp", "derzvp", b, ez).double()
    pp3.copy_(YX(ZY(p3)))
    poisson(ctx, pp3, pc)
    # gradp + cor_vel
    p3z = YZ(XY(pp3)).to(ux.dtype)
    ppi3 = ZY(_apply(ctx, "interzpv", "intzpv", p3z, ez))
    pgz3 = ZY(_apply(ctx, "derzpv", "derzpv", p3z, ez))
    ppi2 = YX(_apply(ctx, "interypv", "intypv", ppi3, ey))
    pgy2 = YX(_apply(ctx, "derypv", "derypv", ppi3, ey))
    pgzi2 = YX(_apply(ctx, "interypv", "intypv", pgz3, ey))
    pg[0].copy_(_apply(ctx, "derxpv", "derxpv", ppi2, ex))
    pg[1].copy_(_apply(ctx, "interxpv", "intxpv", pgy2, ex))
    pg[2].copy_(_apply(ctx, "interxpv", "intxpv", pgzi2, ex))
    for c in range(3):
        u[c].sub_(pg[c])
