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
pencils coincide: 2decomp's 1 x P slabs, z-slabs and y-slabs, are that
case.

Device tensors are C-ordered (z, y, x) views of the Fortran (x, y, z)
layout, with any trailing dimensions carried along (a complex spectrum as
(..., 2) reals).  The exchanges go through torch.distributed: NCCL over
NVLink for CUDA tensors, gloo for CPU tensors.  The packing and unpacking
around them are the library's block-copy kernel on CUDA tensors
(x3d_copy_blocks) and strided tensor views on CPU tensors (gloo ranks); the
line solves and the step's stages are the library's kernels on the
pencils' local extents.
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


# ---- transposes: block plans, the library's packing kernel, one all-to-all ----

@dataclass(frozen=True)
class TransposePlan:
    """One rank's part of a transpose among the members of its group.

    pack: boxes copied from the source pencil into the send buffer, member
    by member (None: the source pencil itself is the send buffer); unpack:
    boxes copied from the receive buffer into the output pencil (None: the
    receive buffer is the output).  A box is (src_offset, dst_offset, nx,
    ny, nz, src_ystride, src_zstride, dst_ystride, dst_zstride) in points
    (x3d_block).  send[i] / recv[i]: points sent to / received from
    members[i]."""
    members: tuple
    pack: tuple | None
    send: tuple
    recv: tuple
    unpack: tuple | None
    out_shape: tuple


def _box(shape, z, y, x):
    """(offset, ystride, zstride) of point (z, y, x) of a C-ordered (nz, ny,
    nx) array, in points."""
    return z * shape[1] * shape[2] + y * shape[2] + x, shape[2], shape[1] * shape[2]


def _to_flat(src_shape, z, y, x, ext, off):
    """A box of extents ext = (nx, ny, nz) at (z, y, x) of the source, to
    offset `off` of a buffer where it lies contiguous."""
    so, sy, sz = _box(src_shape, z, y, x)
    nx, ny, nz = ext
    return (so, off, nx, ny, nz, sy, sz, nx, nx * ny)


def _from_flat(dst_shape, z, y, x, ext, off):
    """A box lying contiguous at offset `off` of a buffer, to (z, y, x) of the
    destination."""
    do, dy, dz = _box(dst_shape, z, y, x)
    nx, ny, nz = ext
    return (off, do, nx, ny, nz, nx, nx * ny, dy, dz)


def plan_transpose(layout: PencilLayout, kind: str) -> TransposePlan | None:
    """The plan of transpose `kind` ('x_to_y', 'y_to_x', 'y_to_z', 'z_to_y')
    for layout.rank, or None when the two pencils coincide (one member).
    As 2decomp's transpose_*: the x <-> y transposes exchange among the
    p_row ranks of a process-grid column, y <-> z among the p_col ranks of a
    row."""
    L = layout
    if kind in ("x_to_y", "y_to_x"):
        if L.p_row == 1:
            return None
        members = tuple(L.xy_members())
    elif kind in ("y_to_z", "z_to_y"):
        if L.p_col == 1:
            return None
        members = tuple(L.yz_members())
    else:
        raise ValueError(f"unknown transpose {kind!r}")
    X, Y, Z = L.tensor_shape("x"), L.tensor_shape("y"), L.tensor_shape("z")
    pack, unpack, send, recv = [], [], [], []
    off_s = off_r = 0
    for m in members:
        if kind == "x_to_y":
            a, b = L.block("y", m)[0]          # m's x range
            ext = (b - a, X[1], X[0])
            pack.append(_to_flat(X, 0, 0, a, ext, off_s))
            ya, yb = L.block("x", m)[1]        # m's y rows
            rext = (Y[2], yb - ya, Y[0])
            unpack.append(_from_flat(Y, 0, ya, 0, rext, off_r))
        elif kind == "y_to_x":
            a, b = L.block("x", m)[1]          # m's y rows
            ext = (Y[2], b - a, Y[0])
            pack.append(_to_flat(Y, 0, a, 0, ext, off_s))
            xa, xb = L.block("y", m)[0]        # m's x range
            rext = (xb - xa, X[1], X[0])
            unpack.append(_from_flat(X, 0, 0, xa, rext, off_r))
        elif kind == "y_to_z":
            a, b = L.block("z", m)[1]          # m's y rows of the Z pencil
            ext = (Y[2], b - a, Y[0])
            pack.append(_to_flat(Y, 0, a, 0, ext, off_s))
            za, zb = L.block("y", m)[2]        # m's z planes: the blocks arrive in z order
            rext = (Z[2], Z[1], zb - za)
        else:  # z_to_y
            a, b = L.block("y", m)[2]          # m's z planes: consecutive ranges of the source
            ext = (Z[2], Z[1], b - a)
            ya, yb = L.block("z", m)[1]        # m's y rows
            rext = (Y[2], yb - ya, Y[0])
            unpack.append(_from_flat(Y, 0, ya, 0, rext, off_r))
        n_s, n_r = ext[0] * ext[1] * ext[2], rext[0] * rext[1] * rext[2]
        send.append(n_s)
        recv.append(n_r)
        off_s += n_s
        off_r += n_r
    out = {"x_to_y": Y, "y_to_x": X, "y_to_z": Z, "z_to_y": Y}[kind]
    return TransposePlan(members, None if kind == "z_to_y" else tuple(pack), tuple(send), tuple(recv),
                         None if kind == "y_to_z" else tuple(unpack), out)


def copy_boxes(ctx, dst, src, boxes, rest=1):
    """Copies `boxes` (x3d_block tuples, in points of `rest` values each)
    from src to dst, both contiguous tensors.  Device tensors go through the
    library's block-copy kernel (x3d_copy_blocks, one launch); host tensors
    (gloo ranks) through strided views of the same boxes."""
    if not boxes:
        return
    if dst.is_cuda:
        if ctx is None or not hasattr(ctx, "copy_blocks"):
            raise ValueError("device pencils are packed by the library: pass its context")
        ctx.copy_blocks(dst, src, dst.element_size() * rest, boxes)
        return
    d, s = dst.reshape(-1), src.reshape(-1)
    for so, do, nx, ny, nz, sy, sz, dy, dz in boxes:
        if nx * ny * nz == 0:
            continue
        sv = s.as_strided((nz, ny, nx, rest), (sz * rest, sy * rest, rest, 1), s.storage_offset() + so * rest)
        dv = d.as_strided((nz, ny, nx, rest), (dz * rest, dy * rest, rest, 1), d.storage_offset() + do * rest)
        dv.copy_(sv)


def _transpose(t, pc: Pencils, kind, src_pencil, ctx=None, out=None):
    import torch
    L = pc.layout
    rest = _check(t, pc, src_pencil)
    if out is not None and (out.dtype != t.dtype or out.device != t.device):
        raise ValueError(f"output pencil is {out.dtype} on {out.device}, the input {t.dtype} on {t.device}")
    plan = plan_transpose(L, kind)
    if plan is None:
        if out is None or out is t:
            return t
        out.copy_(t)
        return out
    group = pc.xy_group if kind in ("x_to_y", "y_to_x") else pc.yz_group
    r = 1
    for v in rest:
        r *= v
    t = t.contiguous()
    if plan.pack is None:
        send = t.view(-1)
    else:
        send = torch.empty(sum(plan.send) * r, dtype=t.dtype, device=t.device)
        copy_boxes(ctx, send, t, plan.pack, r)
    shape = plan.out_shape + rest
    if out is not None and tuple(out.shape) != shape:
        raise ValueError(f"output pencil {tuple(out.shape)} != {shape}")
    if plan.unpack is None and out is not None and out.is_contiguous():
        recv = out.view(-1)
    else:
        recv = torch.empty(sum(plan.recv) * r, dtype=t.dtype, device=t.device)
    import torch.distributed as dist
    dist.all_to_all_single(recv, send, [n * r for n in plan.recv], [n * r for n in plan.send], group=group)
    if plan.unpack is None:
        res = recv.view(shape)
        if out is not None and res.data_ptr() != out.data_ptr():
            out.copy_(res)
            return out
        return res
    res = out if out is not None else torch.empty(shape, dtype=t.dtype, device=t.device)
    copy_boxes(ctx, res, recv, plan.unpack, r)
    return res


def _check(t, pc: Pencils, pencil):
    want = pc.layout.tensor_shape(pencil)
    if tuple(t.shape[:3]) != want:
        raise ValueError(f"not this rank's {pencil} pencil: {tuple(t.shape[:3])} != {want}")
    return tuple(t.shape[3:])


def transpose_x_to_y(t, pc: Pencils, ctx=None, out=None):
    """X pencil -> Y pencil (2decomp's transpose_x_to_y): one all-to-all in
    the rank's process-grid column, packed and unpacked by the library's
    block copies (ctx: the library context, needed for device tensors).
    Returns its input when the two pencils coincide (p_row = 1)."""
    return _transpose(t, pc, "x_to_y", "x", ctx, out)


def transpose_y_to_x(t, pc: Pencils, ctx=None, out=None):
    """Y pencil -> X pencil (2decomp's transpose_y_to_x).  Returns its input
    when the two coincide (p_row = 1)."""
    return _transpose(t, pc, "y_to_x", "y", ctx, out)


def transpose_y_to_z(t, pc: Pencils, ctx=None, out=None):
    """Y pencil -> Z pencil (2decomp's transpose_y_to_z): the blocks arrive
    in z order, so the receive buffer is the Z pencil (no unpacking).
    Returns its input when the two coincide (p_col = 1)."""
    return _transpose(t, pc, "y_to_z", "y", ctx, out)


def transpose_z_to_y(t, pc: Pencils, ctx=None, out=None):
    """Z pencil -> Y pencil (2decomp's transpose_z_to_y): the members' z
    blocks are consecutive ranges of the Z pencil, so it is the send buffer
    (no packing).  Returns its input when the two coincide (p_col = 1)."""
    return _transpose(t, pc, "z_to_y", "z", ctx, out)


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
    XY = lambda a: transpose_x_to_y(a, pc, ctx)  # noqa: E731
    YX = lambda a: transpose_y_to_x(a, pc, ctx)  # noqa: E731
    YZ = lambda a: transpose_y_to_z(a, pc, ctx)  # noqa: E731
    ZY = lambda a: transpose_z_to_y(a, pc, ctx)  # noqa: E731
    out = {0: [_apply(ctx, r, o, field, L.extents("x")) for r, o in SWEEP[0]]}
    fy = XY(field)
    out[1] = [YX(_apply(ctx, r, o, fy, L.extents("y"))) for r, o in SWEEP[1]]
    fz = YZ(fy)
    out[2] = [YX(ZY(_apply(ctx, r, o, fz, L.extents("z")))) for r, o in SWEEP[2]]
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
        spec_y = torch.fft.fft(C(transpose_x_to_y(R(sx), spc, ctx)), dim=1, norm="backward")
    zs = transpose_y_to_z(R(spec_y), spc, ctx)
    (i0, i1), (j0, j1), _ = spc.layout.block("z")
    zc = C(zs) if zs.is_contiguous() else C(zs.contiguous())
    ctx.poisson_zpencil(zc, i1 - i0, i0, j1 - j0, j0)
    back = transpose_z_to_y(R(zc), spc, ctx)
    if L.p_row == 1:
        rhs.copy_(torch.fft.irfft2(C(back), s=(ny, nx), norm="forward"))
    else:
        by = torch.fft.ifft(C(back), dim=1, norm="forward")
        rhs.copy_(torch.fft.irfft(C(transpose_y_to_x(R(by), spc, ctx)), n=nx, dim=2, norm="forward"))
    return rhs


# ---- the step's parts -----------------------------------------------------
#
# Each part runs as the library's fused stage kernel on the pencil
# (x3d_transeq_part, x3d_divergence_part, x3d_gradp_part).  Where the fused
# kernels refuse a pencil (X3D_EUNSUPPORTED: e.g. an FP32 pencil whose x
# extent is not a multiple of 4), the part is composed from the library's
# single-operator routines on the same extents, with the elementwise terms
# as tensor arithmetic.

def _unsupported(e):
    from .api import X3DError
    from ._capi import X3D_EUNSUPPORTED
    return isinstance(e, X3DError) and e.code == X3D_EUNSUPPORTED


def _transeq_part(ctx, d, du, u, add, unew, dt, ext):
    """du_c = add_c + d(u_d u_c)/dx_d + u_d d(u_c)/dx_d (src/transeq.f90:
    101-114 and the y, z blocks); with unew, unew_c = u_c + dt du_c
    (src/time_integrators.f90:41-43)."""
    try:
        return ctx.transeq_part(d, du, u, add, unew, dt, ext)
    except Exception as e:  # noqa: BLE001
        if not _unsupported(e):
            raise
    der = ("derx", "dery", "derz")[d]
    for c in range(3):
        td = _apply(ctx, der, der, u[d] * u[c], ext)
        ta = _apply(ctx, der, der, u[c], ext)
        val = td + u[d] * ta
        du[c].copy_(val if add is None else add[c] + val)
    if unew is not None:  # after every component has read u (unew may be u)
        for c in range(3):
            unew[c].copy_(dt * du[c] + u[c])


def _divergence_part(ctx, d, out, ins, ext):
    """divergence (src/navier.f90:166-202), the stage along d."""
    try:
        return ctx.divergence_part(d, out, ins, ext)
    except Exception as e:  # noqa: BLE001
        if not _unsupported(e):
            raise
    if d == 0:
        out[0].copy_(_apply(ctx, "derxvp", "derxvp", ins[0], ext))
        out[1].copy_(_apply(ctx, "interxvp", "intxvp", ins[1], ext))
        out[2].copy_(_apply(ctx, "interxvp", "intxvp", ins[2], ext))
    elif d == 1:
        out[0].copy_(_apply(ctx, "deryvp", "deryvp", ins[1], ext) + _apply(ctx, "interyvp", "intyvp", ins[0], ext))
        out[1].copy_(_apply(ctx, "interyvp", "intyvp", ins[2], ext))
    else:
        out[0].copy_(_apply(ctx, "interzvp", "intzvp", ins[0], ext).double()
                     + _apply(ctx, "derzvp", "derzvp", ins[1], ext).double())


def _gradp_part(ctx, d, out, ins, ucor, ext):
    """gradp (src/navier.f90:273-304), the stage along d; with ucor the x
    stage also applies cor_vel (:83-87), u_c -= p_c."""
    try:
        return ctx.gradp_part(d, out, ins, ucor, ext)
    except Exception as e:  # noqa: BLE001
        if not _unsupported(e):
            raise
    if d == 2:
        p = ins[0].to(out[0].dtype)
        out[0].copy_(_apply(ctx, "interzpv", "intzpv", p, ext))
        out[1].copy_(_apply(ctx, "derzpv", "derzpv", p, ext))
    elif d == 1:
        out[0].copy_(_apply(ctx, "interypv", "intypv", ins[0], ext))
        out[1].copy_(_apply(ctx, "derypv", "derypv", ins[0], ext))
        out[2].copy_(_apply(ctx, "interypv", "intypv", ins[1], ext))
    else:
        out[0].copy_(_apply(ctx, "derxpv", "derxpv", ins[0], ext))
        out[1].copy_(_apply(ctx, "interxpv", "intxpv", ins[1], ext))
        out[2].copy_(_apply(ctx, "interxpv", "intxpv", ins[2], ext))
        if ucor is not None:
            for c in range(3):
                ucor[c].sub_(out[c])


def euler_step(ctx, u, du, pp3, pg, dt, pc: Pencils):
    """One timestep (src/xcompact3d.f90:80-95) on a box spread over a process
    grid, in the reference's stages, each on its pencil with the transposes
    between: momentum_rhs_eq (src/transeq.f90:44-355) as its z, y and x
    parts, each adding the previous part's terms carried back to its pencil,
    the x part also applying int_time (src/time_integrators.f90:40-44) in
    place; divergence (src/navier.f90:98-236) as its x, y and z parts into
    the FP64 pressure; the pencil Poisson solve; gradp (src/navier.f90:
    249-359) as its z, y and x parts, the x part also applying cor_vel
    (:64-91).  u, du, pg: the three velocity, increment and pressure-gradient
    components as this rank's X pencils; pp3: its FP64 X pencil.  In place,
    like x3d_euler_step."""
    import torch
    L = pc.layout
    ex, ey, ez = L.extents("x"), L.extents("y"), L.extents("z")
    XY = lambda a, out=None: transpose_x_to_y(a, pc, ctx, out)  # noqa: E731
    YX = lambda a, out=None: transpose_y_to_x(a, pc, ctx, out)  # noqa: E731
    YZ = lambda a, out=None: transpose_y_to_z(a, pc, ctx, out)  # noqa: E731
    ZY = lambda a, out=None: transpose_z_to_y(a, pc, ctx, out)  # noqa: E731
    like = u[0]
    Yt = lambda dtype=None: torch.empty(L.tensor_shape("y"), dtype=dtype or like.dtype, device=like.device)  # noqa: E731
    Zt = lambda dtype=None: torch.empty(L.tensor_shape("z"), dtype=dtype or like.dtype, device=like.device)  # noqa: E731
    # calculate_transeq_rhs: z terms, then y terms + z, then x terms + (y + z), u += dt du
    uy = [XY(a) for a in u]
    uz = [YZ(a) for a in uy]
    tz = [Zt() for _ in range(3)]
    _transeq_part(ctx, 2, tz, uz, None, None, dt, ez)
    ty = [ZY(a) for a in tz]
    _transeq_part(ctx, 1, ty, uy, ty, None, dt, ey)
    tx = [YX(a) for a in ty]
    _transeq_part(ctx, 0, du, u, tx, u, dt, ex)
    # divergence
    d1 = [torch.empty_like(like) for _ in range(3)]
    _divergence_part(ctx, 0, d1, u, ex)
    d2 = [Yt() for _ in range(2)]
    _divergence_part(ctx, 1, d2, [XY(a) for a in d1], ey)
    p3 = Zt(torch.float64)
    _divergence_part(ctx, 2, [p3], [YZ(a) for a in d2], ez)
    YX(ZY(p3), out=pp3)
    poisson(ctx, pp3, pc)
    # gradp + cor_vel
    g3 = [Zt() for _ in range(2)]
    _gradp_part(ctx, 2, g3, [YZ(XY(pp3))], None, ez)
    g2 = [Yt() for _ in range(3)]
    _gradp_part(ctx, 1, g2, [ZY(a) for a in g3], None, ey)
    _gradp_part(ctx, 0, pg, [YX(a) for a in g2], u, ex)
