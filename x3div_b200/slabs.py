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

This is the p_row = 1 case of x3div_b200.pencils, with the process group
of the y <-> z transposes passed in directly.  Device tensors are C-ordered
(nz, ny, nx) views of the Fortran (nx, ny, nz) layout, as in the rest of the
package.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import pencils as _pencils
from .pencils import SWEEP, split  # noqa: F401  (re-exported)


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

    def pencils(self, group=None):
        """The 1 x world pencil decomposition this layout is, with `group`
        (default: the default process group) for the y <-> z transposes."""
        return _pencils.Pencils(_pencils.PencilLayout(tuple(self.shape), 1, self.world, self.rank), None, group)


def transpose_y_to_z(zslab, layout: SlabLayout, group=None):
    """X/Y pencil (a (nz_r, ny, nx) tensor) -> Z pencil ((nz, ny_s, nx) on
    rank s): 2decomp's transpose_y_to_z at p_row = 1."""
    return _pencils.transpose_y_to_z(zslab, layout.pencils(group))


def transpose_z_to_y(yslab, layout: SlabLayout, group=None):
    """Z pencil ((nz, ny_r, nx)) -> X/Y pencil ((nz_s, ny, nx) on rank s):
    2decomp's transpose_z_to_y at p_row = 1."""
    return _pencils.transpose_z_to_y(yslab, layout.pencils(group))


def sweep(ctx, field, layout: SlabLayout, group=None):
    """The 18 operator applications of a sweep on one field of a box that is
    spread over the ranks: x and y families on the rank's X/Y pencil, z
    families on its Z pencil (one transpose each way).  ctx is a periodic
    context made for the global box; field is the rank's X/Y pencil.  Returns
    {direction: [six outputs in X/Y-pencil layout]}."""
    return _pencils.sweep(ctx, field, layout.pencils(group))


def poisson(ctx, rhs, layout: SlabLayout, group=None):
    """poisson_000 (src/poisson.f90:276-419) on a box spread over the ranks,
    in place on this rank's X/Y pencil of the FP64 field ((nz_r, ny, nx)):
    2-D x-y transforms of the rank's z planes, the z part on its block of y
    rows after a transpose of the half spectrum (x3d_poisson_zpencil), and
    back."""
    return _pencils.poisson(ctx, rhs, layout.pencils(group))


def euler_step(ctx, u, du, pp3, pg, dt, layout: SlabLayout, group=None):
    """One timestep (src/xcompact3d.f90:80-95) on a box spread over the ranks
    in z-slabs (x3div_b200.pencils.euler_step at p_row = 1).  u, du, pg: the
    three velocity, increment and pressure-gradient components as this
    rank's X/Y pencils; pp3: its FP64 X/Y pencil.  In place."""
    return _pencils.euler_step(ctx, u, du, pp3, pg, dt, layout.pencils(group))
