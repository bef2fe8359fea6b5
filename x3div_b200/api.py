"""Python mirror of the reference's operator interface over the C ABI.

Method names, argument order and meaning follow the reference routines
(``derx(tx, ux, x3dop, nx, ny, nz)`` from src/x3d_derive.f90:111,
``derxvp(tx, ux, x3dop, nx, nxm, ny, nz)`` from src/x3d_staggered.f90:23,
``xthomas(tt, ff, fs, fw, perio, alfa, nx, ny, nz)`` from src/thomas.f90:34,
``poisson(rhs)`` from src/poisson.f90:276, and so on).  A non-zero status
from the library raises :class:`X3DError`, where the reference would call
``decomp_2d_abort``.

Field arguments are device tensors (torch, any layout-compatible view whose
memory is the Fortran-ordered (nx, ny, nz) array -- e.g. a contiguous
``(nz, ny, nx)`` tensor) or host numpy arrays in Fortran order; the library
stages host arrays itself.  Element type is the context precision
(float64 for "f64", float32 for "f32"); pressure fields are float64.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import KIND, OP_NAMES, X3D_F32, X3D_F64


def _torch_current_stream():
    """torch's current CUDA stream when torch is loaded with a device, so that
    library work orders with torch's own work on the same tensors."""
    import sys
    torch = sys.modules.get("torch")
    try:
        if torch is not None and torch.cuda.is_available():
            return torch.cuda.current_stream()
    except Exception:
        return None
    return None


class X3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"x3d status {code}: {msg}")
        self.code = code


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        if not (a.flags.f_contiguous or a.flags.c_contiguous):
            raise ValueError("host arrays must be contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("device tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported field argument {type(a)!r}")


class Operator:
    """Handle on an x3doperator1d living in the library."""

    def __init__(self, ctx: "Context", handle: int, name: str, owned: bool):
        self.ctx, self.handle, self.name, self._owned = ctx, handle, name, owned

    def info(self) -> dict:
        L = _capi.lib()
        meta = (ctypes.c_int * 4)()
        scal = (ctypes.c_double * 5)()
        L.x3d_op_info(self.handle, meta, scal, None, None, None, None)
        n = meta[0]
        arrs = [np.zeros(n) for _ in range(4)]
        L.x3d_op_info(self.handle, meta, scal, *[a.ctypes.data for a in arrs])
        return dict(n=n, kind=meta[1], dir=meta[2], npaire=meta[3], alfa=scal[0], a=scal[1],
                    b=scal[2], c=scal[3], d=scal[4], f=arrs[0], s=arrs[1], w=arrs[2],
                    periodic=arrs[3])

    def close(self):
        if self._owned and self.handle:
            _capi.lib().x3d_op_destroy(self.ctx.handle, self.handle)
            self.handle = None


class Context:
    """An nx*ny*nz box at a 1x1 decomposition (x3d_ctx).  bc, if given, is the
    reference's (nclx1, nclxn, ncly1, nclyn, nclz1, nclzn): 0 periodic, 1 free
    slip, 2 Dirichlet (x3d_ctx_create_bc); by default every direction is
    periodic."""

    def __init__(self, nx, ny, nz, lengths=(1.0, 1.0, 1.0), precision="f64", device=0,
                 stream=None, bc=None):
        self.L = _capi.lib()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.lengths = tuple(float(v) for v in lengths)
        self.precision = precision
        self.fp32 = precision == "f32"
        self.bc = tuple(int(v) for v in bc) if bc is not None else (0,) * 6
        h = ctypes.c_void_p()
        if bc is None:
            rc = self.L.x3d_ctx_create(ctypes.byref(h), self.nx, self.ny, self.nz, *self.lengths,
                                       X3D_F32 if self.fp32 else X3D_F64, int(device))
        else:
            ncl = (ctypes.c_int * 6)(*self.bc)
            rc = self.L.x3d_ctx_create_bc(ctypes.byref(h), self.nx, self.ny, self.nz, *self.lengths,
                                          X3D_F32 if self.fp32 else X3D_F64, int(device), ncl)
        if rc != 0:
            raise X3DError(rc, "x3d_ctx_create failed")
        self.handle = h.value
        nm = [n - 1 if self.bc[2 * d] else n for d, n in enumerate((nx, ny, nz))]
        self.dx, self.dy, self.dz = (l / n for l, n in zip(self.lengths, nm))
        if stream is None:
            stream = _torch_current_stream()
        if stream is not None:
            self.set_stream(stream)
        self._ops = {}

    # -- plumbing ---------------------------------------------------------
    @property
    def np_dtype(self):
        return np.float32 if self.fp32 else np.float64

    def _check(self, rc):
        if rc != 0:
            msg = self.L.x3d_ctx_last_error(self.handle) or b""
            raise X3DError(rc, msg.decode(errors="replace"))

    def set_stream(self, stream):
        """Run on a caller stream: a torch.cuda.Stream or a raw cudaStream_t
        (0 is the legacy default stream)."""
        raw = getattr(stream, "cuda_stream", stream)
        self._check(self.L.x3d_ctx_set_stream(self.handle, raw))

    def selftest_timeout(self, limit_s=0.01):
        """x3d_ctx_selftest_timeout: a bounded device wait that runs out; the
        next sync raises X3DError with code X3D_ETIMEOUT (-5)."""
        self._check(self.L.x3d_ctx_selftest_timeout(self.handle, float(limit_s)))

    def launch_count(self) -> int:
        """Kernels of this library launched on the context so far."""
        out = ctypes.c_ulonglong()
        self._check(self.L.x3d_ctx_launch_count(self.handle, ctypes.byref(out)))
        return out.value

    def last_kernel(self) -> int:
        """x3d_ctx_last_kernel: configuration of the last line-solve or
        fused-stage launch (-1 before the first)."""
        out = ctypes.c_int()
        self._check(self.L.x3d_ctx_last_kernel(self.handle, ctypes.byref(out)))
        return out.value

    def get_stream(self) -> int:
        out = ctypes.c_void_p()
        self._check(self.L.x3d_ctx_get_stream(self.handle, ctypes.byref(out)))
        return out.value or 0

    def sync(self):
        self._check(self.L.x3d_ctx_sync(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            for op in self._ops.values():
                if op._owned:
                    op.close()
            self.L.x3d_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- operators --------------------------------------------------------
    def op(self, name: str) -> Operator:
        """One of the x3d_operator_1d instances (x3d_op_derx ... x3d_op_intzpv,
        plus derxx/deryy/derzz)."""
        name = name.removeprefix("x3d_op_")
        if name not in self._ops:
            h = ctypes.c_void_p()
            self._check(self.L.x3d_op_builtin(self.handle, OP_NAMES.index(name), ctypes.byref(h)))
            self._ops[name] = Operator(self, h.value, name, owned=False)
        return self._ops[name]

    def op_create(self, kind, direction, n, npaire, alfa, f, s, w, periodic, rhs) -> Operator:
        h = ctypes.c_void_p()
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (f, s, w, periodic, rhs)]  # periodic None: a non-periodic operator
        kind = KIND[kind] if isinstance(kind, str) else int(kind)
        self._check(self.L.x3d_op_create(self.handle, kind, int(direction), int(n), int(npaire),
                                         float(alfa), *[None if a is None else a.ctypes.data for a in arrs],
                                         ctypes.byref(h)))
        return Operator(self, h.value, f"user-{kind}-{direction}", owned=True)

    # -- x3d_derive -------------------------------------------------------
    def derx(self, tx, ux, op, nx, ny, nz):
        self._check(self.L.x3d_derx(self.handle, _ptr(tx), _ptr(ux), op.handle, nx, ny, nz))

    def dery(self, ty, uy, op, ppy, nx, ny, nz):
        self._check(self.L.x3d_dery(self.handle, _ptr(ty), _ptr(uy), op.handle, _ptr(ppy), nx, ny, nz))

    def derz(self, tz, uz, op, nx, ny, nz):
        self._check(self.L.x3d_derz(self.handle, _ptr(tz), _ptr(uz), op.handle, nx, ny, nz))

    def derxx(self, tx, ux, op, nx, ny, nz):
        self._check(self.L.x3d_derxx(self.handle, _ptr(tx), _ptr(ux), op.handle, nx, ny, nz))

    def deryy(self, ty, uy, op, nx, ny, nz):
        self._check(self.L.x3d_deryy(self.handle, _ptr(ty), _ptr(uy), op.handle, nx, ny, nz))

    def derzz(self, tz, uz, op, nx, ny, nz):
        self._check(self.L.x3d_derzz(self.handle, _ptr(tz), _ptr(uz), op.handle, nx, ny, nz))

    # -- x3d_staggered ----------------------------------------------------
    def derxvp(self, tx, ux, op, nx, nxm, ny, nz):
        self._check(self.L.x3d_derxvp(self.handle, _ptr(tx), _ptr(ux), op.handle, nx, nxm, ny, nz))

    def interxvp(self, tx, ux, op, nx, nxm, ny, nz):
        self._check(self.L.x3d_interxvp(self.handle, _ptr(tx), _ptr(ux), op.handle, nx, nxm, ny, nz))

    def derxpv(self, tx, ux, op, nxm, nx, ny, nz):
        self._check(self.L.x3d_derxpv(self.handle, _ptr(tx), _ptr(ux), op.handle, nxm, nx, ny, nz))

    def interxpv(self, tx, ux, op, nxm, nx, ny, nz):
        self._check(self.L.x3d_interxpv(self.handle, _ptr(tx), _ptr(ux), op.handle, nxm, nx, ny, nz))

    def interyvp(self, ty, uy, op, nx, ny, nym, nz):
        self._check(self.L.x3d_interyvp(self.handle, _ptr(ty), _ptr(uy), op.handle, nx, ny, nym, nz))

    def deryvp(self, ty, uy, op, ppyi, nx, ny, nym, nz):
        self._check(self.L.x3d_deryvp(self.handle, _ptr(ty), _ptr(uy), op.handle, _ptr(ppyi), nx, ny, nym, nz))

    def interypv(self, ty, uy, op, nx, nym, ny, nz):
        self._check(self.L.x3d_interypv(self.handle, _ptr(ty), _ptr(uy), op.handle, nx, nym, ny, nz))

    def derypv(self, ty, uy, op, ppy, nx, nym, ny, nz):
        self._check(self.L.x3d_derypv(self.handle, _ptr(ty), _ptr(uy), op.handle, _ptr(ppy), nx, nym, ny, nz))

    def derzvp(self, tz, uz, op, nx, ny, nz, nzm):
        self._check(self.L.x3d_derzvp(self.handle, _ptr(tz), _ptr(uz), op.handle, nx, ny, nz, nzm))

    def interzvp(self, tz, uz, op, nx, ny, nz, nzm):
        self._check(self.L.x3d_interzvp(self.handle, _ptr(tz), _ptr(uz), op.handle, nx, ny, nz, nzm))

    def derzpv(self, tz, uz, op, nx, ny, nzm, nz):
        self._check(self.L.x3d_derzpv(self.handle, _ptr(tz), _ptr(uz), op.handle, nx, ny, nzm, nz))

    def interzpv(self, tz, uz, op, nx, ny, nzm, nz):
        self._check(self.L.x3d_interzpv(self.handle, _ptr(tz), _ptr(uz), op.handle, nx, ny, nzm, nz))

    # -- batch ------------------------------------------------------------
    def apply_batch(self, items):
        """items: iterable of (operator, in_field, out_field)."""
        items = list(items)
        arr = (_capi.Work * max(1, len(items)))()
        for k, (op, src, dst) in enumerate(items):
            arr[k].op, arr[k].in_, arr[k].out = op.handle, _ptr(src), _ptr(dst)
        self._check(self.L.x3d_apply_batch(self.handle, arr, len(items)))

    def apply(self, op, src, dst):
        """x3d_apply: dst = op(src) on the context grid."""
        self._check(self.L.x3d_apply(self.handle, op.handle, _ptr(src), _ptr(dst)))

    def autotune(self, max_group=6):
        """Time the kernel configurations on this grid and keep the fastest."""
        self._check(self.L.x3d_autotune(self.handle, int(max_group)))

    def set_kernel(self, cfg):
        """Force a kernel configuration (0..15 and 17..20 chunked, 16 thread per line, -1 default)."""
        self._check(self.L.x3d_ctx_set_kernel(self.handle, int(cfg)))

    def autotune_choice(self, direction, group):
        out = ctypes.c_int()
        self._check(self.L.x3d_autotune_choice(self.handle, int(direction), int(group), ctypes.byref(out)))
        return out.value

    STAGES = ("transeq_x", "transeq_y", "transeq_z", "div_x", "div_y", "div_z",
              "gradp_z", "gradp_y", "gradp_x", "gradp_x_cor")
    # 1 where the autotuner runs a momentum stage as two launches (stages
    # "<name>.b" then "<name>.a"), 0 where as one
    STAGE_SPLITS = ("transeq_x.split", "transeq_y.split", "transeq_z.split")

    def set_stage_choice(self, stage, value):
        """x3d_ctx_set_stage_choice: pin one stage choice (-1 removes it)."""
        self._check(self.L.x3d_ctx_set_stage_choice(self.handle, stage.encode(), int(value)))

    def stage_choices(self):
        """Every autotuned stage choice: the configuration of each stage; where
        a stage runs as several launches, "<stage>.split" (the momentum
        stages: "<stage>.a", "<stage>.b") or "<stage>.parts" (the number of
        launches over disjoint staged inputs: "<stage>.1", ...) and the
        configuration of each launch."""
        out = {s: self.autotune_stage_choice(s) for s in self.STAGES}
        for s in self.STAGE_SPLITS:
            if self.autotune_stage_choice(s) == 1:
                base = s[:-len(".split")]
                out[s] = 1
                for p in ("a", "b"):
                    out[f"{base}.{p}"] = self.autotune_stage_choice(f"{base}.{p}")
        for s in self.STAGES:
            n = self.autotune_stage_choice(s + ".parts")
            if n > 1:
                out[s + ".parts"] = n
                for q in range(1, n + 1):
                    out[f"{s}.{q}"] = self.autotune_stage_choice(f"{s}.{q}")
        return out

    def autotune_stage_choice(self, stage):
        """Configuration the autotuner chose for a fused Euler-step stage (-1: not tuned)."""
        out = ctypes.c_int()
        self._check(self.L.x3d_autotune_stage_choice(self.handle, stage.encode(), ctypes.byref(out)))
        return out.value

    # -- thomas -----------------------------------------------------------
    def _thomas(self, fn, tt, ff, fs, fw, perio, alfa, nx, ny, nz):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (ff, fs, fw, perio)]
        self._check(fn(self.handle, _ptr(tt), *[None if a is None else a.ctypes.data for a in arrs],
                       float(alfa), nx, ny, nz))

    def xthomas(self, tt, ff, fs, fw, perio, alfa, nx, ny, nz):
        self._thomas(self.L.x3d_xthomas, tt, ff, fs, fw, perio, alfa, nx, ny, nz)

    def ythomas(self, tt, ff, fs, fw, perio, alfa, nx, ny, nz):
        self._thomas(self.L.x3d_ythomas, tt, ff, fs, fw, perio, alfa, nx, ny, nz)

    def zthomas(self, tt, ff, fs, fw, perio, alfa, nx, ny, nz):
        self._thomas(self.L.x3d_zthomas, tt, ff, fs, fw, perio, alfa, nx, ny, nz)

    # -- x3d_transpose ----------------------------------------------------
    def transpose_x_to_y(self, src, dst, is_complex=False):
        self._check(self.L.x3d_transpose_x_to_y(self.handle, _ptr(src), _ptr(dst), int(is_complex)))

    def transpose_y_to_z(self, src, dst, is_complex=False):
        self._check(self.L.x3d_transpose_y_to_z(self.handle, _ptr(src), _ptr(dst), int(is_complex)))

    def transpose_z_to_y(self, src, dst, is_complex=False):
        self._check(self.L.x3d_transpose_z_to_y(self.handle, _ptr(src), _ptr(dst), int(is_complex)))

    def transpose_y_to_x(self, src, dst, is_complex=False):
        self._check(self.L.x3d_transpose_y_to_x(self.handle, _ptr(src), _ptr(dst), int(is_complex)))

    # -- poisson / navier / transeq / time --------------------------------
    def poisson(self, rhs):
        self._check(self.L.x3d_poisson(self.handle, _ptr(rhs)))

    def roofline_probe(self, pattern, w, src, outs, ctas_per_sm=0):
        """x3d_roofline_probe: one FP32 field to six with no arithmetic, in a
        flat order (pattern 0) or the y stage kernels' tile order (pattern 1,
        w columns per tile)."""
        nz, ny, nx = src.shape
        arr = (ctypes.c_void_p * 6)(*[o.data_ptr() for o in outs])
        self._check(self.L.x3d_roofline_probe(self.handle, int(pattern), int(w), int(ctas_per_sm), _ptr(src), arr,
                                              nx, ny, nz))

    def poisson_zlines(self, spec, ny_loc, j0):
        """x3d_poisson_zlines: z transforms and mode division on a block of
        y rows of the x-y transformed spectrum (a complex128 CUDA tensor of
        shape (nz, ny_loc, nx//2 + 1))."""
        self._check(self.L.x3d_poisson_zlines(self.handle, _ptr(spec), int(ny_loc), int(j0)))

    def poisson_zpencil(self, spec, nxh_loc, i0, ny_loc, j0):
        """x3d_poisson_zpencil: the same on x modes i0 .. i0 + nxh_loc - 1 and
        y rows j0 .. j0 + ny_loc - 1 (a complex128 CUDA tensor of shape (nz,
        ny_loc, nxh_loc)): the Z pencil of a p_row x p_col decomposition."""
        self._check(self.L.x3d_poisson_zpencil(self.handle, _ptr(spec), int(nxh_loc), int(i0), int(ny_loc),
                                               int(j0)))

    def divergence(self, pp3, ux1, uy1, uz1, nlock=1):
        self._check(self.L.x3d_divergence(self.handle, _ptr(pp3), _ptr(ux1), _ptr(uy1), _ptr(uz1), int(nlock)))

    def gradp(self, px1, py1, pz1, pp3):
        self._check(self.L.x3d_gradp(self.handle, _ptr(px1), _ptr(py1), _ptr(pz1), _ptr(pp3)))

    def cor_vel(self, ux, uy, uz, px, py, pz):
        self._check(self.L.x3d_cor_vel(self.handle, *[_ptr(a) for a in (ux, uy, uz, px, py, pz)]))

    def solve_poisson(self, pp3, px1, py1, pz1, ux1, uy1, uz1):
        self._check(self.L.x3d_solve_poisson(self.handle, *[_ptr(a) for a in (pp3, px1, py1, pz1, ux1, uy1, uz1)]))

    def div_stats(self, pp3):
        out = (ctypes.c_double * 2)()
        self._check(self.L.x3d_div_stats(self.handle, _ptr(pp3), out))
        return out[0], out[1]

    def momentum_rhs_eq(self, dux1, duy1, duz1, ux1, uy1, uz1):
        self._check(self.L.x3d_momentum_rhs_eq(self.handle, *[_ptr(a) for a in (dux1, duy1, duz1, ux1, uy1, uz1)]))

    def int_time(self, ux1, uy1, uz1, dux1, duy1, duz1, gdt):
        self._check(self.L.x3d_int_time(self.handle, *[_ptr(a) for a in (ux1, uy1, uz1, dux1, duy1, duz1)], float(gdt)))

    # -- the step's parts on one pencil of a process grid ---------------------
    @staticmethod
    def _ptrs(fields):
        if fields is None:
            return None
        return (ctypes.c_void_p * len(fields))(*[_ptr(a) for a in fields])

    def transeq_part(self, dir, du, u, add, unew, dt, ext):
        """x3d_transeq_part on a dir-pencil of local extents ext = (nx, ny, nz):
        du[c] = add[c] + d(u_dir u_c)/dx_dir + u_dir d(u_c)/dx_dir, and with
        unew also unew[c] = u[c] + dt du[c] (add, unew: three fields or None)."""
        self._check(self.L.x3d_transeq_part(self.handle, int(dir), self._ptrs(du), self._ptrs(u), self._ptrs(add),
                                            self._ptrs(unew), float(dt), *[int(e) for e in ext]))

    def divergence_part(self, dir, out, ins, ext):
        """x3d_divergence_part: the divergence's stage along dir on a pencil."""
        self._check(self.L.x3d_divergence_part(self.handle, int(dir), self._ptrs(out), self._ptrs(ins),
                                               *[int(e) for e in ext]))

    def gradp_part(self, dir, out, ins, ucor, ext):
        """x3d_gradp_part: the pressure gradient's stage along dir on a pencil
        (dir 0 with ucor: also ucor[c] -= out[c])."""
        self._check(self.L.x3d_gradp_part(self.handle, int(dir), self._ptrs(out), self._ptrs(ins),
                                          self._ptrs(ucor), *[int(e) for e in ext]))

    def copy_blocks(self, dst, src, elem_bytes, blocks):
        """x3d_copy_blocks: blocks is a list of (src_offset, dst_offset, nx, ny,
        nz, src_ystride, src_zstride, dst_ystride, dst_zstride) in elements of
        elem_bytes (4, 8 or 16) bytes; dst and src are device tensors."""
        arr = (_capi.Block * max(1, len(blocks)))(*[_capi.Block(*b) for b in blocks])
        self._check(self.L.x3d_copy_blocks(self.handle, dst.data_ptr(), src.data_ptr(), int(elem_bytes), arr,
                                           len(blocks)))

    def euler_step(self, ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, py1, pz1, dt):
        self._check(self.L.x3d_euler_step(self.handle, *[_ptr(a) for a in (ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, py1, pz1)], float(dt)))

    def step_capture(self, ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, py1, pz1, dt):
        """x3d_step_capture: record one Euler step on these fields into a CUDA graph."""
        self._check(self.L.x3d_step_capture(self.handle, *[_ptr(a) for a in (ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, py1, pz1)], float(dt)))

    def step_launch(self):
        """x3d_step_launch: replay the captured step once."""
        self._check(self.L.x3d_step_launch(self.handle))

    # -- device-resident host arrays ---------------------------------------
    def buf_register(self, host):
        """x3d_buf_register: give a contiguous host numpy array a device mirror;
        returns the mirror's device address."""
        if not isinstance(host, np.ndarray) or not (host.flags.f_contiguous or host.flags.c_contiguous):
            raise ValueError("buf_register takes a contiguous numpy array")
        dev = ctypes.c_void_p()
        self._check(self.L.x3d_buf_register(self.handle, host.ctypes.data, host.nbytes, ctypes.byref(dev)))
        return dev.value

    def buf_unregister(self, host):
        self._check(self.L.x3d_buf_unregister(self.handle, host.ctypes.data))

    def sync_to_device(self, host):
        self._check(self.L.x3d_sync_to_device(self.handle, host.ctypes.data))

    def sync_to_host(self, host):
        self._check(self.L.x3d_sync_to_host(self.handle, host.ctypes.data))

    def vel(self, u, v, w):
        self._check(self.L.x3d_vel(self.handle, _ptr(u), _ptr(v), _ptr(w)))

    def test_rms(self, which, du):
        out = ctypes.c_double()
        self._check(self.L.x3d_test_rms(self.handle, int(which), _ptr(du), ctypes.byref(out)))
        return out.value


def to_device(a: np.ndarray, dtype=None, device="cuda"):
    """Fortran-ordered (nx, ny, nz) numpy field -> contiguous (nz, ny, nx) torch tensor."""
    import torch
    a = np.asarray(a)
    t = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0)))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(device)


def to_host(t) -> np.ndarray:
    """Contiguous (nz, ny, nx) torch tensor -> Fortran-ordered (nx, ny, nz) numpy array."""
    return np.asfortranarray(t.detach().cpu().numpy().transpose(2, 1, 0))


class Batch:
    """Independent periodic boxes swept in one persistent launch (x3d_batch).

    boxes: iterable of (nx, ny, nz) or (nx, ny, nz, xlx, yly, zlz)."""

    def __init__(self, boxes, precision="f32", device=0, stream=None):
        self.L = _capi.lib()
        self.boxes = [tuple(b) + (2 * np.pi,) * (6 - len(b)) for b in boxes]
        arr = (_capi.Box * len(self.boxes))()
        for k, b in enumerate(self.boxes):
            arr[k].nx, arr[k].ny, arr[k].nz = (int(v) for v in b[:3])
            arr[k].xlx, arr[k].yly, arr[k].zlz = (float(v) for v in b[3:])
        h = ctypes.c_void_p()
        rc = self.L.x3d_batch_create(ctypes.byref(h), arr, len(self.boxes),
                                     X3D_F32 if precision == "f32" else X3D_F64, int(device))
        if rc != 0:
            raise X3DError(rc, "x3d_batch_create failed")
        self.handle = h.value
        if stream is None:
            stream = _torch_current_stream()
        if stream is not None:
            self._check(self.L.x3d_batch_set_stream(self.handle, getattr(stream, "cuda_stream", stream)))

    def _check(self, rc):
        if rc != 0:
            msg = self.L.x3d_batch_last_error(self.handle) or b""
            raise X3DError(rc, msg.decode(errors="replace"))

    def bind_sweep(self, fields, outs, nops=6):
        """fields[i][f]: field f of box i; outs[i][f][d][k]: operator family k along d."""
        nf = len(fields[0])
        fin = (ctypes.c_void_p * (len(fields) * nf))()
        fout = (ctypes.c_void_p * (len(fields) * nf * 18))()
        for i, fs in enumerate(fields):
            for f, a in enumerate(fs):
                fin[i * nf + f] = _ptr(a)
                for d in range(3):
                    for k in range(nops):
                        fout[((i * nf + f) * 3 + d) * 6 + k] = _ptr(outs[i][f][d][k])
        self._keep = (fin, fout)
        self._check(self.L.x3d_batch_bind_sweep(self.handle, nf, fin, fout, int(nops)))

    def run(self):
        self._check(self.L.x3d_batch_run(self.handle))

    def capture(self):
        self._check(self.L.x3d_batch_capture(self.handle))

    def replay(self):
        self._check(self.L.x3d_batch_replay(self.handle))

    def sync(self):
        self._check(self.L.x3d_batch_sync(self.handle))

    def info(self):
        p, t = ctypes.c_longlong(), ctypes.c_longlong()
        j, fb = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.x3d_batch_info(self.handle, ctypes.byref(p), ctypes.byref(t), ctypes.byref(j),
                                          ctypes.byref(fb)))
        return dict(points=p.value, tiles=t.value, jobs=j.value, fallback_jobs=fb.value)

    def autotune(self):
        """x3d_batch_autotune: per box shape and direction, the fastest chunk
        length and tile width (overwrites the bound outputs)."""
        self._check(self.L.x3d_batch_autotune(self.handle))

    def choice(self, box, direction):
        """x3d_batch_choice: (chunk length, lines per tile) of box's jobs along direction."""
        c, w = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.x3d_batch_choice(self.handle, int(box), int(direction), ctypes.byref(c), ctypes.byref(w)))
        return c.value, w.value

    def close(self):
        if getattr(self, "handle", None):
            self.L.x3d_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
