"""The C-ABI library loads and exports every symbol include/x3d_b200.h declares
(no GPU needed: nothing here launches a kernel)."""
import ctypes
import os

import pytest

from x3div_b200 import _capi


def test_header_parses():
    syms = _capi.header_symbols()
    assert "x3d_derx" in syms and "x3d_poisson" in syms and "x3d_euler_step" in syms
    assert len(syms) >= 40


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_capi.LIB_PATH)
    missing = [s for s in _capi.header_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(_capi.header_symbols()) <= set(_capi.SIGNATURES), \
        set(_capi.header_symbols()) - set(_capi.SIGNATURES)


def test_null_and_bad_arguments_fail_cleanly():
    L = _capi.lib()
    assert L.x3d_ctx_destroy(None) == _capi.X3D_EINVAL
    assert L.x3d_ctx_sync(None) == _capi.X3D_EINVAL
    assert L.x3d_derx(None, None, None, None, 8, 8, 8) == _capi.X3D_EINVAL
    assert L.x3d_op_info(None, None, None, None, None, None, None) == _capi.X3D_EINVAL
    h = ctypes.c_void_p()
    # lines shorter than the 8-point stencils, and bad precision, are refused before any device work
    assert L.x3d_ctx_create(ctypes.byref(h), 4, 8, 8, 1.0, 1.0, 1.0, 0, 0) == _capi.X3D_EUNSUPPORTED
    assert L.x3d_ctx_create(ctypes.byref(h), 8, 8, 8, 1.0, 1.0, 1.0, 7, 0) == _capi.X3D_EINVAL
    assert L.x3d_ctx_create(ctypes.byref(h), 8, 8, 8, -1.0, 1.0, 1.0, 0, 0) == _capi.X3D_EINVAL
    assert h.value is None


def test_no_device_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _capi.lib()
    h = ctypes.c_void_p()
    assert L.x3d_ctx_create(ctypes.byref(h), 8, 8, 8, 1.0, 1.0, 1.0, 0, 0) == _capi.X3D_ECUDA


def _header_decls(root):
    import re
    with open(os.path.join(root, "include", "x3d_b200.h")) as f:
        header = f.read()
    return {name: len([a for a in args.split(",") if a.strip()])
            for name, args in re.findall(r"^(?:int|const char \*)\s*(x3d_\w+)\(([^;]*?)\);", header, re.M | re.S)}


def test_fortran_interface_module_matches_header():
    """fortran/x3d_b200_bind.f90 declares one bind(C) interface per entry
    point, with the header's argument count (bind(C) matches by position),
    and is exactly what fortran/gen_bind.py writes from the current header."""
    import re
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    decl = _header_decls(root)
    with open(os.path.join(root, "fortran", "x3d_b200_bind.f90")) as f:
        module = f.read()
    iface = {name: len([a for a in args.split(",") if a.strip()])
             for args, name in re.findall(r"function x3d_\w+\(([^)]*)\)[\s&]*bind\(C,[\s&]*name=\"(x3d_\w+)\"\)",
                                          module)}
    assert set(decl) == set(_capi.header_symbols())
    assert iface == decl, {k: (iface.get(k), decl.get(k)) for k in set(iface) | set(decl)
                           if iface.get(k) != decl.get(k)}
    sys.path.insert(0, os.path.join(root, "fortran"))
    import gen_bind
    with open(os.path.join(root, "include", "x3d_b200.h")) as f:
        assert gen_bind.generate(f.read()) == module, "fortran/x3d_b200_bind.f90 is stale: run fortran/gen_bind.py"


def test_fortran_derived_types_have_the_c_layouts():
    """The bind(C) derived types of the module list the C structs' members in
    order with types of the same size, so an array of them has the C
    layout: checked against the ctypes mirrors the Python binding uses."""
    import ctypes as C
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "fortran"))
    import gen_bind
    with open(os.path.join(root, "include", "x3d_b200.h")) as f:
        types = dict(gen_bind.structs(f.read()))
    size = {"integer(c_int)": 4, "integer(c_long_long)": 8, "real(c_double)": 8, "type(c_ptr)": 8}
    mirrors = {"x3d_box": _capi.Box, "x3d_work": _capi.Work, "x3d_block": _capi.Block}
    assert set(types) == set(mirrors)
    for name, fields in types.items():
        cfields = mirrors[name]._fields_
        assert len(fields) == len(cfields), name
        for (ft, _member), (_cname, ctype) in zip(fields, cfields):
            assert size[ft] == C.sizeof(ctype), (name, ft, ctype)


# The reference's staggered routines and their dummy arguments, in order
# (src/x3d_staggered.f90:23-1233), and the abstract derivative interfaces
# (src/x3d_derive.f90:19-52) the re-pointed wrappers must keep.
STAGGERED = {
    "derxvp": "tx,ux,x3dop,nx,nxm,ny,nz", "interxvp": "tx,ux,x3dop,nx,nxm,ny,nz",
    "derxpv": "tx,ux,x3dop,nxm,nx,ny,nz", "interxpv": "tx,ux,x3dop,nxm,nx,ny,nz",
    "interyvp": "ty,uy,x3dop,nx,ny,nym,nz", "deryvp": "ty,uy,x3dop,ppyi,nx,ny,nym,nz",
    "interypv": "ty,uy,x3dop,nx,nym,ny,nz", "derypv": "ty,uy,x3dop,ppy,nx,nym,ny,nz",
    "derzvp": "tz,uz,x3dop,nx,ny,nz,nzm", "interzvp": "tz,uz,x3dop,nx,ny,nz,nzm",
    "derzpv": "tz,uz,x3dop,nx,ny,nzm,nz", "interzpv": "tz,uz,x3dop,nx,ny,nzm,nz",
}
DERIVATIVES = {"derx_b200": "t,u,x3dop,nx,ny,nz", "dery_b200": "t,u,x3dop,pp,nx,ny,nz",
               "derz_b200": "t,u,x3dop,nx,ny,nz", "derxx_b200": "t,u,x3dop,nx,ny,nz",
               "deryy_b200": "t,u,x3dop,nx,ny,nz", "derzz_b200": "t,u,x3dop,nx,ny,nz",
               "poisson_b200": "rhs"}


def _subroutines(path):
    import re
    with open(path) as f:
        text = f.read()
    return {name: ",".join(a.strip() for a in args.split(","))
            for name, args in re.findall(r"^\s*subroutine\s+(\w+)\s*\(([^)]*)\)", text, re.M)}, text


def test_fortran_drop_in_routines_keep_the_reference_interfaces():
    """The staggered drop-in module is named x3d_staggered, exports the twelve
    routines with the reference's argument lists and calls the library entry
    point of each; the derivative and Poisson wrappers keep the reference's
    abstract interfaces, and the re-pointing binds every pointer."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subs, text = _subroutines(os.path.join(root, "fortran", "x3d_staggered_b200.f90"))
    assert "module x3d_staggered\n" in text
    for name, args in STAGGERED.items():
        assert subs.get(name) == args, (name, subs.get(name))
        assert f"x3d_{name}(x3d_ctx" in text, name
    subs, text = _subroutines(os.path.join(root, "fortran", "x3d_b200_derive.f90"))
    for name, args in DERIVATIVES.items():
        assert subs.get(name) == args, (name, subs.get(name))
    for ptr in ("derx", "dery", "derz", "derxx", "deryy", "derzz", "poisson"):
        assert f"{ptr} => {ptr}_b200" in text, ptr
    _, shim = _subroutines(os.path.join(root, "fortran", "decomp_2d_shim.f90"))
    for mod in ("decomp_2d_constants", "decomp_2d_mpi", "decomp_2d", "decomp_2d_fft"):
        assert f"\nmodule {mod}\n" in shim, mod
    for sym in ("alloc_x", "alloc_y", "alloc_z", "transpose_x_to_y", "transpose_y_to_z", "transpose_z_to_y",
                "transpose_y_to_x", "decomp_2d_init", "decomp_info_init", "init_coarser_mesh_statS", "ph1",
                "phG", "xsize", "zstart", "nx_global", "decomp_2d_abort", "decomp_2d_fft_3d"):
        assert sym in shim, sym
