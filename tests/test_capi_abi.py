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


def test_fortran_interface_block_matches_header():
    """INTEGRATION.md's Appendix A declares one bind(C) interface per entry
    point, with the header's argument count (bind(C) matches by position)."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "include", "x3d_b200.h")) as f:
        header = f.read()
    decl = {name: len([a for a in args.split(",") if a.strip()])
            for name, args in re.findall(r"^(?:int|const char \*)\s*(x3d_\w+)\(([^;]*?)\);", header, re.M | re.S)}
    with open(os.path.join(root, "INTEGRATION.md")) as f:
        doc = f.read()
    appendix = doc[doc.index("## Appendix A."):]
    iface = {name: len([a for a in args.split(",") if a.strip()])
             for args, name in re.findall(r"function x3d_\w+\(([^)]*)\)[\s&]*bind\(C,[\s&]*name=\"(x3d_\w+)\"\)",
                                          appendix)}
    assert set(decl) == set(_capi.header_symbols())
    assert iface == decl, {k: (iface.get(k), decl.get(k)) for k in set(iface) | set(decl)
                           if iface.get(k) != decl.get(k)}
