"""ctypes binding of libx3d_b200.so (declared in include/x3d_b200.h).

Loading fails loudly when the shared library has not been built: there is no
CPU or eager fallback behind this package.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libx3d_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "x3d_b200.h")

X3D_OK, X3D_EINVAL, X3D_EUNSUPPORTED, X3D_ECUDA, X3D_ENOMEM, X3D_ETIMEOUT = 0, -1, -2, -3, -4, -5
X3D_F64, X3D_F32 = 0, 1
X3D_DIR_X, X3D_DIR_Y, X3D_DIR_Z = 0, 1, 2
KIND = dict(der=0, der2=1, dervp=2, derpv=3, intvp=4, intpv=5)
OP_NAMES = ["derx", "derxp", "dery", "deryp", "derz", "derzp", "derxvp", "deryvp", "derzvp",
            "derxpv", "derypv", "derzpv", "intxvp", "intyvp", "intzvp", "intxpv", "intypv",
            "intzpv", "derxx", "deryy", "derzz"]

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

# argument signatures, by exported name
SIGNATURES = {
    "x3d_ctx_create": [ctypes.POINTER(_vp), _i, _i, _i, _d, _d, _d, _i, _i],
    "x3d_ctx_create_bc": [ctypes.POINTER(_vp), _i, _i, _i, _d, _d, _d, _i, _i, ctypes.POINTER(_i)],
    "x3d_ctx_destroy": [_vp],
    "x3d_ctx_set_stream": [_vp, _vp],
    "x3d_ctx_get_stream": [_vp, ctypes.POINTER(_vp)],
    "x3d_ctx_launch_count": [_vp, ctypes.POINTER(ctypes.c_ulonglong)],
    "x3d_ctx_last_kernel": [_vp, _ip],
    "x3d_ctx_sync": [_vp],
    "x3d_ctx_last_error": [_vp],
    "x3d_ctx_geometry": [_vp, _ip, _dp, _dp, _ip],
    "x3d_op_builtin": [_vp, _i, ctypes.POINTER(_vp)],
    "x3d_op_create": [_vp, _i, _i, _i, _i, _d, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)],
    "x3d_op_destroy": [_vp, _vp],
    "x3d_op_info": [_vp, _ip, _dp, _vp, _vp, _vp, _vp],
    "x3d_derx": [_vp, _vp, _vp, _vp, _i, _i, _i],
    "x3d_dery": [_vp, _vp, _vp, _vp, _vp, _i, _i, _i],
    "x3d_derz": [_vp, _vp, _vp, _vp, _i, _i, _i],
    "x3d_derxx": [_vp, _vp, _vp, _vp, _i, _i, _i],
    "x3d_deryy": [_vp, _vp, _vp, _vp, _i, _i, _i],
    "x3d_derzz": [_vp, _vp, _vp, _vp, _i, _i, _i],
    "x3d_derxvp": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_interxvp": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_derxpv": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_interxpv": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_interyvp": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_deryvp": [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_interypv": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_derypv": [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_derzvp": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_interzvp": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_derzpv": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_interzpv": [_vp, _vp, _vp, _vp, _i, _i, _i, _i],
    "x3d_apply_batch": [_vp, _vp, _i],
    "x3d_apply": [_vp, _vp, _vp, _vp],
    "x3d_autotune": [_vp, _i],
    "x3d_ctx_set_kernel": [_vp, _i],
    "x3d_autotune_choice": [_vp, _i, _i, _ip],
    "x3d_autotune_stage_choice": [_vp, ctypes.c_char_p, _ip],
    "x3d_ctx_set_stage_choice": [_vp, ctypes.c_char_p, _i],
    "x3d_step_capture": [_vp] + [_vp] * 10 + [ctypes.c_double],
    "x3d_step_launch": [_vp],
    "x3d_ctx_selftest_timeout": [_vp, ctypes.c_double],
    "x3d_poisson_zlines": [_vp, _vp, _i, _i],
    "x3d_poisson_zpencil": [_vp, _vp, _i, _i, _i, _i],
    "x3d_roofline_probe": [_vp, _i, _i, _i, _vp, ctypes.POINTER(_vp), _i, _i, _i],
    "x3d_buf_register": [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(_vp)],
    "x3d_buf_unregister": [_vp, _vp],
    "x3d_sync_to_device": [_vp, _vp],
    "x3d_sync_to_host": [_vp, _vp],
    "x3d_batch_create": [ctypes.POINTER(_vp), _vp, _i, _i, _i],
    "x3d_batch_destroy": [_vp],
    "x3d_batch_set_stream": [_vp, _vp],
    "x3d_batch_last_error": [_vp],
    "x3d_batch_bind_sweep": [_vp, _i, _vp, _vp, _i],
    "x3d_batch_run": [_vp],
    "x3d_batch_capture": [_vp],
    "x3d_batch_replay": [_vp],
    "x3d_batch_sync": [_vp],
    "x3d_batch_info": [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong), _ip, _ip],
    "x3d_batch_autotune": [_vp],
    "x3d_batch_choice": [_vp, _i, _i, _ip, _ip],
    "x3d_xthomas": [_vp, _vp, _vp, _vp, _vp, _vp, _d, _i, _i, _i],
    "x3d_ythomas": [_vp, _vp, _vp, _vp, _vp, _vp, _d, _i, _i, _i],
    "x3d_zthomas": [_vp, _vp, _vp, _vp, _vp, _vp, _d, _i, _i, _i],
    "x3d_transpose_x_to_y": [_vp, _vp, _vp, _i],
    "x3d_transpose_y_to_z": [_vp, _vp, _vp, _i],
    "x3d_transpose_z_to_y": [_vp, _vp, _vp, _i],
    "x3d_transpose_y_to_x": [_vp, _vp, _vp, _i],
    "x3d_poisson": [_vp, _vp],
    "x3d_divergence": [_vp, _vp, _vp, _vp, _vp, _i],
    "x3d_divergence_noalloc": [_vp, _vp, _vp, _vp, _vp],
    "x3d_gradp": [_vp, _vp, _vp, _vp, _vp],
    "x3d_cor_vel": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "x3d_solve_poisson": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "x3d_div_stats": [_vp, _vp, _dp],
    "x3d_momentum_rhs_eq": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "x3d_int_time": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _d],
    "x3d_euler_step": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d],
    "x3d_copy_blocks": [_vp, _vp, _vp, _i, _vp, _i],
    "x3d_transeq_part": [_vp, _i, _vp, _vp, _vp, _vp, _d, _i, _i, _i],
    "x3d_divergence_part": [_vp, _i, _vp, _vp, _i, _i, _i],
    "x3d_gradp_part": [_vp, _i, _vp, _vp, _vp, _i, _i, _i],
    "x3d_vel": [_vp, _vp, _vp, _vp],
    "x3d_test_rms": [_vp, _i, _vp, _dp],
}

class Box(ctypes.Structure):
    """x3d_box: one periodic box of a batch."""
    _fields_ = [("nx", _i), ("ny", _i), ("nz", _i), ("xlx", _d), ("yly", _d), ("zlz", _d)]


class Block(ctypes.Structure):
    """x3d_block: one box of an x3d_copy_blocks list (elements)."""
    _fields_ = [("src_offset", ctypes.c_longlong), ("dst_offset", ctypes.c_longlong), ("nx", _i), ("ny", _i),
                ("nz", _i), ("src_ystride", ctypes.c_longlong), ("src_zstride", ctypes.c_longlong),
                ("dst_ystride", ctypes.c_longlong), ("dst_zstride", ctypes.c_longlong)]


class Work(ctypes.Structure):
    """x3d_work: one item of an x3d_apply_batch work-list."""
    _fields_ = [("op", _vp), ("in_", _vp), ("out", _vp)]


_lib = None


def header_symbols(path: str = HEADER) -> list[str]:
    """Names of every function declared in include/x3d_b200.h."""
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(x3d_\w+)\s*\(", text, re.M)))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                "g.build()'` (or make -C x3div_b200/csrc); there is no fallback implementation")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_char_p if name.endswith("_last_error") else ctypes.c_int
        _lib = L
    return _lib
