"""ctypes binding of libainv_b200.so (the C-ABI declared in include/ainv_b200.h).

The library is built in-tree (``make -C mld-ainv_b200``).  There is no
fallback: importing this module without the library raises, and every
compute entry point runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_DIR, "libainv_b200.so")

SUCCESS = 0
ERR_ARG = 30
ERR_ALLOC = 4025
ERR_INTERNAL = 4000
ERR_CUDA = 4100
ERR_NOT_BUILT = 4101
ERR_BREAKDOWN = 4102
ERR_NONFINITE = 4103
ERR_NOCONV = 4104
ERR_UNSUPPORTED = 4105
ERR_TIMEOUT = 4106

PREC = {"FP64": 0, "FP32": 1, "BF16": 2, "FP32_ACC64": 3, "BF16_ACC64": 4}
KRYLOV = {"CG": 0, "BICGSTAB": 1}
AINV_ALG = {"LLK": 0, "SYM-LLK": 1, "STAB-LLK": 2, "LLK-NOTH": 3, "MLK": 4}

# (name, restype, argtypes) for every symbol the header declares.
_vp, _i, _d, _c = C.c_void_p, C.c_int, C.c_double, C.c_char
_ip, _dp, _ll = C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_longlong
_llp = C.POINTER(C.c_longlong)
SIGNATURES = [
    ("ainv_last_error", C.c_char_p, []),
    ("ainv_version", C.c_char_p, []),
    ("ainv_gpu_create", _i, [C.POINTER(_vp), _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i]),
    ("ainv_gpu_apply", _i, [_vp, _c, _d, _vp, _d, _vp, _vp]),
    ("ainv_gpu_apply_stage", _i, [_vp, _c, _i, _d, _vp, _d, _vp, _vp]),
    ("ainv_gpu_apply_host", _i, [_vp, _c, _d, _vp, _d, _vp]),
    ("ainv_gpu_destroy", _i, [_vp]),
    ("ainv_gpu_check", _i, [_vp]),
    ("ainv_gpu_sizeof", C.c_size_t, [_vp]),
    ("ainv_gpu_get_nzeros", _ll, [_vp]),
    ("ainv_gpu_get_n", _i, [_vp]),
    ("ainv_gpu_get_prec", _i, [_vp]),
    ("ainv_gpu_layout_info", _i, [_vp, _i, _llp, _llp, _llp, _ip, _ip]),
    ("ainv_gpu_apply_csr_noalloc", _i, [_i, _vp, _vp, _vp, _ll, _vp, _vp, _vp, _ll, _vp, _d,
                                        _vp, _d, _vp, _vp]),
    ("ainv_csr_create", _i, [C.POINTER(_vp), _i, _vp, _vp, _vp, _i]),
    ("ainv_csr_spmv", _i, [_vp, _d, _vp, _d, _vp, _vp]),
    ("ainv_csr_destroy", _i, [_vp]),
    ("ainv_csr_check", _i, [_vp]),
    ("ainv_csr_solve_info", _i, [_vp, _ip, _ip]),
    ("ainv_csr_solve_history", _i, [_vp, _vp, _i, _ip]),
    ("ainv_gpu_solve", _i, [_vp, _vp, _vp, _vp, _i, _d, _i, _ip, _dp, _vp]),
    ("ainv_gpu_update_a", _i, [_vp, _vp, _vp, _vp]),
    ("mld_d_solver_update_a", _i, [_vp, _vp, _i]),
    ("mld_d_solver_load", _i, [_vp, C.c_char_p]),
    ("mld_d_solver_save", _i, [_vp, C.c_char_p]),
    ("mld_d_solver_restore", _i, [_vp, C.c_char_p]),
    ("ainv_gpu_block_solve", _i, [_vp, _vp, _i, _vp, _i, _vp, _i, _d, _i, _vp, _vp, _vp, _vp]),
    ("mld_d_solver_create", _i, [C.POINTER(_vp), C.c_char_p]),
    ("mld_d_solver_destroy", _i, [_vp]),
    ("mld_d_solver_default", _i, [_vp]),
    ("mld_d_solver_cseti", _i, [_vp, C.c_char_p, _i]),
    ("mld_d_solver_csetr", _i, [_vp, C.c_char_p, _d]),
    ("mld_d_solver_csetc", _i, [_vp, C.c_char_p, C.c_char_p]),
    ("mld_d_solver_check", _i, [_vp]),
    ("mld_d_solver_build", _i, [_vp, _i, _vp, _vp, _vp, _i]),
    ("mld_d_solver_cnv", _i, [_vp, _i]),
    ("mld_d_solver_apply", _i, [_vp, _d, _vp, _d, _vp, _c, _vp]),
    ("mld_d_solver_apply_host", _i, [_vp, _d, _vp, _d, _vp, _c]),
    ("mld_d_solver_handle", _vp, [_vp]),
    ("mld_d_solver_get_factors", _i, [_vp, _ip, _llp, _llp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("mld_d_solver_clone", _i, [_vp, C.POINTER(_vp)]),
    ("mld_d_solver_clone_settings", _i, [_vp, _vp]),
    ("mld_d_solver_free", _i, [_vp]),
    ("mld_d_solver_sizeof", C.c_size_t, [_vp]),
    ("mld_d_solver_get_nzeros", _ll, [_vp]),
    ("mld_d_solver_get_wrksz", _i, []),
    ("mld_d_solver_descr", _i, [_vp, C.c_char_p, C.c_size_t]),
    ("mld_d_solver_dump", _i, [_vp, C.c_char_p]),
    ("ainv_server_create", _i, [C.POINTER(_vp), _i, C.c_size_t, _i]),
    ("ainv_server_add_operator", _i, [_vp, _vp, _vp, _ip]),
    ("ainv_server_submit", _i, [_vp, _i, _vp, _vp, _d, _i, _llp]),
    ("ainv_server_wait", _i, [_vp, _ll, _d, _vp]),
    ("ainv_server_stats", _i, [_vp, _vp]),
    ("ainv_server_destroy", _i, [_vp]),
    ("ainv_server_request_bytes", C.c_size_t, [_i]),
    ("ainv_server_plan", _i, [_i, _vp, _i, _vp, _vp]),
]


class Result(C.Structure):
    """ainv_result"""
    _fields_ = [("id", C.c_longlong), ("op", C.c_int), ("status", C.c_int),
                ("iter", C.c_int), ("err", C.c_double), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double)]


class ServerInfo(C.Structure):
    """ainv_server_info"""
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("graph_launches", C.c_longlong), ("kernel_launches", C.c_longlong),
                ("active", C.c_int), ("queued", C.c_int), ("peak_active", C.c_int),
                ("max_slots", C.c_int), ("grid", C.c_int), ("iters_per_launch", C.c_int),
                ("arena_bytes", C.c_size_t), ("arena_used", C.c_size_t),
                ("arena_peak", C.c_size_t), ("clock", C.c_double)]


class AinvError(RuntimeError):
    def __init__(self, info: int, msg: str):
        super().__init__(f"[info={info}] {msg}")
        self.info = info


_lib = None


def lib():
    """Load libainv_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                "(there is no fallback path)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().ainv_last_error().decode()


def check(info: int) -> int:
    if info != SUCCESS:
        raise AinvError(info, last_error())
    return info
