"""ctypes binding of libfmgpu.so (the C-ABI declared in include/fmgpu.h).

The library is built in-tree (``gnu_femlisp_b200/libfmgpu.so``).  There is no
CPU fallback: if the library or a CUDA device is missing every call raises.
"""
from __future__ import annotations

import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfmgpu.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "fmgpu.h")

FMG_OK = 0
FMG_K_CONST, FMG_K_CELL, FMG_F_CONST, FMG_F_IP, FMG_LAMBDA_MU_CELL, FMG_F_VEC = 0, 1, 2, 3, 4, 5
FMG_JACOBI, FMG_SOR, FMG_SSC, FMG_PSC = 0, 1, 2, 3
FMG_ASSEMBLE_REDISCRETIZE, FMG_ASSEMBLE_GALERKIN = 0, 1
FMG_CSR, FMG_CCS = 0, 1
FMG_METHOD_MG, FMG_METHOD_CG_MG, FMG_METHOD_CG = 0, 1, 2
FMG_MULTIPLICATIVE, FMG_ADDITIVE = 0, 1
FMG_MXK_RESIDUAL, FMG_MXK_SMOOTH, FMG_MXK_MATVEC64 = 1, 2, 3
FMG_MXK_RESTRICT, FMG_MXK_PROLONG, FMG_MXK_PRESMOOTH = 4, 5, 6

_ERRNAMES = {-1: "FMG_ERR_ARG", -2: "FMG_ERR_CUDA", -3: "FMG_ERR_STATE", -4: "FMG_ERR_NOMEM",
             -5: "FMG_ERR_NUMERIC", -6: "FMG_ERR_UNSUPPORTED", -7: "FMG_ERR_IO"}

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class FmgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class SolveCfg(ctypes.Structure):
    """fmg_solve_cfg: the initargs of <geometric-cs>/<cg> and the
    success/failure forms of <linear-solver>."""
    _fields_ = [
        ("method", ctypes.c_int),
        ("smoother", ctypes.c_int),
        ("damp", ctypes.c_double),
        ("pre_steps", ctypes.c_int),
        ("post_steps", ctypes.c_int),
        ("gamma", ctypes.c_int),
        ("compat_alias", ctypes.c_int),
        ("coarse_damp", ctypes.c_double),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("maxsteps", ctypes.c_int),
        ("combination", ctypes.c_int),
        ("fmg", ctypes.c_int),
    ]


class MixedCfg(ctypes.Structure):
    """fmg_mixed_cfg: inner tolerance and limits of the mixed-precision solve."""
    _fields_ = [
        ("inner_rtol", ctypes.c_double),
        ("max_inner", ctypes.c_int),
        ("max_outer", ctypes.c_int),
        ("matrix_free", ctypes.c_int),
        ("judge", ctypes.c_int),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "fmg_init": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "fmg_finalize": (ctypes.c_int, [_vp]),
    "fmg_last_error": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int]),
    "fmg_synchronize": (ctypes.c_int, [_vp]),
    "fmg_get_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "fmg_launch_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_longlong)]),
    "fmg_grid_create": (ctypes.c_int, [_vp] + [ctypes.c_int] * 7 + [ctypes.POINTER(_vp)]),
    "fmg_grid_create_algebraic": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
                                                 ctypes.POINTER(_vp)]),
    "fmg_set_interpolation": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int), _dp, ctypes.c_long, ctypes.c_long]),
    "fmg_grid_destroy": (ctypes.c_int, [_vp]),
    "fmg_grid_nnodes": (ctypes.c_long, [_vp, ctypes.c_int]),
    "fmg_grid_nslots": (ctypes.c_int, [_vp]),
    "fmg_set_coefficient": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_long]),
    "fmg_assemble": (ctypes.c_int, [_vp]),
    "fmg_get_matrix": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "fmg_set_matrix": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), _dp, ctypes.c_long]),
    "fmg_set_rhs": (ctypes.c_int, [_vp, _dp, ctypes.c_long]),
    "fmg_get_rhs": (ctypes.c_int, [_vp, _dp]),
    "fmg_set_node_damping": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_long]),
    "fmg_vec_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "fmg_vec_destroy": (ctypes.c_int, [_vp]),
    "fmg_vec_set": (ctypes.c_int, [_vp, _dp, ctypes.c_long]),
    "fmg_vec_get": (ctypes.c_int, [_vp, _dp, ctypes.c_long]),
    "fmg_vec_fill": (ctypes.c_int, [_vp, ctypes.c_double]),
    "fmg_copy": (ctypes.c_int, [_vp, _vp]),
    "fmg_axpy": (ctypes.c_int, [ctypes.c_double, _vp, _vp]),
    "fmg_dot": (ctypes.c_int, [_vp, _vp, _dp]),
    "fmg_l2_norm": (ctypes.c_int, [_vp, _dp]),
    "fmg_matvec": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "fmg_residual": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "fmg_matvec_mf": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "fmg_batch_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "fmg_batch_load": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "fmg_batch_solve": (ctypes.c_int, [_vp, ctypes.c_void_p, _vp, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "fmg_restrict": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "fmg_prolongate": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "fmg_jacobi": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp, _vp]),
    "fmg_sor": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp, _vp, _vp]),
    "fmg_ssc": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp, _vp, _vp]),
    "fmg_psc": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp, _vp]),
    "fmg_coarse_solve": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp]),
    "fmg_vcycle": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), _vp, _vp, _vp]),
    "fmg_solve": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), _vp, _dp, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "fmg_dot_noalloc": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_long, _vp]),
    "fmg_mixed_top_kernel": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "fmg_wait_selftest": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_longlong]),
    "fmg_cg_start": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), _vp]),
    "fmg_cg_step": (ctypes.c_int, [_vp, _vp, _vp, _dp]),
    "fmg_assemble_levels": (ctypes.c_int, [_vp, ctypes.c_int]),
    "fmg_solve_mixed": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), ctypes.POINTER(MixedCfg), _vp, _dp,
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "fmg_net_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(_vp)]),
    "fmg_net_destroy": (ctypes.c_int, [_vp]),
    "fmg_net_nparams": (ctypes.c_long, [_vp]),
    "fmg_net_get_params": (ctypes.c_int, [_vp, _fp, ctypes.c_long]),
    "fmg_net_set_params": (ctypes.c_int, [_vp, _fp, ctypes.c_long]),
    "fmg_net_get_grads": (ctypes.c_int, [_vp, _fp, ctypes.c_long]),
    "fmg_net_zero_grads": (ctypes.c_int, [_vp]),
    "fmg_net_adam": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "fmg_net_save": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "fmg_net_load": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]),
    "fmg_net_damping": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _dp]),
    "fmg_net_apply": (ctypes.c_int, [_vp, _vp]),
    "fmg_net_backward": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _dp]),
    "fmg_learn_loss": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), _vp, _dp, _dp]),
    "fmg_learned_judge": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), _dp, _dp, ctypes.POINTER(ctypes.c_int)]),
    "fmg_learned_judge_mixed": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), ctypes.POINTER(MixedCfg), _dp, _dp,
                                               ctypes.POINTER(ctypes.c_int)]),
    "fmg_learned_status": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), _dp, _dp, ctypes.POINTER(ctypes.c_int)]),
    "fmg_learn_loss_levels": (ctypes.c_int, [_vp, ctypes.POINTER(SolveCfg), _vp, ctypes.c_int, _dp, _dp]),
    "fmg_learn_step": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(SolveCfg), ctypes.c_int, ctypes.c_ulonglong,
                                      ctypes.c_int, _dp]),
}

_lib = None


def header_symbols(path: str = HEADER) -> list[str]:
    """Every function declared in include/fmgpu.h."""
    with open(path) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmg_[a-z0-9_]+)\s*\(", text)))


def load(path: str = LIB_PATH):
    """Load libfmgpu.so; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FmgError(-6, f"{path} not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a):
    import numpy as np
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def fptr(a):
    import numpy as np
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_fp)
