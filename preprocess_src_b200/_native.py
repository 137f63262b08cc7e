"""ctypes binding of the C ABI in include/rbc_step.h.

The library is built in-tree by ``python -m preprocess_src_b200.build`` into
``preprocess_src_b200/_lib/libpreprocess_src_b200.so``.  There is no fallback:
if the library is missing or fails to load, importing raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libpreprocess_src_b200.so"

RBC_OK, RBC_ERR_ARG, RBC_ERR_CUDA, RBC_ERR_UNSUPPORTED = 0, 1, 2, 3
RBC_ERR_TOPOLOGY, RBC_ERR_NOT_CONVERGED, RBC_ERR_NONFINITE, RBC_ERR_STATE, RBC_ERR_NO_DEVICE = 4, 5, 6, 7, 8
RBC_COMP, RBC_BUFF, RBC_WALL = 0, 1, 2
RBC_STORE_F32, RBC_STORE_F16 = 0, 1
RBC_FLOW_CHANNEL, RBC_FLOW_SHEAR = 0, 1
RBC_WALLS_BOTH, RBC_WALLS_TOP = 0, 1
RBC_NOALLOC_MAX_CELLS = 4096
RBC_NOALLOC_MAX_VERTEX = 4096
RBC_SHAPE_LBM_PLANES = 1
RBC_NUM_KERNELS = 8
RBC_KERNEL_NAMES = ("step_begin", "membrane", "spread", "lbm_collide_stream", "force_reset", "advect", "vof", "volume")
RBC_FLAG_VC_NOT_CONVERGED, RBC_FLAG_NONFINITE, RBC_FLAG_SPREAD_OVERFLOW, RBC_FLAG_SOLVE_RESIDUAL = 1, 2, 4, 8
RBC_FLAG_VOF_NOT_CONVERGED = 16


class RbcParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dt", C.c_double), ("tau", C.c_double), ("Cr", C.c_double),
                ("P", C.c_double), ("B", C.c_double), ("flowstart", C.c_int), ("freq", C.c_double),
                ("LX", C.c_double), ("LZ", C.c_double), ("xmin", C.c_double), ("xmax", C.c_double),
                ("zmin", C.c_double), ("zmax", C.c_double), ("C", C.c_double), ("rgs", C.c_double),
                ("law", C.c_int), ("br", C.c_double), ("M", C.c_int), ("rk_order", C.c_int),
                ("storage", C.c_int), ("membrane_fp64", C.c_int), ("solver_iters", C.c_int),
                ("device", C.c_int), ("flow", C.c_int), ("sr", C.c_double), ("walls", C.c_int),
                ("tube_r", C.c_double), ("bend_spont", C.c_int), ("lambda1", C.c_double), ("vof_k", C.c_int),
                ("vof_residual", C.c_double), ("vof_itrmax", C.c_int)]


class RbcMesh(C.Structure):
    _fields_ = [("ncell", C.c_int), ("vertex", C.c_int), ("element", C.c_int),
                ("tri", C.POINTER(C.c_int)), ("xr", C.POINTER(C.c_double))]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_H = C.c_void_p

# name -> argtypes (all return int unless listed in _RESTYPE)
_SIGS = {
    "rbc_create": [C.POINTER(RbcParams), C.POINTER(RbcMesh), _IP, C.POINTER(_H)],
    "rbc_destroy": [_H],
    "rbc_last_error": [_H],
    "rbc_import_ref_lattice": [_H, _DP],
    "rbc_export_ref_lattice": [_H, _DP, _DP, _DP, _DP, _DP],
    "rbc_export_ref_force": [_H, _DP, _DP, _DP],
    "rbc_import_ref_cells": [_H, _DP, _DP, _DP, _DP, _DP, _DP, _DP],
    "rbc_import_ref_vertex_force": [_H, _DP, _DP, _DP],
    "rbc_export_ref_cells": [_H, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP],
    "rbc_set_iter": [_H, C.c_int],
    "rbc_get_iter": [_H, _IP],
    "rbc_stress": [_H],
    "rbc_ibm_st1": [_H],
    "rbc_lbm_d3q19": [_H],
    "rbc_ibm_st2": [_H],
    "rbc_volume_correction": [_H, _IP],
    "rbc_step": [_H, C.c_int],
    "rbc_get_status": [_H, _IP, _IP],
    "rbc_cell_metrics": [_H, _DP, _DP, _DP],
    "rbc_cell_metrics_async": [_H, _DP],
    "rbc_synchronize": [_H],
    "rbc_launch_count": [_H, C.POINTER(C.c_longlong)],
    "rbc_dims": [_H, _IP, _IP, _IP, _IP, _IP, _IP],
    "rbc_get_stream": [_H, C.POINTER(C.c_void_p)],
    "rbc_profile_steps": [_H, C.c_int, _DP],
    "rbc_set_launch_shape": [_H, C.c_int, C.c_int],
    "rbc_get_launch_shape": [_H, C.c_int, _IP],
    "rbc_cell_metrics_noalloc": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p,
                                 _DP, _DP, _DP],
    "rbc_batch_create": [C.POINTER(_H), C.c_int, C.POINTER(_H)],
    "rbc_batch_destroy": [_H],
    "rbc_batch_set_form": [_H, C.c_int],
    "rbc_batch_get_form": [_H, _IP, C.POINTER(C.c_char_p)],
    "rbc_batch_set_shape": [_H, C.c_int, C.c_int, C.c_int],
    "rbc_batch_get_shape": [_H, _IP, _IP, _IP],
    "rbc_batch_launch_count": [_H, C.POINTER(C.c_longlong)],
    "rbc_batch_last_error": [_H],
    "rbc_batch_step": [_H, C.c_int],
    "rbc_batch_synchronize": [_H],
    "rbc_batch_get_stream": [_H, C.POINTER(C.c_void_p)],
    "rbc_batch_set_chain": [_H, C.c_int],
    "rbc_batch_get_chain": [_H, _IP],
    "rbc_batch_autotune": [_H, C.c_int, _IP],
    "rbc_adjoint_record": [_H, C.c_int, C.c_int],
    "rbc_adjoint_record_binomial": [_H, C.c_int, C.c_int, C.c_int],
    "rbc_adjoint_schedule": [_H, _IP, _IP, _IP, C.POINTER(C.c_longlong)],
    "rbc_adjoint_binomial_plan": [C.c_int, C.c_int, _IP, _IP, C.c_int, _IP],
    "rbc_adjoint_backward": [_H, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, C.POINTER(C.c_float)],
    "rbc_set_coefficients": [_H, C.c_double, C.c_double, C.c_double],
    "rbc_set_output_interval": [_H, C.c_int],
    "rbc_write_restart": [_H, C.c_char_p, C.c_int],
    "rbc_read_restart": [_H, C.c_char_p, _IP],
    "rbc_write_cell_file": [_H, C.c_char_p],
    "rbc_write_prof_file": [_H, C.c_char_p],
    "rbc_write_center_file": [_H, C.c_char_p],
    "rbc_read_center_file": [_H, C.c_char_p],
    "rbc_thinc_wlic": [_H],
    "rbc_front_tracking": [_H, _IP],
    "rbc_export_ref_vof": [_H, _DP, _DP],
    "rbc_import_ref_vof": [_H, _DP, _DP],
    "rbc_add_wbc": [_H, C.POINTER(RbcMesh), C.c_double, C.c_double],
    "rbc_wbc_dims": [_H, _IP, _IP, _IP],
    "rbc_import_ref_wbc": [_H, _DP, _DP, _DP, _DP, _DP, _DP, _DP],
    "rbc_export_ref_wbc": [_H, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP],
    "rbc_wbc_metrics": [_H, _DP, _DP, _DP],
}
_RESTYPE = {"rbc_last_error": C.c_char_p, "rbc_batch_last_error": C.c_char_p}

# every entry point declared in include/rbc_step.h
EXPORTED = tuple(_SIGS)

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m preprocess_src_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


class RbcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rbc error {code}: {msg}")
        self.code = code


def check(code: int, handle=None) -> None:
    if code != RBC_OK:
        msg = lib().rbc_last_error(handle)
        raise RbcError(code, msg.decode() if msg else "")


def params_struct(d: dict) -> RbcParams:
    p = RbcParams()
    for name, _ in RbcParams._fields_:
        setattr(p, name, d.get(name, -1) if name == "device" else d[name])
    return p
