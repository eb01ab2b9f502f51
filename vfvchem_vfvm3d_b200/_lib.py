"""ctypes binding of libvfvgpu.so (the C ABI declared in include/vfv_gpu.h).

The shared library is built in-tree (``make -C vfvchem_vfvm3d_b200``). Loading fails loudly when
it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvfvgpu.so")

VFV_OK, VFV_NOT_CONVERGED, VFV_NONFINITE, VFV_BAD_INPUT, VFV_CUDA_ERROR, VFV_TIMEOUT = range(6)
PRECOND_NONE, PRECOND_JACOBI, PRECOND_ILU0, PRECOND_BJ4 = 0, 1, 2, 3
FP64, MIXED = 0, 1
ILU_MULTICOLOR, ILU_NATURAL = 0, 1
ORTHO_CGS2, ORTHO_DGKS, ORTHO_CGS = 0, 1, 2
ENGINE_PERSISTENT, ENGINE_GRAPH, ENGINE_OVERLAP = 0, 1, 2
BC_TEMP, BC_FLUX = 0, 1


class GmresOpts(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("restart", C.c_int32),
        ("max_outer", C.c_int32),
        ("precond", C.c_int32),
        ("precision", C.c_int32),
        ("ilu_order", C.c_int32),
        ("engine", C.c_int32),
        ("inner_rtol", C.c_double),
        ("wait_limit", C.c_int64),
        ("ilu_sweeps", C.c_int32),
        ("ilu_sweeps_upper", C.c_int32),
        ("ortho", C.c_int32),
        ("ilu_sweep_half", C.c_int32),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("iters", C.c_int32),
        ("cycles", C.c_int32),
        ("levels", C.c_int32),
        ("relres", C.c_double),
        ("bnorm", C.c_double),
    ]


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_I64P = C.POINTER(C.c_int64)
_I32P = C.POINTER(C.c_int32)
_U64P = C.POINTER(C.c_uint64)
_DP = C.POINTER(C.c_double)

# (name, restype, argtypes) for every symbol of include/vfv_gpu.h
SIGNATURES = [
    ("vfv_gmres_default_opts", None, [C.POINTER(GmresOpts)]),
    ("vfv_ctx_create", C.c_int, [C.c_int, _PP]),
    ("vfv_ctx_destroy", None, [_P]),
    ("vfv_last_error", C.c_char_p, [_P]),
    ("vfv_ctx_synchronize", C.c_int, [_P]),
    ("vfv_ctx_stream", C.c_void_p, [_P]),
    ("vfv_ctx_launch_count", C.c_int64, [_P]),
    ("vfv_pattern_from_triplets", C.c_int, [_P, C.c_int64, C.c_int64, _U64P, _U64P, _PP]),
    ("vfv_pattern_from_csr", C.c_int, [_P, C.c_int64, _I32P, _I32P, _PP]),
    ("vfv_pattern_destroy", None, [_P]),
    ("vfv_pattern_info", C.c_int, [_P, _I64P, _I64P, _I64P]),
    ("vfv_values_from_triplets", C.c_int, [_P, _P, _DP]),
    ("vfv_values_set", C.c_int, [_P, _P, _P, C.c_int]),
    ("vfv_csr_export", C.c_int, [_P, _P, _I32P, _I32P, _DP]),
    ("vfv_solve", C.c_int, [_P, _P, _DP, _DP, _DP, C.POINTER(GmresOpts), C.POINTER(SolveInfo)]),
    ("vfv_solve_device", C.c_int, [_P, _P, _P, _P, _P, C.POINTER(GmresOpts), C.POINTER(SolveInfo)]),
    ("vfv_spmv_device", C.c_int, [_P, _P, _P, _P]),
    ("vfv_spmv_device_f32", C.c_int, [_P, _P, _P, _P]),
    ("vfv_ilu0_apply_device", C.c_int, [_P, _P, C.c_int, _P, _P, _I32P]),
    ("vfv_ilu0_apply_device_f32", C.c_int, [_P, _P, C.c_int, _P, _P, _P, _I32P]),
    ("vfv_ilu0_sweep_apply_device", C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P]),
    ("vfv_ilu0_sweep_apply_device_f32", C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P]),
    ("vfv_ilu0_sweep_apply_device_f16", C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P]),
    ("vfv_ilu0_sweep_layout", C.c_int, [_P, C.c_int, _I32P]),
    ("vfv_pattern_autotune", C.c_int, [_P, _P, _I32P, _I32P]),
    ("vfv_pattern_set_spmv_lanes", C.c_int, [_P, _P, C.c_int32, C.c_int32]),
    ("vfv_pattern_spmv_shape", C.c_int, [_P, _I32P, _I32P, _I32P, _I32P]),
    ("vfv_ilu0_ordering", C.c_int, [_P, _P, C.c_int, _I32P, _I32P, _I32P]),
    ("vfv_ilu0_apply_device_noalloc", C.c_int, [_P, _P, C.c_int, _P, _P, _I32P]),
    ("vfv_mesh_jitter_cube", C.c_int, [C.c_int, C.c_uint64, C.c_double, _PP]),
    ("vfv_mesh_from_vertices", C.c_int, [C.c_int64, C.c_int64, _DP, _I32P, _PP]),
    ("vfv_mesh_destroy", None, [_P]),
    ("vfv_mesh_dual_device", C.c_int, [_P, _P]),
    ("vfv_mesh_jitter_cubes_device_dual", C.c_int, [_P, C.c_int, _I32P, _U64P, C.c_double, C.POINTER(C.c_void_p)]),
    ("vfv_mesh_jitter_cubes", C.c_int, [C.c_int, _I32P, _U64P, C.c_double, C.POINTER(C.c_void_p)]),
    ("vfv_mesh_info", C.c_int, [_P, _I64P, _I64P, _I64P, _I64P, _I64P]),
    ("vfv_mesh_export", C.c_int, [_P, _DP, _I32P, _I32P]),
    ("vfv_mesh_write_vtu", C.c_int, [_P, _DP, C.c_int, C.c_char_p]),
    ("vfv_mesh_write_csv", C.c_int, [_P, _DP, C.c_int, C.c_char_p]),
    ("vfv_points_write_vtu", C.c_int, [C.c_int64, _DP, _DP, C.c_int, C.c_char_p]),
    ("vfv_points_write_csv", C.c_int, [C.c_int64, _DP, _DP, C.c_int, C.c_char_p]),
    ("vfv_mesh_export_dual", C.c_int, [_P, _I64P, _I32P, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _I64P, _I32P, _I32P, _DP, _DP, _DP]),
    ("vfv_heat_create", C.c_int, [_P, _P, C.c_int32, _I32P, _PP]),
    ("vfv_heat_destroy", None, [_P]),
    ("vfv_heat_pattern", C.c_void_p, [_P]),
    ("vfv_heat_assemble", C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.c_int, _DP]),
    ("vfv_heat_rhs_device", C.c_void_p, [_P]),
    ("vfv_update_grad", C.c_int, [_P, _P, _DP, _DP]),
    ("vfv_transport_create", C.c_int, [_P, C.c_int, C.POINTER(C.c_void_p), C.c_double, _PP]),
    ("vfv_transport_destroy", None, [_P]),
    ("vfv_transport_pattern", C.c_void_p, [_P]),
    ("vfv_transport_info", C.c_int, [_P, _I64P, _I64P, _I32P, _I64P]),
    ("vfv_transport_assemble", C.c_int, [_P, _P, _P, _P, C.c_int]),
    ("vfv_transport_run", C.c_int, [_P, _P, _DP, C.c_int, C.POINTER(GmresOpts), _DP, _I32P]),
    ("vfv_transport_mesh_steps", C.c_int, [_P, _I64P]),
    ("vfv_transport_adjoint_D", C.c_int, [_P, _P, _DP, C.c_int, C.c_int, _DP, C.POINTER(GmresOpts), _DP, _DP, _I32P]),
    ("vfv_flow_pattern_host", C.c_int, [_P, C.c_int64, _I64P, _I64P, _I32P, _I32P]),
    ("vfv_flow_create", C.c_int, [_P, _P, _DP, _DP, _DP, _DP, C.c_int64, C.c_double, C.POINTER(C.c_void_p)]),
    ("vfv_flow_destroy", None, [_P]),
    ("vfv_flow_pattern", _P, [_P]),
    ("vfv_flow_info", C.c_int, [_P, _I64P, _I64P, _I64P]),
    ("vfv_flow_assemble", C.c_int, [_P, _P, _DP, _DP]),
    ("vfv_flow_assemble_device", C.c_int, [_P, _P, C.c_void_p, C.c_void_p]),
    ("vfv_flow_picard", C.c_int, [_P, _P, _DP, C.c_int, C.c_double, C.c_double, C.POINTER(GmresOpts), _DP, _I32P, _I32P, _DP]),
    ("vfv_heat_adjoint", C.c_int, [_P, _P, _DP, _DP, C.POINTER(GmresOpts), _DP, _DP, _DP, C.POINTER(SolveInfo)]),
]

_lib = None


def load() -> C.CDLL:
    """Load libvfvgpu.so and bind every declared symbol; raises if the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libvfvgpu.so not built: run `make -C {_HERE}` (no CPU fallback exists)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)
