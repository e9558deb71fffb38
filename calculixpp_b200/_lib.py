"""ctypes binding of libcxg.so (declared in include/cxg.h).

The library is built in-tree by calculixpp_b200.build. Loading fails loudly when it is
missing: there is no CPU fallback for anything in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcxg.so")

CXG_OK = 0
CXG_ERR_INVALID_ARGUMENT = 1
CXG_ERR_CUDA = 2
CXG_ERR_OUT_OF_MEMORY = 3
CXG_ERR_NEGATIVE_JACOBIAN = 4
CXG_ERR_UNSUPPORTED = 5
CXG_ERR_UNKNOWN_NODE = 6
CXG_ERR_NO_GPU = 7
CXG_ERR_NOT_CONVERGED = 8

FP64, MIXED = 0, 1
SOLVER_DIRECT, SOLVER_CG, SOLVER_IC0_CG = 0, 1, 2
COMMITTED, TRIAL = 0, 1
ACCUMULATE = 1

_vp = C.c_void_p


class CxgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cxg error {code}: {msg}")
        self.code = code


class CxgMaterial(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("n_plastic", C.c_int32),
                ("eqplastic", _vp), ("yield_", _vp), ("hardening", C.c_int32),
                ("h_kin", C.c_double)]


class CxgMeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_elems", C.c_int64), ("elem_type", C.c_int32),
                ("coords", _vp), ("conn", _vp), ("young", _vp), ("poisson", _vp),
                ("elem_mat", _vp), ("n_materials", C.c_int32), ("materials", _vp)]


class CxgDofmapDesc(C.Structure):
    _fields_ = [("dof_eq", _vp), ("prescribed", _vp), ("n_free", C.c_int32)]


class CxgPlanInfo(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_elems", C.c_int64), ("elem_type", C.c_int32),
                ("n_free", C.c_int32), ("nnz", C.c_int64), ("n_gauss_points", C.c_int64),
                ("precision", C.c_int32), ("device", C.c_int32), ("device_bytes", C.c_int64)]


class CxgBatchModelInfo(C.Structure):
    _fields_ = [("elem_type", C.c_int32), ("group", C.c_int32), ("n_nodes", C.c_int64), ("n_elems", C.c_int64),
                ("n_free", C.c_int32), ("nnz", C.c_int64), ("vals_offset", C.c_int64), ("rhs_offset", C.c_int64),
                ("node_offset", C.c_int64)]


class CxgBatchInfo(C.Structure):
    _fields_ = [("n_models", C.c_int32), ("n_groups", C.c_int32), ("n_nodes", C.c_int64), ("n_elems", C.c_int64),
                ("n_free", C.c_int64), ("nnz", C.c_int64), ("device_bytes", C.c_int64)]


# name -> (restype, argtypes)
SIGNATURES = {
    "cxg_last_error": (C.c_char_p, []),
    "cxg_abi_version": (C.c_int, []),
    "cxg_nodes_per_element": (C.c_int, [C.c_int32]),
    "cxg_gauss_points_per_element": (C.c_int, [C.c_int32]),
    "cxg_plan_create": (C.c_int, [C.POINTER(CxgMeshDesc), C.POINTER(CxgDofmapDesc), C.c_int32,
                                  C.POINTER(_vp)]),
    "cxg_plan_destroy": (C.c_int, [_vp]),
    "cxg_plan_get_info": (C.c_int, [_vp, C.POINTER(CxgPlanInfo)]),
    "cxg_plan_set_precision": (C.c_int, [_vp, C.c_int32]),
    "cxg_plan_get_pattern": (C.c_int, [_vp, _vp, _vp]),
    "cxg_plan_pattern_device": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp)]),
    "cxg_plan_update_coords": (C.c_int, [_vp, _vp]),
    "cxg_plan_update_young": (C.c_int, [_vp, _vp]),
    "cxg_plan_check": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "cxg_plan_set_launch_config": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "cxg_plan_set_j2_fp32_return": (C.c_int, [_vp, C.c_int32]),
    "cxg_plan_set_thermal_strain": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cxg_thermal_strain_load": (C.c_int, [_vp, _vp, _vp]),
    "cxg_thermal_plan_set_films": (C.c_int, [_vp, C.c_int64, _vp, _vp, _vp, _vp]),
    "cxg_plan_set_ring_bytes": (C.c_int, [_vp, C.c_int64]),
    "cxg_plan_create_mpc": (C.c_int, [_vp, _vp, _vp, C.c_int32, _vp]),
    "cxg_solve_sparse": (C.c_int, [C.c_int32, C.c_int64, _vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_double, C.c_int32,
                                   _vp, _vp]),
    "cxg_batch_assemble_tangent": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cxg_batch_commit": (C.c_int, [_vp, _vp]),
    "cxg_batch_get_state": (C.c_int, [_vp, C.c_int32, C.c_int32, _vp]),
    "cxg_plan_use_reference_pattern": (C.c_int, [_vp, C.c_int32]),
    "cxg_plan_get_windows": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "cxg_assemble_linear": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cxg_assemble_linear_ex": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int32, _vp]),
    "cxg_assemble_tangent": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cxg_assemble_mass": (C.c_int, [_vp, _vp, C.c_int32, _vp, _vp]),
    "cxg_assemble_geometric": (C.c_int, [_vp, _vp, _vp, _vp]),
    "cxg_thermal_plan_create": (C.c_int, [C.POINTER(CxgMeshDesc), _vp, _vp, C.c_int32, C.POINTER(_vp)]),
    "cxg_assemble_conduction": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "cxg_recover_gauss_stress": (C.c_int, [_vp, _vp, _vp, _vp]),
    "cxg_recover_fields": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cxg_state_get": (C.c_int, [_vp, C.c_int32, _vp]),
    "cxg_state_set": (C.c_int, [_vp, C.c_int32, _vp]),
    "cxg_state_commit": (C.c_int, [_vp, _vp]),
    "cxg_element_stiffness": (C.c_int, [C.c_int32, C.c_int64, _vp, _vp, _vp, C.c_int32, _vp, _vp]),
    "cxg_element_tangent_force": (C.c_int, [C.c_int32, C.c_int64, _vp, _vp, C.POINTER(CxgMaterial),
                                            _vp, _vp, C.c_int32, _vp, _vp, _vp]),
    "cxg_adjoint_compliance": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cxg_spmv": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cxg_solve_cg": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                               C.POINTER(C.c_double), _vp]),
    "cxg_element_tangent_force_noalloc": (C.c_int, [C.c_int32, C.c_int64, _vp, _vp, C.POINTER(CxgMaterial),
                                                    _vp, _vp, C.c_int32, _vp, _vp, _vp]),
    "cxg_batch_create": (C.c_int, [C.c_int32, C.POINTER(CxgMeshDesc), C.POINTER(CxgDofmapDesc), C.c_int32,
                                   C.POINTER(_vp)]),
    "cxg_batch_destroy": (C.c_int, [_vp]),
    "cxg_batch_get_info": (C.c_int, [_vp, C.POINTER(CxgBatchInfo)]),
    "cxg_batch_get_model_info": (C.c_int, [_vp, C.c_int32, C.POINTER(CxgBatchModelInfo)]),
    "cxg_batch_get_pattern": (C.c_int, [_vp, C.c_int32, _vp, _vp]),
    "cxg_batch_set_precision": (C.c_int, [_vp, C.c_int32]),
    "cxg_batch_set_launch": (C.c_int, [_vp, C.c_int32]),
    "cxg_batch_get_launch": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "cxg_batch_assemble": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cxg_batch_graph_launch": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cxg_batch_check": (C.c_int, [_vp]),
    "cxg_batch_tune": (C.c_int, [_vp, _vp, _vp, _vp, C.c_char_p, _vp]),
    "cxg_batch_group_config": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "cxg_batch_set_group_config": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
}

_LIB = None


def load():
    """Load libcxg.so once; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with python -m calculixpp_b200.build")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def check(rc):
    if rc != CXG_OK:
        msg = load().cxg_last_error()
        raise CxgError(rc, msg.decode() if msg else "")
