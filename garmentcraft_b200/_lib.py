"""Loads the in-tree device library and declares the C ABI signatures.

There is no fallback: if libklon3d_b200.so is missing, importing the solver
raises. Build it with ``python -m garmentcraft_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_native", "libklon3d_b200.so")

# every entry point include/klon3d_step.h and include/klon3d_mesh.h declare
EXPORTS = [
    "k3d_abi_version", "k3d_params_default", "k3d_simparams_default", "k3d_build_scene",
    "k3d_built_scene_view", "k3d_built_scene_free", "k3d_solver_create", "k3d_solver_destroy",
    "k3d_last_error", "k3d_solver_name", "k3d_upload_scene", "k3d_frame", "k3d_frames_resident",
    "k3d_upload_state", "k3d_download_state", "k3d_operator", "k3d_system_for", "k3d_solve", "k3d_solve_contacts",
    "k3d_residual", "k3d_read_load", "k3d_read_warm_start", "k3d_last_frame_ms", "k3d_last_solve_ms", "k3d_kernel_launches",
    "k3d_pcg_blocks",
    "k3d_operator_noalloc", "k3d_selfcollision_pairs", "k3d_selfcollision_hash", "k3d_selfcollision_springs",
    "k3d_adjoint_forward", "k3d_adjoint_backward",
    "k3d_mesh_create", "k3d_mesh_destroy", "k3d_mesh_last_error", "k3d_mesh_update", "k3d_mesh_get_info",
    "k3d_mesh_tables", "k3d_mesh_nearest", "k3d_mesh_penetration", "k3d_mesh_sdf", "k3d_mesh_set_velocity",
    "k3d_mesh_velocity_at",
]

_lib = None


class K3dError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m garmentcraft_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    st = C.c_int
    L.k3d_abi_version.restype = C.c_int32
    L.k3d_params_default.argtypes = [C.POINTER(_abi.K3dParams)]
    L.k3d_simparams_default.argtypes = [C.POINTER(_abi.K3dSimparams)]
    L.k3d_build_scene.argtypes = [C.POINTER(_abi.K3dPattern), C.POINTER(P)]
    L.k3d_build_scene.restype = st
    L.k3d_built_scene_view.argtypes = [P, C.POINTER(_abi.K3dScene)]
    L.k3d_built_scene_view.restype = st
    L.k3d_built_scene_free.argtypes = [P]
    L.k3d_solver_create.argtypes = [C.POINTER(_abi.K3dParams), C.c_int32]
    L.k3d_solver_create.restype = P
    L.k3d_solver_destroy.argtypes = [P]
    L.k3d_last_error.argtypes = [P]
    L.k3d_last_error.restype = C.c_char_p
    L.k3d_solver_name.argtypes = [P]
    L.k3d_solver_name.restype = C.c_char_p
    L.k3d_upload_scene.argtypes = [P, C.POINTER(_abi.K3dScene)]
    L.k3d_upload_scene.restype = st
    L.k3d_frame.argtypes = [P, C.POINTER(_abi.K3dScene), C.POINTER(_abi.K3dStats)]
    L.k3d_frame.restype = st
    L.k3d_frames_resident.argtypes = [P, C.c_int32, C.POINTER(_abi.K3dStats)]
    L.k3d_frames_resident.restype = st
    L.k3d_adjoint_forward.argtypes = [P, C.c_int32, C.c_int32, C.POINTER(_abi.K3dStats)]
    L.k3d_adjoint_forward.restype = st
    L.k3d_adjoint_backward.argtypes = [P, dp, dp, dp, dp, dp, dp, C.POINTER(_abi.K3dAdjointStats)]
    L.k3d_adjoint_backward.restype = st
    L.k3d_upload_state.argtypes = [P, dp, dp]
    L.k3d_upload_state.restype = st
    L.k3d_download_state.argtypes = [P, dp, dp]
    L.k3d_download_state.restype = st
    L.k3d_operator.argtypes = [P, dp, dp]
    L.k3d_operator.restype = st
    L.k3d_system_for.argtypes = [P, C.POINTER(_abi.K3dSystemReadback)]
    L.k3d_system_for.restype = st
    L.k3d_solve.argtypes = [P, dp, C.POINTER(_abi.K3dCgResult)]
    L.k3d_solve.restype = st
    L.k3d_solve_contacts.argtypes = [P, C.POINTER(_abi.K3dContactSet), dp, C.POINTER(_abi.K3dCgResult)]
    L.k3d_solve_contacts.restype = st
    L.k3d_residual.argtypes = [P, dp, dp]
    L.k3d_residual.restype = st
    L.k3d_read_load.argtypes = [P, dp]
    L.k3d_read_load.restype = st
    L.k3d_read_warm_start.argtypes = [P, dp]
    L.k3d_read_warm_start.restype = st
    L.k3d_last_frame_ms.argtypes = [P]
    L.k3d_last_frame_ms.restype = C.c_double
    L.k3d_last_solve_ms.argtypes = [P]
    L.k3d_last_solve_ms.restype = C.c_double
    L.k3d_kernel_launches.argtypes = [P]
    L.k3d_kernel_launches.restype = C.c_int64
    L.k3d_pcg_blocks.argtypes = [P]
    L.k3d_pcg_blocks.restype = C.c_int32
    L.k3d_operator_noalloc.argtypes = [C.POINTER(_abi.K3dParams), C.POINTER(_abi.K3dScene), C.c_void_p,
                                       C.c_void_p, C.c_void_p]
    L.k3d_operator_noalloc.restype = st
    u32p = C.POINTER(C.c_uint32)
    L.k3d_selfcollision_pairs.argtypes = [P, C.c_int64, C.POINTER(C.c_int32), u32p, dp, dp, dp, dp]
    L.k3d_selfcollision_pairs.restype = C.c_int64
    L.k3d_selfcollision_hash.argtypes = [P, C.c_int32, C.c_int64, u32p, C.c_int64, u32p, C.POINTER(C.c_int64)]
    L.k3d_selfcollision_hash.restype = C.c_int64
    L.k3d_selfcollision_springs.argtypes = [P, C.c_int64, dp, dp]
    L.k3d_selfcollision_springs.restype = C.c_int64
    i32p = C.POINTER(C.c_int32)
    L.k3d_mesh_create.argtypes = [dp, C.c_int64, u32p, C.c_int64, C.c_double, C.c_int32, C.POINTER(P), C.c_char_p,
                                  C.c_int64]
    L.k3d_mesh_create.restype = st
    L.k3d_mesh_destroy.argtypes = [P]
    L.k3d_mesh_last_error.argtypes = [P]
    L.k3d_mesh_last_error.restype = C.c_char_p
    L.k3d_mesh_update.argtypes = [P, dp]
    L.k3d_mesh_update.restype = st
    L.k3d_mesh_get_info.argtypes = [P, C.POINTER(_abi.K3dMeshInfo)]
    L.k3d_mesh_get_info.restype = st
    L.k3d_mesh_tables.argtypes = [P, dp, dp, u32p, dp]
    L.k3d_mesh_tables.restype = st
    L.k3d_mesh_nearest.argtypes = [P, dp, C.c_int64, C.c_double, dp, dp, dp, i32p, i32p]
    L.k3d_mesh_nearest.restype = st
    L.k3d_mesh_penetration.argtypes = [P, dp, dp, C.c_int64, i32p, dp, dp]
    L.k3d_mesh_penetration.restype = st
    L.k3d_mesh_sdf.argtypes = [P, i32p, dp, C.c_double, C.c_double, C.POINTER(C.c_float)]
    L.k3d_mesh_sdf.restype = st
    L.k3d_mesh_set_velocity.argtypes = [P, dp]
    L.k3d_mesh_set_velocity.restype = st
    L.k3d_mesh_velocity_at.argtypes = [P, i32p, dp, C.c_int64, dp, dp]
    L.k3d_mesh_velocity_at.restype = st
    if L.k3d_abi_version() != _abi.K3D_ABI_VERSION:
        raise RuntimeError("libklon3d_b200.so ABI version mismatch")
    _lib = L
    return L
