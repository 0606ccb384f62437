"""ctypes declarations of the C ABI in include/mgsb.h.

The shared library is built in-tree (``python -m multigridsoftbody_b200.build``).
Loading fails loudly when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmgsb.so")

SOLVER_REFERENCE_JACOBI = 0
SOLVER_MULTIGRID = 1
PRECISION_FP32 = 0
PRECISION_MIXED = 1

STATUS = {
    0: "ok", 1: "invalid argument", 2: "degenerate tetrahedron", 3: "CUDA error", 4: "diverged",
    5: "timeout", 6: "not supported", 7: "out of memory", 8: "I/O error",
}


class MgsbError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"mgsb status {status} ({STATUS.get(status, '?')}): {msg}")


class Params(C.Structure):
    _fields_ = [
        ("solver", C.c_int32),
        ("iterations", C.c_int32),
        ("dt", C.c_float),
        ("damping", C.c_float),
        ("gravity", C.c_float * 3),
        ("volume_stiffness", C.c_float),
        ("collision_stiffness", C.c_float),
        ("cheb_rho", C.c_float),
        ("relaxation", C.c_float),
        ("density", C.c_float),
        ("youngs_modulus", C.c_float),
        ("poisson_ratio", C.c_float),
        ("contact_stiffness", C.c_float),
        ("levels", C.c_int32),
        ("pre_sweeps", C.c_int32),
        ("post_sweeps", C.c_int32),
        ("jacobi_omega", C.c_float),
        ("precision", C.c_int32),
        ("refinement_passes", C.c_int32),
        ("use_graph", C.c_int32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
    ]


class Mesh(C.Structure):
    _fields_ = [
        ("num_verts", C.c_int32),
        ("num_tets", C.c_int32),
        ("positions", C.POINTER(C.c_float)),
        ("tets", C.POINTER(C.c_int32)),
        ("grid_dims", C.c_int32 * 3),
    ]


class MeshData(C.Structure):
    _fields_ = [
        ("num_verts", C.c_int32),
        ("num_tets", C.c_int32),
        ("positions", C.POINTER(C.c_float)),
        ("tets", C.POINTER(C.c_int32)),
        ("num_tris", C.c_int32),
        ("tris", C.POINTER(C.c_int32)),
        ("tri_opposite", C.POINTER(C.c_int32)),
        ("grid_dims", C.c_int32 * 3),
    ]


# (name, restype, argtypes) of every exported entry point
_P = C.c_void_p
_FP = C.POINTER(C.c_float)
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
_U8P = C.POINTER(C.c_uint8)
SIGNATURES = [
    ("mgsb_default_params", C.c_int, [C.c_int32, C.POINTER(Params)]),
    ("mgsb_create", C.c_int, [C.POINTER(Mesh), C.POINTER(Params), C.POINTER(_P)]),
    ("mgsb_batch_create", C.c_int, [C.c_int32, C.POINTER(Mesh), C.POINTER(Params), C.POINTER(_P)]),
    ("mgsb_destroy", C.c_int, [_P]),
    ("mgsb_num_bodies", C.c_int, [_P, _IP]),
    ("mgsb_num_verts", C.c_int, [_P, C.c_int32, _IP]),
    ("mgsb_num_tets", C.c_int, [_P, C.c_int32, _IP]),
    ("mgsb_set_material", C.c_int, [_P, C.c_int32, _FP, _FP]),
    ("mgsb_set_params", C.c_int, [_P, C.POINTER(Params)]),
    ("mgsb_get_params", C.c_int, [_P, C.POINTER(Params)]),
    ("mgsb_set_fixed", C.c_int, [_P, C.c_int32, _U8P]),
    ("mgsb_set_tool_capsule", C.c_int, [_P, C.c_int32, _FP, _FP, C.c_float]),
    ("mgsb_set_tool_capsules", C.c_int, [_P, _FP, _FP, _FP]),
    ("mgsb_set_tool_spheres", C.c_int, [_P, C.c_int32, _FP, _FP, _U8P]),
    ("mgsb_step", C.c_int, [_P]),
    ("mgsb_step_n", C.c_int, [_P, C.c_int32]),
    ("mgsb_synchronize", C.c_int, [_P]),
    ("mgsb_get_positions", C.c_int, [_P, C.c_int32, _FP]),
    ("mgsb_get_velocities", C.c_int, [_P, C.c_int32, _FP]),
    ("mgsb_get_all_positions", C.c_int, [_P, _FP]),
    ("mgsb_get_positions_f64", C.c_int, [_P, C.c_int32, _DP]),
    ("mgsb_get_contact_flags", C.c_int, [_P, C.c_int32, _IP]),
    ("mgsb_get_all_contact_flags", C.c_int, [_P, _IP]),
    ("mgsb_get_contacts", C.c_int, [_P, C.c_int32, _IP, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("mgsb_get_collision_depth", C.c_int, [_P, C.c_int32, _FP]),
    ("mgsb_get_device_positions", C.c_int, [_P, C.c_int32, C.POINTER(_FP)]),
    ("mgsb_get_normals", C.c_int, [_P, C.c_int32, _FP]),
    ("mgsb_get_normals_noalloc", C.c_int, [_P, C.c_int32, _FP]),
    ("mgsb_set_learned_smoother", C.c_int, [_P, _P, C.c_float]),
    ("mgsb_learned_stats", C.c_int, [_P, C.POINTER(C.c_uint64)]),
    ("mgsb_learned_cycle_norms", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                           C.POINTER(C.c_int32)]),
    ("mgsb_smoother_pairs", C.c_int, [_P, C.c_int32, _FP, _FP, C.c_int64, C.POINTER(C.c_int64)]),
    ("mgsb_vcycle_residuals", C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    ("mgsb_mg2_create", C.c_int, [C.POINTER(Mesh), C.POINTER(Mesh), C.POINTER(Params), C.POINTER(_P)]),
    ("mgsb_mg2_destroy", C.c_int, [_P]),
    ("mgsb_mg2_last_error", C.c_char_p, [_P]),
    ("mgsb_mg2_level", C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    ("mgsb_mg2_set_fixed", C.c_int, [_P, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]),
    ("mgsb_mg2_set_tool_spheres", C.c_int, [_P, C.c_int32, _FP, _FP, C.POINTER(C.c_uint8)]),
    ("mgsb_mg2_step", C.c_int, [_P]),
    ("mgsb_mg2_get_positions", C.c_int, [_P, C.c_int32, _FP]),
    ("mgsb_mlp_num_params", C.c_int32, []),
    ("mgsb_mlp_create", C.c_int, [C.c_int32, C.c_uint64, C.POINTER(_P)]),
    ("mgsb_mlp_destroy", C.c_int, [_P]),
    ("mgsb_mlp_last_error", C.c_char_p, [_P]),
    ("mgsb_mlp_set_params", C.c_int, [_P, _FP, C.c_int32]),
    ("mgsb_mlp_get_params", C.c_int, [_P, _FP, C.c_int32]),
    ("mgsb_mlp_forward", C.c_int, [_P, _FP, C.c_int32, _FP]),
    ("mgsb_mlp_loss_grad", C.c_int, [_P, _FP, _FP, C.c_int32, _FP, _FP]),
    ("mgsb_mlp_train", C.c_int, [_P, _FP, _FP, C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _FP]),
    ("mgsb_set_state", C.c_int, [_P, C.c_int32, _FP, _FP]),
    ("mgsb_get_energy", C.c_int, [_P, C.c_int32, _DP]),
    ("mgsb_last_frame_ms", C.c_int, [_P, _FP]),
    ("mgsb_launches_per_frame", C.c_int, [_P, _IP]),
    ("mgsb_profile_frame", C.c_int, [_P, C.c_int32, C.c_char_p, _FP, _IP, _IP]),
    ("mgsb_time_kernel", C.c_int, [_P, C.c_char_p, C.c_int32, _FP, _IP]),
    ("mgsb_get_precompute", C.c_int, [_P, _FP, _FP, _FP, _FP, _FP]),
    ("mgsb_level_size", C.c_int, [_P, C.c_int32, _IP, _IP]),
    ("mgsb_body_level_size", C.c_int, [_P, C.c_int32, C.c_int32, _IP]),
    ("mgsb_level_info", C.c_int, [_P, C.c_int32, _IP]),
    ("mgsb_autotune", C.c_int, [_P, C.c_int32, _IP]),
    ("mgsb_set_kernel_shape", C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    ("mgsb_set_coarse_split", C.c_int, [_P, C.c_int32]),
    ("mgsb_get_coarse_split", C.c_int, [_P, _IP]),
    ("mgsb_set_launch_overlap", C.c_int, [_P, C.c_int32]),
    ("mgsb_set_fused_prolongation", C.c_int, [_P, C.c_int32]),
    ("mgsb_set_fused_restriction", C.c_int, [_P, C.c_int32]),
    ("mgsb_get_frame", C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int32)]),
    ("mgsb_get_frame_view", C.c_int, [_P, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.POINTER(C.c_int32))]),
    ("mgsb_set_surface_contact", C.c_int, [_P, C.c_int32]),
    ("mgsb_set_coarse_dense", C.c_int, [_P, C.c_int32]),
    ("mgsb_get_coarse_dense", C.c_int, [_P, _IP]),
    ("mgsb_set_broad_phase", C.c_int, [_P, C.c_int32]),
    ("mgsb_inspect_level", C.c_int, [C.POINTER(Mesh), C.POINTER(Params), _U8P, C.c_int32, _IP, _IP, _IP, _FP, _FP, _IP,
                                     _IP, _FP]),
    ("mgsb_last_error_string", C.c_char_p, [_P]),
    ("mgsb_status_string", C.c_char_p, [C.c_int]),
    ("mgsb_mesh_box", C.c_int, [C.c_int32, C.c_int32, C.c_int32, _FP, _FP, C.POINTER(C.POINTER(MeshData))]),
    ("mgsb_mesh_blob", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_float, _FP, C.c_float, C.c_float, C.c_uint64,
                                 C.POINTER(C.POINTER(MeshData))]),
    ("mgsb_mesh_read_msh", C.c_int, [C.c_char_p, C.POINTER(C.POINTER(MeshData))]),
    ("mgsb_mesh_extract_surface", C.c_int, [C.POINTER(MeshData)]),
    ("mgsb_mesh_free", C.c_int, [C.POINTER(MeshData)]),
    ("mgsb_value_noise", C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64]),
]

_lib = None


def load() -> C.CDLL:
    """Load libmgsb.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m multigridsoftbody_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
