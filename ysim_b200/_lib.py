"""ctypes binding of the C ABI declared in include/ysim_b200.h.

The shared library is built in-tree (ysim_b200/lib/libysim_b200.so) by
``ysim_b200.build``.  There is no fallback: importing this module without the
library, or calling into it without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libysim_b200.so")

# status codes / flags (ysim_b200.h)
YS_OK = 0
YS_ERR_BAD_ARG = -1  # include/ysim_b200.h
FLAG_NONFINITE = 1
FLAG_STACK_OVF = 2
FLAG_PAIR_OVF = 4
FLAG_ITER_CAP = 8
FLAG_CONTACT_OVF = 16

TRIANGULAR_CLOTH = 0
FAST_GRID_CLOTH = 1
RIGID = 3
FLOAT = 4
KINEMATIC = 7

MESH_STATIC = 1
MESH_COLLIDABLE = 2
MESH_SELF_COLLIDE = 4

SELF_OFF = 0
SELF_HASH = 1
SELF_BVH = 2
TREE_REFERENCE = 0  # Morton normalisation per axis, node for node the reference's tree
TREE_CUBE = 1       # one scale for all axes (default)

BUILD_KARRAS = 0    # buildTree_Tri + bottom-up boxes (reference default)
BUILD_APETREI = 1   # agglomerativeBuild_Tri: topology and boxes in one pass

# ColliderKind (ys_analytic_shape.kind)
COLLIDER_MESH = 0
COLLIDER_SPHERE = 1
COLLIDER_BOX = 2
COLLIDER_CYLINDER = 3
COLLIDER_PLANE = 4


ORDER_VERTEX = 0
ORDER_MORTON = 1
ORDER_TILE = 2
ORDER_NAMES = ("vertex", "morton", "tile")


class FusedClass(C.Structure):
    _fields_ = [("max_mesh_vertices", C.c_uint32), ("meshes", C.c_uint32), ("vertices", C.c_uint32),
                ("ctas_per_sm", C.c_int32), ("thread_order", C.c_int32), ("ms", (C.c_float * 3) * 3)]


class SimParams(C.Structure):
    _fields_ = [
        ("subh", C.c_float), ("kair", C.c_float), ("kd", C.c_float),
        ("gravity", C.c_float * 3),
        ("margin", C.c_float), ("radius", C.c_float),
        ("substeps", C.c_uint32), ("rebuild_frames", C.c_uint32),
        ("self_mode", C.c_uint32), ("cols_per_point", C.c_uint32),
    ]


class MeshDesc(C.Structure):
    _fields_ = [
        ("behavior", C.c_uint32), ("flags", C.c_uint32),
        ("num_vertices", C.c_uint32), ("num_facets", C.c_uint32),
        ("x", C.c_void_p), ("v", C.c_void_p), ("mass", C.c_void_p), ("mask", C.c_void_p),
        ("facets", C.c_void_p),
        ("kstretch", C.c_float), ("kshear", C.c_float), ("kbend", C.c_float), ("thickness", C.c_float),
        ("grid_n", C.c_uint32), ("grid_rest", C.c_float * 6), ("group", C.c_uint32),
    ]


class YsError(RuntimeError):
    pass


_lib = None

_PROTOS = {
    "ys_last_error": (C.c_char_p, []),
    "ys_version": (C.c_char_p, []),
    "ys_scene_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(SimParams), C.c_int]),
    "ys_scene_destroy": (C.c_int, [C.c_void_p]),
    "ys_scene_add_mesh": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(C.c_int)]),
    "ys_scene_pack": (C.c_int, [C.c_void_p]),
    "ys_frame_preamble": (C.c_int, [C.c_void_p]),
    "ys_broad_refit": (C.c_int, [C.c_void_p]),
    "ys_broad_detect": (C.c_int, [C.c_void_p]),
    "ys_narrow_and_sort": (C.c_int, [C.c_void_p]),
    "ys_snapshot_xprev": (C.c_int, [C.c_void_p]),
    "ys_system_update": (C.c_int, [C.c_void_p]),
    "ys_scene_step_staged": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ys_scene_step": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ys_scene_set_record": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_set_tree_layout": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_set_fused_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_set_thread_order": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_autotune_classes": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]),
    "ys_scene_wide_tree": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_uint32, C.c_void_p]),
    "ys_scene_set_tree_builder": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_lbvh_set_builder": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_set_collider": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ys_scene_colliders": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "ys_narrow_analytic": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                     C.c_uint32, C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_void_p,
                                     C.c_uint64, C.c_void_p, C.c_void_p]),
    "ys_scene_autotune": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "ys_scene_sync": (C.c_int, [C.c_void_p]),
    "ys_scene_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "ys_scene_get_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "ys_scene_set_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "ys_scene_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "ys_scene_clear_flags": (C.c_int, [C.c_void_p]),
    "ys_scene_totals": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "ys_scene_set_external_forces": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ys_scene_read_positions_async": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ys_scene_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_scene_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "ys_scene_rows": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ys_scene_contacts": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ys_scene_tree": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_uint32)]),
    "ys_shff_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_uint32, C.c_int, C.c_void_p]),
    "ys_shff_destroy": (C.c_int, [C.c_void_p]),
    "ys_shff_detect": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                 C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_int, C.c_void_p, C.c_uint64,
                                 C.c_void_p]),
    "ys_shff_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ys_lbvh_set_split": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_lbvh_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_uint32, C.c_int, C.c_void_p]),
    "ys_lbvh_destroy": (C.c_int, [C.c_void_p]),
    "ys_lbvh_build": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "ys_lbvh_refit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int]),
    "ys_lbvh_query": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_int, C.c_void_p, C.c_uint64,
                                C.c_void_p]),
    "ys_lbvh_arrays": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_void_p), C.POINTER(C.c_uint32)]),
    "ys_shash_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]),
    "ys_shash_destroy": (C.c_int, [C.c_void_p]),
    "ys_shash_build": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float]),
    "ys_shash_query": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p, C.c_uint64,
                                 C.c_void_p]),
    "ys_shash_entries": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "ys_scene_set_grid_springs": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "ys_adjoint_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.c_uint32, C.c_uint32]),
    "ys_adjoint_destroy": (C.c_int, [C.c_void_p]),
    "ys_adjoint_num_springs": (C.c_uint32, [C.c_void_p]),
    "ys_adjoint_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ys_adjoint_forward": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ys_adjoint_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ys_adjoint_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "ys_adjoint_set_params_f64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ys_adjoint_forward_f64": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ys_adjoint_backward_f64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ys_morton_codes": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    "ys_radix_sort_scratch_bytes": (C.c_size_t, [C.c_uint32]),
    "ys_radix_sort_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "ys_radix_sort_pairs_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
}

# every symbol the header declares (tests check the library exports them all)
EXPORTED = tuple(_PROTOS)


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"ysim_b200 CUDA library not found at {path}; build it with "
            "`python -m ysim_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(path)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = "") -> None:
    if status != YS_OK:
        msg = _lib.ys_last_error().decode() if _lib is not None else ""
        raise YsError(f"{what} failed with status {status}: {msg}")
