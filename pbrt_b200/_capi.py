"""ctypes declarations of the C ABI in include/pbrt_b200.h.

Loading fails loudly: there is no CPU fallback for anything this library computes.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbrt_b200.so")

PBRT_MISS = 0xFFFFFFFF

STATUS = {
    0: "PBRT_OK",
    1: "PBRT_ERR_INVALID_ARGUMENT",
    2: "PBRT_ERR_OUT_OF_MEMORY",
    3: "PBRT_ERR_CUDA",
    4: "PBRT_ERR_DEVICE_BUDGET",
    5: "PBRT_ERR_CAPACITY",
    6: "PBRT_ERR_UNSUPPORTED",
}

SHAPE_MESH, SHAPE_SPHERE, SHAPE_CYLINDER, SHAPE_RECTANGLE, SHAPE_AABOX, SHAPE_PLANE, SHAPE_CSG = 0, 1, 2, 3, 4, 5, 6
CSG_UNION, CSG_INTERSECTION, CSG_SUBTRACTION = 0, 1, 2
TEXTURE_COLOR, TEXTURE_CHECKERBOARD = 0, 1
NODE_SIMPLE, NODE_TRANSFORMED, NODE_COMPOUND = 0, 1, 2
MAT_LAMBERTIAN, MAT_METAL, MAT_DIELECTRIC, MAT_DIFFUSE_LIGHT = 0, 1, 2, 3
LIGHT_POINT, LIGHT_UNIFORM_INFINITE, LIGHT_BACKGROUND_INFINITE, LIGHT_AREA = 0, 1, 2, 3


class MeshDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32), ("indices", C.c_void_p),
                ("triangle_count", C.c_uint32), ("face_materials", C.c_void_p)]


class MaterialDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("color", C.c_float * 3), ("fuzz", C.c_float), ("ior", C.c_float),
                ("texture", C.c_uint32), ("color2", C.c_float * 3), ("scale", C.c_float)]


class ObjectDesc(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("mesh", C.c_uint32), ("radius", C.c_float), ("height", C.c_float),
                ("material", C.c_uint32), ("transformed", C.c_uint32), ("to_world", C.c_float * 12),
                ("to_local", C.c_float * 12), ("extent", C.c_float * 3), ("csg_op", C.c_uint32),
                ("csg_first", C.c_uint32), ("csg_count", C.c_uint32)]


class CsgElemDesc(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("mesh", C.c_uint32), ("radius", C.c_float), ("height", C.c_float),
                ("extent", C.c_float * 3), ("to_world", C.c_float * 12), ("to_local", C.c_float * 12)]


class NodeDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("object", C.c_uint32), ("first", C.c_uint32), ("count", C.c_uint32),
                ("to_world", C.c_float * 12), ("to_local", C.c_float * 12)]


class LightDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("position", C.c_float * 3), ("radiance", C.c_float * 3),
                ("bottom", C.c_float * 3), ("top", C.c_float * 3), ("object", C.c_uint32)]


class SceneDesc(C.Structure):
    _fields_ = [("meshes", C.POINTER(MeshDesc)), ("mesh_count", C.c_uint32),
                ("materials", C.POINTER(MaterialDesc)), ("material_count", C.c_uint32),
                ("objects", C.POINTER(ObjectDesc)), ("object_count", C.c_uint32),
                ("lights", C.POINTER(LightDesc)), ("light_count", C.c_uint32),
                ("bvh_bins", C.c_uint32), ("bvh_max_leaf", C.c_uint32),
                ("nodes", C.POINTER(NodeDesc)), ("node_count", C.c_uint32),
                ("node_children", C.POINTER(C.c_uint32)), ("child_count", C.c_uint32),
                ("roots", C.POINTER(C.c_uint32)), ("root_count", C.c_uint32), ("device_build", C.c_uint32),
                ("csg_elems", C.POINTER(CsgElemDesc)), ("csg_elem_count", C.c_uint32)]


class SceneInfo(C.Structure):
    _fields_ = [("triangle_count", C.c_uint64), ("mesh_node_count", C.c_uint64), ("mesh_leaf_count", C.c_uint64),
                ("mesh_max_depth", C.c_uint32), ("mesh_max_leaf_tris", C.c_uint32), ("object_count", C.c_uint64),
                ("device_bytes", C.c_uint64)]


class CameraDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("fov", C.c_float), ("near", C.c_float),
                ("far", C.c_float), ("position", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("thin_lens", C.c_uint32), ("lens_radius", C.c_float), ("focal_distance", C.c_float)]


class RenderParams(C.Structure):
    _fields_ = [("camera", CameraDesc), ("spp", C.c_uint32), ("max_depth", C.c_uint32), ("rr_start", C.c_uint32),
                ("sample_offset", C.c_uint32), ("seed", C.c_uint64), ("integrator", C.c_uint32),
                ("pixel_stride", C.c_uint32)]


class CacheParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("learning_rate", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("epsilon", C.c_float), ("scene_min", C.c_float * 3), ("scene_max", C.c_float * 3),
                ("terminate_bounce", C.c_uint32), ("train_samples", C.c_uint32), ("train_steps", C.c_uint32)]


class StageOptions(C.Structure):
    _fields_ = [("base_dir", C.c_char_p), ("width", C.c_uint32), ("height", C.c_uint32), ("fov_deg", C.c_double),
                ("near", C.c_double), ("far", C.c_double), ("no_loader_lights", C.c_uint32),
                ("bvh_bins", C.c_uint32), ("bvh_max_leaf", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("wave_paths", C.c_uint32), ("trace_threads", C.c_uint32), ("trace_blocks_per_sm", C.c_uint32),
                ("shade_threads", C.c_uint32), ("shade_blocks_per_sm", C.c_uint32)]


# Every symbol the header declares, with its signature. tests/test_capi_symbols.py checks
# the library exports each of them.
SIGNATURES = {
    "pbrt_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "pbrt_ctx_destroy": (None, [C.c_void_p]),
    "pbrt_last_error": (C.c_char_p, [C.c_void_p]),
    "pbrt_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pbrt_ctx_sync": (C.c_int, [C.c_void_p]),
    "pbrt_scene_create": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]),
    "pbrt_scene_destroy": (None, [C.c_void_p]),
    "pbrt_scene_create_many": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.c_uint32, C.c_uint32, C.c_void_p]),
    "pbrt_scene_get_info": (C.c_int, [C.c_void_p, C.POINTER(SceneInfo)]),
    "pbrt_mesh_bvh_build_host": (C.c_int, [C.POINTER(MeshDesc), C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64,
                                           C.c_void_p, C.POINTER(C.c_uint64)]),
    "pbrt_mesh_bvh_build_device": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.c_uint32, C.c_uint32, C.c_void_p,
                                             C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p]),
    "pbrt_trace_closest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pbrt_trace_closest_instrumented": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                                  C.c_void_p]),
    "pbrt_trace_any": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "pbrt_trace_closest_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "pbrt_trace_closest_counted": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p]),
    "pbrt_trace_any_counted": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "pbrt_stage_parse": (C.c_int, [C.c_char_p, C.POINTER(StageOptions), C.POINTER(C.c_void_p), C.c_char_p,
                                   C.c_size_t]),
    "pbrt_stage_describe": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(CameraDesc), C.c_void_p]),
    "pbrt_stage_destroy": (None, [C.c_void_p]),
    "pbrt_scene_load": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(StageOptions), C.POINTER(C.c_void_p),
                                  C.POINTER(CameraDesc)]),
    "pbrt_ply_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_uint32),
                                C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint32), C.c_char_p, C.c_size_t]),
    "pbrt_free": (None, [C.c_void_p]),
    "pbrt_render": (C.c_int, [C.c_void_p, C.POINTER(RenderParams), C.c_void_p]),
    "pbrt_cache_create": (C.c_int, [C.c_void_p, C.POINTER(CacheParams), C.POINTER(C.c_void_p)]),
    "pbrt_cache_destroy": (None, [C.c_void_p]),
    "pbrt_cache_reset": (C.c_int, [C.c_void_p]),
    "pbrt_cache_get_weights": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pbrt_cache_set_weights": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pbrt_cache_query": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "pbrt_cache_gradient": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "pbrt_cache_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "pbrt_cache_save": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "pbrt_cache_load": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "pbrt_render_cached": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(RenderParams), C.c_uint32, C.c_void_p]),
    "pbrt_ctx_render_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pbrt_ctx_set_tuning": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pbrt_ctx_get_tuning": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pbrt_batch_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(RenderParams), C.c_uint32, C.POINTER(C.c_void_p)]),
    "pbrt_batch_render": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "pbrt_batch_destroy": (None, [C.c_void_p]),
    "pbrt_render_batch": (C.c_int, [C.c_void_p, C.POINTER(RenderParams), C.c_uint32, C.c_void_p]),
    "pbrt_ctx_set_batch_kernel": (C.c_int, [C.c_void_p, C.c_int]),
    "pbrt_ctx_set_batch_branches": (C.c_int, [C.c_void_p, C.c_uint32]),
    "pbrt_film_to_rgba8": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]),
    "pbrt_write_png": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libpbrt_b200.so (raises if it is missing: build it with pbrt_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing; build it with `python -m pbrt_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class PbrtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code
