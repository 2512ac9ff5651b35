"""Host-side mirror of the reference's scene API, lowered to include/pbrt_b200.h.

Names and argument meanings follow the Rust crate:
  TriangleMesh::new(vertices, indices, ..)   src/shapes/triangle_mesh/triangle_mesh.rs:27-41
  Sphere::new(r)                             src/shapes/sphere.rs:16-18
  Cylinder::new(radius, height)              src/shapes/cylinder.rs:13-19
  Simple::new(shape, material)               src/objects/simple.rs:16-21
  Transformed::new(object, transform)        src/objects/transformed.rs:15-20
  Transform::translation / rotation_*        src/geom/transform.rs:43-72
  Lambertian / Metal / Dielectric / DiffuseLight   src/materials/*.rs
  Scene::new / add_object / add_light / commit     src/scene.rs:80-115
  Scene::intersect / intersect_p (batched)         src/scene.rs:118-150
Errors the reference reports by panicking (an empty mesh, an index out of range) raise
PbrtError here; "no hit" is PBRT_MISS in the returned id array, as `None` is in Rust.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _capi
from ._capi import PbrtError

try:  # torch is only plumbing: device buffers for callers that already hold them
    import torch
except Exception:  # pragma: no cover
    torch = None


# ------------------------------------------------------------------------------------------
# Context
# ------------------------------------------------------------------------------------------
class Context:
    """A CUDA device context (pbrt_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = _capi.load()
        h = C.c_void_p()
        rc = self.lib.pbrt_ctx_create(device, C.byref(h))
        if rc != 0:
            raise PbrtError(rc, f"pbrt_ctx_create(device={device}) failed (a B200 / sm_100 GPU is required)")
        self.h = h
        self.device = device

    def check(self, rc: int, what: str = ""):
        if rc != 0:
            raise PbrtError(rc, f"{what}: {self.lib.pbrt_last_error(self.h).decode()}")

    def set_stream(self, stream_ptr: Optional[int]):
        self.check(self.lib.pbrt_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)), "pbrt_ctx_set_stream")

    def sync(self):
        self.check(self.lib.pbrt_ctx_sync(self.h), "pbrt_ctx_sync")

    def close(self):
        if getattr(self, "h", None):
            self.lib.pbrt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ------------------------------------------------------------------------------------------
# Transforms (src/geom/transform.rs). Kept in float64 on the host, handed over as FP32 3x4.
# ------------------------------------------------------------------------------------------
class Transform:
    def __init__(self, mat: np.ndarray, inv: np.ndarray):
        self.mat = np.asarray(mat, np.float64)
        self.inv = np.asarray(inv, np.float64)

    @staticmethod
    def identity() -> "Transform":
        return Transform(np.eye(4), np.eye(4))

    @staticmethod
    def translation(p: Sequence[float]) -> "Transform":
        m, i = np.eye(4), np.eye(4)
        m[:3, 3] = p
        i[:3, 3] = [-p[0], -p[1], -p[2]]
        return Transform(m, i)

    @staticmethod
    def _rot(axis: int, a: float) -> "Transform":
        s, c = math.sin(a), math.cos(a)
        m = np.eye(4)
        j, k = [(1, 2), (0, 2), (0, 1)][axis]
        if axis == 1:  # Matrix4::rotation_y (matrix4.rs:54-60)
            m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
        else:
            m[j, j], m[j, k], m[k, j], m[k, k] = c, -s, s, c
        return Transform(m, m.T.copy())

    @staticmethod
    def rotation_x(a: float) -> "Transform":
        return Transform._rot(0, a)

    @staticmethod
    def rotation_y(a: float) -> "Transform":
        return Transform._rot(1, a)

    @staticmethod
    def rotation_z(a: float) -> "Transform":
        return Transform._rot(2, a)

    def __mul__(self, o: "Transform") -> "Transform":  # transform.rs:119-127
        return Transform(self.mat @ o.mat, o.inv @ self.inv)


# ------------------------------------------------------------------------------------------
# Shapes, materials, objects
# ------------------------------------------------------------------------------------------
class TriangleMesh:
    def __init__(self, vertices, indices):
        v = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
        i = np.ascontiguousarray(np.asarray(indices, np.uint32).reshape(-1, 3))
        if i.shape[0] == 0:
            raise PbrtError(1, "a TriangleMesh needs at least one triangle")
        self.vertices, self.indices = v, i

    @property
    def triangle_count(self) -> int:
        return int(self.indices.shape[0])


@dataclass
class Sphere:
    r: float


@dataclass
class Cylinder:
    radius: float
    height: float


@dataclass
class Lambertian:
    albedo: Sequence[float]


@dataclass
class Metal:
    fuzz: float
    albedo: Sequence[float]


@dataclass
class Dielectric:
    ref_idx: float
    albedo: Sequence[float] = (1.0, 1.0, 1.0)


@dataclass
class DiffuseLight:
    emitted: Sequence[float]


@dataclass
class Simple:
    shape: object
    material: object = field(default_factory=lambda: Lambertian((0.5, 0.5, 0.5)))


@dataclass
class Transformed:
    object: Simple
    transform: Transform


# ------------------------------------------------------------------------------------------
# Buffers
# ------------------------------------------------------------------------------------------
def _is_torch(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor)


def _ptr(a) -> int:
    if _is_torch(a):
        assert a.is_contiguous()
        return a.data_ptr()
    return a.ctypes.data


def _as_rays(rays):
    """Rays as 8 SoA planes (8, n) of float32: ox oy oz dx dy dz tmin tmax."""
    if _is_torch(rays):
        assert rays.dtype == torch.float32 and rays.dim() == 2 and rays.shape[0] == 8
        return rays.contiguous(), int(rays.shape[1])
    r = np.ascontiguousarray(rays, dtype=np.float32)
    assert r.ndim == 2 and r.shape[0] == 8, "rays are 8 SoA planes: ox oy oz dx dy dz tmin tmax"
    return r, int(r.shape[1])


def _empty_like(ref, n: int, dtype: str):
    if _is_torch(ref):
        td = {"u32": torch.int32, "f32": torch.float32, "u8": torch.uint8}[dtype]
        return torch.empty(n, dtype=td, device=ref.device)
    nd = {"u32": np.uint32, "f32": np.float32, "u8": np.uint8}[dtype]
    return np.empty(n, nd)


# ------------------------------------------------------------------------------------------
# Scene
# ------------------------------------------------------------------------------------------
class Scene:
    """Scene::new / add_object / add_light / commit; commit() builds and uploads."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx
        self.objects: List[object] = []
        self.lights: List[object] = []
        self.h = None
        self._keep = []

    def add_object(self, obj) -> "Scene":
        self.objects.append(obj)
        return self

    def add_light(self, light) -> "Scene":
        self.lights.append(light)
        return self

    def commit(self, bvh_bins: int = 8, bvh_max_leaf: int = 1) -> "Scene":
        if self.ctx is None:
            self.ctx = default_context()
        self.release()
        meshes, mesh_ids, materials, mat_ids, objs = [], {}, [], {}, []

        def mat_index(m):
            key = id(m)
            if key not in mat_ids:
                d = _capi.MaterialDesc()
                if isinstance(m, Lambertian):
                    d.kind, col = _capi.MAT_LAMBERTIAN, m.albedo
                elif isinstance(m, Metal):
                    d.kind, col, d.fuzz = _capi.MAT_METAL, m.albedo, m.fuzz
                elif isinstance(m, Dielectric):
                    d.kind, col, d.ior = _capi.MAT_DIELECTRIC, m.albedo, m.ref_idx
                elif isinstance(m, DiffuseLight):
                    d.kind, col = _capi.MAT_DIFFUSE_LIGHT, m.emitted
                else:
                    raise TypeError(f"unknown material {m!r}")
                d.color[:] = [float(c) for c in col]
                mat_ids[key] = len(materials)
                materials.append(d)
            return mat_ids[key]

        for o in self.objects:
            xf = None
            if isinstance(o, Transformed):
                xf, o = o.transform, o.object
            if not isinstance(o, Simple):
                raise TypeError("objects are Simple or Transformed(Simple)")
            d = _capi.ObjectDesc()
            shp = o.shape
            if isinstance(shp, TriangleMesh):
                if id(shp) not in mesh_ids:
                    md = _capi.MeshDesc(_ptr(shp.vertices), shp.vertices.shape[0], _ptr(shp.indices),
                                        shp.indices.shape[0])
                    mesh_ids[id(shp)] = len(meshes)
                    meshes.append(md)
                    self._keep.append(shp)
                d.shape, d.mesh = _capi.SHAPE_MESH, mesh_ids[id(shp)]
            elif isinstance(shp, Sphere):
                d.shape, d.radius = _capi.SHAPE_SPHERE, shp.r
            elif isinstance(shp, Cylinder):
                d.shape, d.radius, d.height = _capi.SHAPE_CYLINDER, shp.radius, shp.height
            else:
                raise TypeError(f"unknown shape {shp!r}")
            d.material = mat_index(o.material)
            if xf is not None:
                d.transformed = 1
                d.to_world[:] = [float(x) for x in xf.mat[:3, :].reshape(-1)]
                d.to_local[:] = [float(x) for x in xf.inv[:3, :].reshape(-1)]
            objs.append(d)

        desc = _capi.SceneDesc()
        MA = _capi.MeshDesc * max(1, len(meshes))
        TA = _capi.MaterialDesc * max(1, len(materials))
        OA = _capi.ObjectDesc * max(1, len(objs))
        self._arrays = (MA(*meshes), TA(*materials), OA(*objs))
        desc.meshes, desc.mesh_count = C.cast(self._arrays[0], C.POINTER(_capi.MeshDesc)), len(meshes)
        desc.materials, desc.material_count = C.cast(self._arrays[1], C.POINTER(_capi.MaterialDesc)), len(materials)
        desc.objects, desc.object_count = C.cast(self._arrays[2], C.POINTER(_capi.ObjectDesc)), len(objs)
        desc.lights, desc.light_count = None, 0
        desc.bvh_bins, desc.bvh_max_leaf = bvh_bins, bvh_max_leaf
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.pbrt_scene_create(self.ctx.h, C.byref(desc), C.byref(h)), "pbrt_scene_create")
        self.h = h
        return self

    def info(self) -> dict:
        inf = _capi.SceneInfo()
        self.ctx.check(self.ctx.lib.pbrt_scene_get_info(self.h, C.byref(inf)), "pbrt_scene_get_info")
        return {k: getattr(inf, k) for k, _ in _capi.SceneInfo._fields_}

    def _need(self):
        if self.h is None:
            raise PbrtError(1, "Scene::commit must run before a query")

    def intersect(self, rays, with_object: bool = False):
        """Nearest hit for a batch of rays: (prim_id, t[, object_id])."""
        self._need()
        r, n = _as_rays(rays)
        prim, t = _empty_like(r, n, "u32"), _empty_like(r, n, "f32")
        obj = _empty_like(r, n, "u32") if with_object else None
        self.ctx.check(self.ctx.lib.pbrt_trace_closest(self.h, _ptr(r), n, _ptr(prim), _ptr(t),
                                                       _ptr(obj) if obj is not None else None),
                       "pbrt_trace_closest")
        return (prim, t, obj) if with_object else (prim, t)

    def intersect_instrumented(self, rays):
        """Nearest hit plus the summed traversal counters (nodes, box tests, triangle tests)."""
        self._need()
        r, n = _as_rays(rays)
        prim, t = _empty_like(r, n, "u32"), _empty_like(r, n, "f32")
        stats = (C.c_uint64 * 3)()
        self.ctx.check(self.ctx.lib.pbrt_trace_closest_instrumented(self.h, _ptr(r), n, _ptr(prim), _ptr(t), stats),
                       "pbrt_trace_closest_instrumented")
        return prim, t, dict(nodes_visited=stats[0], box_tests=stats[1], triangle_tests=stats[2])

    def intersect_p(self, rays):
        """Occlusion per ray within its [tmin, tmax] (uint8 0/1)."""
        self._need()
        r, n = _as_rays(rays)
        occ = _empty_like(r, n, "u8")
        self.ctx.check(self.ctx.lib.pbrt_trace_any(self.h, _ptr(r), n, _ptr(occ)), "pbrt_trace_any")
        return occ

    def release(self):
        if self.h is not None and self.ctx is not None and self.ctx.h is not None:
            self.ctx.lib.pbrt_scene_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------
# Host-only tree inspection (no GPU needed)
# ------------------------------------------------------------------------------------------
GPU_NODE_DTYPE = np.dtype([("bmin", np.float32, 3), ("left_first", np.uint32), ("bmax", np.float32, 3),
                           ("count", np.uint32)])


def build_mesh_bvh_host(vertices, indices, bvh_bins: int = 8, bvh_max_leaf: int = 1):
    """The flattened mesh BVH pbrt_scene_create would upload: (nodes, tri_order).

    nodes use GPU numbering (0 = root, 1 = padding, sibling pairs at even indices)."""
    lib = _capi.load()
    v = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
    i = np.ascontiguousarray(np.asarray(indices, np.uint32).reshape(-1, 3))
    md = _capi.MeshDesc(v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0])
    cnt = C.c_uint64()
    rc = lib.pbrt_mesh_bvh_build_host(C.byref(md), bvh_bins, bvh_max_leaf, None, 0, None, C.byref(cnt))
    if rc != 0:
        raise PbrtError(rc, "pbrt_mesh_bvh_build_host")
    nodes = np.zeros(cnt.value, GPU_NODE_DTYPE)
    order = np.zeros(i.shape[0], np.uint32)
    rc = lib.pbrt_mesh_bvh_build_host(C.byref(md), bvh_bins, bvh_max_leaf, nodes.ctypes.data, cnt.value,
                                      order.ctypes.data, C.byref(cnt))
    if rc != 0:
        raise PbrtError(rc, "pbrt_mesh_bvh_build_host")
    return nodes, order
