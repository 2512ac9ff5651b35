"""Host-side mirror of the reference's scene API, lowered to include/pbrt_b200.h.

Names and argument meanings follow the Rust crate:
  TriangleMesh::new(vertices, indices, ..)   src/shapes/triangle_mesh/triangle_mesh.rs:27-41
  Sphere::new(r)                             src/shapes/sphere.rs:16-18
  Cylinder::new(radius, height)              src/shapes/cylinder.rs:13-19
  Rectangle::new(width, height)              src/shapes/rectangle.rs:14-21
  AABox::new(extent)                         src/shapes/aabox.rs:14-22
  Plane::new()                               src/shapes/plane.rs:11-15
  PlainColor / CheckerBoard::new(c1, c2, scale)   src/textures/*.rs
  Simple::new(shape, material)               src/objects/simple.rs:16-21
  Transformed::new(object, transform)        src/objects/transformed.rs:15-20
  Compound::new(objects)                     src/objects/compound.rs:15-19
  Transform::translation / rotation_*        src/geom/transform.rs:43-72
  Lambertian / Metal / Dielectric / DiffuseLight   src/materials/*.rs
  PointLight / UniformInfiniteLight / BackgroundInfiniteLight   src/lights/*.rs
  AreaLight — the reference's planned light (ideas/area_light.md), on an emissive object
  Scene::new / add_object / add_light / commit     src/scene.rs:80-115
  Scene::intersect / intersect_p (batched)         src/scene.rs:118-150
  Scene::intersect[_p]_instrumented (batched)      src/scene.rs:124-153
  renderers::mt::render (mean radiance film)       src/renderers/mt.rs:23-130
Errors the reference reports by panicking (an empty mesh, an index out of range) raise
PbrtError here; "no hit" is PBRT_MISS in the returned id array, as `None` is in Rust.

A scene lowers to a plain description dict (Scene.describe), the same one the CPU oracle
consumes in the tests; Scene.from_description builds a scene from such a dict.
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

    def set_tuning(self, wave_paths: int = 0, trace_threads: int = 0, trace_blocks_per_sm: int = 0,
                   shade_threads: int = 0, shade_blocks_per_sm: int = 0):
        """Launch shape of the wavefront (zeros: defaults); applies to later renders/batches."""
        t = _capi.Tuning(int(wave_paths), int(trace_threads), int(trace_blocks_per_sm), int(shade_threads),
                         int(shade_blocks_per_sm))
        self.check(self.lib.pbrt_ctx_set_tuning(self.h, C.byref(t)), "pbrt_ctx_set_tuning")

    def set_batch_kernel(self, kind: str):
        """How batches created afterwards run a frame: "wavefront" (the default; waves of
        paths through queues, one kernel per stage and bounce) or "persistent" (one
        persistent launch, each lane running a path to its end). Films are the same."""
        kinds = {"wavefront": 0, "persistent": 1}
        if kind not in kinds:
            raise ValueError(f"batch kernel must be one of {sorted(kinds)}")
        self.check(self.lib.pbrt_ctx_set_batch_kernel(self.h, kinds[kind]), "pbrt_ctx_set_batch_kernel")

    def set_batch_branches(self, branches: int):
        """Concurrent branches (streams inside the frame's graph, each with its own wave
        buffers) of the wavefront frame of batches created afterwards, 1..8. A scene's waves
        stay on one branch; films are the same for any count."""
        self.check(self.lib.pbrt_ctx_set_batch_branches(self.h, int(branches)), "pbrt_ctx_set_batch_branches")

    def tuning(self) -> dict:
        t = _capi.Tuning()
        self.check(self.lib.pbrt_ctx_get_tuning(self.h, C.byref(t)), "pbrt_ctx_get_tuning")
        return {k: getattr(t, k) for k, _ in _capi.Tuning._fields_}

    def render_stats(self) -> dict:
        """Rays, shadow rays and paths of the last render on this context."""
        out = np.zeros(3, np.uint64)
        self.check(self.lib.pbrt_ctx_render_stats(self.h, out.ctypes.data), "pbrt_ctx_render_stats")
        return dict(rays=int(out[0]), shadow_rays=int(out[1]), paths=int(out[2]))

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
        return Transform(_matmul4(self.mat, o.mat), _matmul4(o.inv, self.inv))

    def rows(self):
        """(to_world, to_local) as 12 float64 values each (row-major 3x4); the scene
        description rounds them to FP32."""
        return (self.mat[:3, :].reshape(-1).copy(), self.inv[:3, :].reshape(-1).copy())


def _matmul4(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Matrix4 * Matrix4 as the reference sums it (matrix4.rs:216-232): m[i][j] starts at 0 and
    adds a[i][k] * b[k][j] for k = 0..3 in turn (no fused or reordered sums)."""
    m = np.zeros((4, 4))
    for i in range(4):
        for j in range(4):
            acc = 0.0
            for k in range(4):
                acc += float(a[i, k]) * float(b[k, j])
            m[i, j] = acc
    return m


# ------------------------------------------------------------------------------------------
# Shapes, materials, objects, lights
# ------------------------------------------------------------------------------------------
class TriangleMesh:
    """Triangles sharing one BVH. `face_materials` (optional) gives each triangle its own
    material: a list of materials and, per triangle, an index into it; the triangles then
    ignore the material of the object that holds the mesh."""

    def __init__(self, vertices, indices, face_materials=None):
        v = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
        i = np.ascontiguousarray(np.asarray(indices, np.uint32).reshape(-1, 3))
        if i.shape[0] == 0:
            raise PbrtError(1, "a TriangleMesh needs at least one triangle")
        self.vertices, self.indices = v, i
        self.face_materials = None
        if face_materials is not None:
            mats, per_face = face_materials
            per_face = np.ascontiguousarray(np.asarray(per_face, np.uint32).reshape(-1))
            if per_face.shape[0] != i.shape[0] or (per_face.size and int(per_face.max()) >= len(mats)):
                raise PbrtError(1, "face_materials: one index per triangle into the material list")
            self.face_materials = (list(mats), per_face)

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
class Rectangle:
    """Rectangle::new(width, height): y = 0, |x| <= width/2, |z| <= height/2, facing +y."""
    width: float
    height: float


@dataclass
class AABox:
    """AABox::new(extent): the box [-extent/2, extent/2]."""
    extent: Sequence[float]


@dataclass
class Plane:
    """The y = 0 plane (unbounded: kept out of the scene's BVH, tested first)."""


@dataclass
class Csg:
    """csg::Union / Intersection / Substraction (src/shapes/csg/*.rs): op is "union",
    "intersection" or "subtraction"; elements are (plain shape, Transform) pairs (csg::Elem) in
    the order the solid holds them: elements[0] is the piece the others are subtracted from. A
    scene file lists a solid's elements in the reverse of that order (the scene builder pops
    them, loader/visitors/scene_builder.rs:117-143)."""
    op: str
    elements: List[tuple]


@dataclass
class CheckerBoard:
    """CheckerBoard::new(c1, c2, scale): a texture usable wherever a material takes a colour."""
    c1: Sequence[float]
    c2: Sequence[float]
    scale: float


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
    object: object  # Simple, Transformed or Compound
    transform: Transform


@dataclass
class Compound:
    """Several objects as one primitive: the nearest member's hit, the first on a tie."""
    objects: List[object]


@dataclass
class PointLight:
    """PointLight::new(transform, i): a point at transform·(0,0,0) with intensity I."""
    position: Sequence[float]
    i: Sequence[float]


@dataclass
class UniformInfiniteLight:
    i: Sequence[float]


@dataclass
class BackgroundInfiniteLight:
    """Gradient f (downwards) → t (upwards) on the direction's y (background_infinite_light.rs)."""
    f: Sequence[float]
    t: Sequence[float]


@dataclass
class AreaLight:
    """The emissive surface of an object already added to the scene (its material is a
    DiffuseLight); sampled by area for next-event estimation (ideas/area_light.md)."""
    object: object


_NO_MATERIAL = object()  # a csg element's shape carries no material of its own


def _texture(c) -> dict:
    if isinstance(c, CheckerBoard):
        return dict(color=tuple(c.c1), texture=_capi.TEXTURE_CHECKERBOARD, color2=tuple(c.c2), scale=float(c.scale))
    return dict(color=tuple(c))


def _material_desc(m) -> dict:
    if isinstance(m, Lambertian):
        return dict(kind=_capi.MAT_LAMBERTIAN, fuzz=0.0, ior=1.0, **_texture(m.albedo))
    if isinstance(m, Metal):
        return dict(kind=_capi.MAT_METAL, fuzz=float(m.fuzz), ior=1.0, **_texture(m.albedo))
    if isinstance(m, Dielectric):
        return dict(kind=_capi.MAT_DIELECTRIC, fuzz=0.0, ior=float(m.ref_idx), **_texture(m.albedo))
    if isinstance(m, DiffuseLight):
        return dict(kind=_capi.MAT_DIFFUSE_LIGHT, fuzz=0.0, ior=1.0, **_texture(m.emitted))
    raise TypeError(f"unknown material {m!r}")


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


def camera_desc(camera: dict) -> _capi.CameraDesc:
    """A camera dict: width, height, fov (radians), near, far, position, look_at, up; with
    kind = "thin_lens" also lens_radius and focal_distance (ThinLensCamera)."""
    c = _capi.CameraDesc()
    c.width, c.height = int(camera["width"]), int(camera["height"])
    c.fov, c.near, c.far = float(camera["fov"]), float(camera["near"]), float(camera["far"])
    c.position[:] = [float(x) for x in camera["position"]]
    c.look_at[:] = [float(x) for x in camera["look_at"]]
    c.up[:] = [float(x) for x in camera["up"]]
    if camera.get("kind") == "thin_lens":
        c.thin_lens = 1
        c.lens_radius, c.focal_distance = float(camera["lens_radius"]), float(camera["focal_distance"])
    return c


INTEGRATORS = {"path": 0, "naive": 1, "normal": 2}


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
        self._desc = None

    @classmethod
    def from_description(cls, desc: dict, ctx: Optional[Context] = None) -> "Scene":
        s = cls(ctx)
        s._desc = desc
        return s

    def add_object(self, obj) -> "Scene":
        self.objects.append(obj)
        return self

    def add_light(self, light) -> "Scene":
        self.lights.append(light)
        return self

    def describe(self, bvh_bins: int = 8, bvh_max_leaf: int = 1) -> dict:
        """The plain description dict of this scene (see the module docstring). Scenes whose
        objects are all Simple or Transformed(Simple) list them as objects; any other nesting
        (Compound, Transformed of a Transformed) adds the object tree (nodes, roots)."""
        if self._desc is not None:
            return self._desc
        meshes, mesh_ids, materials, mat_ids, objs, obj_ids = [], {}, [], {}, [], {}

        def mat_index(m):
            if id(m) not in mat_ids:
                mat_ids[id(m)] = len(materials)
                materials.append(_material_desc(m))
            return mat_ids[id(m)]

        def simple_desc(o: Simple) -> dict:  # noqa: C901
            d = dict(shape=0, mesh=0, radius=0.0, height=0.0, material=0, to_world=None, to_local=None)
            shp = o.shape
            if isinstance(shp, TriangleMesh):
                if id(shp) not in mesh_ids:
                    mesh_ids[id(shp)] = len(meshes)
                    md = dict(vertices=shp.vertices, indices=shp.indices)
                    if shp.face_materials is not None:
                        glob = [mat_index(m) for m in shp.face_materials[0]]
                        md["face_materials"] = np.asarray(glob, np.uint32)[shp.face_materials[1]]
                    meshes.append(md)
                d.update(shape=_capi.SHAPE_MESH, mesh=mesh_ids[id(shp)])
            elif isinstance(shp, Sphere):
                d.update(shape=_capi.SHAPE_SPHERE, radius=float(shp.r))
            elif isinstance(shp, Cylinder):
                d.update(shape=_capi.SHAPE_CYLINDER, radius=float(shp.radius), height=float(shp.height))
            elif isinstance(shp, Rectangle):
                d.update(shape=_capi.SHAPE_RECTANGLE, radius=float(shp.width), height=float(shp.height))
            elif isinstance(shp, AABox):
                d.update(shape=_capi.SHAPE_AABOX, extent=tuple(float(x) for x in shp.extent))
            elif isinstance(shp, Plane):
                d.update(shape=_capi.SHAPE_PLANE)
            elif isinstance(shp, Csg):
                ops = {"union": _capi.CSG_UNION, "intersection": _capi.CSG_INTERSECTION,
                       "subtraction": _capi.CSG_SUBTRACTION}
                elems = []
                for es, ex in shp.elements:
                    if isinstance(es, Csg):
                        raise TypeError("a csg element is a plain shape")
                    e = plain(es)
                    e["to_world"], e["to_local"] = ex.rows()
                    elems.append(e)
                d.update(shape=_capi.SHAPE_CSG, csg=dict(op=ops[shp.op], elements=elems))
            else:
                raise TypeError(f"unknown shape {shp!r}")
            if o.material is not _NO_MATERIAL:
                d["material"] = mat_index(o.material)
            return d

        def plain(shp) -> dict:
            return simple_desc(Simple(shp, _NO_MATERIAL))

        flat = all(isinstance(o, Simple) or (isinstance(o, Transformed) and isinstance(o.object, Simple))
                   for o in self.objects)
        nodes, roots = None, None
        if flat:
            for o in self.objects:
                top, xf = o, None
                if isinstance(o, Transformed):
                    xf, o = o.transform, o.object
                d = simple_desc(o)
                if xf is not None:
                    d["to_world"], d["to_local"] = xf.rows()
                obj_ids[id(top)] = len(objs)
                objs.append(d)
        else:
            nodes, node_ids, simple_ids = [], {}, {}

            def node(o) -> int:
                if id(o) in node_ids:  # a shared object stays one node
                    return node_ids[id(o)]
                if isinstance(o, Simple):
                    if id(o) not in simple_ids:
                        simple_ids[id(o)] = len(objs)
                        objs.append(simple_desc(o))
                    n = dict(kind=_capi.NODE_SIMPLE, object=simple_ids[id(o)])
                elif isinstance(o, Transformed):
                    w, l = o.transform.rows()
                    n = dict(kind=_capi.NODE_TRANSFORMED, children=[node(o.object)], to_world=w, to_local=l)
                elif isinstance(o, Compound):
                    n = dict(kind=_capi.NODE_COMPOUND, children=[node(c) for c in o.objects])
                else:
                    raise TypeError(f"unknown object {o!r}")
                node_ids[id(o)] = len(nodes)
                nodes.append(n)
                return node_ids[id(o)]

            roots = [node(o) for o in self.objects]
            for o in self.objects:  # an area light names a top-level Simple or Transformed(Simple)
                inner = o.object if isinstance(o, Transformed) else o
                if isinstance(inner, Simple) and id(inner) in simple_ids:
                    obj_ids[id(o)] = simple_ids[id(inner)]
        lights = []
        for l in self.lights:
            if isinstance(l, PointLight):
                lights.append(dict(kind=_capi.LIGHT_POINT, position=tuple(l.position), radiance=tuple(l.i)))
            elif isinstance(l, UniformInfiniteLight):
                lights.append(dict(kind=_capi.LIGHT_UNIFORM_INFINITE, radiance=tuple(l.i)))
            elif isinstance(l, BackgroundInfiniteLight):
                lights.append(dict(kind=_capi.LIGHT_BACKGROUND_INFINITE, bottom=tuple(l.f), top=tuple(l.t)))
            elif isinstance(l, AreaLight):
                if id(l.object) not in obj_ids:
                    raise PbrtError(1, "an AreaLight's object must be added to the scene")
                lights.append(dict(kind=_capi.LIGHT_AREA, object=obj_ids[id(l.object)]))
            else:
                raise TypeError(f"unknown light {l!r}")
        out = dict(meshes=meshes, materials=materials, objects=objs, lights=lights, bvh_bins=bvh_bins,
                   bvh_max_leaf=bvh_max_leaf)
        if nodes is not None:
            out.update(nodes=nodes, roots=roots)
        return out

    def commit(self, bvh_bins: int = 8, bvh_max_leaf: int = 1, device_build: bool = False) -> "Scene":
        """Scene::commit: builds (the meshes' BVHs on the GPU with device_build) and uploads."""
        if self.ctx is None:
            self.ctx = default_context()
        self.release()
        desc = self.describe(bvh_bins, bvh_max_leaf)
        if device_build:
            desc = dict(desc, device_build=True)
        sd, keep = _lower_description(desc, bvh_bins, bvh_max_leaf)
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.pbrt_scene_create(self.ctx.h, C.byref(sd), C.byref(h)), "pbrt_scene_create")
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

    def intersect_counted(self, rays):
        """Scene::intersect_instrumented over a batch: (prim_id, t, object_id, {nodes, boxes,
        objects}) with the scene accelerator's counters summed over the rays."""
        self._need()
        r, n = _as_rays(rays)
        prim, t, obj = _empty_like(r, n, "u32"), _empty_like(r, n, "f32"), _empty_like(r, n, "u32")
        stats = (C.c_uint64 * 3)()
        self.ctx.check(self.ctx.lib.pbrt_trace_closest_counted(self.h, _ptr(r), n, _ptr(prim), _ptr(t), _ptr(obj),
                                                               stats), "pbrt_trace_closest_counted")
        return prim, t, obj, dict(nodes=stats[0], boxes=stats[1], objects=stats[2])

    def intersect_p_counted(self, rays):
        """Scene::intersect_p_instrumented over a batch: (occluded, {nodes, boxes, objects})."""
        self._need()
        r, n = _as_rays(rays)
        occ = _empty_like(r, n, "u8")
        stats = (C.c_uint64 * 3)()
        self.ctx.check(self.ctx.lib.pbrt_trace_any_counted(self.h, _ptr(r), n, _ptr(occ), stats),
                       "pbrt_trace_any_counted")
        return occ, dict(nodes=stats[0], boxes=stats[1], objects=stats[2])

    def render(self, camera: dict, spp: int, max_depth: int, seed: int = 1, rr_start: int = 0,
               sample_offset: int = 0, integrator: str = "path", film=None, pixel_stride: int = 1):
        """Mean radiance per pixel, (height, width, 3) float64; `film` may be a CUDA tensor.
        pixel_stride s > 1 renders only the pixels (s*i, s*j), exactly as a full render does,
        into a (ceil(height/s), ceil(width/s), 3) film."""
        self._need()
        p = _capi.RenderParams()
        p.camera = camera_desc(camera)
        p.spp, p.max_depth, p.rr_start, p.sample_offset = int(spp), int(max_depth), int(rr_start), int(sample_offset)
        p.seed, p.integrator, p.pixel_stride = int(seed), INTEGRATORS[integrator], int(pixel_stride)
        if film is None:
            film = np.zeros(film_shape(camera, pixel_stride), np.float64)
        self.ctx.check(self.ctx.lib.pbrt_render(self.h, C.byref(p), _ptr(film)), "pbrt_render")
        return film

    def render_cached(self, cache, camera: dict, spp: int, max_depth: int, seed: int = 1, rr_start: int = 0,
                      sample_offset: int = 0, train_rounds: int = 1, film=None, pixel_stride: int = 1):
        """`train_rounds` rounds of online training of `cache` (a pbrt_b200.cache.RadianceCache),
        then `spp` samples per pixel whose paths end into it; returns the film (None when
        spp is 0)."""
        self._need()
        p = _capi.RenderParams()
        p.camera = camera_desc(camera)
        p.spp, p.max_depth, p.rr_start, p.sample_offset = int(spp), int(max_depth), int(rr_start), int(sample_offset)
        p.seed, p.integrator, p.pixel_stride = int(seed), 0, int(pixel_stride)
        if film is None and spp > 0:
            film = np.zeros(film_shape(camera, pixel_stride), np.float64)
        self.ctx.check(self.ctx.lib.pbrt_render_cached(self.h, cache.h, C.byref(p), int(train_rounds),
                                                       _ptr(film) if film is not None else None),
                       "pbrt_render_cached")
        return film

    def release(self):
        if self.h is not None and self.ctx is not None and self.ctx.h is not None:
            self.ctx.lib.pbrt_scene_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def _lower_description(desc: dict, bvh_bins: int = 8, bvh_max_leaf: int = 1):
    """The C pbrt_scene_desc of a description dict, with the arrays it points into."""
    keep = []
    meshes = []
    for m in desc["meshes"]:
        v = np.ascontiguousarray(m["vertices"], np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(m["indices"], np.uint32).reshape(-1, 3)
        keep += [v, i]
        fm = None
        if m.get("face_materials") is not None:
            fm = np.ascontiguousarray(m["face_materials"], np.uint32)
            keep.append(fm)
        meshes.append(_capi.MeshDesc(v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0],
                                     fm.ctypes.data if fm is not None else None))
    mats = []
    for m in desc["materials"]:
        d = _capi.MaterialDesc()
        d.kind = int(m["kind"])
        d.color[:] = [float(c) for c in m["color"]]
        d.fuzz, d.ior = float(m.get("fuzz", 0.0)), float(m.get("ior", 1.0))
        d.texture = int(m.get("texture", 0))
        d.color2[:] = [float(c) for c in m.get("color2", (0.0, 0.0, 0.0))]
        d.scale = float(m.get("scale", 1.0))
        mats.append(d)

    def xf(dst, m):  # float64 (or float32) 3x4 rows, rounded to FP32
        dst[:] = [float(x) for x in np.asarray(np.asarray(m, np.float64).reshape(-1)[:12], np.float32)]

    objs, celems = [], []
    for o in desc["objects"]:
        d = _capi.ObjectDesc()
        d.shape, d.mesh = int(o["shape"]), int(o.get("mesh", 0))
        d.radius, d.height = float(o.get("radius", 0.0)), float(o.get("height", 0.0))
        d.extent[:] = [float(x) for x in o.get("extent", (0.0, 0.0, 0.0))]
        d.material = int(o["material"])
        if o.get("to_world") is not None:
            d.transformed = 1
            xf(d.to_world, o["to_world"])
            xf(d.to_local, o["to_local"])
        if o.get("csg") is not None:
            d.csg_op, d.csg_first, d.csg_count = int(o["csg"]["op"]), len(celems), len(o["csg"]["elements"])
            for e in o["csg"]["elements"]:
                c = _capi.CsgElemDesc()
                c.shape, c.mesh = int(e["shape"]), int(e.get("mesh", 0))
                c.radius, c.height = float(e.get("radius", 0.0)), float(e.get("height", 0.0))
                c.extent[:] = [float(x) for x in e.get("extent", (0.0, 0.0, 0.0))]
                xf(c.to_world, e["to_world"])
                xf(c.to_local, e["to_local"])
                celems.append(c)
        objs.append(d)
    nodes, kids = [], []
    for n in desc.get("nodes") or []:
        d = _capi.NodeDesc()
        d.kind, d.object = int(n["kind"]), int(n.get("object", 0))
        ch = [int(c) for c in n.get("children", [])]
        d.first, d.count = len(kids), len(ch)
        kids += ch
        if n.get("to_world") is not None:
            xf(d.to_world, n["to_world"])
            xf(d.to_local, n["to_local"])
        nodes.append(d)
    roots = [int(r) for r in desc.get("roots", [])] if nodes else []
    lights = []
    for l in desc["lights"]:
        d = _capi.LightDesc()
        d.kind = int(l["kind"])
        for k in ("position", "radiance", "bottom", "top"):
            getattr(d, k)[:] = [float(x) for x in l.get(k, (0.0, 0.0, 0.0))]
        d.object = int(l.get("object", 0))
        lights.append(d)
    arrays = ((_capi.MeshDesc * max(1, len(meshes)))(*meshes), (_capi.MaterialDesc * max(1, len(mats)))(*mats),
              (_capi.ObjectDesc * max(1, len(objs)))(*objs), (_capi.LightDesc * max(1, len(lights)))(*lights))
    sd = _capi.SceneDesc()
    sd.meshes, sd.mesh_count = C.cast(arrays[0], C.POINTER(_capi.MeshDesc)), len(meshes)
    sd.materials, sd.material_count = C.cast(arrays[1], C.POINTER(_capi.MaterialDesc)), len(mats)
    sd.objects, sd.object_count = C.cast(arrays[2], C.POINTER(_capi.ObjectDesc)), len(objs)
    sd.lights, sd.light_count = C.cast(arrays[3], C.POINTER(_capi.LightDesc)), len(lights)
    sd.bvh_bins, sd.bvh_max_leaf = int(desc.get("bvh_bins", bvh_bins)), int(desc.get("bvh_max_leaf", bvh_max_leaf))
    sd.device_build = 1 if desc.get("device_build") else 0
    if celems:
        ca = (_capi.CsgElemDesc * len(celems))(*celems)
        sd.csg_elems, sd.csg_elem_count = C.cast(ca, C.POINTER(_capi.CsgElemDesc)), len(celems)
        keep.append(ca)
    if nodes:
        tree = ((_capi.NodeDesc * len(nodes))(*nodes), (C.c_uint32 * max(1, len(kids)))(*kids),
                (C.c_uint32 * max(1, len(roots)))(*roots))
        sd.nodes, sd.node_count = C.cast(tree[0], C.POINTER(_capi.NodeDesc)), len(nodes)
        sd.node_children, sd.child_count = C.cast(tree[1], C.POINTER(C.c_uint32)), len(kids)
        sd.roots, sd.root_count = C.cast(tree[2], C.POINTER(C.c_uint32)), len(roots)
        keep.append(tree)
    keep.append(arrays)
    return sd, keep


def create_scenes(descs, ctx: Optional[Context] = None, threads: int = 0, bvh_bins: int = 8,
                  bvh_max_leaf: int = 1, device_build: bool = False) -> list:
    """Committed Scenes of many descriptions at once: the host-side BVH builds run on
    `threads` threads (0: all cores) inside pbrt_scene_create_many; with device_build the
    meshes' BVHs are built on the GPU instead."""
    ctx = ctx or default_context()
    if device_build:
        descs = [dict(d, device_build=True) for d in descs]
    lowered = [_lower_description(d, bvh_bins, bvh_max_leaf) for d in descs]
    arr = (_capi.SceneDesc * len(lowered))(*[sd for sd, _ in lowered])
    hs = (C.c_void_p * len(lowered))()
    ctx.check(ctx.lib.pbrt_scene_create_many(ctx.h, arr, len(lowered), int(threads), hs), "pbrt_scene_create_many")
    out = []
    for d, h in zip(descs, hs):
        sc = Scene.from_description(d, ctx)
        sc.h = C.c_void_p(h)
        out.append(sc)
    return out


def render_params(camera: dict, spp: int, max_depth: int, seed: int = 1, rr_start: int = 0, sample_offset: int = 0,
                  integrator: str = "path", pixel_stride: int = 1) -> "_capi.RenderParams":
    p = _capi.RenderParams()
    p.camera = camera_desc(camera)
    p.spp, p.max_depth, p.rr_start, p.sample_offset = int(spp), int(max_depth), int(rr_start), int(sample_offset)
    p.seed, p.integrator, p.pixel_stride = int(seed), INTEGRATORS[integrator], int(pixel_stride)
    return p


class Batch:
    """Many committed scenes rendered together (pbrt_batch): one wavefront over all their
    paths, or one persistent launch (Context.set_batch_kernel), a frame's launches recorded
    once in a CUDA graph. `params` are render_params() per scene."""

    def __init__(self, scenes, params, ctx: Optional[Context] = None):
        self.ctx = ctx or scenes[0].ctx
        self.scenes = list(scenes)  # kept alive: the batch refers to their device data
        self.params = list(params)
        hs = (C.c_void_p * len(scenes))(*[s.h.value if isinstance(s.h, C.c_void_p) else s.h for s in scenes])
        ps = (_capi.RenderParams * len(params))(*params)
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.pbrt_batch_create(self.ctx.h, hs, ps, len(scenes), C.byref(h)), "pbrt_batch_create")
        self.h = h

    def film_shapes(self):
        out = []
        for p in self.params:
            s = max(1, p.pixel_stride)
            out.append((-(-p.camera.height // s), -(-p.camera.width // s), 3))
        return out

    def render(self, frame: int = 0, films=None, scene_times: bool = False):
        """Films (numpy float64 by default, or the given host/device arrays) and, with
        scene_times, each scene's completion time in ms from the frame's start."""
        if films is None:
            films = [np.zeros(sh, np.float64) for sh in self.film_shapes()]
        fp = (C.c_void_p * len(films))(*[_ptr(f) if f is not None else None for f in films])
        ms = (C.c_float * len(self.scenes))() if scene_times else None
        self.ctx.check(self.ctx.lib.pbrt_batch_render(self.h, int(frame), fp, ms), "pbrt_batch_render")
        return (films, list(ms)) if scene_times else films

    def close(self):
        if getattr(self, "h", None) is not None and self.ctx.h is not None:
            self.ctx.lib.pbrt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def film_shape(camera: dict, pixel_stride: int = 1):
    """(rows, columns, 3) of the film a render with this camera and pixel stride fills."""
    s = max(1, int(pixel_stride))
    return (-(-int(camera["height"]) // s), -(-int(camera["width"]) // s), 3)


def write_png(path: str, rgba: np.ndarray):
    """image_write (src/renderers/mt.rs:152-167): an (h, w, 4) uint8 image as an RGBA PNG."""
    a = np.ascontiguousarray(rgba, np.uint8)
    rc = _capi.load().pbrt_write_png(path.encode(), a.ctypes.data, a.shape[1], a.shape[0])
    if rc != 0:
        raise PbrtError(rc, f"pbrt_write_png({path})")


def film_to_png(film: np.ndarray, path: str):
    """The renderer's output file: gamma, clip, 8 bits (film_to_rgba8), then write_png."""
    write_png(path, film_to_rgba8(film))


def film_to_rgba8(film: np.ndarray) -> np.ndarray:
    """Spectrum::gamma_correct + to_rgb (src/spectrum.rs:13-25): (h, w, 4) uint8."""
    f = np.ascontiguousarray(film, np.float64)
    h, w = f.shape[0], f.shape[1]
    out = np.zeros((h, w, 4), np.uint8)
    rc = _capi.load().pbrt_film_to_rgba8(f.ctypes.data, w, h, out.ctypes.data)
    if rc != 0:
        raise PbrtError(rc, "pbrt_film_to_rgba8")
    return out


# ------------------------------------------------------------------------------------------
# Host-only tree inspection (no GPU needed)
# ------------------------------------------------------------------------------------------
GPU_NODE_DTYPE = np.dtype([("bmin", np.float32, 3), ("left_first", np.uint32), ("bmax", np.float32, 3),
                           ("count", np.uint32)])


def build_mesh_bvh_device(vertices, indices, bvh_bins: int = 8, bvh_max_leaf: int = 1,
                          ctx: Optional["Context"] = None):
    """build_mesh_bvh_host on the GPU (pbrt_mesh_bvh_build_device): (nodes, tri_order,
    build milliseconds). vertices / indices may be numpy arrays or CUDA tensors."""
    ctx = ctx or default_context()
    if _is_torch(vertices):
        v = vertices.contiguous()
        nv = v.numel() // 3
    else:
        v = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
        nv = v.shape[0]
    if _is_torch(indices):
        i = indices.contiguous()
        nt = i.numel() // 3
    else:
        i = np.ascontiguousarray(np.asarray(indices, np.uint32).reshape(-1, 3))
        nt = i.shape[0]
    md = _capi.MeshDesc(_ptr(v), nv, _ptr(i), nt)
    cnt = C.c_uint64()
    ms = C.c_float()
    ctx.check(ctx.lib.pbrt_mesh_bvh_build_device(ctx.h, C.byref(md), bvh_bins, bvh_max_leaf, None, 0, None,
                                                 C.byref(cnt), None), "pbrt_mesh_bvh_build_device")
    nodes = np.zeros(cnt.value, GPU_NODE_DTYPE)
    order = np.zeros(nt, np.uint32)
    ctx.check(ctx.lib.pbrt_mesh_bvh_build_device(ctx.h, C.byref(md), bvh_bins, bvh_max_leaf, nodes.ctypes.data,
                                                 cnt.value, order.ctypes.data, C.byref(cnt), C.byref(ms)),
              "pbrt_mesh_bvh_build_device")
    return nodes, order, float(ms.value)


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
