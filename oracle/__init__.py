"""CPU oracle for the pbrt_b200 hot path — TEST INFRASTRUCTURE, NOT THE PRODUCT.

A C++ restatement (pbrt_oracle.hpp) of nmichel/pbrt's CPU traversal, intersection and
path-integration code, loaded here through ctypes. It is the checker of the CUDA path:
only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py may use it,
and nothing on the product path calls into it.

Parity pinning: the FP64 instantiation reproduces, to the unit, the hit counts and the
per-ray box/triangle test counts that the reference publishes for its mesh-mode traversal
benchmark (docs/mesures_bvh.md:706-713, produced by src/bin/bvh_stats.rs:345-401); see
tests/test_oracle_kat.py and tests/golden/bvh_stats_published.json.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

MISS = 0xFFFFFFFF


def build(force: bool = False) -> str:
    """Compile liboracle.so from its sources with the Makefile beside it."""
    srcs = [os.path.join(_HERE, f) for f in os.listdir(_HERE) if f.endswith((".cpp", ".hpp"))]
    if force or not os.path.exists(_LIB_PATH) or any(
        os.path.getmtime(s) > os.path.getmtime(_LIB_PATH) for s in srcs
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    vp, sz, i32, u32 = C.c_void_p, C.c_size_t, C.c_int, C.c_uint32
    L.oracle_last_error.restype = C.c_char_p
    L.oracle_ply_read.argtypes = [C.c_char_p, i32, C.POINTER(C.POINTER(C.c_double)), C.POINTER(sz),
                                  C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(sz)]
    L.oracle_free.argtypes = [vp]
    for suf in ("f64", "f32"):
        getattr(L, f"oracle_mesh_new_{suf}").restype = vp
        getattr(L, f"oracle_mesh_new_{suf}").argtypes = [vp, sz, vp, sz, i32, u32]
        getattr(L, f"oracle_mesh_free_{suf}").argtypes = [vp]
        getattr(L, f"oracle_mesh_build_stats_{suf}").argtypes = [vp, vp]
        getattr(L, f"oracle_mesh_node_count_{suf}").restype = sz
        getattr(L, f"oracle_mesh_node_count_{suf}").argtypes = [vp]
        getattr(L, f"oracle_mesh_nodes_{suf}").argtypes = [vp, vp, vp, vp]
        getattr(L, f"oracle_mesh_tri_idx_{suf}").argtypes = [vp, vp]
        getattr(L, f"oracle_mesh_trace_{suf}").argtypes = [vp, vp, sz, vp, vp, vp, i32]
        getattr(L, f"oracle_mesh_occluded_{suf}").argtypes = [vp, vp, sz, vp, i32]
        getattr(L, f"oracle_mesh_brute_{suf}").argtypes = [vp, vp, sz, vp, vp, i32]
        getattr(L, f"oracle_mesh_orbit_rays_{suf}").argtypes = [vp, vp]
        getattr(L, f"oracle_box_hit_{suf}").argtypes = [vp, vp, C.c_double if suf == "f64" else C.c_float,
                                                        C.c_double if suf == "f64" else C.c_float, vp]
        getattr(L, f"oracle_make_ray_{suf}").argtypes = [vp, vp, vp]
    L.oracle_slab_widening_f64.restype = C.c_double
    L.oracle_slab_widening_f32.restype = C.c_float


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def read_ply(path: str, reverse: bool = False):
    """Vertices (f64, values of the f32 text) and flat triangle indices of an ASCII PLY."""
    L = lib()
    vp = C.POINTER(C.c_double)()
    ip = C.POINTER(C.c_uint32)()
    nv, ni = C.c_size_t(), C.c_size_t()
    if L.oracle_ply_read(path.encode(), int(reverse), C.byref(vp), C.byref(nv), C.byref(ip), C.byref(ni)) != 0:
        raise IOError(L.oracle_last_error().decode())
    verts = np.ctypeslib.as_array(vp, shape=(max(1, nv.value * 3),))[: nv.value * 3].copy()
    idx = np.ctypeslib.as_array(ip, shape=(max(1, ni.value),))[: ni.value].copy()
    L.oracle_free(C.cast(vp, C.c_void_p))
    L.oracle_free(C.cast(ip, C.c_void_p))
    return verts.reshape(-1, 3), idx.reshape(-1, 3)


class MeshBVH:
    """The reference's mesh BVH (src/shapes/triangle_mesh/bvh.rs), built and traversed on
    the CPU in f64 (`dtype=np.float64`) or in the f32 restatement (`np.float32`).

    bins=8, max_leaf=1 is the reference's own build; bins=16, max_leaf=4 is the
    GPU configuration of the 327,680-triangle ray-cast workload."""

    def __init__(self, vertices, indices, dtype=np.float64, bins: int = 8, max_leaf: int = 1):
        self.dtype = np.dtype(dtype)
        self.suf = "f64" if self.dtype == np.float64 else "f32"
        self._v = np.ascontiguousarray(vertices, dtype=self.dtype).reshape(-1)
        self._i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
        L = lib()
        self._h = getattr(L, f"oracle_mesh_new_{self.suf}")(_ptr(self._v), self._v.size // 3, _ptr(self._i),
                                                            self._i.size // 3, bins, max_leaf)
        if not self._h:
            raise ValueError(L.oracle_last_error().decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            getattr(_lib, f"oracle_mesh_free_{self.suf}")(h)
            self._h = None

    def build_stats(self) -> dict:
        out = np.zeros(5, np.uint64)
        getattr(lib(), f"oracle_mesh_build_stats_{self.suf}")(self._h, _ptr(out))
        keys = ("node_count", "leaf_count", "max_depth", "max_leaf_tri_count", "total_leaf_tri_count")
        return {k: int(v) for k, v in zip(keys, out)}

    def nodes(self):
        n = getattr(lib(), f"oracle_mesh_node_count_{self.suf}")(self._h)
        boxes = np.zeros((n, 6), self.dtype)
        lf = np.zeros(n, np.uint64)
        cnt = np.zeros(n, np.uint64)
        getattr(lib(), f"oracle_mesh_nodes_{self.suf}")(self._h, _ptr(boxes), _ptr(lf), _ptr(cnt))
        return boxes, lf, cnt

    def tri_idx(self):
        out = np.zeros(self._i.size // 3, np.uint32)
        getattr(lib(), f"oracle_mesh_tri_idx_{self.suf}")(self._h, _ptr(out))
        return out

    def _rays(self, rays):
        rays = np.ascontiguousarray(rays, dtype=self.dtype)
        assert rays.ndim == 2 and rays.shape[0] == 8, "rays are 8 SoA planes: ox oy oz dx dy dz tmin tmax"
        return rays

    def trace(self, rays, threads: int = os.cpu_count() or 1):
        """Nearest hit per ray: (prim_id uint32 with 0xFFFFFFFF for a miss, t, counters)."""
        rays = self._rays(rays)
        n = rays.shape[1]
        prim = np.empty(n, np.uint32)
        t = np.empty(n, self.dtype)
        stats = np.zeros(3, np.uint64)
        if getattr(lib(), f"oracle_mesh_trace_{self.suf}")(self._h, _ptr(rays), n, _ptr(prim), _ptr(t),
                                                             _ptr(stats), threads) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return prim, t, dict(nodes_visited=int(stats[0]), box_tests=int(stats[1]), triangle_tests=int(stats[2]))

    def occluded(self, rays, threads: int = os.cpu_count() or 1):
        rays = self._rays(rays)
        n = rays.shape[1]
        occ = np.empty(n, np.uint8)
        if getattr(lib(), f"oracle_mesh_occluded_{self.suf}")(self._h, _ptr(rays), n, _ptr(occ), threads) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return occ

    def brute_force(self, rays, threads: int = os.cpu_count() or 1):
        rays = self._rays(rays)
        n = rays.shape[1]
        prim = np.empty(n, np.uint32)
        t = np.empty(n, self.dtype)
        getattr(lib(), f"oracle_mesh_brute_{self.suf}")(self._h, _ptr(rays), n, _ptr(prim), _ptr(t), threads)
        return prim, t

    def orbit_rays(self):
        """The mesh-mode ray set of src/bin/bvh_stats.rs:345-382 (240,000 rays)."""
        out = np.zeros((8, 6 * 200 * 200), self.dtype)
        getattr(lib(), f"oracle_mesh_orbit_rays_{self.suf}")(self._h, _ptr(out))
        return out


def box_hit(bmin, bmax, origin, direction, tmin, tmax, dtype=np.float64):
    """AABoundingBox::hit (src/geom/aabound.rs:323-355): entry distance or None. The
    direction is used as given (the reference's Ray::new normalises it; use make_ray)."""
    dt = np.dtype(dtype)
    suf = "f64" if dt == np.float64 else "f32"
    box = np.array(list(bmin) + list(bmax), dt)
    ray = np.array(list(origin) + list(direction), dt)
    entry = np.zeros(1, dt)
    hit = getattr(lib(), f"oracle_box_hit_{suf}")(_ptr(box), _ptr(ray), float(tmin), float(tmax), _ptr(entry))
    return float(entry[0]) if hit else None


def make_ray(origin, direction, dtype=np.float64):
    """Ray::new (src/geom/ray.rs:10-18): (origin, normalised direction)."""
    dt = np.dtype(dtype)
    suf = "f64" if dt == np.float64 else "f32"
    o = np.array(origin, dt)
    d = np.array(direction, dt)
    out = np.zeros(6, dt)
    getattr(lib(), f"oracle_make_ray_{suf}")(_ptr(o), _ptr(d), _ptr(out))
    return out[:3].copy(), out[3:].copy()


# ------------------------------------------------------------------------------------------
# Scenes and rendering (pbrt_oracle_pt.hpp)
#
# A scene is described by a plain dict, the same one the tests lower into the product:
#   meshes:    [{"vertices": (n,3) float32, "indices": (m,3) uint32}]
#   materials: [{"kind": 0 lambertian | 1 metal | 2 dielectric | 3 diffuse light,
#                "color": (3,), "fuzz": f, "ior": f,
#                optional "texture": 1 checkerboard with "color2": (3,), "scale": f}]
#   objects:   [{"shape": 0 mesh | 1 sphere | 2 cylinder | 3 rectangle | 4 aabox | 5 plane | 6 csg,
#                "mesh": i, "radius": r, "height": h, "extent": (3,), "material": i,
#                "to_world": (12,) or None, "to_local": (12,) or None,
#                csg: "csg": {"op": 0 union | 1 intersection | 2 subtraction,
#                             "elements": [{"shape", "mesh", "radius", "height", "extent",
#                                           "to_world", "to_local"}]}}]
#              (rectangle: radius = width, height = height; aabox: extent = full size)
#   lights:    [{"kind": 0 point | 1 uniform infinite | 2 background | 3 area, "position": (3,),
#                "radiance": (3,), "bottom": (3,), "top": (3,), "object": i}]
#   optional object tree: "nodes": [{"kind": 0 simple | 1 transformed | 2 compound,
#                "object": i (simple), "children": [node, ...], "to_world", "to_local"
#                (transformed)}], "roots": [node, ...] (the scene's primitives, in order)
#   bvh_bins, bvh_max_leaf
# Transforms are float64 here (the f64 oracle keeps them; the f32 oracle and the product
# round them to float32).
# camera: {"width", "height", "fov" (radians), "near", "far", "position", "look_at", "up"}
# ------------------------------------------------------------------------------------------
class _OMesh(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32), ("indices", C.c_void_p),
                ("triangle_count", C.c_uint32), ("face_materials", C.c_void_p)]


class _OMaterial(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("color", C.c_float * 3), ("fuzz", C.c_float), ("ior", C.c_float),
                ("texture", C.c_uint32), ("color2", C.c_float * 3), ("scale", C.c_float)]


class _OObject(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("mesh", C.c_uint32), ("radius", C.c_double), ("height", C.c_double),
                ("extent", C.c_double * 3), ("material", C.c_uint32), ("transformed", C.c_uint32),
                ("to_world", C.c_double * 12), ("to_local", C.c_double * 12), ("csg_op", C.c_uint32),
                ("csg_first", C.c_uint32), ("csg_count", C.c_uint32)]


class _OCsgElem(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("mesh", C.c_uint32), ("radius", C.c_double), ("height", C.c_double),
                ("extent", C.c_double * 3), ("to_world", C.c_double * 12), ("to_local", C.c_double * 12)]


class _ONode(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("object", C.c_uint32), ("first", C.c_uint32), ("count", C.c_uint32),
                ("to_world", C.c_double * 12), ("to_local", C.c_double * 12)]


class _OLight(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("position", C.c_float * 3), ("radiance", C.c_float * 3),
                ("bottom", C.c_float * 3), ("top", C.c_float * 3), ("object", C.c_uint32)]


class _OScene(C.Structure):
    _fields_ = [("meshes", C.c_void_p), ("mesh_count", C.c_uint32), ("materials", C.c_void_p),
                ("material_count", C.c_uint32), ("objects", C.c_void_p), ("object_count", C.c_uint32),
                ("lights", C.c_void_p), ("light_count", C.c_uint32), ("bvh_bins", C.c_uint32),
                ("bvh_max_leaf", C.c_uint32), ("nodes", C.c_void_p), ("node_count", C.c_uint32),
                ("children", C.c_void_p), ("child_count", C.c_uint32), ("roots", C.c_void_p),
                ("root_count", C.c_uint32), ("csg_elems", C.c_void_p), ("csg_elem_count", C.c_uint32)]


class _OCamera(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("fov", C.c_double), ("near", C.c_double),
                ("far", C.c_double), ("position", C.c_double * 3), ("look_at", C.c_double * 3),
                ("up", C.c_double * 3), ("thin_lens", C.c_uint32), ("lens_radius", C.c_double),
                ("focal_distance", C.c_double)]


class _ORender(C.Structure):
    _fields_ = [("camera", _OCamera), ("spp", C.c_uint32), ("max_depth", C.c_uint32), ("rr_start", C.c_uint32),
                ("sample_offset", C.c_uint32), ("seed", C.c_uint64), ("integrator", C.c_uint32)]


def _camera(cam: dict) -> _OCamera:
    c = _OCamera()
    c.width, c.height = int(cam["width"]), int(cam["height"])
    c.fov, c.near, c.far = float(cam["fov"]), float(cam["near"]), float(cam["far"])
    c.position[:] = [float(x) for x in cam["position"]]
    c.look_at[:] = [float(x) for x in cam["look_at"]]
    c.up[:] = [float(x) for x in cam["up"]]
    if cam.get("kind") == "thin_lens":  # ThinLensCamera (src/cameras/thin_lens.rs)
        c.thin_lens = 1
        c.lens_radius, c.focal_distance = float(cam["lens_radius"]), float(cam["focal_distance"])
    return c


def _declare_scene(L):
    vp, sz = C.c_void_p, C.c_size_t
    for suf in ("f64", "f32"):
        getattr(L, f"oracle_scene_new_{suf}").restype = vp
        getattr(L, f"oracle_scene_new_{suf}").argtypes = [C.POINTER(_OScene)]
        getattr(L, f"oracle_scene_free_{suf}").argtypes = [vp]
        getattr(L, f"oracle_scene_trace_{suf}").argtypes = [vp, vp, sz, vp, vp, vp, C.c_int]
        getattr(L, f"oracle_scene_occluded_{suf}").argtypes = [vp, vp, sz, vp, C.c_int]
        getattr(L, f"oracle_render_{suf}").argtypes = [vp, C.POINTER(_ORender), vp, C.c_int]
        getattr(L, f"oracle_render_counted_{suf}").argtypes = [vp, C.POINTER(_ORender), vp, C.c_int, vp]
        getattr(L, f"oracle_render_cached_{suf}").argtypes = [vp, C.POINTER(_ORender), vp, vp, C.c_uint32, vp,
                                                              C.c_int]
        getattr(L, f"oracle_camera_rays_{suf}").argtypes = [C.POINTER(_OCamera), vp]
        getattr(L, f"oracle_scene_bvh_{suf}").argtypes = [vp, vp, vp, vp, vp]
        getattr(L, f"oracle_scene_bvh_nodes_{suf}").restype = sz
        getattr(L, f"oracle_scene_bvh_nodes_{suf}").argtypes = [vp]
        getattr(L, f"oracle_scene_trace_stats_{suf}").argtypes = [vp, vp, sz, vp, vp, vp, C.c_int, vp]
        getattr(L, f"oracle_scene_occluded_stats_{suf}").argtypes = [vp, vp, sz, vp, C.c_int, vp]
        getattr(L, f"oracle_scene_cast_sets_{suf}").argtypes = [vp, C.POINTER(_OCamera), vp, C.c_double,
                                                                C.c_double, C.c_double, vp, vp]
        getattr(L, f"oracle_scene_counts_{suf}").argtypes = [vp, vp]


def _xf12(m):
    """A transform given as 12 row-major values or a 3x4 / 4x4 matrix, as 12 float64."""
    return [float(x) for x in np.asarray(m, np.float64).reshape(-1)[:12]]


class Scene:
    """The reference's Scene (src/scene.rs) with its objects, materials and lights, in f64
    or in the f32 restatement; renders with the path or naive integrator."""

    def __init__(self, desc: dict, dtype=np.float32):
        L = lib()
        if not getattr(L, "_scene_declared", False):
            _declare_scene(L)
            L._scene_declared = True
        self.dtype = np.dtype(dtype)
        self.suf = "f64" if self.dtype == np.float64 else "f32"
        self._keep = []
        ms = []
        for m in desc.get("meshes", []):
            v = np.ascontiguousarray(m["vertices"], np.float32).reshape(-1, 3)
            i = np.ascontiguousarray(m["indices"], np.uint32).reshape(-1, 3)
            self._keep += [v, i]
            fm = None
            if m.get("face_materials") is not None:
                fm = np.ascontiguousarray(m["face_materials"], np.uint32)
                self._keep.append(fm)
            ms.append(_OMesh(v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0],
                             fm.ctypes.data if fm is not None else None))
        mats = []
        for m in desc.get("materials", []):
            d = _OMaterial()
            d.kind = int(m["kind"])
            d.color[:] = [float(c) for c in m.get("color", (0, 0, 0))]
            d.fuzz, d.ior = float(m.get("fuzz", 0.0)), float(m.get("ior", 1.0))
            d.texture = int(m.get("texture", 0))
            d.color2[:] = [float(c) for c in m.get("color2", (0, 0, 0))]
            d.scale = float(m.get("scale", 1.0))
            mats.append(d)
        objs, celems = [], []
        for o in desc.get("objects", []):
            d = _OObject()
            d.shape, d.mesh = int(o["shape"]), int(o.get("mesh", 0))
            d.radius, d.height = float(o.get("radius", 0.0)), float(o.get("height", 0.0))
            d.extent[:] = [float(x) for x in o.get("extent", (0.0, 0.0, 0.0))]
            d.material = int(o["material"])
            if o.get("to_world") is not None:
                d.transformed = 1
                d.to_world[:] = _xf12(o["to_world"])
                d.to_local[:] = _xf12(o["to_local"])
            if o.get("csg") is not None:
                d.csg_op, d.csg_first, d.csg_count = int(o["csg"]["op"]), len(celems), len(o["csg"]["elements"])
                for e in o["csg"]["elements"]:
                    c = _OCsgElem()
                    c.shape, c.mesh = int(e["shape"]), int(e.get("mesh", 0))
                    c.radius, c.height = float(e.get("radius", 0.0)), float(e.get("height", 0.0))
                    c.extent[:] = [float(x) for x in e.get("extent", (0.0, 0.0, 0.0))]
                    c.to_world[:] = _xf12(e["to_world"])
                    c.to_local[:] = _xf12(e["to_local"])
                    celems.append(c)
            objs.append(d)
        nodes, kids = [], []
        for n in desc.get("nodes", []) or []:
            d = _ONode()
            d.kind = int(n["kind"])
            d.object = int(n.get("object", 0))
            ch = [int(c) for c in n.get("children", [])]
            d.first, d.count = len(kids), len(ch)
            kids += ch
            if n.get("to_world") is not None:
                d.to_world[:] = _xf12(n["to_world"])
                d.to_local[:] = _xf12(n["to_local"])
            nodes.append(d)
        roots = [int(r) for r in desc.get("roots", [])] if nodes else []
        lts = []
        for l in desc.get("lights", []):
            d = _OLight()
            d.kind = int(l["kind"])
            for k in ("position", "radiance", "bottom", "top"):
                getattr(d, k)[:] = [float(x) for x in l.get(k, (0, 0, 0))]
            d.object = int(l.get("object", 0))
            lts.append(d)
        arrs = [(_OMesh * max(1, len(ms)))(*ms), (_OMaterial * max(1, len(mats)))(*mats),
                (_OObject * max(1, len(objs)))(*objs), (_OLight * max(1, len(lts)))(*lts),
                (_ONode * max(1, len(nodes)))(*nodes), (C.c_uint32 * max(1, len(kids)))(*kids),
                (C.c_uint32 * max(1, len(roots)))(*roots), (_OCsgElem * max(1, len(celems)))(*celems)]
        self._keep += arrs
        sd = _OScene(C.addressof(arrs[0]), len(ms), C.addressof(arrs[1]), len(mats), C.addressof(arrs[2]), len(objs),
                     C.addressof(arrs[3]), len(lts), int(desc.get("bvh_bins", 8)), int(desc.get("bvh_max_leaf", 1)),
                     C.addressof(arrs[4]) if nodes else None, len(nodes), C.addressof(arrs[5]), len(kids),
                     C.addressof(arrs[6]), len(roots), C.addressof(arrs[7]), len(celems))
        self._h = getattr(L, f"oracle_scene_new_{self.suf}")(C.byref(sd))
        if not self._h:
            raise ValueError(L.oracle_last_error().decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            getattr(_lib, f"oracle_scene_free_{self.suf}")(h)
            self._h = None

    def trace(self, rays, threads: int = os.cpu_count() or 1):
        """Scene::intersect per ray: (prim, object, t); prim is the triangle index (0 for an
        analytic shape), both MISS on a miss."""
        rays = np.ascontiguousarray(rays, dtype=self.dtype)
        n = rays.shape[1]
        prim, obj, t = np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty(n, self.dtype)
        getattr(lib(), f"oracle_scene_trace_{self.suf}")(self._h, _ptr(rays), n, _ptr(prim), _ptr(obj), _ptr(t),
                                                         threads)
        return prim, obj, t

    def occluded(self, rays, threads: int = os.cpu_count() or 1):
        rays = np.ascontiguousarray(rays, dtype=self.dtype)
        occ = np.empty(rays.shape[1], np.uint8)
        getattr(lib(), f"oracle_scene_occluded_{self.suf}")(self._h, _ptr(rays), rays.shape[1], _ptr(occ), threads)
        return occ

    def trace_instrumented(self, rays, threads: int = os.cpu_count() or 1):
        """trace plus the scene query's counters summed over the rays: {nodes, boxes, objects}
        as Scene::intersect_instrumented counts them (src/scene.rs:124-128)."""
        rays = np.ascontiguousarray(rays, dtype=self.dtype)
        n = rays.shape[1]
        prim, obj, t = np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty(n, self.dtype)
        st = np.zeros(3, np.uint64)
        getattr(lib(), f"oracle_scene_trace_stats_{self.suf}")(self._h, _ptr(rays), n, _ptr(prim), _ptr(obj),
                                                               _ptr(t), threads, _ptr(st))
        return prim, obj, t, dict(zip(("nodes", "boxes", "objects"), (int(x) for x in st)))

    def occluded_instrumented(self, rays, threads: int = os.cpu_count() or 1):
        """occluded plus Scene::intersect_p_instrumented's counters (src/scene.rs:148-153)."""
        rays = np.ascontiguousarray(rays, dtype=self.dtype)
        occ = np.empty(rays.shape[1], np.uint8)
        st = np.zeros(3, np.uint64)
        getattr(lib(), f"oracle_scene_occluded_stats_{self.suf}")(self._h, _ptr(rays), rays.shape[1], _ptr(occ),
                                                                  threads, _ptr(st))
        return occ, dict(zip(("nodes", "boxes", "objects"), (int(x) for x in st)))

    def counts(self) -> dict:
        """{bounded primitives (the BVH's), unbounded primitives, BVH nodes}."""
        out = np.zeros(3, np.uint64)
        getattr(lib(), f"oracle_scene_counts_{self.suf}")(self._h, _ptr(out))
        return dict(zip(("primitives", "unbounded", "nodes"), (int(x) for x in out)))

    def cast_sets(self, camera: dict, target=(0.0, 2.0, 1.0), near: float = 1e-4, far: float = 1000.0,
                  shadow_near: float = 1e-5, shadow_rays: bool = False):
        """The scene mode of the reference's traversal benchmark (src/bin/bvh_stats.rs:254-286):
        pixel-centre primary rays, and from each hit a shadow ray towards `target`. Returns
        {"primary": {rays, hits, nodes, boxes, objects}, "shadow": {...}} and, with
        shadow_rays=True, the shadow rays (8 x pixels SoA, NaN rows for primary misses)."""
        L = lib()
        c = _camera(camera)
        out = np.zeros(10, np.uint64)
        tgt = np.asarray(target, np.float64)
        n = int(camera["width"]) * int(camera["height"])
        sr = np.zeros((8, n), self.dtype) if shadow_rays else None
        getattr(L, f"oracle_scene_cast_sets_{self.suf}")(self._h, C.byref(c), _ptr(tgt), near, far, shadow_near,
                                                         _ptr(out), _ptr(sr) if sr is not None else None)
        keys = ("rays", "hits", "nodes", "boxes", "objects")
        res = {"primary": {k: int(v) for k, v in zip(keys, out[:5])},
               "shadow": {k: int(v) for k, v in zip(keys, out[5:])}}
        return (res, sr) if shadow_rays else res

    def bvh(self):
        n = getattr(lib(), f"oracle_scene_bvh_nodes_{self.suf}")(self._h)
        boxes = np.zeros((n, 6), self.dtype)
        lf, cnt = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        order = np.zeros(max(1, n), np.uint32)
        getattr(lib(), f"oracle_scene_bvh_{self.suf}")(self._h, _ptr(boxes), _ptr(lf), _ptr(cnt), _ptr(order))
        return boxes, lf, cnt, order

    def render(self, camera: dict, spp: int, max_depth: int, seed: int = 1, rr_start: int = 0,
               sample_offset: int = 0, integrator: str = "path", threads: int = os.cpu_count() or 1):
        """Mean radiance per pixel, (height, width, 3) float64 (renderers/mt.rs:112-130)."""
        p = _ORender()
        p.camera = _camera(camera)
        p.spp, p.max_depth, p.rr_start, p.sample_offset = spp, max_depth, rr_start, sample_offset
        p.seed, p.integrator = seed, {"path": 0, "naive": 1, "normal": 2}[integrator]
        film = np.zeros((int(camera["height"]), int(camera["width"]), 3), np.float64)
        if getattr(lib(), f"oracle_render_{self.suf}")(self._h, C.byref(p), _ptr(film), threads) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return film

    def render_counted(self, camera: dict, spp: int, max_depth: int, seed: int = 1, rr_start: int = 0,
                       sample_offset: int = 0, threads: int = os.cpu_count() or 1):
        """render() with the path integrator, plus its work summed over every scene query:
        (film, {rays, shadow_rays, top_boxes, objects, mesh_boxes, triangles, shapes})."""
        p = _ORender()
        p.camera = _camera(camera)
        p.spp, p.max_depth, p.rr_start, p.sample_offset = spp, max_depth, rr_start, sample_offset
        p.seed, p.integrator = seed, 0
        film = np.zeros((int(camera["height"]), int(camera["width"]), 3), np.float64)
        out = np.zeros(7, np.uint64)
        if getattr(lib(), f"oracle_render_counted_{self.suf}")(self._h, C.byref(p), _ptr(film), threads,
                                                                _ptr(out)) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        keys = ("rays", "shadow_rays", "top_boxes", "objects", "mesh_boxes", "triangles", "shapes")
        return film, {k: int(v) for k, v in zip(keys, out)}

    def render_cached(self, camera: dict, spp: int, max_depth: int, weights, bounds, terminate_bounce: int = 2,
                      seed: int = 1, rr_start: int = 0, sample_offset: int = 0,
                      threads: int = os.cpu_count() or 1):
        """The path integrator ending paths into the network `weights` (BF16-emulating) at hit
        terminate_bounce + 1, as the GPU's cached render does after its training rounds."""
        p = _ORender()
        p.camera = _camera(camera)
        p.spp, p.max_depth, p.rr_start, p.sample_offset = spp, max_depth, rr_start, sample_offset
        p.seed, p.integrator = seed, 0
        w = np.ascontiguousarray(weights, np.float32)
        b = np.ascontiguousarray(bounds, np.float32).reshape(6)
        film = np.zeros((int(camera["height"]), int(camera["width"]), 3), np.float64)
        fn = getattr(lib(), f"oracle_render_cached_{self.suf}")
        if fn(self._h, C.byref(p), _ptr(w), _ptr(b), terminate_bounce + 1, _ptr(film), threads) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return film


def camera_rays(camera: dict, dtype=np.float32):
    """Pixel-centre primary rays of PinHoleCamera (src/cameras/pin_hole.rs:42-50), row-major."""
    L = lib()
    if not getattr(L, "_scene_declared", False):
        _declare_scene(L)
        L._scene_declared = True
    dt = np.dtype(dtype)
    n = int(camera["width"]) * int(camera["height"])
    out = np.zeros((8, n), dt)
    c = _camera(camera)
    getattr(L, f"oracle_camera_rays_{'f64' if dt == np.float64 else 'f32'}")(C.byref(c), _ptr(out))
    return out


# ------------------------------------------------------------------------------------------
# The radiance cache's network (mlp_oracle.hpp)
# ------------------------------------------------------------------------------------------
MLP_PARAMS = 23552


def _declare_mlp(L):
    vp = C.c_void_p
    L.oracle_mlp_forward.argtypes = [vp, vp, vp, C.c_size_t, vp, C.c_int, C.c_int]
    L.oracle_mlp_gradient.argtypes = [vp, vp, vp, vp, C.c_size_t, vp, vp, C.c_int]
    L.oracle_mlp_forward_f64.argtypes = [vp, vp, vp, C.c_size_t, vp]
    L.oracle_mlp_forward_margins.argtypes = [vp, vp, vp, C.c_size_t, vp, vp, vp, C.c_int]
    L.oracle_mlp_adam.argtypes = [vp, vp, vp, vp, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float]
    L.oracle_mlp_encode.argtypes = [vp, vp, C.c_size_t, vp]


def _mlp_lib():
    L = lib()
    if not getattr(L, "_mlp_declared", False):
        _declare_mlp(L)
        L._mlp_declared = True
    return L


def mlp_encode(bounds, records):
    """The network's input features (n, 96) of query records (n, 16) (mlp_oracle.hpp encode)."""
    b = np.ascontiguousarray(bounds, np.float32).reshape(6)
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 16)
    out = np.zeros((r.shape[0], 96), np.float32)
    _mlp_lib().oracle_mlp_encode(_ptr(b), _ptr(r), r.shape[0], _ptr(out))
    return out


def mlp_forward(weights, bounds, records, emulate=True, threads: int = os.cpu_count() or 1):
    """Network outputs (n, 3); bounds = (min xyz, max xyz) of the position normalisation."""
    w = np.ascontiguousarray(weights, np.float32)
    b = np.ascontiguousarray(bounds, np.float32).reshape(6)
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 16)
    out = np.zeros((r.shape[0], 3), np.float32)
    _mlp_lib().oracle_mlp_forward(_ptr(w), _ptr(b), _ptr(r), r.shape[0], _ptr(out), int(emulate), threads)
    return out


def mlp_forward_margins(weights, bounds, records, threads: int = os.cpu_count() or 1):
    """BF16-emulating outputs (n, 3), per record the smallest BF16 rounding margin of its
    forward pass (distance of a BF16-rounded value to a rounding boundary, in units of 2^-24
    times the magnitude sum of the terms that formed it), and the outputs' magnitude sums (n, 3)."""
    w = np.ascontiguousarray(weights, np.float32)
    b = np.ascontiguousarray(bounds, np.float32).reshape(6)
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 16)
    n = r.shape[0]
    out = np.zeros((n, 3), np.float32)
    margin = np.zeros(n, np.float64)
    scale = np.zeros((n, 3), np.float64)
    _mlp_lib().oracle_mlp_forward_margins(_ptr(w), _ptr(b), _ptr(r), n, _ptr(out), _ptr(margin), _ptr(scale), threads)
    return out, margin, scale


def mlp_forward_f64(weights, bounds, records):
    """Exact-mode network outputs (n, 3) in float64."""
    w = np.ascontiguousarray(weights, np.float32)
    b = np.ascontiguousarray(bounds, np.float32).reshape(6)
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 16)
    out = np.zeros((r.shape[0], 3), np.float64)
    _mlp_lib().oracle_mlp_forward_f64(_ptr(w), _ptr(b), _ptr(r), r.shape[0], _ptr(out))
    return out


def mlp_gradient(weights, bounds, records, targets, emulate=True):
    """(gradient (23552,) float64, mean loss) of the relative-L2 loss over the batch."""
    w = np.ascontiguousarray(weights, np.float32)
    b = np.ascontiguousarray(bounds, np.float32).reshape(6)
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 16)
    t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
    g = np.zeros(MLP_PARAMS, np.float64)
    loss = np.zeros(1, np.float64)
    _mlp_lib().oracle_mlp_gradient(_ptr(w), _ptr(b), _ptr(r), _ptr(t), r.shape[0], _ptr(g), _ptr(loss), int(emulate))
    return g, float(loss[0])


def mlp_adam(w, m, v, g, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step in place on float32 arrays."""
    for a in (w, m, v):
        assert a.dtype == np.float32 and a.flags.c_contiguous
    gg = np.ascontiguousarray(g, np.float32)
    _mlp_lib().oracle_mlp_adam(_ptr(w), _ptr(m), _ptr(v), _ptr(gg), step, lr, b1, b2, eps)
