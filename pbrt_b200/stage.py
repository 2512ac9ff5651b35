"""Scene files: the reference's `Loader::load_scene` (src/loader.rs:29-45) over the library's
C++ `.stage` parser and PLY reader (pbrt_stage_parse / pbrt_scene_load / pbrt_ply_read).

    scene, camera = load_scene(open("test_files/cornell_box_canonical.stage").read(),
                               fov_deg=60, far=2000, base_dir="/path/to/pbrt")
    film = scene.render(camera, spp=16, max_depth=8)

Options are the Config fields the reference's loader reads (src/config.rs:112-129): the
output size, the field of view in degrees, the near and far planes. Mesh file names in a
scene file are read relative to `base_dir` (the reference reads them relative to its
working directory). Like the reference's loader, every scene gets a point light at (0, 2, 1)
of intensity 15 and a white-to-(0.5, 0.7, 1.0) background unless loader_lights=False.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _capi
from ._capi import PbrtError
from .scene import Context, Scene, default_context


def _options(base_dir, width, height, fov_deg, near, far, loader_lights, bvh_bins, bvh_max_leaf):
    o = _capi.StageOptions()
    o.base_dir = base_dir.encode() if base_dir else None
    o.width, o.height = int(width), int(height)
    o.fov_deg, o.near, o.far = float(fov_deg), float(near), float(far)
    o.no_loader_lights = 0 if loader_lights else 1
    o.bvh_bins, o.bvh_max_leaf = int(bvh_bins), int(bvh_max_leaf)
    return o


def _camera_dict(c: _capi.CameraDesc) -> dict:
    d = dict(width=c.width, height=c.height, fov=c.fov, near=c.near, far=c.far, position=tuple(c.position),
             look_at=tuple(c.look_at), up=tuple(c.up))
    if c.thin_lens:
        d.update(kind="thin_lens", lens_radius=c.lens_radius, focal_distance=c.focal_distance)
    return d


class Stage:
    """A parsed scene file (host memory): its description and camera."""

    def __init__(self, text: str, base_dir: Optional[str] = None, width: int = 800, height: int = 600,
                 fov_deg: float = 90.0, near: float = 0.0001, far: float = 1000.0, loader_lights: bool = True,
                 bvh_bins: int = 8, bvh_max_leaf: int = 1):
        self.lib = _capi.load()
        self.h = C.c_void_p()
        err = C.create_string_buffer(512)
        opt = _options(base_dir, width, height, fov_deg, near, far, loader_lights, bvh_bins, bvh_max_leaf)
        rc = self.lib.pbrt_stage_parse(text.encode(), C.byref(opt), C.byref(self.h), err, len(err))
        if rc != 0:
            self.h = None
            raise PbrtError(rc, err.value.decode())
        self.sd = _capi.SceneDesc()
        self.cam = _capi.CameraDesc()
        self._lens = (C.c_float * 2)()
        self.lib.pbrt_stage_describe(self.h, C.byref(self.sd), C.byref(self.cam), self._lens)

    @property
    def camera(self) -> dict:
        """The camera as a dict for Scene.render (kind "thin_lens" with lens_radius and
        focal_distance for a thin_lens camera)."""
        return _camera_dict(self.cam)

    @property
    def lens(self) -> Tuple[float, float]:
        """A thin_lens camera's (radius, focal distance); (0, 0) for a pin_hole camera."""
        return (float(self._lens[0]), float(self._lens[1]))

    def describe(self) -> dict:
        """The scene description dict (copies of the parsed arrays; transforms as FP32 rows)."""
        sd = self.sd
        meshes = []
        for i in range(sd.mesh_count):
            m = sd.meshes[i]
            v = np.ctypeslib.as_array(C.cast(m.vertices, C.POINTER(C.c_float)), shape=(max(1, m.vertex_count * 3),))
            ix = np.ctypeslib.as_array(C.cast(m.indices, C.POINTER(C.c_uint32)),
                                       shape=(max(1, m.triangle_count * 3),))
            meshes.append(dict(vertices=v[: m.vertex_count * 3].reshape(-1, 3).copy(),
                               indices=ix[: m.triangle_count * 3].reshape(-1, 3).copy()))
        mats = []
        for i in range(sd.material_count):
            m = sd.materials[i]
            d = dict(kind=m.kind, color=tuple(m.color), fuzz=m.fuzz, ior=m.ior)
            if m.texture:
                d.update(texture=m.texture, color2=tuple(m.color2), scale=m.scale)
            mats.append(d)
        objs = []
        for i in range(sd.object_count):
            o = sd.objects[i]
            d = dict(shape=o.shape, mesh=o.mesh, radius=o.radius, height=o.height, extent=tuple(o.extent),
                     material=o.material, to_world=None, to_local=None)
            if o.transformed:
                d.update(to_world=np.array(o.to_world, np.float32), to_local=np.array(o.to_local, np.float32))
            if o.shape == _capi.SHAPE_CSG:
                elems = []
                for k in range(o.csg_first, o.csg_first + o.csg_count):
                    e = sd.csg_elems[k]
                    elems.append(dict(shape=e.shape, mesh=e.mesh, radius=e.radius, height=e.height,
                                      extent=tuple(e.extent), to_world=np.array(e.to_world, np.float32),
                                      to_local=np.array(e.to_local, np.float32)))
                d["csg"] = dict(op=o.csg_op, elements=elems)
            objs.append(d)
        nodes = []
        for i in range(sd.node_count):
            n = sd.nodes[i]
            d = dict(kind=n.kind)
            if n.kind == _capi.NODE_SIMPLE:
                d["object"] = n.object
            else:
                cnt = 1 if n.kind == _capi.NODE_TRANSFORMED else n.count
                d["children"] = [int(sd.node_children[n.first + k]) for k in range(cnt)]
            if n.kind == _capi.NODE_TRANSFORMED:
                d.update(to_world=np.array(n.to_world, np.float32), to_local=np.array(n.to_local, np.float32))
            nodes.append(d)
        lights = []
        for i in range(sd.light_count):
            l = sd.lights[i]
            lights.append(dict(kind=l.kind, position=tuple(l.position), radiance=tuple(l.radiance),
                               bottom=tuple(l.bottom), top=tuple(l.top), object=l.object))
        out = dict(meshes=meshes, materials=mats, objects=objs, lights=lights, bvh_bins=sd.bvh_bins or 8,
                   bvh_max_leaf=sd.bvh_max_leaf or 1, camera=self.camera)
        if nodes:
            out.update(nodes=nodes, roots=[int(sd.roots[k]) for k in range(sd.root_count)])
        return out

    def scene(self, ctx: Optional[Context] = None) -> Scene:
        """The committed Scene of this file (pbrt_scene_create on its description)."""
        s = Scene(ctx or default_context())
        h = C.c_void_p()
        s.ctx.check(s.ctx.lib.pbrt_scene_create(s.ctx.h, C.byref(self.sd), C.byref(h)), "pbrt_scene_create")
        s.h = h
        return s

    def close(self):
        if self.h is not None:
            self.lib.pbrt_stage_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_scene(text: str, ctx: Optional[Context] = None, **options) -> Tuple[Scene, dict]:
    """Loader::load_scene: (the committed Scene, its camera dict). Options as Stage."""
    st = Stage(text, **options)
    try:
        return st.scene(ctx), st.camera
    finally:
        st.close()


def read_ply(path: str, reverse: bool = False):
    """load_ply_mesh's geometry (src/loader/mesh_loader.rs:13-24): (vertices (n, 3) float32,
    indices (m, 3) uint32), faces reversed when `reverse`."""
    lib = _capi.load()
    vp = C.POINTER(C.c_float)()
    ip = C.POINTER(C.c_uint32)()
    nv, nt = C.c_uint32(), C.c_uint32()
    err = C.create_string_buffer(512)
    rc = lib.pbrt_ply_read(path.encode(), int(reverse), C.byref(vp), C.byref(nv), C.byref(ip), C.byref(nt), err,
                           len(err))
    if rc != 0:
        raise PbrtError(rc, err.value.decode())
    try:
        v = np.ctypeslib.as_array(vp, shape=(max(1, nv.value * 3),))[: nv.value * 3].reshape(-1, 3).copy()
        i = np.ctypeslib.as_array(ip, shape=(max(1, nt.value * 3),))[: nt.value * 3].reshape(-1, 3).copy()
    finally:
        lib.pbrt_free(C.cast(vp, C.c_void_p))
        lib.pbrt_free(C.cast(ip, C.c_void_p))
    return v, i
