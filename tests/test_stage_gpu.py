"""The reference's scene files through the library's loader and the GPU, against the oracle.

Scene mode of the reference's traversal benchmark (src/bin/bvh_stats.rs:254-286) on its own
scene files: the GPU's nearest-hit and any-hit scene queries must give the FP32 oracle's
answers bit for bit — object, primitive (triangle, box face, cylinder piece), distance,
occlusion — and the same scene-accelerator counters (nodes visited, box tests, object tests).
(The FP64 oracle reproduces the published counters exactly; tests/test_stage_oracle.py.)
Rendered images of the files match the oracle's renders of the same sample streams.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import pbrt_b200 as pb
from conftest import fixture_mesh_loader, stage_text
from oracle.stage import load_stage
from pbrt_b200 import workloads as W
from pbrt_b200.scene import Batch, render_params

pytestmark = pytest.mark.gpu

TRACE_SCENES = ["cornell_box_canonical.stage", "many_spheres.stage", "many_meshes.stage", "default.stage",
                "cube_mesh.stage", "cornell_box.stage", "csg_union_spheres.stage"]

CSG_SCENE = """camera pin_hole pos 0.5 1.2 5 look 0 0 0 up 0 1 0
scene
  object transformed object simple csg intersection {
      elem sphere 1 transform { translate -0.3 0 0 }
      elem aabox 1.2 1.2 1.2 transform { rotate_y 0.5 translate 0.2 0 0 }
      elem cylinder 0.7 3 transform { rotate_x 0.4 } }
    lambertian checkerboard 0.9 0.2 0.2 0.2 0.9 0.2 4
    transform { translate -1.2 0.3 0 }
  object transformed object simple csg substraction {
      elem aabox 1.4 1.4 1.4 transform { }
      elem sphere 0.9 transform { translate 0.4 0.4 0.4 }
      elem cylinder 0.3 3 transform { rotate_z 1.5708 } }
    metal 0.2 color 0.8 0.8 0.9
    transform { rotate_y 0.6 translate 1.3 0.2 -0.5 }
  object simple csg union {
      elem mesh file "test_files/cube.ply" reverse transform { translate 0 -0.2 1.5 }
      elem sphere 0.5 transform { translate 0.4 0.3 1.5 }
      elem plane transform { translate 0 -1 0 } }
    lambertian color 0.6 0.6 0.6
  object transformed object simple rectangle 2 2 diffuse_light color 6 6 6
    transform { rotate_x 3.14159 translate 0 3 0 }
"""

TREE_SCENE = """camera pin_hole pos 0.3 1.5 6 look 0 0 0 up 0 1 0
scene
  object transformed object simple aabox 1 2 1.5 lambertian color 0.5 0.5 0.5
    transform { rotate_y 0.7 rotate_x 0.2 translate -1 0.2 0 }
  object transformed object transformed object simple rectangle 2 1 metal 0.1 color 0.9 0.9 0.9
    transform { rotate_z 0.3 } transform { translate 1.2 0.5 -0.5 rotate_x 1.2 }
  object transformed object compound {
      object simple sphere 0.4 dielectric 1.5 color 1 1 1
      object transformed object simple cylinder 0.3 0.8 lambertian color 0.2 0.8 0.2
        transform { translate 0.5 0 0 } }
    transform { translate 0 1.2 0.8 }
  object transformed object simple mesh file "test_files/cube.ply" reverse
      lambertian checkerboard 0.9 0.1 0.1 0.1 0.1 0.9 3
    transform { rotate_y 0.4 translate 1.5 -0.4 1 }
  object transformed object simple plane lambertian checkerboard 0.8 0.8 0.8 0.2 0.2 0.2 1.5
    transform { translate 0 -1 0 }
  object transformed object simple rectangle 1 1 diffuse_light color 4 4 4
    transform { rotate_x 3.14159 translate 0 3 0 }
"""


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref * ref + 1e-2)))


def _pair(text, golden_meshes, mesh_dir, **opts):
    st = pb.Stage(text, base_dir=mesh_dir, **opts)
    want = load_stage(text, fixture_mesh_loader(golden_meshes), **opts)
    return st, st.scene(), want, oracle.Scene(want, np.float32)


def _check_scene_mode(st, scene, want, osc):
    rays = oracle.camera_rays(want["camera"], np.float32)
    prim, t, obj, gst = scene.intersect_counted(rays)
    oprim, oobj, ot, ost = osc.trace_instrumented(rays)
    np.testing.assert_array_equal(obj, oobj)
    np.testing.assert_array_equal(prim, oprim)
    np.testing.assert_array_equal(t, ot)
    assert gst == ost
    res, srays = osc.cast_sets(want["camera"], shadow_rays=True)
    sr = np.ascontiguousarray(srays[:, ~np.isnan(srays[0])])
    occ, gsst = scene.intersect_p_counted(sr)
    oocc, osst = osc.occluded_instrumented(sr)
    np.testing.assert_array_equal(occ, oocc)
    assert gsst == osst
    assert int(occ.sum()) == res["shadow"]["hits"]
    assert (obj != pb.PBRT_MISS).sum() == res["primary"]["hits"]
    # the plain queries agree with the counted ones
    p2, t2, o2 = scene.intersect(rays, with_object=True)
    np.testing.assert_array_equal(o2, obj)
    np.testing.assert_array_equal(t2, t)
    np.testing.assert_array_equal(scene.intersect_p(sr), occ)
    return gst, gsst, rays.shape[1], sr.shape[1]


@pytest.mark.parametrize("name", TRACE_SCENES)
def test_scene_mode_bit_exact(name, golden_meshes, mesh_dir, published_scenes):
    st, scene, want, osc = _pair(stage_text(name), golden_meshes, mesh_dir, width=200, height=150)
    gp, gs, n, m = _check_scene_mode(st, scene, want, osc)
    if name in published_scenes:  # FP32 against the published FP64 figures, for the record
        pub = published_scenes[name]
        print(name, "primary", [round(v / n, 2) for v in gp.values()], pub["primary"],
              "shadow", [round(v / m, 2) for v in gs.values()], pub["shadow"])


def test_csg_bit_exact_and_render(golden_meshes, mesh_dir):
    """Union (with a mesh and an unbounded plane), Intersection and Substraction of mixed
    shapes: identical hits, pieces and counters, and the image."""
    st, scene, want, osc = _pair(CSG_SCENE, golden_meshes, mesh_dir, width=96, height=72)
    assert scene.info()["object_count"] == 4
    _check_scene_mode(st, scene, want, osc)
    img = scene.render(st.camera, spp=32, max_depth=6, seed=2)
    ref = osc.render(want["camera"], 32, 6, seed=2)
    assert relmse(img, ref) < 5e-3


def test_object_tree_bit_exact(golden_meshes, mesh_dir):
    """Compound, nested Transformed, AABox, Rectangle, Cylinder, a reversed mesh and an
    unbounded Plane, on rays from inside and outside the scene."""
    st, scene, want, osc = _pair(TREE_SCENE, golden_meshes, mesh_dir, width=96, height=72)
    assert scene.info()["object_count"] == 6
    _check_scene_mode(st, scene, want, osc)
    rng = np.random.default_rng(3)
    n = 20000
    o = rng.uniform(-3, 3, (3, n)).astype(np.float32)
    d = rng.normal(size=(3, n))
    d = (d / np.linalg.norm(d, axis=0)).astype(np.float32)
    dn = d * (np.float32(1) / np.sqrt((d * d).sum(0, dtype=np.float32)))
    rays = np.concatenate([o, dn, np.full((1, n), 1e-4, np.float32), np.full((1, n), 1e3, np.float32)])
    prim, t, obj, gst = scene.intersect_counted(rays)
    oprim, oobj, ot, ost = osc.trace_instrumented(rays)
    np.testing.assert_array_equal(obj, oobj)
    np.testing.assert_array_equal(prim, oprim)
    np.testing.assert_array_equal(t, ot)
    assert gst == ost
    occ, g2 = scene.intersect_p_counted(rays)
    oocc, o2 = osc.occluded_instrumented(rays)
    np.testing.assert_array_equal(occ, oocc)
    assert g2 == o2


@pytest.mark.parametrize("name,opts,spp,depth,tol", [
    ("cornell_box_canonical.stage", dict(fov_deg=60.0, far=2000.0), 64, 8, 5e-3),
    ("default.stage", dict(), 32, 8, 5e-3),
    ("many_spheres.stage", dict(), 16, 8, 5e-3),
])
def test_render_matches_oracle(name, opts, spp, depth, tol, golden_meshes, mesh_dir):
    st, scene, want, osc = _pair(stage_text(name), golden_meshes, mesh_dir, width=64, height=48, **opts)
    img = scene.render(st.camera, spp=spp, max_depth=depth, seed=4)
    ref = osc.render(want["camera"], spp, depth, seed=4)
    assert np.all(np.isfinite(img)) and img.mean() > 0
    err = relmse(img, ref)
    print(name, "relMSE", err)
    assert err < tol, err


def test_tree_scene_render_matches_oracle(golden_meshes, mesh_dir):
    st, scene, want, osc = _pair(TREE_SCENE, golden_meshes, mesh_dir, width=64, height=48)
    img = scene.render(st.camera, spp=32, max_depth=8, seed=9)
    ref = osc.render(want["camera"], 32, 8, seed=9)
    assert relmse(img, ref) < 5e-3


def test_load_scene_one_call(golden_meshes, mesh_dir):
    scene, cam = pb.load_scene(stage_text("cornell_box_canonical.stage"), base_dir=mesh_dir, width=40, height=30,
                               fov_deg=60.0, far=2000.0)
    img = scene.render(cam, spp=4, max_depth=4, seed=1)
    assert img.shape == (30, 40, 3) and np.all(np.isfinite(img)) and img.mean() > 0


def test_api_built_tree_equals_loaded(golden_meshes, mesh_dir):
    """The Python mirror (Compound, Transformed, Rectangle, AABox, Plane, CheckerBoard) lowers
    to the same scene as the loader: identical hits."""
    T = pb.Transform
    box = pb.Simple(pb.AABox((1.0, 2.0, 1.5)), pb.Lambertian((0.5, 0.5, 0.5)))
    rect = pb.Simple(pb.Rectangle(2.0, 1.0), pb.Metal(0.1, (0.9, 0.9, 0.9)))
    ball = pb.Simple(pb.Sphere(0.4), pb.Dielectric(1.5, (1.0, 1.0, 1.0)))
    cyl = pb.Simple(pb.Cylinder(0.3, 0.8), pb.Lambertian((0.2, 0.8, 0.2)))
    v, i = golden_meshes["cube_vertices"], golden_meshes["cube_indices"][:, ::-1]
    cube = pb.Simple(pb.TriangleMesh(v, i), pb.Lambertian(pb.CheckerBoard((0.9, 0.1, 0.1), (0.1, 0.1, 0.9), 3.0)))
    floor = pb.Simple(pb.Plane(), pb.Lambertian(pb.CheckerBoard((0.8, 0.8, 0.8), (0.2, 0.2, 0.2), 1.5)))
    lamp = pb.Simple(pb.Rectangle(1.0, 1.0), pb.DiffuseLight((4.0, 4.0, 4.0)))
    s = pb.Scene()
    I = T.identity()  # a transform block folds its steps onto the identity
    # scene files list objects in reverse; add them in the loaded order
    s.add_object(pb.Transformed(lamp, I * T.translation((0, 3, 0)) * T.rotation_x(3.14159)))
    s.add_object(pb.Transformed(floor, I * T.translation((0, -1, 0))))
    s.add_object(pb.Transformed(cube, I * T.translation((1.5, -0.4, 1)) * T.rotation_y(0.4)))
    s.add_object(pb.Transformed(pb.Compound([pb.Transformed(cyl, I * T.translation((0.5, 0, 0))), ball]),
                                I * T.translation((0, 1.2, 0.8))))
    s.add_object(pb.Transformed(pb.Transformed(rect, I * T.rotation_z(0.3)),
                                I * T.rotation_x(1.2) * T.translation((1.2, 0.5, -0.5))))
    s.add_object(pb.Transformed(box, I * T.translation((-1, 0.2, 0)) * T.rotation_x(0.2) * T.rotation_y(0.7)))
    s.commit()
    loaded = pb.Stage(TREE_SCENE, base_dir=mesh_dir, width=96, height=72)
    ls = loaded.scene()
    rays = oracle.camera_rays(load_stage(TREE_SCENE, fixture_mesh_loader(golden_meshes), width=96, height=72)["camera"],
                              np.float32)
    a = s.intersect_counted(rays)
    b = ls.intersect_counted(rays)
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[0], b[0])
    assert a[3] == b[3]


def test_api_built_csg_equals_loaded(golden_meshes, mesh_dir):
    T = pb.Transform
    I = T.identity()
    text = """camera pin_hole pos 0 0.5 4 look 0 0 0 up 0 1 0
    scene
      object simple csg substraction {
          elem sphere 1 transform { translate 0.5 0.5 0.5 }
          elem aabox 2 2 2 transform { rotate_y 0.3 } }
        lambertian color 0.5 0.5 0.5
    """
    # the file's elements, popped by the scene builder, come out reversed: the box is the base piece
    shp = pb.Csg("subtraction", [(pb.AABox((2.0, 2.0, 2.0)), I * T.rotation_y(0.3)),
                                 (pb.Sphere(1.0), I * T.translation((0.5, 0.5, 0.5)))])
    s = pb.Scene().add_object(pb.Simple(shp, pb.Lambertian((0.5, 0.5, 0.5)))).commit()
    loaded = pb.Stage(text, width=64, height=48)
    rays = oracle.camera_rays(load_stage(text, fixture_mesh_loader(golden_meshes), width=64, height=48)["camera"],
                              np.float32)
    a = s.intersect_counted(rays)
    b = loaded.scene().intersect_counted(rays)
    for k in range(3):
        np.testing.assert_array_equal(a[k], b[k])
    assert a[3] == b[3]
    hit = a[0] != pb.PBRT_MISS
    assert hit.mean() > 0.04 and set(np.unique(a[0][hit] >> 24)) == {0, 1}  # box faces and the cavity


def test_batch_mixing_solids_and_plain_scenes_equals_single_renders(mesh_dir):
    """A batch that holds a scene with constructive solids runs every scene through the
    kernels built with the solids' code, while a scene without solids rendered alone takes
    the build without it: the films must still be equal."""
    st = pb.Stage(CSG_SCENE, base_dir=mesh_dir, width=48, height=36)
    csg = st.scene()
    d, cam = W.cornell_box(32, 24)
    plain = pb.Scene.from_description(d).commit()
    kw = dict(spp=3, max_depth=5, seed=4)
    singles = [csg.render(st.camera, **kw), plain.render(cam, **kw)]
    b = Batch([csg, plain], [render_params(st.camera, **kw), render_params(cam, **kw)])
    films = b.render(0)
    for f, s in zip(films, singles):
        np.testing.assert_allclose(f, s, rtol=1e-12, atol=1e-15)
    b.close()


def _csg_grid_text(nx=8, nz=6):
    """nx * nz constructive solids (union of a sphere and a box, each placed by its own
    transform): a top-level tree deep enough for the persistent walk, with solids in it."""
    objs = []
    for i in range(nx):
        for k in range(nz):
            x, z = -3.5 + i, -2.5 + k
            objs.append(f"""  object transformed object simple csg union {{
      elem sphere 0.45 transform {{ }}
      elem aabox 0.6 0.6 0.6 transform {{ rotate_y 0.{i + k} translate 0.25 0 0 }} }}
    lambertian color 0.{i + 1} 0.5 0.{k + 2}
    transform {{ translate {x} 0 {z} }}""")
    return ("camera pin_hole pos 0 3 4.5 look 0 0 0 up 0 1 0\nscene\n" + "\n".join(objs) +
            "\n  object transformed object simple rectangle 4 4 diffuse_light color 4 4 4\n"
            "    transform { rotate_x 3.14159 translate 0 5 0 }\n")


def test_walk_over_many_solids(golden_meshes, mesh_dir):
    """Many constructive solids: the nearest-hit walk built with the solids' code renders
    them. Primary hits are bit-exact against the oracle, and the normal integrator (a
    function of the first hit only) agrees with the oracle's within 1e-5."""
    st, scene, want, osc = _pair(_csg_grid_text(), golden_meshes, mesh_dir, width=96, height=64)
    assert scene.info()["object_count"] == 49
    _check_scene_mode(st, scene, want, osc)
    img = scene.render(st.camera, spp=2, max_depth=1, seed=3, integrator="normal")
    ref = osc.render(want["camera"], 2, 1, seed=3, integrator="normal")
    np.testing.assert_allclose(img, ref, rtol=0, atol=1e-5)
    assert (img.sum(axis=2) > 0).mean() > 0.2
