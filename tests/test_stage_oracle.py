"""The oracle's scene loader and scene traversal, pinned to the reference's published figures.

The reference's traversal benchmark, run on its own scene files (src/bin/bvh_stats.rs:220-286),
publishes per scene the primitive count and, for the camera's 200 x 150 pixel-centre rays and the
shadow rays cast from their hits, the nodes / box tests / object tests per ray and the exact hit
count (docs/mesures_bvh.md:715-738). The FP64 oracle — its restatement of the `.stage` parser and
scene builder, of Rectangle / AABox / Transformed / Compound, of Scene::commit and of the scene
BVH's query / query_p — must reproduce every one of those figures, the counts to the unit.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from oracle.stage import StageError, Xf, load_stage, matmul4, tokenize
from conftest import fixture_mesh_loader, stage_text

FIXTURE_SCENES = ["cornell_box_canonical.stage", "many_spheres.stage", "many_meshes.stage"]


def _cast(desc):
    s = oracle.Scene(desc, np.float64)
    return s, s.cast_sets(desc["camera"])


def _check_published(name, s, res, pub):
    assert s.counts()["primitives"] + s.counts()["unbounded"] == pub["primitives"], name
    for key in ("primary", "shadow"):
        got = res[key]
        n = got["rays"]
        nodes, boxes, objects, touches = pub[key]
        assert got["hits"] == touches, (name, key)
        assert round(got["nodes"] / n, 2) == pytest.approx(nodes, abs=1e-9), (name, key)
        assert round(got["boxes"] / n, 2) == pytest.approx(boxes, abs=1e-9), (name, key)
        assert round(got["objects"] / n, 2) == pytest.approx(objects, abs=1e-9), (name, key)
    assert res["primary"]["rays"] == 200 * 150
    assert res["shadow"]["rays"] == res["primary"]["hits"]


@pytest.mark.parametrize("name", FIXTURE_SCENES)
def test_published_scene_counts(name, golden_meshes, published_scenes):
    desc = load_stage(stage_text(name), fixture_mesh_loader(golden_meshes), width=200, height=150)
    s, res = _cast(desc)
    _check_published(name, s, res, published_scenes[name])


def test_published_scene_counts_bunny(golden_meshes, published_scenes, reference_test_files):
    name = "bunny_mesh.stage"
    desc = load_stage(stage_text(name), fixture_mesh_loader(golden_meshes, reference_test_files), width=200,
                      height=150)
    s, res = _cast(desc)
    _check_published(name, s, res, published_scenes[name])


def test_tokens():
    """lexer.rs:379-440: numbers with sign and optional decimals, keywords, strings, comments."""
    for text, val in (("10", 10.0), ("10.", 10.0), ("10.0", 10.0), ("1234.56", 1234.56), ("+1234.56", 1234.56),
                      ("-1234.56", -1234.56)):
        assert tokenize(text) == [("num", val)]
    toks = tokenize('camera pin_hole # a comment\n  pos 1.6 2.3 3.4 { } "file.ply" foo_1')
    assert toks == [("kw", "camera"), ("kw", "pin_hole"), ("kw", "pos"), ("num", 1.6), ("num", 2.3), ("num", 3.4),
                    ("sym", "{"), ("sym", "}"), ("str", "file.ply"), ("id", "foo_1")]
    assert tokenize("1 .5 2") == [("num", 1.0)]  # '.' starts no token: the stream ends there


def test_scene_order_and_transform_fold(golden_meshes):
    """Objects come out in reverse file order (scene_builder.rs:56-61); a transform block is
    identity * last * ... * first (scene_builder.rs:200-212), so the first step acts first."""
    text = """camera pin_hole pos 0 0 5 look 0 0 0 up 0 1 0
    scene
      object simple sphere 1 lambertian color 1 0 0
      object transformed object simple aabox 1 2 3 metal 0.5 color 0 1 0
        transform { rotate_y 0.5 translate 1 2 3 }
      object compound { object simple sphere 2 lambertian color 0 0 1
                        object simple rectangle 4 6 diffuse_light color 5 5 5 }
    """
    d = load_stage(text, fixture_mesh_loader(golden_meshes))
    roots = [d["nodes"][r] for r in d["roots"]]
    assert [n["kind"] for n in roots] == [2, 1, 0]
    comp = roots[0]
    assert [d["objects"][d["nodes"][k]["object"]]["shape"] for k in comp["children"]] == [3, 1]
    xf = Xf.translation(1.0, 2.0, 3.0) * Xf.rotation("y", 0.5)
    w, l = xf.rows()
    np.testing.assert_array_equal(roots[1]["to_world"], w)
    np.testing.assert_array_equal(roots[1]["to_local"], l)
    assert w[3] == 1.0 and w[7] == 2.0 and w[11] == 3.0 and w[0] == math.cos(0.5)
    rect = d["objects"][d["nodes"][comp["children"][0]]["object"]]
    assert rect["radius"] == 4.0 and rect["height"] == 6.0  # Rectangle::new(width, height)
    assert d["camera"]["fov"] == 90.0 * math.pi / 180.0 and d["camera"]["near"] == 0.0001
    assert [l["kind"] for l in d["lights"]] == [0, 2]  # loader.rs:36-42


def test_matrix_product_is_sequential():
    a = [[0.1 * (i + 1) + 0.01 * j for j in range(4)] for i in range(4)]
    b = [[0.3 / (i + j + 1) for j in range(4)] for i in range(4)]
    m = matmul4(a, b)
    for i in range(4):
        for j in range(4):
            acc = 0.0
            for k in range(4):
                acc = acc + a[i][k] * b[k][j]
            assert m[i][j] == acc


@pytest.mark.parametrize("text", [
    "scene object simple sphere 1 lambertian color 1 1 1",                     # no camera
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object simple cone 1",  # unknown shape
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object simple sphere 1 lambertian",
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object transformed object simple sphere 1 "
    "lambertian color 1 1 1 transform { scale 2 }",
])
def test_rejected_files(text, golden_meshes):
    with pytest.raises(StageError):
        load_stage(text, fixture_mesh_loader(golden_meshes))


def test_every_fixture_scene_loads(golden_meshes):
    for name in ("cornell_box.stage", "cube_mesh.stage", "default.stage", "cornell_box_canonical.stage",
                 "many_spheres.stage", "many_meshes.stage"):
        d = load_stage(stage_text(name), fixture_mesh_loader(golden_meshes))
        s = oracle.Scene(d, np.float32)
        assert s.counts()["primitives"] == len(d["roots"])
    d = load_stage(stage_text("csg_union_spheres.stage"), fixture_mesh_loader(golden_meshes))
    csg = [o for o in d["objects"] if o["shape"] == 6]
    assert len(csg) == 1 and csg[0]["csg"]["op"] == 0 and len(csg[0]["csg"]["elements"]) == 9


def test_shapes_against_brute_force(golden_meshes):
    """Scene::intersect through the BVH equals testing every primitive (scene.rs:356-413), in
    both precisions, on a scene of every shape kind, a compound and nested transforms."""
    text = """camera pin_hole pos 0.3 1.5 6 look 0 0 0 up 0 1 0
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
      object transformed object simple plane lambertian color 0.7 0.7 0.7
        transform { translate 0 -1 0 }
    """
    d = load_stage(text, fixture_mesh_loader(golden_meshes), width=48, height=36)
    for dt in (np.float64, np.float32):
        s = oracle.Scene(d, dt)
        assert s.counts()["unbounded"] == 1
        rays = oracle.camera_rays(d["camera"], dt)
        prim, obj, t = s.trace(rays)
        assert (obj != oracle.MISS).mean() > 0.5
        # brute force: every root on its own, nearest with the earlier root winning ties
        best_t = np.full(rays.shape[1], np.inf)
        best_o = np.full(rays.shape[1], oracle.MISS, np.uint32)
        order = d["roots"]
        for r in order:
            sub = dict(d, roots=[r])
            _, o1, t1 = oracle.Scene(sub, dt).trace(rays)
            better = (o1 != oracle.MISS) & (t1 < best_t)
            best_t[better], best_o[better] = t1[better], o1[better]
        hit = obj != oracle.MISS
        np.testing.assert_array_equal(hit, best_o != oracle.MISS)
        np.testing.assert_array_equal(t[hit], best_t[hit].astype(dt))
        occ = s.occluded(rays)
        np.testing.assert_array_equal(occ.astype(bool), hit)


def _csg_scene(op, elements, extra=()):
    """One constructive solid (and optional plain spheres) as a scene description."""
    objs = [dict(shape=6, material=0, csg=dict(op=op, elements=[
        dict(shape=sh, radius=r, to_world=w, to_local=l) for sh, r, (w, l) in elements]))]
    for r, xf in extra:
        w, l = xf.rows()
        objs.append(dict(shape=1, radius=r, material=0, to_world=w, to_local=l))
    return dict(meshes=[], materials=[dict(kind=0, color=(0.5, 0.5, 0.5))], objects=objs, lights=[])


def _rays(n, seed, dt):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-3, 3, (3, n))
    d = rng.normal(size=(3, n))
    d /= np.linalg.norm(d, axis=0)
    return np.concatenate([o, d, np.full((1, n), 1e-4), np.full((1, n), 1e3)]).astype(dt)


def test_csg_bound_of_a_sphere_cut_by_a_plane():
    """intersection.rs:  the half-sphere is bounded by the sphere's box, in either order."""
    ident = Xf.identity().rows()
    for els in ([(1, 1.0, ident), (5, 0.0, ident)], [(5, 0.0, ident), (1, 1.0, ident)]):
        s = oracle.Scene(_csg_scene(1, els), np.float64)
        assert s.counts() == dict(primitives=1, unbounded=0, nodes=1)
        boxes = s.bvh()[0]
        np.testing.assert_array_equal(boxes[0], [-1, -1, -1, 1, 1, 1])


def test_csg_union_of_disjoint_spheres_is_their_compound():
    xs = [Xf.translation(x, 0.0, 0.0) for x in (-1.5, 0.0, 1.5)]
    u = oracle.Scene(_csg_scene(0, [(1, 0.5, x.rows()) for x in xs]), np.float64)
    c = oracle.Scene(_csg_scene(0, [], extra=[(0.5, x) for x in xs]), np.float64)
    rays = _rays(20000, 3, np.float64)
    _, ou, tu = u.trace(rays)
    _, oc, tc = c.trace(rays)
    hit = oc != oracle.MISS
    np.testing.assert_array_equal(ou != oracle.MISS, hit)
    np.testing.assert_array_equal(tu[hit], tc[hit])


def test_csg_intersection_and_subtraction_geometry():
    a, b = Xf.translation(-0.3, 0, 0).rows(), Xf.translation(0.3, 0, 0).rows()
    rays = _rays(60000, 4, np.float64)
    o, d = rays[0:3], rays[3:6]
    for op in (1, 2):
        s = oracle.Scene(_csg_scene(op, [(1, 1.0, a), (1, 0.8, b)]), np.float64)
        _, obj, t = s.trace(rays)
        hit = obj != oracle.MISS
        assert hit.sum() > 300
        p = o[:, hit] + d[:, hit] * t[hit]
        da = np.linalg.norm(p - np.array([[-0.3], [0], [0]]), axis=0)
        db = np.linalg.norm(p - np.array([[0.3], [0], [0]]), axis=0)
        if op == 1:  # on one sphere, inside the other
            assert np.all(((np.abs(da - 1) < 1e-9) & (db <= 0.8 + 1e-9)) | ((np.abs(db - 0.8) < 1e-9) & (da <= 1 + 1e-9)))
        else:  # on the base outside the hole, or on the hole inside the base
            assert np.all(((np.abs(da - 1) < 1e-9) & (db >= 0.8 - 1e-9)) | ((np.abs(db - 0.8) < 1e-9) & (da <= 1 + 1e-9)))
        assert np.array_equal(s.occluded(rays).astype(bool), hit)
