"""The library's C++ scene-file loader against the oracle's restatement (no GPU needed).

pbrt_stage_parse must build, from the reference's own scene files, exactly the description the
oracle's loader builds: the same objects in the same (reversed) order, the same object tree,
transforms equal to the oracle's f64 compositions rounded to FP32, the same materials,
textures, camera and loader lights; pbrt_ply_read must read the same vertices and faces as the
oracle's PLY reader.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
import pbrt_b200 as pb
from conftest import fixture_mesh_loader, stage_text
from oracle.stage import load_stage
from pbrt_b200 import PbrtError

SCENES = ["cornell_box_canonical.stage", "cornell_box.stage", "default.stage", "cube_mesh.stage",
          "many_spheres.stage", "many_meshes.stage", "csg_union_spheres.stage"]


def _f32(x):
    return np.asarray(np.asarray(x, np.float64), np.float32)


def _compare(got: dict, want: dict):
    assert len(got["meshes"]) == len(want["meshes"])
    for a, b in zip(got["meshes"], want["meshes"]):
        np.testing.assert_array_equal(a["vertices"], _f32(b["vertices"]))
        np.testing.assert_array_equal(a["indices"], np.asarray(b["indices"], np.uint32))
    assert len(got["materials"]) == len(want["materials"])
    for a, b in zip(got["materials"], want["materials"]):
        assert a["kind"] == b["kind"]
        np.testing.assert_array_equal(_f32(a["color"]), _f32(b["color"]))
        assert a.get("texture", 0) == b.get("texture", 0)
        if b.get("texture", 0):
            np.testing.assert_array_equal(_f32(a["color2"]), _f32(b["color2"]))
            assert np.float32(a["scale"]) == np.float32(b["scale"])
        for k in ("fuzz", "ior"):
            if k in b:
                assert np.float32(a[k]) == np.float32(b[k])
    assert len(got["objects"]) == len(want["objects"])
    for a, b in zip(got["objects"], want["objects"]):
        assert a["shape"] == b["shape"] and a["material"] == b["material"]
        assert a["mesh"] == b.get("mesh", 0) or b["shape"] != 0
        for k in ("radius", "height"):
            assert np.float32(a[k]) == np.float32(b.get(k, 0.0))
        np.testing.assert_array_equal(_f32(a["extent"]), _f32(b.get("extent", (0, 0, 0))))
        assert ("csg" in a) == ("csg" in b)
        if "csg" in b:
            assert a["csg"]["op"] == b["csg"]["op"]
            assert len(a["csg"]["elements"]) == len(b["csg"]["elements"])
            for ea, eb in zip(a["csg"]["elements"], b["csg"]["elements"]):
                assert ea["shape"] == eb["shape"] and np.float32(ea["radius"]) == np.float32(eb.get("radius", 0))
                np.testing.assert_array_equal(ea["to_world"], _f32(eb["to_world"]))
                np.testing.assert_array_equal(ea["to_local"], _f32(eb["to_local"]))
    assert len(got["nodes"]) == len(want["nodes"])
    for a, b in zip(got["nodes"], want["nodes"]):
        assert a["kind"] == b["kind"]
        assert a.get("object") == b.get("object") and a.get("children") == b.get("children")
        if b["kind"] == 1:
            np.testing.assert_array_equal(a["to_world"], _f32(b["to_world"]))
            np.testing.assert_array_equal(a["to_local"], _f32(b["to_local"]))
    assert got["roots"] == want["roots"]
    assert [l["kind"] for l in got["lights"]] == [l["kind"] for l in want["lights"]]
    for a, b in zip(got["lights"], want["lights"]):
        for k in ("position", "radiance", "bottom", "top"):
            if k in b:
                np.testing.assert_array_equal(_f32(a[k]), _f32(b[k]))
    gc, wc = got["camera"], want["camera"]
    assert (gc["width"], gc["height"]) == (wc["width"], wc["height"])
    for k in ("fov", "near", "far"):
        assert np.float32(gc[k]) == np.float32(wc[k]), k
    for k in ("position", "look_at", "up"):
        np.testing.assert_array_equal(_f32(gc[k]), _f32(wc[k]))


@pytest.mark.parametrize("name", SCENES)
def test_loader_matches_oracle(name, golden_meshes, mesh_dir):
    text = stage_text(name)
    opts = dict(width=200, height=150, fov_deg=60.0, far=2000.0)
    got = pb.Stage(text, base_dir=mesh_dir, **opts).describe()
    want = load_stage(text, fixture_mesh_loader(golden_meshes), **opts)
    _compare(got, want)


def test_loader_defaults_and_options(golden_meshes, mesh_dir):
    text = stage_text("default.stage")
    d = pb.Stage(text, base_dir=mesh_dir).describe()
    c = d["camera"]
    assert (c["width"], c["height"]) == (800, 600)
    assert np.float32(c["fov"]) == np.float32(np.pi / 2) and np.float32(c["near"]) == np.float32(1e-4)
    assert [l["kind"] for l in d["lights"]] == [0, 2]
    assert pb.Stage(text, loader_lights=False).describe()["lights"] == []


def test_thin_lens_camera_is_parsed():
    text = ("camera thin_lens pos 0 0 5 look 0 0 0 up 0 1 0 radius 0.1 focal_length 4.5\n"
            "scene object simple sphere 1 lambertian color 0.5 0.5 0.5")
    st = pb.Stage(text)
    assert st.lens == pytest.approx((0.1, 4.5))
    assert st.camera["position"] == (0.0, 0.0, 5.0)


@pytest.mark.parametrize("text", [
    "scene object simple sphere 1 lambertian color 1 1 1",
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object simple cone 1",
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object simple sphere 1 lambertian",
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object transformed object simple sphere 1 "
    "lambertian color 1 1 1 transform { scale 2 }",
    "camera pin_hole pos 0 0 0 look 0 0 1 up 0 1 0 scene object simple mesh file \"missing.ply\" "
    "lambertian color 1 1 1",
])
def test_loader_rejects_what_the_reference_rejects(text):
    with pytest.raises(PbrtError):
        pb.Stage(text)


def test_nested_csg_is_refused_as_unsupported():
    text = ("camera pin_hole pos 0 0 5 look 0 0 0 up 0 1 0 scene object simple csg union { elem csg union { "
            "elem sphere 1 transform { } } transform { } } lambertian color 1 1 1")
    with pytest.raises(PbrtError) as e:
        pb.Stage(text)
    assert e.value.code == 6  # PBRT_ERR_UNSUPPORTED


def test_ply_reader_matches_oracle(mesh_dir, golden_meshes):
    for key in ("cube", "bun_zipper_res4"):
        path = os.path.join(mesh_dir, "test_files", key + ".ply")
        for rev in (False, True):
            v, i = pb.read_ply(path, rev)
            ov, oi = oracle.read_ply(path, rev)
            np.testing.assert_array_equal(v, ov.astype(np.float32))
            np.testing.assert_array_equal(i, oi)
        np.testing.assert_array_equal(pb.read_ply(path)[1], golden_meshes[key + "_indices"])


def test_ply_reader_on_reference_files(reference_test_files):
    for name in ("cube.ply", "bun_zipper_res4.ply", "bunny.ply"):
        path = os.path.join(reference_test_files, name)
        v, i = pb.read_ply(path, True)
        ov, oi = oracle.read_ply(path, True)
        np.testing.assert_array_equal(v, ov.astype(np.float32))
        np.testing.assert_array_equal(i, oi)


def test_ply_reader_errors(tmp_path):
    bad = tmp_path / "quad.ply"
    bad.write_text("ply\nformat ascii 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty float z\n"
                   "element face 1\nproperty list uchar int vertex_indices\nend_header\n"
                   "0 0 0\n1 0 0\n1 1 0\n0 1 0\n4 0 1 2 3\n")
    with pytest.raises(PbrtError):
        pb.read_ply(str(bad))
    binary = tmp_path / "bin.ply"
    binary.write_text("ply\nformat binary_little_endian 1.0\nend_header\n")
    with pytest.raises(PbrtError):
        pb.read_ply(str(binary))
    oob = tmp_path / "oob.ply"
    oob.write_text("ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nproperty float z\n"
                   "element face 1\nproperty list uchar int vertex_indices\nend_header\n0 0 0\n3 0 1 2\n")
    with pytest.raises(PbrtError):
        pb.read_ply(str(oob))
