"""The mesh BVH built on the GPU equals the host build bit for bit: the same nodes (boxes,
counts, children, numbering) and the same triangle order in every leaf — the reference's
binned-SAH tree (src/shapes/triangle_mesh/bvh.rs:221-309, 609-735), whose leaf order comes
from its forward-swap partition. Scenes built with device_build render and trace exactly as
host-built ones."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import pbrt_b200 as pb
from conftest import unbuilt_grid_mesh
from pbrt_b200 import workloads
from pbrt_b200.scene import build_mesh_bvh_device, build_mesh_bvh_host

pytestmark = pytest.mark.gpu


def _same(v, i, bins, max_leaf):
    hn, ho = build_mesh_bvh_host(v, i, bins, max_leaf)
    dn, do, ms = build_mesh_bvh_device(v, i, bins, max_leaf)
    assert dn.shape == hn.shape
    np.testing.assert_array_equal(dn.view(np.uint32).reshape(-1, 8), hn.view(np.uint32).reshape(-1, 8))
    np.testing.assert_array_equal(do, ho)
    return ms


def _meshes():
    yield "grid6", unbuilt_grid_mesh(6)
    yield "grid12", unbuilt_grid_mesh(12)  # 1,728 slanted triangles: large and small nodes
    for lvl in (3, 5, 6):
        v, i = workloads.displaced_icosphere(lvl)
        yield f"ico{lvl}", (v, i)
    v, i = workloads.torus_knot(segments=300, sides=12)
    yield "knot", (v, i)


@pytest.mark.parametrize("bins,max_leaf", [(8, 1), (16, 4), (2, 1), (64, 2), (8, 600)])
def test_device_build_equals_host_build(bins, max_leaf, golden_meshes):
    for name, (v, i) in _meshes():
        _same(v, i, bins, max_leaf)
    for key in ("cube", "bun_zipper_res4"):
        _same(golden_meshes[key + "_vertices"], golden_meshes[key + "_indices"], bins, max_leaf)


def test_degenerate_meshes():
    # every centroid equal: no axis can be split, the root stays a leaf
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    i = np.tile(np.array([[0, 1, 2]], np.uint32), (2000, 1))
    _same(v, i, 8, 1)
    # centroids distinct along x only, with duplicates and zero coordinates of both signs
    rng = np.random.default_rng(5)
    xs = np.repeat(rng.integers(-3, 4, 700).astype(np.float32), 3)
    v = np.stack([xs, np.tile(np.array([0.0, -0.0, 0.5], np.float32), 700), np.zeros(2100, np.float32)], 1)
    i = np.arange(2100, dtype=np.uint32).reshape(-1, 3)
    _same(v, i, 16, 1)
    # a single triangle
    _same(v[:3], i[:1], 8, 1)


def test_large_mesh_and_speed():
    v, i = workloads.displaced_icosphere(8)  # 1,310,720 triangles
    ms = _same(v, i, 16, 4)
    print("device build of 1.31M triangles:", ms, "ms")


def test_bad_input_is_refused():
    v = np.zeros((3, 3), np.float32)
    i = np.array([[0, 1, 7]], np.uint32)
    with pytest.raises(pb.PbrtError):
        build_mesh_bvh_device(v, i)
    v = np.array([[0, 0, 0], [1, np.inf, 0], [0, 1, 0]], np.float32)
    with pytest.raises(pb.PbrtError):
        build_mesh_bvh_device(v, np.array([[0, 1, 2]], np.uint32))


def test_device_arrays_in():
    torch = pytest.importorskip("torch")
    v, i = workloads.displaced_icosphere(5)
    hn, ho = build_mesh_bvh_host(v, i, 16, 4)
    dn, do, _ = build_mesh_bvh_device(torch.from_numpy(np.asarray(v, np.float32)).cuda(),
                                      torch.from_numpy(np.asarray(i, np.int32)).cuda(), 16, 4)
    np.testing.assert_array_equal(dn.view(np.uint32), hn.view(np.uint32))
    np.testing.assert_array_equal(do, ho)


def test_scene_device_build_renders_identically():
    desc, cam = workloads.cornell_box(48, 48)
    a = pb.Scene.from_description(desc).commit(bvh_bins=16, bvh_max_leaf=4)
    b = pb.Scene.from_description(desc).commit(bvh_bins=16, bvh_max_leaf=4, device_build=True)
    np.testing.assert_array_equal(a.render(cam, spp=8, max_depth=6, seed=3), b.render(cam, spp=8, max_depth=6, seed=3))
    v, i = workloads.displaced_icosphere(6)
    m = pb.Simple(pb.TriangleMesh(v, i))
    s1 = pb.Scene().add_object(m).commit(bvh_bins=16, bvh_max_leaf=4)
    s2 = pb.Scene().add_object(m).commit(bvh_bins=16, bvh_max_leaf=4, device_build=True)
    rays = workloads.incoherent_rays(200_000, v.min(0), v.max(0), seed=4)
    p1, t1, st1 = s1.intersect_instrumented(rays)
    p2, t2, st2 = s2.intersect_instrumented(rays)
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(t1, t2)
    assert st1 == st2
    assert s1.info()["mesh_node_count"] == s2.info()["mesh_node_count"]


def test_create_scenes_with_device_builds():
    from pbrt_b200.scene import create_scenes
    specs = workloads.batch_scenes(3, seed=11, width=32, height=32, levels=(3, 6))
    host = create_scenes([d for d, _, _ in specs], bvh_max_leaf=2)
    dev = create_scenes([d for d, _, _ in specs], bvh_max_leaf=2, device_build=True)
    for a, b, (_, cam, spp) in zip(host, dev, specs):
        np.testing.assert_array_equal(a.render(cam, spp=2, max_depth=4, seed=1), b.render(cam, spp=2, max_depth=4, seed=1))
