"""The oracle is pinned to the reference's own published figures.

The FP64 instantiation of the oracle must reproduce, to the unit, the hit counts of the
reference's mesh-mode traversal benchmark and, to the published two decimals, its ray/box
and ray/triangle tests per ray, plus the exact node and leaf counts of the built tree
(docs/mesures_bvh.md:706-713; ray set of src/bin/bvh_stats.rs:345-401).
"""
import os

import numpy as np
import pytest

import oracle


def _check(name, v, i, pub):
    m = oracle.MeshBVH(v, i, np.float64, bins=8, max_leaf=1)
    bs = m.build_stats()
    assert bs["node_count"] == pub["nodes"], name
    assert bs["leaf_count"] == pub["leaves"], name
    assert bs["total_leaf_tri_count"] == pub["triangles"], "every triangle belongs to exactly one leaf"
    rays = m.orbit_rays()
    prim, t, st = m.trace(rays)
    n = rays.shape[1]
    assert n == 240000
    assert int((prim != oracle.MISS).sum()) == pub["hits"], name
    assert round(st["box_tests"] / n, 2) == pytest.approx(pub["box_per_ray"], abs=1e-9), name
    assert round(st["triangle_tests"] / n, 2) == pytest.approx(pub["tri_per_ray"], abs=1e-9), name


@pytest.mark.parametrize("key,name", [("cube", "cube.ply"), ("bun_zipper_res4", "bun_zipper_res4.ply"),
                                      ("dragon_vrip_res4", "dragon_vrip_res4.ply")])
def test_published_counts_from_fixtures(golden_meshes, published, key, name):
    _check(name, golden_meshes[key + "_vertices"], golden_meshes[key + "_indices"], published[name])


@pytest.mark.parametrize("name", ["dragon_vrip_res3.ply", "bunny.ply"])
def test_published_counts_from_reference_meshes(reference_test_files, published, name):
    v, i = oracle.read_ply(os.path.join(reference_test_files, name))
    _check(name, v, i, published[name])


def test_fixture_matches_reference_ply(reference_test_files, golden_meshes):
    for key in ("cube", "bun_zipper_res4", "dragon_vrip_res4"):
        v, i = oracle.read_ply(os.path.join(reference_test_files, key + ".ply"))
        assert np.array_equal(v, golden_meshes[key + "_vertices"])
        assert np.array_equal(i, golden_meshes[key + "_indices"])
