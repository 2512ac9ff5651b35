"""The reference's own unit tests for this path, restated against the oracle.

Sources: src/shapes/triangle_mesh/bvh.rs:896-995 (tree vs brute force, intersect_p vs
query, separated triangles) and src/geom/aabound.rs:475-682 (slab test edge cases). Each is
run in both instantiations (f64 = the reference's precision, f32 = the GPU's).
"""
import numpy as np
import pytest

import oracle
from conftest import grid_ray_set, unbuilt_grid_mesh

DTYPES = [np.float64, np.float32]


@pytest.mark.parametrize("dtype", DTYPES)
def test_query_matches_brute_force(dtype):
    v, i = unbuilt_grid_mesh(3)
    m = oracle.MeshBVH(v, i, dtype)
    rays = grid_ray_set(v, i, oracle.make_ray, dtype)
    prim, t, _ = m.trace(rays)
    bprim, bt = m.brute_force(rays)
    assert np.array_equal(prim, bprim)
    hit = prim != oracle.MISS
    assert np.array_equal(t[hit], bt[hit])
    assert hit.sum() > 20


@pytest.mark.parametrize("dtype", DTYPES)
def test_intersect_p_agrees_with_query(dtype):
    v, i = unbuilt_grid_mesh(3)
    m = oracle.MeshBVH(v, i, dtype)
    rays = grid_ray_set(v, i, oracle.make_ray, dtype)
    prim, t, _ = m.trace(rays)
    assert np.array_equal(m.occluded(rays).astype(bool), prim != oracle.MISS)
    hit = prim != oracle.MISS
    assert hit.sum() > 20
    for factor in (0.5, 0.99, 0.999999, 1.0, 1.000001):
        r = rays[:, hit].copy()
        r[7] = (t[hit] * factor).astype(dtype)
        p2, _, _ = m.trace(r)
        assert np.array_equal(m.occluded(r).astype(bool), p2 != oracle.MISS), factor


def test_separated_triangles_land_in_distinct_leaves():
    v, i = unbuilt_grid_mesh(4)
    bs = oracle.MeshBVH(v, i, np.float64).build_stats()
    assert bs["total_leaf_tri_count"] == 64
    assert bs["max_leaf_tri_count"] <= 4


def test_max_leaf_caps_leaves_and_keeps_every_triangle():
    v, i = unbuilt_grid_mesh(4)
    for ml in (1, 2, 4, 8):
        bs = oracle.MeshBVH(v, i, np.float32, bins=16, max_leaf=ml).build_stats()
        assert bs["total_leaf_tri_count"] == 64
        assert bs["max_leaf_tri_count"] <= max(ml, 1)


@pytest.mark.parametrize("dtype", DTYPES)
def test_box_collide(dtype):
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    cases = [
        ((0, 0, 0), (0, 0, 1), True), ((0, 0, 0), (0, 1, 0), True), ((0, 0, 0), (1, 0, 0), True),
        ((0, 0, 0), (0, 0, -1), True), ((0, 0, 0), (0, -1, 0), True), ((0, 0, 0), (-1, 0, 0), True),
        ((1.01, 0, 0), (0, 0, 1), False), ((0, 0, -1.1), (0, 1, 0), False), ((0, 0, 1.01), (1, 0, 0), False),
        ((-1.01, 0, 0), (0, 0, -1), False), ((1.01, 0, -1.01), (0, -1, 0), False), ((1.10, 1.01, 0), (-1, 0, 0), False),
        ((0.5, -0.5, 0), (1, -1, 1), True), ((0.5, -0.5, 0), (-0.63, -1, 2.13), True),
        ((0.5, -0.5, 0), (12.2, 0.004, -0.0003), True), ((-2, 0, 0), (3, 1, 0), True), ((-2, 0, 0), (3, 1, -2), True),
    ]
    for o, d, expect in cases:
        ro, rd = oracle.make_ray(o, d, dtype)
        assert (oracle.box_hit(lo, hi, ro, rd, 0.0, 1000.0, dtype) is not None) == expect, (o, d)


@pytest.mark.parametrize("dtype", DTYPES)
def test_box_flat_and_grazing(dtype):
    lo, hi = (-1.0, 0.0, -1.0), (1.0, 0.0, 1.0)
    crossing = [((0, 1, 0), (0, -1, 0)), ((0, -1, 0), (0, 1, 0)), ((-0.5, 1, -0.5), (0.3, -1, 0.2)),
                ((-0.5, 0, 0), (1, 0, 0))]
    missing = [((-0.5, 0.5, 0), (1, 0, 0)), ((2, 1, 0), (0, -1, 0)), ((0, 1, 0), (0, 1, 0))]
    for o, d in crossing:
        assert oracle.box_hit(lo, hi, *oracle.make_ray(o, d, dtype), 0.0, 1000.0, dtype) is not None, (o, d)
    for o, d in missing:
        assert oracle.box_hit(lo, hi, *oracle.make_ray(o, d, dtype), 0.0, 1000.0, dtype) is None, (o, d)
    g = oracle.make_ray((-2, 1, 0), (1, 0, 0), dtype)
    assert oracle.box_hit((-1, -1, -1), (1, 1, 1), *g, 0.0, 1000.0, dtype) is not None


def test_rounding_bound_magnitude():
    u64 = np.finfo(np.float64).eps / 2
    w64 = oracle.lib().oracle_slab_widening_f64()
    assert 6 * u64 < w64 < 8 * u64 and w64 < 1e-15
    u32 = np.finfo(np.float32).eps / 2
    w32 = oracle.lib().oracle_slab_widening_f32()
    assert 6 * u32 < w32 < 8 * u32
