"""The product's host BVH builder produces the oracle's tree, node for node (no GPU needed).

The GPU traversal is bit-exact only if it walks the very tree the FP32 restatement of the
reference builds (src/shapes/triangle_mesh/bvh.rs:221-309, 609-735): same splits, same
child order, same triangle order inside leaves, same FP32 boxes.
"""
import numpy as np
import pytest

import oracle
from conftest import unbuilt_grid_mesh
from pbrt_b200 import workloads
from pbrt_b200.scene import build_mesh_bvh_host


def _compare(v, i, bins, max_leaf):
    nodes, order = build_mesh_bvh_host(v, i, bins, max_leaf)
    m = oracle.MeshBVH(v, i, np.float32, bins=bins, max_leaf=max_leaf)
    boxes, lf, cnt = m.nodes()
    n = boxes.shape[0]
    assert nodes.shape[0] == n + 1, "GPU numbering adds one padding slot"
    g = np.concatenate([[0], np.arange(2, n + 1)])  # ref index k -> GPU index
    gn = nodes[g]
    assert np.array_equal(gn["bmin"], boxes[:, :3])
    assert np.array_equal(gn["bmax"], boxes[:, 3:])
    assert np.array_equal(gn["count"].astype(np.uint64), cnt)
    leaf = cnt > 0
    assert np.array_equal(gn["left_first"][leaf].astype(np.uint64), lf[leaf])
    assert np.array_equal(gn["left_first"][~leaf].astype(np.uint64), lf[~leaf] + 1)
    assert np.all(gn["left_first"][~leaf] % 2 == 0), "sibling pairs start at even indices"
    assert np.array_equal(order, m.tri_idx())


@pytest.mark.parametrize("bins,max_leaf", [(8, 1), (16, 4), (12, 2)])
def test_builder_matches_oracle_on_icosphere(bins, max_leaf):
    v, f = workloads.displaced_icosphere(4, seed=3)
    _compare(v, f, bins, max_leaf)


def test_builder_matches_oracle_on_reference_mesh(golden_meshes):
    v = golden_meshes["bun_zipper_res4_vertices"].astype(np.float32)
    _compare(v, golden_meshes["bun_zipper_res4_indices"], 8, 1)
    _compare(v, golden_meshes["bun_zipper_res4_indices"], 16, 4)


def test_builder_matches_oracle_on_grid():
    v, i = unbuilt_grid_mesh(4)
    _compare(v.astype(np.float32), i, 8, 1)


def test_builder_rejects_bad_meshes():
    from pbrt_b200 import PbrtError
    v, i = unbuilt_grid_mesh(2)
    with pytest.raises(PbrtError):
        build_mesh_bvh_host(v, np.zeros((0, 3), np.uint32))
    bad = i.copy()
    bad[0, 0] = 10_000
    with pytest.raises(PbrtError):
        build_mesh_bvh_host(v, bad)
    vn = v.copy()
    vn[0, 0] = np.nan
    with pytest.raises(PbrtError):
        build_mesh_bvh_host(vn, i)
