"""Per-face materials in the oracle restatement (CPU)."""
from __future__ import annotations

import numpy as np

import oracle
from pbrt_b200.workloads import cornell_box, radiance_cache_scene, torus_knot


def test_uniform_face_materials_equal_object_material():
    desc, cam = cornell_box(16, 16)
    plain = oracle.Scene(desc, np.float32).render(cam, 4, 6, seed=2, threads=4)
    # the red wall's mesh names the red material per face while its object names grey
    d2 = {**desc, "meshes": [dict(m) for m in desc["meshes"]], "objects": [dict(o) for o in desc["objects"]]}
    d2["meshes"][1]["face_materials"] = np.full(d2["meshes"][1]["indices"].shape[0], 1, np.uint32)
    d2["objects"][1]["material"] = 0
    faced = oracle.Scene(d2, np.float32).render(cam, 4, 6, seed=2, threads=4)
    np.testing.assert_array_equal(plain, faced)


def test_torus_knot_counts_and_winding():
    v, f = torus_knot(segments=10627, sides=41)
    assert f.shape == (871_414, 3) and v.shape == (435_707, 3)
    assert int(f.max()) < v.shape[0]
    desc, _ = radiance_cache_scene(32, 18, segments=300, sides=10)
    knot = desc["meshes"][-1]
    assert knot["face_materials"].shape[0] == knot["indices"].shape[0]
    kinds = {desc["materials"][m]["kind"] for m in np.unique(knot["face_materials"])}
    assert kinds == {0, 1}  # diffuse and glossy faces


def test_cached_oracle_with_zero_network_cuts_paths():
    desc, cam = cornell_box(16, 16)
    s = oracle.Scene(desc, np.float32)
    w = np.zeros(oracle.MLP_PARAMS, np.float32)
    b = np.array([-0.5, -0.5, -0.5, 0.5, 0.5, 0.5], np.float32)
    cached = s.render_cached(cam, 4, 16, w, b, terminate_bounce=2, seed=3, threads=4)
    cut = s.render(cam, 4, 3, seed=3, threads=4)
    np.testing.assert_array_equal(cached, cut)
