"""Generates the golden fixtures under tests/golden/ from the reference checkout.

Run from the repository root, in a container where the reference is mounted:

    python tests/golden/make_golden.py /path/to/nmichel-pbrt

(or with the checkout's location in PBRT_REFERENCE_ROOT and no argument).

Writes:
  meshes.npz — the three smallest PLY meshes of the reference's test_files/ (cube.ply,
      bun_zipper_res4.ply, dragon_vrip_res4.ply) parsed with the reference's PLY semantics
      (f32 text widened to f64, src/loader/ply/ply_loader.rs:137 and :40), so the oracle's
      known-answer tests and the GPU tests use real reference geometry on a machine without
      the reference.
  bvh_stats_published.json — the mesh-mode figures the reference publishes for its own
      traversal benchmark (docs/mesures_bvh.md:706-713, produced by
      src/bin/bvh_stats.rs:345-401): hit counts (exact), box and triangle tests per ray
      (two decimals), node and leaf counts of the tree; and the scene-mode figures
      (docs/mesures_bvh.md:729-738, src/bin/bvh_stats.rs:220-286): per scene file and ray set
      (primary, shadow), nodes / boxes / objects per ray and the exact hit ("touches") count.
  stage/*.stage — verbatim copies of the reference's scene files that need no mesh beyond
      meshes.npz (test_files/*.stage), the inputs of the scene-mode figures and of the
      loader tests. bunny_mesh.stage is copied too; its bunny.ply (2.9 MB) is not, so the
      tests that need it read the reference checkout when one is mounted.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# docs/mesures_bvh.md:706-713 — mesh, tris, nodes (leaves), box/ray, tri/ray, hits.
PUBLISHED = {
    "cube.ply": dict(triangles=12, nodes=11, leaves=6, box_per_ray=5.83, tri_per_ray=1.19, hits=116004),
    "bun_zipper_res4.ply": dict(triangles=948, nodes=1811, leaves=906, box_per_ray=10.04, tri_per_ray=0.77,
                                hits=47693),
    "dragon_vrip_res4.ply": dict(triangles=11102, nodes=21137, leaves=10569, box_per_ray=12.01, tri_per_ray=0.63,
                                 hits=42797),
    "dragon_vrip_res3.ply": dict(triangles=47794, nodes=92929, leaves=46465, box_per_ray=13.75, tri_per_ray=0.60,
                                 hits=43451),
    "bunny.ply": dict(triangles=69451, nodes=138881, leaves=69441, box_per_ray=14.19, tri_per_ray=0.58,
                      hits=46904),
}


# docs/mesures_bvh.md:715-720 (primitives) and :729-738 — per set: rays, nodes/ray, box/ray,
# object/ray, touches. 200 x 150 pixel-centre primary rays (config defaults: fov 90, near 1e-4,
# far 1000); one shadow ray per primary hit towards (0, 2, 1) on [1e-5, |target - p|].
PUBLISHED_SCENES = {
    "cornell_box_canonical.stage": dict(primitives=8, primary=(1.39, 3.42, 0.18, 5027), shadow=(7.90, 13.00, 1.62, 1043)),
    "bunny_mesh.stage": dict(primitives=4, primary=(3.77, 7.00, 0.77, 16336), shadow=(3.20, 6.97, 0.20, 444)),
    "many_spheres.stage": dict(primitives=445, primary=(7.54, 14.59, 0.75, 16296), shadow=(22.40, 38.67, 2.29, 9991)),
    "many_meshes.stage": dict(primitives=100, primary=(6.62, 13.18, 0.53, 6831), shadow=(9.16, 16.31, 1.01, 2070)),
}
STAGES = ("cornell_box_canonical.stage", "bunny_mesh.stage", "many_spheres.stage", "many_meshes.stage",
          "cornell_box.stage", "cube_mesh.stage", "default.stage", "csg_union_spheres.stage")


def main(ref_root: str):
    out = {}
    for name in ("cube.ply", "bun_zipper_res4.ply", "dragon_vrip_res4.ply"):
        v, i = oracle.read_ply(os.path.join(ref_root, "test_files", name))
        key = name.replace(".ply", "")
        out[key + "_vertices"] = v
        out[key + "_indices"] = i
    np.savez_compressed(os.path.join(HERE, "meshes.npz"), **out)
    with open(os.path.join(HERE, "bvh_stats_published.json"), "w") as f:
        json.dump({"source": "docs/mesures_bvh.md:706-713 (Apple M2 Pro, 1 thread, f64, 6 orbit views x 200x200 "
                             "pixel-centre rays, near 1e-4, far 1000)", "meshes": PUBLISHED,
                   "scene_source": "docs/mesures_bvh.md:715-738 (src/bin/bvh_stats.rs scene mode: 200x150 "
                                   "pixel-centre rays, fov 90, near 1e-4, far 1000; shadow rays to (0, 2, 1) "
                                   "from 1e-5); per set (nodes/ray, box/ray, object/ray, touches)",
                   "scenes": PUBLISHED_SCENES}, f, indent=1)
    os.makedirs(os.path.join(HERE, "stage"), exist_ok=True)
    for name in STAGES:
        with open(os.path.join(ref_root, "test_files", name), "rb") as src:
            data = src.read()
        with open(os.path.join(HERE, "stage", name), "wb") as dst:
            dst.write(data)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PBRT_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set PBRT_REFERENCE_ROOT)")
    main(root)
