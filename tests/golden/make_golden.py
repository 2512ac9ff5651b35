"""Generates the golden fixtures under tests/golden/ from the reference checkout.

Run from the repository root, in a container where the reference is mounted:

    python tests/golden/make_golden.py /path/to/nmichel-pbrt

Writes:
  meshes.npz — the two smallest PLY meshes of the reference's test_files/ (cube.ply,
      bun_zipper_res4.ply) parsed with the reference's PLY semantics (f32 text widened to
      f64, src/loader/ply/ply_loader.rs:137 and :40), so GPU tests can use real reference
      geometry on a machine without the reference.
  bvh_stats_published.json — the mesh-mode figures the reference publishes for its own
      traversal benchmark (docs/mesures_bvh.md:706-713, produced by
      src/bin/bvh_stats.rs:345-401): hit counts (exact), box and triangle tests per ray
      (two decimals), node and leaf counts of the tree.
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


def main(ref_root: str):
    out = {}
    for name in ("cube.ply", "bun_zipper_res4.ply"):
        v, i = oracle.read_ply(os.path.join(ref_root, "test_files", name))
        key = name.replace(".ply", "")
        out[key + "_vertices"] = v
        out[key + "_indices"] = i
    np.savez_compressed(os.path.join(HERE, "meshes.npz"), **out)
    with open(os.path.join(HERE, "bvh_stats_published.json"), "w") as f:
        json.dump({"source": "docs/mesures_bvh.md:706-713 (Apple M2 Pro, 1 thread, f64, 6 orbit views x 200x200 "
                             "pixel-centre rays, near 1e-4, far 1000)", "meshes": PUBLISHED}, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
