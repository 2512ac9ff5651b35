"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on a CPU-only host."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference checkout, for the few tests that read its larger meshes; they skip without it.
REFERENCE_ROOT = os.environ.get("PBRT_REFERENCE_ROOT")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built libpbrt_b200.so")


@pytest.fixture(scope="session")
def golden_meshes():
    d = np.load(os.path.join(GOLDEN, "meshes.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def published():
    with open(os.path.join(GOLDEN, "bvh_stats_published.json")) as f:
        return json.load(f)["meshes"]


@pytest.fixture(scope="session")
def published_scenes():
    with open(os.path.join(GOLDEN, "bvh_stats_published.json")) as f:
        return json.load(f)["scenes"]


def stage_text(name: str) -> str:
    """A scene file of the reference's test_files/ (copied under tests/golden/stage/)."""
    with open(os.path.join(GOLDEN, "stage", name)) as f:
        return f.read()


def fixture_mesh_loader(meshes: dict, reference_dir=None):
    """load_ply_mesh(file, reverse) for scene files: the meshes of meshes.npz, else the
    reference checkout's test_files/ when `reference_dir` is given. Faces reversed as
    src/loader/mesh_loader.rs:60-70 does."""
    import oracle

    def load(name: str, reverse: bool):
        key = os.path.basename(name).replace(".ply", "")
        if key + "_vertices" in meshes:
            v, i = meshes[key + "_vertices"], meshes[key + "_indices"]
            return v, (i[:, ::-1] if reverse else i)
        if reference_dir is None:
            pytest.skip(f"{name} is not among the fixtures")
        return oracle.read_ply(os.path.join(reference_dir, os.path.basename(name)), reverse)

    return load


def write_ply(path, v, i):
    """An ASCII PLY whose float text reads back to exactly these float32 values."""
    v = np.asarray(v, np.float32).reshape(-1, 3)
    i = np.asarray(i, np.uint32).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f"ply\nformat ascii 1.0\ncomment written by the tests\nelement vertex {len(v)}\n"
                "property float x\nproperty float y\nproperty float z\n"
                f"element face {len(i)}\nproperty list uchar int vertex_indices\nend_header\n")
        for p in v:
            f.write(" ".join(repr(float(x)) for x in p) + "\n")
        for t in i:
            f.write("3 " + " ".join(str(int(x)) for x in t) + "\n")


@pytest.fixture(scope="session")
def mesh_dir(tmp_path_factory, golden_meshes):
    """A directory with test_files/cube.ply and test_files/bun_zipper_res4.ply written from the
    fixtures, for scene files that name them."""
    d = tmp_path_factory.mktemp("stage")
    os.makedirs(d / "test_files")
    for key in ("cube", "bun_zipper_res4"):
        write_ply(d / "test_files" / f"{key}.ply", golden_meshes[key + "_vertices"], golden_meshes[key + "_indices"])
    return str(d)


@pytest.fixture(scope="session")
def reference_test_files():
    if not REFERENCE_ROOT:
        pytest.skip("PBRT_REFERENCE_ROOT (the reference checkout) is not set")
    p = os.path.join(REFERENCE_ROOT, "test_files")
    if not os.path.isdir(p):
        pytest.skip(f"{p} does not exist")
    return p


def unbuilt_grid_mesh(side: int):
    """side³ small slanted triangles, one per grid cell (src/shapes/triangle_mesh/bvh.rs:746-766)."""
    verts, idx = [], []
    for ix in range(side):
        for iy in range(side):
            for iz in range(side):
                x, y, z = float(ix), float(iy), float(iz)
                first = len(verts)
                verts += [[x, y, z], [x + 0.4, y + 0.1, z], [x + 0.1, y + 0.4, z + 0.3]]
                idx.append([first, first + 1, first + 2])
    return np.array(verts, np.float64), np.array(idx, np.uint32)


def grid_ray_set(vertices, indices, make_ray, dtype):
    """Rays aimed at every centroid from three origins plus axis pencils
    (src/shapes/triangle_mesh/bvh.rs:828-854), normalised with the oracle's Ray::new."""
    origins = [(-6.0, -7.0, -8.0), (9.0, -6.0, 7.0), (-5.0, 8.0, -9.0)]
    rays = []
    dt = np.dtype(dtype)
    v = vertices.astype(dt)
    for tri in indices:
        # tri_centroid: ((v0 + v1) + v2) * (1/3) in the working precision (bvh.rs:578-584)
        c = ((v[tri[0]] + v[tri[1]]) + v[tri[2]]) * (dt.type(1) / dt.type(3))
        for o in origins:
            oo = np.array(o, dt)
            rays.append(make_ray(oo, c - oo, dt))
    for a in range(7):
        for b in range(7):
            u, w = -1.0 + a * 0.7, -1.0 + b * 0.7
            rays.append(make_ray((-5.0, u, w), (1.0, 0.0, 0.0), dt))
            rays.append(make_ray((u, -5.0, w), (0.0, 1.0, 0.0), dt))
            rays.append(make_ray((u, w, -5.0), (0.0, 0.0, 1.0), dt))
    out = np.zeros((8, len(rays)), dt)
    for k, (o, d) in enumerate(rays):
        out[0:3, k] = o
        out[3:6, k] = d
    out[6] = dt.type(0.0001)
    out[7] = dt.type(1000.0)
    return out
