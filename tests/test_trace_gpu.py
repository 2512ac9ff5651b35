"""GPU parity of the ray-cast path against the FP32 oracle (bit-exact ids and t).

The oracle restates the reference's traversal (src/shapes/triangle_mesh/bvh.rs:381-526)
and Möller–Trumbore (triangle_mesh.rs:183-217) in FP32 without FMA; the CUDA kernels walk
the same tree in the same order with the same roundings, so the nearest triangle, its t,
the occlusion answer and even the work counters must be identical.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import grid_ray_set, unbuilt_grid_mesh
import pbrt_b200 as pb
from pbrt_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _scene(v, f, bins=8, max_leaf=1):
    s = pb.Scene()
    s.add_object(pb.Simple(pb.TriangleMesh(v, f)))
    return s.commit(bvh_bins=bins, bvh_max_leaf=max_leaf)


def _assert_parity(scene, m, rays, counters=True):
    prim, t, st = scene.intersect_instrumented(rays) if counters else (*scene.intersect(rays), None)
    oprim, ot, ost = m.trace(rays)
    assert np.array_equal(prim, oprim), f"{(prim != oprim).sum()} ids differ"
    hit = oprim != oracle.MISS
    assert np.array_equal(t[hit], ot[hit]), "t must be bit-identical on hits"
    assert np.all(np.isinf(t[~hit]))
    if counters:
        assert st == ost, (st, ost)
    occ = scene.intersect_p(rays)
    assert np.array_equal(occ, m.occluded(rays))
    return hit


def test_grid_fixture_parity():
    v, i = unbuilt_grid_mesh(3)
    v = v.astype(np.float32)
    rays = grid_ray_set(v, i, oracle.make_ray, np.float32)
    s = _scene(v, i)
    m = oracle.MeshBVH(v, i, np.float32)
    hit = _assert_parity(s, m, rays)
    assert hit.sum() > 20
    # far swept across the nearest hit (bvh.rs:937-975)
    prim, t = s.intersect(rays)
    h = prim != pb.PBRT_MISS
    for factor in (0.5, 0.99, 0.999999, 1.0, 1.000001):
        r = rays[:, h].copy()
        r[7] = (t[h] * factor).astype(np.float32)
        _assert_parity(s, m, r)


@pytest.mark.parametrize("bins,max_leaf", [(8, 1), (16, 4)])
def test_reference_mesh_orbit_rays(golden_meshes, bins, max_leaf):
    v = golden_meshes["bun_zipper_res4_vertices"].astype(np.float32)
    i = golden_meshes["bun_zipper_res4_indices"]
    m = oracle.MeshBVH(v, i, np.float32, bins=bins, max_leaf=max_leaf)
    rays = m.orbit_rays()
    hit = _assert_parity(_scene(v, i, bins, max_leaf), m, rays)
    assert hit.sum() > 40_000


@pytest.mark.parametrize("bins,max_leaf", [(16, 4), (8, 1)])
def test_displaced_icosphere_incoherent(bins, max_leaf):
    v, f = W.displaced_icosphere(6, seed=11)
    rays = W.incoherent_rays(1 << 20, v.min(0), v.max(0), seed=12)
    # plus rays aimed into the mesh so most of them traverse deep
    rng = np.random.default_rng(13)
    aim = rays[:, : 1 << 18].copy()
    tgt = (rng.random((3, aim.shape[1])) - 0.5).astype(np.float32)
    aim[3:6] = W.normalize_f32(tgt - aim[0:3])
    rays = np.concatenate([rays, aim], axis=1)
    m = oracle.MeshBVH(v, f, np.float32, bins=bins, max_leaf=max_leaf)
    hit = _assert_parity(_scene(v, f, bins, max_leaf), m, rays)
    assert hit.sum() > 100_000


def test_headline_mesh_level7_incoherent():
    """The ray-cast workload's own mesh and tree (icosphere level 7, 327,680 triangles, 16
    bins, leaves of at most 4) with 4M incoherent rays of its distribution plus 1M rays aimed
    into the mesh: ids, t, occlusion and work counters identical to the FP32 oracle's."""
    v, f = W.displaced_icosphere(7, seed=1)
    assert f.shape[0] == 327_680
    rays = W.incoherent_rays(1 << 22, v.min(0), v.max(0), seed=71)
    rng = np.random.default_rng(72)
    aim = rays[:, : 1 << 20].copy()
    tgt = (rng.random((3, aim.shape[1])) - 0.5).astype(np.float32)
    aim[3:6] = W.normalize_f32(tgt - aim[0:3])
    rays = np.concatenate([rays, aim], axis=1)
    m = oracle.MeshBVH(v, f, np.float32, bins=16, max_leaf=4)
    s = _scene(v, f, 16, 4)
    hit = _assert_parity(s, m, rays)
    assert hit.sum() > 1_000_000
    # the timed path (persistent traversal over device buffers) gives the same answers
    dp, dt = s.intersect(torch.from_numpy(rays).cuda())
    oprim, ot, _ = m.trace(rays)
    assert np.array_equal(dp.cpu().numpy().view(np.uint32), oprim)
    assert np.array_equal(dt.cpu().numpy()[hit], ot[hit])


def test_host_and_device_buffers_agree_across_chunks():
    v, f = W.displaced_icosphere(5, seed=21)
    n = (1 << 21) * 2 + 12345  # five 1M-ray pipelined chunks over three staging slots, the last one partial
    rays = W.incoherent_rays(n, v.min(0), v.max(0), seed=22)
    s = _scene(v, f, 16, 4)
    hp, ht = s.intersect(rays)
    dr = torch.from_numpy(rays).cuda()
    dp, dt = s.intersect(dr)
    assert np.array_equal(hp, dp.cpu().numpy().view(np.uint32))
    assert np.array_equal(ht, dt.cpu().numpy())
    occ_h = s.intersect_p(rays)
    occ_d = s.intersect_p(dr).cpu().numpy()
    assert np.array_equal(occ_h, occ_d)
    m = oracle.MeshBVH(v, f, np.float32, bins=16, max_leaf=4)
    op, ot, _ = m.trace(rays)
    assert np.array_equal(hp, op)


def test_edge_cases():
    v, f = W.displaced_icosphere(3, seed=31)
    s = _scene(v, f)
    m = oracle.MeshBVH(v, f, np.float32)
    rays = []
    # axis-aligned directions (zero components take the parallel-slab branch)
    for d in [(1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (0, -1, 0), (0, 0, -1)]:
        for o in [(-3, 0.1, 0.05), (0.1, -3, 0.05), (0.05, 0.1, -3), (3, 0.1, 0.05), (0, 0, 0), (2, 2, 2)]:
            rays.append((o, d, 1e-4, 1e30))
    # starting inside the mesh, empty interval, interval ending before the surface, negative far
    rays += [((0, 0, 0), (0.3, 0.4, 0.5), 1e-4, 1e30), ((0, 0, 0), (0.3, 0.4, 0.5), 5.0, 1.0),
             ((0, 0, 0), (0.3, 0.4, 0.5), 1e-4, 0.5), ((-3, 0, 0), (1, 0, 0), 1e-4, -1.0),
             ((0, 0, -5), (0, 0, 1), 0.0, 1e30)]
    arr = np.zeros((8, len(rays)), np.float32)
    for k, (o, d, a, b) in enumerate(rays):
        ro, rd = oracle.make_ray(o, d, np.float32)
        arr[0:3, k], arr[3:6, k], arr[6, k], arr[7, k] = ro, rd, a, b
    _assert_parity(s, m, arr)
    # n = 0 is a no-op
    p, t = s.intersect(np.zeros((8, 0), np.float32))
    assert p.size == 0 and t.size == 0


def test_unsupported_and_invalid_inputs_raise():
    with pytest.raises(pb.PbrtError):
        pb.Scene().add_object(pb.Simple(pb.TriangleMesh(np.zeros((3, 3), np.float32), np.zeros((0, 3))))).commit()
    v, f = W.icosphere(1)
    bad = f.copy()
    bad[0, 0] = 9999
    with pytest.raises(pb.PbrtError):
        pb.Scene().add_object(pb.Simple(pb.TriangleMesh(v, bad))).commit()


_DENSE_SCRIPT = """
import sys, numpy as np, torch
sys.path.insert(0, {root!r})
import pbrt_b200 as pb
from pbrt_b200 import workloads as W
v, f = W.displaced_icosphere(6, seed=41)
s = pb.Scene()
s.add_object(pb.Simple(pb.TriangleMesh(v, f)))
s = s.commit(bvh_bins=16, bvh_max_leaf=4)
n = (1 << 21) + 1028  # device buffers: 2,050 chunks of 1,024 rays, the last one of 4
rays = W.incoherent_rays(n, v.min(0), v.max(0), seed=42)
rng = np.random.default_rng(43)
aim = rays[:, : 1 << 18]
aim[3:6] = W.normalize_f32((rng.random((3, aim.shape[1])) - 0.5).astype(np.float32) - aim[0:3])
dp, dt = s.intersect(torch.from_numpy(rays).cuda())
hp, ht = s.intersect(rays[:, : (1 << 20) + 3 * 1024 + 8])  # host buffers: two pipelined chunks, the second ragged
np.savez({out!r}, rays=rays, dp=dp.cpu().numpy().view(np.uint32), dt=dt.cpu().numpy(), hp=hp, ht=ht)
"""


_FORMS = {
    "default": {},
    "dense results": {"PBRT_TRACE_DENSE": "1"},
    "cull by direct loads": {"PBRT_CULL_BULK": "0"},
    "cull by direct loads, 256-thread blocks": {"PBRT_CULL_BULK": "0", "PBRT_CULL_THREADS": "256"},
    "drained-queue schedule as the bulk's": {"PBRT_TRACE_SCHEDULE": "8,8,8"},
    "drained-queue schedule 1, 2": {"PBRT_TRACE_SCHEDULE": "8,8,8,1,2"},
}


@pytest.mark.parametrize("form", list(_FORMS))
def test_two_stage_forms_match_oracle(tmp_path, form):
    """Every form of the two-stage pass gives the oracle's ids and t, on device buffers with a
    partial last chunk and on host buffers: the cull's miss answers plus scattered hit stores;
    the survivor bitmask, results by queue slot and the ray-order pass; the cull's rays
    staged by bulk copies (the default) or read directly, in 128- or 256-thread blocks; other schedules once the queue is
    drained. The switches are read once per process: a child per form."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = str(tmp_path / "form.npz")
    env = {k: v for k, v in os.environ.items() if not k.startswith(("PBRT_TRACE_", "PBRT_CULL_"))}
    env.update(_FORMS[form])
    subprocess.run([sys.executable, "-c", _DENSE_SCRIPT.format(root=root, out=out)], env=env, check=True,
                   timeout=600)
    z = np.load(out)
    rays = z["rays"]
    v, f = W.displaced_icosphere(6, seed=41)
    m = oracle.MeshBVH(v, f, np.float32, bins=16, max_leaf=4)
    op, ot, _ = m.trace(rays)
    hit = op != oracle.MISS
    assert hit.sum() > 200_000
    assert np.array_equal(z["dp"], op), f"{int((z['dp'] != op).sum())} ids differ"
    assert np.array_equal(z["dt"][hit], ot[hit]) and np.all(np.isinf(z["dt"][~hit]))
    k = z["hp"].shape[0]
    assert np.array_equal(z["hp"], op[:k]) and np.array_equal(z["ht"][hit[:k]], ot[:k][hit[:k]])
    assert np.all(np.isinf(z["ht"][~hit[:k]]))
