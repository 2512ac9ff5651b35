"""The synthetic workload generators: sizes, determinism, winding and ray normalisation."""
import numpy as np

import oracle
from pbrt_b200 import workloads as W


def test_icosphere_counts_and_closed_surface():
    for level in range(0, 5):
        v, f = W.icosphere(level)
        assert f.shape[0] == 20 * 4 ** level
        assert v.shape[0] == 10 * 4 ** level + 2
        e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
        _, counts = np.unique(e, axis=0, return_counts=True)
        assert np.all(counts == 2), "every edge is shared by exactly two faces"


def test_level7_is_the_raycast_mesh_size():
    v, f = W.displaced_icosphere(7)
    assert f.shape == (327_680, 3) and v.dtype == np.float32
    r = np.linalg.norm(v.astype(np.float64), axis=1)
    assert r.min() >= 0.9 - 1e-6 and r.max() <= 1.1 + 1e-6, "radial displacement of amplitude 0.1·r"


def test_reference_normal_points_outward():
    v, f = W.displaced_icosphere(3)
    v = v.astype(np.float64)
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    n = np.cross(p2 - p1, p1 - p0)
    assert np.all((n * (p0 + p1 + p2)).sum(1) > 0)


def test_rays_are_deterministic_and_normalised_like_ray_new():
    v, f = W.displaced_icosphere(2)
    a = W.incoherent_rays(1000, v.min(0), v.max(0), seed=5)
    b = W.incoherent_rays(1000, v.min(0), v.max(0), seed=5)
    assert np.array_equal(a, b)
    for k in range(0, 1000, 97):
        _, d = oracle.make_ray(a[0:3, k], a[3:6, k], np.float32)
        raw = a[3:6, k]
        # the generator applies the same FP32 normalisation to the raw direction
        assert np.allclose(d, raw, rtol=0, atol=2e-7)
    assert np.all(a[6] == np.float32(1e-4)) and np.all(a[7] == np.float32(1e30))


def test_batch_scenes_are_seeded_and_in_range():
    from pbrt_b200 import workloads as W
    a = W.batch_scenes(n=6, levels=(3, 5), spp=(4, 64))
    b = W.batch_scenes(n=6, levels=(3, 5), spp=(4, 64))
    assert [(d["level"], s) for d, _, s in a] == [(d["level"], s) for d, _, s in b]
    for d, cam, s in a:
        assert 3 <= d["level"] <= 5 and 4 <= s <= 64
        assert cam["width"] == 512 and cam["height"] == 512
        assert d["meshes"][-1]["indices"].shape[0] == 20 * 4 ** d["level"]
        v = d["meshes"][-1]["vertices"]
        assert v.min() > -0.5 and v.max() < 0.5  # inside the box
