"""The path tracer ending paths into the learned radiance cache, on the GPU.

- With all-zero weights the cache answers 0, so the cached render must equal, bit for bit,
  the plain render cut at the same hit (same random streams, same arithmetic).
- With trained weights, the GPU's cached render matches the oracle's restatement (the same
  path prefix, the network in its BF16-emulating mode) within the tolerance of the other
  image parity tests.
- What the trained network gains: against a converged plain render, the cached image at a
  few samples per pixel is much closer than the same paths cut at the cache's hit without
  the network, and than plain path tracing at the same sample count.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from pbrt_b200 import PbrtError, Scene
from pbrt_b200.cache import PARAMS, RadianceCache
from pbrt_b200.workloads import cornell_box, radiance_cache_scene

pytestmark = pytest.mark.gpu

TERM = 2  # paths end into the cache at hit TERM + 1


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref * ref + 1e-2)))


def _box_bounds(desc):
    v = np.concatenate([np.asarray(m["vertices"], np.float32).reshape(-1, 3) for m in desc["meshes"]])
    return v.min(0), v.max(0)


@pytest.fixture(scope="module")
def cornell():
    desc, cam = cornell_box(48, 48)
    return desc, cam, Scene.from_description(desc).commit(bvh_bins=8, bvh_max_leaf=1)


@pytest.fixture(scope="module")
def trained(cornell):
    desc, cam, scene = cornell
    lo, hi = _box_bounds(desc)
    cache = RadianceCache(lo, hi, seed=3, terminate_bounce=TERM, train_samples=1 << 14, train_steps=4)
    scene.render_cached(cache, cam, spp=0, max_depth=16, seed=11, train_rounds=40)
    return cache


def test_zero_network_equals_cut_paths(cornell):
    desc, cam, scene = cornell
    lo, hi = _box_bounds(desc)
    cache = RadianceCache(lo, hi, terminate_bounce=TERM)
    cache.set_weights(np.zeros(PARAMS, np.float32))
    got = scene.render_cached(cache, cam, spp=8, max_depth=16, seed=5, train_rounds=0)
    want = scene.render(cam, spp=8, max_depth=TERM + 1, seed=5)
    np.testing.assert_array_equal(got, want)


def test_training_only_call(cornell):
    desc, cam, scene = cornell
    lo, hi = _box_bounds(desc)
    cache = RadianceCache(lo, hi, terminate_bounce=TERM, train_samples=4096)
    w0 = cache.weights()
    assert scene.render_cached(cache, cam, spp=0, max_depth=16, train_rounds=2) is None
    assert not np.array_equal(cache.weights(), w0)


def test_cached_render_matches_oracle(cornell, trained):
    desc, cam, scene = cornell
    lo, hi = _box_bounds(desc)
    w = trained.weights()
    got = scene.render_cached(trained, cam, spp=32, max_depth=16, seed=7, train_rounds=0)
    ref = oracle.Scene(desc, np.float32).render_cached(cam, 32, 16, w, np.concatenate([lo, hi]), TERM, seed=7)
    assert np.all(np.isfinite(got))
    err = relmse(got, ref)
    assert err < 5e-3, err


def test_trained_cache_gain(cornell, trained):
    desc, cam, scene = cornell
    judge = scene.render(cam, spp=4096, max_depth=16, seed=99)
    out = {}
    for spp in (8, 256):
        cached = scene.render_cached(trained, cam, spp=spp, max_depth=16, seed=3, train_rounds=0)
        cut = scene.render(cam, spp=spp, max_depth=TERM + 1, seed=3)
        plain = scene.render(cam, spp=spp, max_depth=16, seed=3)
        out[spp] = {k: (relmse(v, judge), float(v.mean() / judge.mean() - 1.0))
                    for k, v in (("cached", cached), ("cut", cut), ("plain", plain))}
        print(spp, "spp: relMSE / energy bias", out[spp])
    # energy: pixel noise averages out over the image, what remains is bias
    b = out[256]
    assert abs(b["cached"][1]) < 0.25 * abs(b["cut"][1])
    # the cut paths' missing light dominates their error; the network brings it back
    assert b["cached"][0] < 0.5 * b["cut"][0]
    assert out[8]["cached"][0] < out[8]["plain"][0]


def test_rejects_naive_integrator_and_foreign_cache(cornell):
    desc, cam, scene = cornell
    lo, hi = _box_bounds(desc)
    cache = RadianceCache(lo, hi)
    with pytest.raises(PbrtError):
        p_film = np.zeros((48, 48, 3))
        import ctypes as C
        from pbrt_b200 import _capi
        from pbrt_b200.scene import camera_desc
        p = _capi.RenderParams()
        p.camera = camera_desc(cam)
        p.spp, p.max_depth, p.integrator = 1, 4, 1
        scene.ctx.check(scene.ctx.lib.pbrt_render_cached(scene.h, cache.h, C.byref(p), 0, p_film.ctypes.data),
                        "pbrt_render_cached")


def test_knot_scene_face_materials():
    """The cache workload's mesh carries per-face materials; a small knot renders and the
    glossy/diffuse faces differ in the image."""
    desc, cam = radiance_cache_scene(64, 36, segments=400, sides=12)
    scene = Scene.from_description(desc).commit(bvh_bins=16, bvh_max_leaf=4)
    img = scene.render(cam, spp=16, max_depth=8, seed=1)
    ref = oracle.Scene(desc, np.float32).render(cam, 16, 8, seed=1)
    assert np.all(np.isfinite(img))
    assert relmse(img, ref) < 5e-3


def test_training_beside_the_frame(cornell):
    """A call that trains and renders runs its rounds beside the frame: the frame reads the
    weights the call started with (so its film is that of a render-only call with those
    weights), and the call leaves the weights its rounds trained. The rounds' training
    vertices are recorded in whatever order the GPU schedules them, so their weights are not
    compared bit for bit with a separate training call."""
    desc, cam, scene = cornell
    lo, hi = _box_bounds(desc)
    kw = dict(terminate_bounce=TERM, train_samples=4096, train_steps=4, seed=7)
    a, b = RadianceCache(lo, hi, **kw), RadianceCache(lo, hi, **kw)
    for frame in range(3):
        w0 = a.weights()
        b.set_weights(w0)
        got = scene.render_cached(a, cam, spp=4, max_depth=16, seed=20 + frame, train_rounds=1)
        want = scene.render_cached(b, cam, spp=4, max_depth=16, seed=20 + frame, train_rounds=0)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-15)
        w1 = a.weights()
        assert np.isfinite(w1).all() and not np.array_equal(w1, w0)
