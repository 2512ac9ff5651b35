"""Batched multi-scene rendering (pbrt_batch): one wavefront over many scenes, replayed as a
CUDA graph. Each scene's paths are the paths pbrt_render traces for it alone (same sample
streams, same kernels), so every film must equal the scene's own render, whatever the wave
size and launch shape."""
from __future__ import annotations

import numpy as np
import pytest

import pbrt_b200 as pb
from pbrt_b200 import PbrtError
from pbrt_b200 import workloads as W
from pbrt_b200.scene import Batch, create_scenes, render_params

pytestmark = pytest.mark.gpu


def _specs():
    d0, c0 = W.cornell_box(32, 24)
    d1, c1 = W.many_spheres(300, width=40, height=30)
    d2, c2 = W.radiance_cache_scene(48, 27, segments=200, sides=10)
    d3, c3 = W.cornell_box(20, 20)
    return [(d0, c0, dict(spp=3, max_depth=6)), (d1, c1, dict(spp=2, max_depth=8, rr_start=3)),
            (d2, c2, dict(spp=2, max_depth=5, pixel_stride=2)), (d3, c3, dict(spp=4, max_depth=4, integrator="naive"))]


@pytest.fixture(scope="module")
def built():
    specs = _specs()
    scenes = create_scenes([d for d, _, _ in specs])
    singles = [s.render(cam, seed=5, **kw) for s, (_, cam, kw) in zip(scenes, specs)]
    params = [render_params(cam, seed=5, **kw) for _, cam, kw in specs]
    return specs, scenes, singles, params


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)


def test_batch_films_equal_single_renders(built):
    specs, scenes, singles, params = built
    b = Batch(scenes, params)
    films, ms = b.render(0, scene_times=True)
    for f, s in zip(films, singles):
        assert f.shape == s.shape
        _close(f, s)
    assert all(t > 0 for t in ms)
    # scenes run cheapest first (pixels x spp x max depth, ties in the given order)
    cost = [cam["width"] * cam["height"] * kw["spp"] * kw["max_depth"] for _, cam, kw in specs]
    order = sorted(range(len(specs)), key=lambda i: (cost[i], i))
    assert order != list(range(len(specs)))  # the fixture exercises a reordering
    assert all(ms[order[i]] <= ms[order[i + 1]] + 1e-3 for i in range(len(order) - 1))
    # replaying the graph gives the same frame
    again = b.render(0)
    for f, s in zip(again, singles):
        _close(f, s)
    b.close()


def test_frames_continue_the_sample_sequence(built):
    specs, scenes, singles, params = built
    b = Batch(scenes, params)
    films = b.render(2)
    for sc, f, (_, cam, kw) in zip(scenes, films, specs):
        ref = sc.render(cam, seed=5, sample_offset=2 * kw["spp"], **kw)
        _close(f, ref)
    b.close()


@pytest.mark.parametrize("tuning", [dict(wave_paths=4096), dict(trace_threads=64, trace_blocks_per_sm=32),
                                    dict(trace_threads=256, trace_blocks_per_sm=4, shade_threads=256,
                                         shade_blocks_per_sm=2)])
def test_results_do_not_depend_on_the_launch_shape(built, tuning):
    specs, scenes, singles, params = built
    ctx = scenes[0].ctx
    ctx.set_tuning(**tuning)
    try:
        b = Batch(scenes, params)
        for f, s in zip(b.render(0), singles):
            _close(f, s)
        b.close()
        # single-scene renders follow the context's tuning too
        _close(scenes[0].render(specs[0][1], seed=5, **specs[0][2]), singles[0])
    finally:
        ctx.set_tuning()


def test_device_films_and_one_shot(built):
    torch = pytest.importorskip("torch")
    specs, scenes, singles, params = built
    b = Batch(scenes, params)
    films = [torch.zeros(sh, dtype=torch.float64, device="cuda") for sh in b.film_shapes()]
    b.render(0, films)
    for f, s in zip(films, singles):
        _close(f.cpu().numpy(), s)
    b.close()
    import ctypes as C
    from pbrt_b200 import _capi
    ctx = scenes[0].ctx
    hs = (C.c_void_p * 2)(scenes[0].h.value, scenes[1].h.value)
    ps = (_capi.RenderParams * 2)(params[0], params[1])
    outs = [np.zeros(s.shape) for s in singles[:2]]
    fp = (C.c_void_p * 2)(outs[0].ctypes.data, outs[1].ctypes.data)
    ctx.check(ctx.lib.pbrt_render_batch(hs, ps, 2, fp), "pbrt_render_batch")
    _close(outs[0], singles[0])
    _close(outs[1], singles[1])


def test_invalid_batches_and_tuning_are_refused(built):
    specs, scenes, singles, params = built
    other = pb.Context(0)
    with pytest.raises(PbrtError):
        Batch(scenes[:2], params[:2], ctx=other)
    with pytest.raises(PbrtError):
        other.set_tuning(trace_threads=48)
    with pytest.raises(PbrtError):
        other.set_tuning(wave_paths=10)
    bad = render_params(specs[0][1], spp=0, max_depth=4)
    with pytest.raises(PbrtError):
        Batch(scenes[:1], [bad])
    other.close()


def test_batch_render_stats(built):
    specs, scenes, singles, params = built
    b = Batch(scenes, params)
    b.render(0)
    st = scenes[0].ctx.render_stats()
    want = sum(int(np.prod(sh[:2])) * p.spp for sh, p in zip(b.film_shapes(), params))
    assert st["paths"] == want
    b.close()


def test_batch_with_deferred_meshes_equals_single_renders():
    """Scenes whose large mesh is answered by the deferred passes, mixed with plain ones, in
    waves small enough that some span several scenes (per-path scene lookup) and some hold
    one scene (the single-scene kernels): every film equals the scene's own render."""
    specs = [(d, c, dict(spp=s, max_depth=6)) for d, c, s in
             W.batch_scenes(3, seed=13, width=40, height=30, levels=(5, 6), spp=(2, 4))]
    d0, c0 = W.cornell_box(24, 20)
    specs.insert(1, (d0, c0, dict(spp=3, max_depth=6)))
    scenes = create_scenes([d for d, _, _ in specs])
    singles = [s.render(cam, seed=5, **kw) for s, (_, cam, kw) in zip(scenes, specs)]
    params = [render_params(cam, seed=5, **kw) for _, cam, kw in specs]
    ctx = scenes[0].ctx
    ctx.set_tuning(wave_paths=3000)
    try:
        for branches in (1, 3):  # the deferred passes' fetch counters belong to each branch
            ctx.set_batch_branches(branches)
            b = Batch(scenes, params)
            for f, s in zip(b.render(0), singles):
                _close(f, s)
            b.close()
    finally:
        ctx.set_batch_branches(2)  # the default
        ctx.set_tuning()
    # the persistent launch answers the large meshes inside each path's query
    ctx.set_batch_kernel("persistent")
    try:
        b = Batch(scenes, params)
        for f, s in zip(b.render(0), singles):
            _close(f, s)
        b.close()
    finally:
        ctx.set_batch_kernel("wavefront")


@pytest.mark.parametrize("branches", [2, 3, 8])
@pytest.mark.parametrize("wave_paths", [0, 3000])
def test_concurrent_branches_equal_single_renders(built, branches, wave_paths):
    """A frame whose waves run on several streams inside the graph (each branch its own wave
    buffers): every film equals the scene's own render, in later frames too, whether each
    scene is a group of its own waves (small waves) or scenes share waves; the work counters
    equal the single-branch frame's; every scene reports a completion time."""
    specs, scenes, singles, params = built
    ctx = scenes[0].ctx
    ctx.set_tuning(wave_paths=wave_paths)
    try:
        ctx.set_batch_branches(1)
        one = Batch(scenes, params)
        one.render(0)
        one_stats = ctx.render_stats()
        one.close()
        ctx.set_batch_branches(branches)
        b = Batch(scenes, params)
        films, ms = b.render(0, scene_times=True)
        for f, s in zip(films, singles):
            _close(f, s)
        assert ctx.render_stats() == one_stats
        assert all(np.isfinite(t) and t > 0 for t in ms)
        for sc, f, (_, cam, kw) in zip(scenes, b.render(2), specs):
            _close(f, sc.render(cam, seed=5, sample_offset=2 * kw["spp"], **kw))
        b.close()
    finally:
        ctx.set_batch_branches(2)  # the default
        ctx.set_tuning()
    for bad in (0, 9):
        with pytest.raises(PbrtError):
            ctx.set_batch_branches(bad)


def test_persistent_batch_equals_single_renders(built):
    """One persistent launch over the batch (each lane runs a path to its end with the
    wavefront's shading code): every film equals the scene's own render, in later frames too;
    the scenes complete cheapest first on the GPU clock; the work counters equal the
    wavefront batch's."""
    specs, scenes, singles, params = built
    ctx = scenes[0].ctx
    wave = Batch(scenes, params)
    wave.render(0)
    wave_stats = ctx.render_stats()
    wave.close()
    ctx.set_batch_kernel("persistent")
    try:
        b = Batch(scenes, params)
        films, ms = b.render(0, scene_times=True)
        for f, s in zip(films, singles):
            _close(f, s)
        assert ctx.render_stats() == wave_stats
        # (paths are taken in table order, but a scene's last path may still finish after a
        # later scene's, so the times are not ordered)
        assert all(np.isfinite(t) and t > 0 for t in ms)
        for sc, f, (_, cam, kw) in zip(scenes, b.render(2), specs):
            _close(f, sc.render(cam, seed=5, sample_offset=2 * kw["spp"], **kw))
        b.close()
    finally:
        ctx.set_batch_kernel("wavefront")
    with pytest.raises(ValueError):
        ctx.set_batch_kernel("megakernel")


_TIGHT_SCRIPT = """
import sys, numpy as np
sys.path.insert(0, {root!r})
import pbrt_b200 as pb
from pbrt_b200 import workloads as W
from pbrt_b200.scene import Batch, create_scenes, render_params
(d0, c0), (d1, c1) = W.cornell_box(24, 20), W.many_spheres(200, width=32, height=24)
scenes = create_scenes([d0, d1])
params = [render_params(c0, spp=3, max_depth=6, seed=9), render_params(c1, spp=2, max_depth=8, rr_start=3, seed=9)]
singles = [scenes[0].render(c0, spp=3, max_depth=6, seed=9), scenes[1].render(c1, spp=2, max_depth=8, rr_start=3, seed=9)]
scenes[0].ctx.set_batch_kernel("persistent")
films = Batch(scenes, params).render(0)
np.savez({out!r}, f0=films[0], f1=films[1], s0=singles[0], s1=singles[1])
"""


@pytest.mark.parametrize("env", [{"PBRT_BATCH_TIGHT": "0"}, {"PBRT_BATCH_REFILL": "1"}, {"PBRT_BATCH_REFILL": "32"}])
def test_persistent_batch_builds_and_refill(tmp_path, env):
    """The 96-register build of the persistent batch kernel, and refills at every idle lane or
    only when the whole warp is idle, give the scenes' own films (switches read once per
    process: a child each)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = str(tmp_path / "films.npz")
    subprocess.run([sys.executable, "-c", _TIGHT_SCRIPT.format(root=root, out=out)], env=dict(os.environ, **env),
                   check=True, timeout=300)
    z = np.load(out)
    _close(z["f0"], z["s0"])
    _close(z["f1"], z["s1"])


@pytest.mark.parametrize("wave_paths", [0, 1 << 19])
def test_waves_along_scene_boundaries(wave_paths):
    """Scenes of at least 2^20 paths get waves of their own (split into several by a
    2^19-path wave size) on the least-loaded branch, the small scenes around them are packed
    into shared waves: every film equals the scene's own render, and each scene's completion
    time is reported."""
    specs = [(W.cornell_box(32, 24), dict(spp=2, max_depth=5)),
             (W.cornell_box(512, 512), dict(spp=4, max_depth=4)),  # 1,048,576 paths
             (W.many_spheres(200, width=40, height=30), dict(spp=3, max_depth=6, rr_start=3)),
             (W.cornell_box(512, 512), dict(spp=8, max_depth=3)),  # 2,097,152 paths
             (W.cornell_box(20, 20), dict(spp=5, max_depth=6))]
    scenes = create_scenes([d for (d, _), _ in specs])
    singles = [s.render(cam, seed=9, **kw) for s, ((_, cam), kw) in zip(scenes, specs)]
    params = [render_params(cam, seed=9, **kw) for (_, cam), kw in specs]
    ctx = scenes[0].ctx
    ctx.set_tuning(wave_paths=wave_paths)
    try:
        b = Batch(scenes, params)
        films, ms = b.render(0, scene_times=True)
        for f, s in zip(films, singles):
            _close(f, s)
        assert all(t > 0 for t in ms)
        b.close()
    finally:
        ctx.set_tuning()
