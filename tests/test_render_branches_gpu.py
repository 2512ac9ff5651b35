"""A render's paths split over concurrent streams (each part a chain of waves with its own
wave buffers, forked from the call's stream and joined back to it): films must not depend on
the number of parts, and the fork and join must hold inside a captured CUDA graph."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

import pbrt_b200 as pb
from pbrt_b200 import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SCRIPT = """
import sys, numpy as np
sys.path.insert(0, {root!r})
import pbrt_b200 as pb
from pbrt_b200 import workloads as W
d, cam = W.cornell_box(40, 30)
scene = pb.Scene.from_description(d, pb.Context(0)).commit(bvh_bins=8, bvh_max_leaf=1)
np.save({out!r}, scene.render(cam, spp=5, max_depth=7, seed=9, rr_start=3))
"""


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)


def _scene(ctx=None):
    d, cam = W.cornell_box(40, 30)
    return pb.Scene.from_description(d, ctx or pb.Context(0)).commit(bvh_bins=8, bvh_max_leaf=1), cam


@pytest.mark.parametrize("branches", ["1", "3", "8"])
def test_films_do_not_depend_on_the_branch_count(tmp_path, branches):
    """6,000 paths in 1, 3 or 8 concurrent parts (another process, PBRT_RENDER_BRANCHES)
    against this process's default of 2: the same film."""
    scene, cam = _scene()
    ref = scene.render(cam, spp=5, max_depth=7, seed=9, rr_start=3)
    out = str(tmp_path / "film.npy")
    subprocess.run([sys.executable, "-c", _SCRIPT.format(root=ROOT, out=out)],
                   env=dict(os.environ, PBRT_RENDER_BRANCHES=branches), check=True, timeout=300)
    _close(np.load(out), ref)


def test_render_captured_in_a_cuda_graph():
    """pbrt_render on a caller's stream recorded into a CUDA graph: the branches' fork and
    join become edges of the graph, and each replay renders the same film as a direct call."""
    torch = pytest.importorskip("torch")
    scene, cam = _scene()
    ctx = scene.ctx
    ref = scene.render(cam, spp=4, max_depth=6, seed=5)
    s = torch.cuda.Stream()
    film = torch.zeros((cam["height"], cam["width"], 3), dtype=torch.float64, device="cuda")
    ctx.set_stream(s.cuda_stream)
    try:
        with torch.cuda.stream(s):
            scene.render(cam, spp=4, max_depth=6, seed=5, film=film)  # allocates the buffers
        s.synchronize()
        _close(film.cpu().numpy(), ref)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
            scene.render(cam, spp=4, max_depth=6, seed=5, film=film)
        for _ in range(2):
            film.fill_(-1.0)
            g.replay()
            torch.cuda.synchronize()
            _close(film.cpu().numpy(), ref)
        del g
    finally:
        ctx.set_stream(None)
