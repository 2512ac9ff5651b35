"""The oracle's measurement helpers: the counted render (the work tally behind the render
path's algorithmic bytes) and the network's BF16 rounding margins (behind the forward-pass
parity test). Both must leave the oracle's answers unchanged."""
import numpy as np

import oracle
from pbrt_b200 import workloads as W
from pbrt_b200.cache import PARAMS, random_records


def test_counted_render_equals_render_and_counts_the_work():
    desc, cam = W.cornell_box(48, 32)
    o = oracle.Scene(desc, np.float32)
    plain = o.render(cam, 2, 8, seed=3)
    film, work = o.render_counted(cam, 2, 8, seed=3)
    np.testing.assert_array_equal(film, plain)
    assert work["rays"] >= 48 * 32 * 2  # every sample traces at least its camera ray
    assert 0 < work["shadow_rays"] <= work["rays"]
    assert work["top_boxes"] > 0 and work["mesh_boxes"] > work["rays"] and work["triangles"] > 0
    assert work["shapes"] == 0  # the closed box is made of meshes only
    d2, c2 = W.many_spheres(200, width=24, height=16)
    _, w2 = oracle.Scene(d2, np.float32).render_counted(c2, 1, 6, seed=1, rr_start=4)
    assert w2["shapes"] > 0 and w2["triangles"] == 0


def test_margins_leave_the_forward_unchanged():
    lo, hi = (-1.0, -0.5, -2.0), (1.0, 1.5, 0.0)
    b = np.array(lo + hi, np.float32)
    w = ((np.random.default_rng(1).random(PARAMS) - 0.5) * 0.3).astype(np.float32)
    r = random_records(3000, lo, hi, seed=3)
    out, margin, scale = oracle.mlp_forward_margins(w, b, r)
    np.testing.assert_array_equal(out, oracle.mlp_forward(w, b, r))
    assert np.all(margin >= 0) and np.all(scale >= np.abs(out) - 1e-6)
    # a sizeable share of rows clears every rounding boundary by 16 accumulation units
    assert 0.05 < (margin > 16).mean() < 0.95
