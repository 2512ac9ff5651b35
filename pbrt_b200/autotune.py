"""Autotuner of the batched wavefront renderer: picks the BVH leaf size, the wave size
(paths in flight, i.e. the queues' capacity; by default only the largest is tried) and the
launch shape (threads per block and resident blocks per SM) of the traversal and shading
kernels by timing trial batches.

Search: a sample of the batch's scenes (spread over the list), rendered at `trial_spp`
samples per pixel as one graph-replayed batch; each trial's cost is the device time until the
last scene's last wave finished (median of `reps` frames). Leaf size first (it changes the
scenes' trees, so the sample is rebuilt per candidate), then the wave size, then the
traversal and shading shapes, one coordinate at a time, keeping the best so far.
"""
from __future__ import annotations

import json
import statistics
from typing import Optional

from .scene import Batch, Context, create_scenes, default_context, render_params

LEAF_SIZES = (1, 2, 4, 8)
# Wave size candidates: only the largest by default. A trial batch (a few scenes at 1-2 spp)
# holds fewer paths than one wave, so it cannot show the wave size's effect; at frame scale
# fewer, larger waves leave fewer per-bounce kernel tails (10,000 spheres at 1024x768x64 spp:
# 139.7 ms a frame at 2^22 paths per wave, 103.7 ms at 2^26).
WAVES = (1 << 26,)
SHAPES = ((64, 32), (128, 16), (256, 8), (128, 8), (256, 4))


def _trial(ctx: Context, scenes, params, tuning: dict, reps: int) -> float:
    ctx.set_tuning(**tuning)
    b = Batch(scenes, params, ctx)
    try:
        none = [None] * len(scenes)
        b.render(0, none, scene_times=True)  # warm-up
        times = [max(b.render(f + 1, none, scene_times=True)[1]) for f in range(reps)]
    finally:
        b.close()
    return statistics.median(times)


def autotune(specs, ctx: Optional[Context] = None, sample: int = 8, trial_spp: int = 2, reps: int = 3,
             leaf_sizes=LEAF_SIZES, waves=WAVES, shapes=SHAPES, out_json: Optional[str] = None) -> dict:
    """specs: [(description, camera, spp)] with max depth in each description's
    'max_depth' key (8 when absent). Returns the chosen parameters and every trial."""
    ctx = ctx or default_context()
    idx = sorted({round(i * (len(specs) - 1) / max(1, sample - 1)) for i in range(min(sample, len(specs)))})
    picked = [specs[i] for i in idx]
    params = [render_params(cam, trial_spp, d.get("max_depth", 8), seed=11) for d, cam, _ in picked]
    trials = []
    best = {"wave_paths": 1 << 26, "trace_threads": 128, "trace_blocks_per_sm": 16, "shade_threads": 128,
            "shade_blocks_per_sm": 16}

    best_leaf, best_ms, best_scenes = None, None, None
    for leaf in leaf_sizes:
        descs = [dict(d, bvh_max_leaf=leaf) for d, _, _ in picked]
        scenes = create_scenes(descs, ctx)
        ms = _trial(ctx, scenes, params, best, reps)
        trials.append({"leaf": leaf, **best, "ms": ms})
        if best_ms is None or ms < best_ms:
            best_leaf, best_ms, best_scenes = leaf, ms, scenes
        else:
            for s in scenes:
                s.release()

    def descend(keys, candidates):
        nonlocal best_ms
        for cand in candidates:
            t = dict(best)
            t.update(dict(zip(keys, cand if isinstance(cand, tuple) else (cand,))))
            if t == best:
                continue
            ms = _trial(ctx, best_scenes, params, t, reps)
            trials.append({"leaf": best_leaf, **t, "ms": ms})
            if ms < best_ms:
                best.update(t)
                best_ms = ms

    descend(("wave_paths",), waves)
    descend(("trace_threads", "trace_blocks_per_sm"), shapes)
    descend(("shade_threads", "shade_blocks_per_sm"), shapes)
    ctx.set_tuning(**best)
    for s in best_scenes:
        s.release()
    result = {"leaf": best_leaf, **best, "trial_ms": best_ms, "sample_scenes": idx, "trial_spp": trial_spp,
              "trials": trials}
    if out_json:
        with open(out_json, "w") as f:
            json.dump(result, f, indent=1)
    return result
