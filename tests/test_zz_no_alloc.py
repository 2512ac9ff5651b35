"""pbrt_trace_closest_noalloc: the nearest-hit entry point for callers that cannot call
cudaMalloc (a host that owns every device allocation through its own pool and budget, or a
latency-critical path that cannot afford cudaMalloc's synchronisation and cost).

It must return exactly what pbrt_trace_closest returns, on consecutive calls that reuse its
static scratch array, and allocate no device memory while doing so. This file is collected
last so that a run stopping at the first failure has already run every other test; it also
passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import pbrt_b200 as pb
from pbrt_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_RAYS = 1 << 20  # PBRT_NOALLOC_MAX_RAYS


def _free_bytes():
    free, _ = torch.cuda.mem_get_info()
    return free


def test_noalloc_matches_trace_closest_on_consecutive_calls():
    v, f = W.displaced_icosphere(5, seed=41)
    scene = pb.Scene(pb.Context(0)).add_object(pb.Simple(pb.TriangleMesh(v, f))).commit(bvh_bins=16, bvh_max_leaf=4)
    lib, ctx = scene.ctx.lib, scene.ctx
    batches = []
    for seed, n in ((42, MAX_RAYS), (43, 300_001)):  # a full batch, then a ragged one
        rays = W.incoherent_rays(n, v.min(0), v.max(0), seed=seed)
        aim = rays[:, : n // 2].copy()
        aim[3:6] = W.normalize_f32(-aim[0:3])  # half of them aimed at the mesh
        rays[:, : n // 2] = aim
        batches.append(torch.from_numpy(rays).cuda())

    expected = []
    for r in batches:  # the existing entry point, whose lazily allocated scratch is set up here
        n = r.shape[1]
        p = torch.empty(n, dtype=torch.int32, device="cuda")
        t = torch.empty(n, dtype=torch.float32, device="cuda")
        ctx.check(lib.pbrt_trace_closest(scene.h, r.data_ptr(), n, p.data_ptr(), t.data_ptr(), None), "trace")
        expected.append((p.cpu(), t.cpu()))

    # Output buffers are allocated up front, so that only the entry point runs while the
    # free device memory is watched.
    order = (0, 1, 0)
    outs = [(torch.full((batches[k].shape[1],), 7, dtype=torch.int32, device="cuda"),
             torch.full((batches[k].shape[1],), 7.0, dtype=torch.float32, device="cuda")) for k in order]
    torch.cuda.synchronize()

    def noalloc(k, out):
        r = batches[k]
        p, t = out
        ctx.check(lib.pbrt_trace_closest_noalloc(scene.h, r.data_ptr(), r.shape[1], p.data_ptr(), t.data_ptr()),
                  "pbrt_trace_closest_noalloc")

    noalloc(order[0], outs[0])  # first call: its kernels may load now (lazy module loading)
    free_before = _free_bytes()
    noalloc(order[1], outs[1])  # two more calls in a row reuse the array as the last one left it
    noalloc(order[2], outs[2])
    torch.cuda.synchronize()
    assert _free_bytes() == free_before, "the no-alloc entry point must not allocate device memory"

    for (p, t), k in zip(outs, order):
        ep, et = expected[k]
        assert torch.equal(p.cpu(), ep), "ids differ from pbrt_trace_closest"
        assert torch.equal(t.cpu(), et), "distances differ from pbrt_trace_closest (bit-exact expected)"
    assert int((expected[0][0] != -1).sum()) > MAX_RAYS // 4


def test_noalloc_rejects_oversized_and_host_batches():
    v, f = W.displaced_icosphere(3, seed=44)
    scene = pb.Scene(pb.Context(0)).add_object(pb.Simple(pb.TriangleMesh(v, f))).commit()
    lib = scene.ctx.lib
    n = MAX_RAYS + 1
    rays = torch.zeros((8, n), dtype=torch.float32, device="cuda")
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    rc = lib.pbrt_trace_closest_noalloc(scene.h, rays.data_ptr(), n, p.data_ptr(), t.data_ptr())
    assert rc == 5  # PBRT_ERR_CAPACITY
    assert b"exceeds its fixed scratch capacity" in lib.pbrt_last_error(scene.ctx.h)
    hr = np.zeros((8, 16), np.float32)
    hp = np.zeros(16, np.uint32)
    ht = np.zeros(16, np.float32)
    rc = lib.pbrt_trace_closest_noalloc(scene.h, hr.ctypes.data, 16, hp.ctypes.data, ht.ctypes.data)
    assert rc == 1  # PBRT_ERR_INVALID_ARGUMENT: device buffers only
    assert lib.pbrt_trace_closest_noalloc(scene.h, None, 0, None, None) == 0


def test_noalloc_refuses_a_capturing_stream_and_accepts_empty_batches():
    """The entry point waits for its results, so on a stream under capture it must refuse
    before enqueuing anything and leave the caller's capture intact; n = 0 is a no-op on any
    scene, as for pbrt_trace_closest."""
    v, f = W.displaced_icosphere(3, seed=45)
    ctx = pb.Context(0)
    scene = pb.Scene(ctx).add_object(pb.Simple(pb.TriangleMesh(v, f))).commit()
    lib = ctx.lib
    n = 1024
    rays = torch.from_numpy(W.incoherent_rays(n, v.min(0), v.max(0), seed=46)).cuda()
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    x = torch.zeros(4, device="cuda")
    s = torch.cuda.Stream()
    ctx.set_stream(s.cuda_stream)
    g = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(g, stream=s):
        x.add_(1.0)
        rcs.append(lib.pbrt_trace_closest_noalloc(scene.h, rays.data_ptr(), n, p.data_ptr(), t.data_ptr()))
    assert rcs == [6]  # PBRT_ERR_UNSUPPORTED
    assert b"stream being captured" in lib.pbrt_last_error(ctx.h)
    g.replay()  # the capture survived the refusal
    torch.cuda.synchronize()
    assert torch.equal(x.cpu(), torch.ones(4))
    del g
    # outside a capture the same call on the same stream works
    ctx.check(lib.pbrt_trace_closest_noalloc(scene.h, rays.data_ptr(), n, p.data_ptr(), t.data_ptr()), "noalloc")
    ctx.set_stream(None)
    # n = 0 returns PBRT_OK even on a scene the entry point does not trace (two meshes)
    two = pb.Scene(ctx).add_object(pb.Simple(pb.TriangleMesh(v, f))).add_object(
        pb.Simple(pb.TriangleMesh(v + 3.0, f))).commit()
    assert lib.pbrt_trace_closest_noalloc(two.h, None, 0, None, None) == 0
