"""The learned radiance cache (pbrt_cache in include/pbrt_b200.h): a small MLP trained online
on the path tracer's own radiance estimates, with tcgen05 forward and backward kernels."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import CacheParams, PbrtError  # noqa: F401
from .scene import Context, default_context

PARAMS = 23552
RECORD = 16


class RadianceCache:
    def __init__(self, scene_min: Sequence[float], scene_max: Sequence[float], seed: int = 1,
                 learning_rate: float = 1e-2, terminate_bounce: int = 2, train_samples: int = 1 << 16,
                 train_steps: int = 4, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        p = CacheParams()
        p.seed, p.learning_rate = seed, learning_rate
        p.scene_min[:] = [float(x) for x in scene_min]
        p.scene_max[:] = [float(x) for x in scene_max]
        p.terminate_bounce, p.train_samples, p.train_steps = terminate_bounce, train_samples, train_steps
        self.params = p
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.pbrt_cache_create(self.ctx.h, C.byref(p), C.byref(h)), "pbrt_cache_create")
        self.h = h

    @property
    def bounds(self):
        return np.array(list(self.params.scene_min) + list(self.params.scene_max), np.float32)

    def weights(self) -> np.ndarray:
        w = np.zeros(PARAMS, np.float32)
        self.ctx.check(self.ctx.lib.pbrt_cache_get_weights(self.h, w.ctypes.data), "pbrt_cache_get_weights")
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self.ctx.check(self.ctx.lib.pbrt_cache_set_weights(self.h, w.ctypes.data), "pbrt_cache_set_weights")

    def reset(self):
        self.ctx.check(self.ctx.lib.pbrt_cache_reset(self.h), "pbrt_cache_reset")

    def query(self, records):
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD)
        out = np.zeros((r.shape[0], 3), np.float32)
        self.ctx.check(self.ctx.lib.pbrt_cache_query(self.h, r.ctypes.data, r.shape[0], out.ctypes.data),
                       "pbrt_cache_query")
        return out

    def gradient(self, records, targets):
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        g = np.zeros(PARAMS, np.float32)
        loss = C.c_float()
        self.ctx.check(self.ctx.lib.pbrt_cache_gradient(self.h, r.ctypes.data, t.ctypes.data, r.shape[0],
                                                        g.ctypes.data, C.byref(loss)), "pbrt_cache_gradient")
        return g, loss.value

    def train_step(self, records, targets) -> float:
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        loss = C.c_float()
        self.ctx.check(self.ctx.lib.pbrt_cache_train_step(self.h, r.ctypes.data, t.ctypes.data, r.shape[0],
                                                          C.byref(loss)), "pbrt_cache_train_step")
        return loss.value

    def save(self) -> bytes:
        n = C.c_uint64()
        self.ctx.check(self.ctx.lib.pbrt_cache_save(self.h, None, 0, C.byref(n)), "pbrt_cache_save")
        buf = (C.c_uint8 * n.value)()
        self.ctx.check(self.ctx.lib.pbrt_cache_save(self.h, buf, n.value, C.byref(n)), "pbrt_cache_save")
        return bytes(buf)

    def load(self, data: bytes):
        buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
        self.ctx.check(self.ctx.lib.pbrt_cache_load(self.h, buf, len(data)), "pbrt_cache_load")

    def close(self):
        if getattr(self, "h", None) is not None and self.ctx.h is not None:
            self.ctx.lib.pbrt_cache_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_records(n: int, lo, hi, seed: int = 0) -> np.ndarray:
    """Query records with positions in [lo, hi], unit directions and normals, albedo, roughness."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    r = np.zeros((n, RECORD), np.float32)
    r[:, 0:3] = lo + rng.random((n, 3)) * (hi - lo)
    r[:, 3] = rng.random(n)
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    r[:, 8:11] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    r[:, 12:15] = rng.random((n, 3))
    return r
