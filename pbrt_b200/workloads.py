"""Seeded synthetic workloads of the hot path (no public suite or dataset exists for it).

incoherent_raycast(): the ray-cast workload — an icosphere subdivided to level 7
(327,680 triangles, FP32) whose vertices are displaced radially by a seeded 3-octave value
noise of amplitude 0.1·r, and 16,777,216 incoherent rays: origins uniform in a cube three
times the mesh bounds, directions uniform on the sphere and normalised the way the
reference's Ray::new does (src/geom/ray.rs:10-18), near 1e-4, far 1e30.
"""
from __future__ import annotations

import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0


def icosphere(level: int):
    """Unit icosphere with 20·4^level triangles. Faces are wound so that the reference's
    mesh normal cross(dpdv, dpdu) = (p2−p1)×(p1−p0) (triangle_mesh.rs:119 with the default
    uvs) points outward."""
    v = np.array([[-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0], [0, -1, _PHI], [0, 1, _PHI],
                  [0, -1, -_PHI], [0, 1, -_PHI], [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1]],
                 np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    verts = [v]
    nverts = v.shape[0]
    for _ in range(level):
        # midpoint of every edge, shared between the two faces that own it
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.minimum(e[:, 0], e[:, 1]) * (1 << 32) + np.maximum(e[:, 0], e[:, 1])
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq >> 32, uniq & 0xFFFFFFFF
        allv = np.concatenate(verts)
        mid = allv[a] + allv[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        verts = [allv, mid]
        m = inv.reshape(3, -1).T + nverts  # midpoints of (v0v1, v1v2, v2v0) per face
        nverts += mid.shape[0]
        v0, v1, v2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([v0, m01, m20], 1), np.stack([v1, m12, m01], 1), np.stack([v2, m20, m12], 1),
                            np.stack([m01, m12, m20], 1)])
    verts = np.concatenate(verts)
    # (p2−p1)×(p1−p0) must point outward: flip faces where it points inward.
    p0, p1, p2 = verts[f[:, 0]], verts[f[:, 1]], verts[f[:, 2]]
    n = np.cross(p2 - p1, p1 - p0)
    inward = (n * (p0 + p1 + p2)).sum(1) < 0
    f[inward] = f[inward][:, ::-1]
    return verts, f.astype(np.uint32)


def _hash3(ix, iy, iz, seed: int):
    h = (ix.astype(np.uint64) * np.uint64(0x9E3779B185EBCA87) ^ iy.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F)
         ^ iz.astype(np.uint64) * np.uint64(0x165667B19E3779F9) ^ np.uint64(seed * 0x27D4EB2F165667C5 & (2**64 - 1)))
    h ^= h >> np.uint64(29)
    h *= np.uint64(0xBF58476D1CE4E5B9)
    h ^= h >> np.uint64(32)
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise in [0, 1) with smoothstep weights on an integer lattice."""
    p = np.asarray(p, np.float64)
    i = np.floor(p).astype(np.int64)
    fr = p - i
    w = fr * fr * (3.0 - 2.0 * fr)
    out = np.zeros(p.shape[0])
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                h = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += h * wx * wy * wz
    return out


def displaced_icosphere(level: int, seed: int = 1, radius: float = 1.0, amplitude: float = 0.1,
                        frequency: float = 2.0):
    """Icosphere of `radius` displaced radially by 3-octave value noise, amplitude·radius."""
    v, f = icosphere(level)
    n = np.zeros(v.shape[0])
    norm = 0.0
    for o in range(3):
        a = 0.5 ** o
        n += a * value_noise(v * frequency * (2 ** o), seed + 7919 * o)
        norm += a
    n = 2.0 * (n / norm) - 1.0  # [-1, 1)
    v = v * (radius * (1.0 + amplitude * n))[:, None]
    return v.astype(np.float32), f


def normalize_f32(d: np.ndarray) -> np.ndarray:
    """Ray::new normalisation in FP32: d * (1 / sqrt((x*x + y*y) + z*z)) (vector3.rs:69-74)."""
    d = d.astype(np.float32)
    nrm = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]
    inv = np.float32(1.0) / np.sqrt(nrm)
    return d * inv


def incoherent_rays(n: int, lo: np.ndarray, hi: np.ndarray, seed: int = 2, near: float = 1e-4,
                    far: float = 1e30) -> np.ndarray:
    """n rays as (8, n) float32 SoA planes; origins uniform in the cube of side 3× the largest
    extent of [lo, hi] around its centre, directions uniform on S²."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = (np.asarray(lo, np.float64) + np.asarray(hi, np.float64)) * 0.5
    side = 3.0 * float(np.max(np.asarray(hi, np.float64) - np.asarray(lo, np.float64)))
    rays = np.empty((8, n), np.float32)
    rays[0:3] = (c[:, None] + (rng.random((3, n)) - 0.5) * side).astype(np.float32)
    z = rng.random(n) * 2.0 - 1.0
    phi = rng.random(n) * (2.0 * np.pi)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([s * np.cos(phi), s * np.sin(phi), z]).astype(np.float32)
    rays[3:6] = normalize_f32(d)
    rays[6] = np.float32(near)
    rays[7] = np.float32(far)
    return rays


def raycast_workload(level: int = 7, n_rays: int = 1 << 24, seed: int = 1):
    """(vertices, triangles, rays) of the incoherent ray-cast workload."""
    v, f = displaced_icosphere(level, seed=seed)
    rays = incoherent_rays(n_rays, v.min(0), v.max(0), seed=seed + 1)
    return v, f, rays
