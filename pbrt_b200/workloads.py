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


# ------------------------------------------------------------------------------------------
# Path-tracing scenes, as plain description dicts (pbrt_b200.Scene.from_description) plus a
# camera dict. Triangles are wound so that the reference's mesh normal
# (p2−p1)×(p1−p0) faces the lit side (into the room, out of the boxes).
# ------------------------------------------------------------------------------------------
def _quad(p0, p1, p2, p3, normal):
    p = [np.asarray(x, np.float64) for x in (p0, p1, p2, p3)]
    tris = [[p[0], p[1], p[2]], [p[0], p[2], p[3]]]
    out = []
    for a, b, c in tris:
        n = np.cross(c - b, b - a)
        out.append([a, b, c] if np.dot(n, normal) > 0 else [c, b, a])
    return out


def _box(center, half, angle):
    c, h = np.asarray(center, np.float64), np.asarray(half, np.float64)
    s, co = np.sin(angle), np.cos(angle)
    rot = np.array([[co, 0, s], [0, 1, 0], [-s, 0, co]])  # Matrix4::rotation_y (matrix4.rs:54-60)

    def corner(sx, sy, sz):
        return c + rot @ (h * np.array([sx, sy, sz], np.float64))

    tris = []
    for axis in range(3):
        for sign in (-1, 1):
            n = np.zeros(3)
            n[axis] = sign
            u, v = [a for a in range(3) if a != axis]
            cs = []
            for su, sv in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                q = np.zeros(3)
                q[axis], q[u], q[v] = sign, su, sv
                cs.append(corner(*q))
            tris += _quad(*cs, rot @ n)
    return tris


def _mesh(tris):
    v = np.asarray(tris, np.float64).reshape(-1, 3).astype(np.float32)
    return dict(vertices=v, indices=np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3))


def cornell_box(width: int = 256, height: int = 256):
    """Closed box of triangles: five Lambertian walls of a unit cube (grey 0.73, red left,
    green right), two 12-triangle boxes rotated ±18° about y, a 0.25-wide quad light of 2
    triangles at the ceiling centre emitting (17, 12, 4). No loader lights."""
    L = 0.5
    white = [*_quad((-L, -L, -L), (L, -L, -L), (L, -L, L), (-L, -L, L), (0, 1, 0)),   # floor
             *_quad((-L, L, -L), (L, L, -L), (L, L, L), (-L, L, L), (0, -1, 0)),      # ceiling
             *_quad((-L, -L, -L), (L, -L, -L), (L, L, -L), (-L, L, -L), (0, 0, 1)),   # back
             *_box((0.17, -0.35, 0.10), (0.15, 0.15, 0.15), -np.pi / 10),            # short box, -18°
             *_box((-0.17, -0.20, -0.15), (0.15, 0.30, 0.15), np.pi / 10)]           # tall box, +18°
    red = _quad((-L, -L, -L), (-L, L, -L), (-L, L, L), (-L, -L, L), (1, 0, 0))
    green = _quad((L, -L, -L), (L, L, -L), (L, L, L), (L, -L, L), (-1, 0, 0))
    y, s = L - 1e-3, 0.125
    light = _quad((-s, y, -s), (s, y, -s), (s, y, s), (-s, y, s), (0, -1, 0))
    desc = dict(
        meshes=[_mesh(white), _mesh(red), _mesh(green), _mesh(light)],
        materials=[dict(kind=0, color=(0.73, 0.73, 0.73)), dict(kind=0, color=(0.65, 0.05, 0.05)),
                   dict(kind=0, color=(0.12, 0.45, 0.15)), dict(kind=3, color=(17.0, 12.0, 4.0))],
        objects=[dict(shape=0, mesh=k, material=k, to_world=None, to_local=None) for k in range(4)],
        lights=[dict(kind=3, object=3)],
        bvh_bins=8, bvh_max_leaf=1,
    )
    camera = dict(width=width, height=height, fov=np.deg2rad(40.0), near=1e-4, far=1000.0,
                  position=(0.0, 0.0, 1.85), look_at=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0))
    return desc, camera


def _translation_rows(c):
    tw = np.array([[1, 0, 0, c[0]], [0, 1, 0, c[1]], [0, 0, 1, c[2]]], np.float32).reshape(-1)
    tl = np.array([[1, 0, 0, -c[0]], [0, 1, 0, -c[1]], [0, 0, 1, -c[2]]], np.float32).reshape(-1)
    return tw, tl


def many_spheres(n: int = 10_000, seed: int = 3, width: int = 1024, height: int = 768, extent: float = 10.0):
    """n non-overlapping spheres, radius U[0.05, 0.3], centres U in a (2·extent)³ box, each a
    Transformed(translation) of Simple(Sphere); materials in equal thirds: Lambertian
    (albedo U[0.1, 0.9]³), metal (fuzz U[0, 0.3], albedo U[0.5, 0.95]³ — the metal albedo is
    not specified, this is the choice), dielectric (IOR 1.5). Lights: the white → (0.5, 0.7,
    1.0) sky gradient (BackgroundInfiniteLight) and one spherical area light."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cell = 0.6
    grid = {}
    centres, radii = [], []
    while len(centres) < n:
        c = (rng.random(3) * 2.0 - 1.0) * extent
        r = 0.05 + 0.25 * rng.random()
        key = tuple(np.floor(c / cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        if np.sum((centres[j] - c) ** 2) <= (radii[j] + r) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            grid.setdefault(key, []).append(len(centres))
            centres.append(c)
            radii.append(r)
    materials, objects = [], []
    for k, (c, r) in enumerate(zip(centres, radii)):
        kind = k % 3
        if kind == 0:
            materials.append(dict(kind=0, color=tuple(0.1 + 0.8 * rng.random(3))))
        elif kind == 1:
            materials.append(dict(kind=1, color=tuple(0.5 + 0.45 * rng.random(3)), fuzz=0.3 * rng.random()))
        else:
            materials.append(dict(kind=2, color=(1.0, 1.0, 1.0), ior=1.5))
        tw, tl = _translation_rows(c)
        objects.append(dict(shape=1, radius=float(r), material=k, to_world=tw, to_local=tl))
    materials.append(dict(kind=3, color=(8.0, 8.0, 8.0)))
    tw, tl = _translation_rows((0.0, extent + 5.0, 0.0))
    objects.append(dict(shape=1, radius=2.5, material=len(materials) - 1, to_world=tw, to_local=tl))
    desc = dict(meshes=[], materials=materials, objects=objects,
                lights=[dict(kind=2, bottom=(1.0, 1.0, 1.0), top=(0.5, 0.7, 1.0)),
                        dict(kind=3, object=len(objects) - 1)],
                bvh_bins=8, bvh_max_leaf=1)
    camera = dict(width=width, height=height, fov=np.deg2rad(45.0), near=1e-4, far=1000.0,
                  position=(0.0, 0.6 * extent, 3.2 * extent), look_at=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0))
    return desc, camera


def torus_knot(segments: int = 10627, sides: int = 41, p: int = 2, q: int = 3, scale: float = 0.105,
               tube: float = 0.045, amplitude: float = 0.25, seed: int = 4):
    """A (p, q) torus-knot tube of 2·segments·sides triangles (871,414 by default), its
    surface displaced along the tube normal by seeded 3-octave value noise of amplitude
    `amplitude`·tube. The knot lies in the xy plane around the origin. Faces are wound so
    that (p2−p1)×(p1−p0) points out of the tube."""
    t = np.arange(segments, dtype=np.float64) * (2.0 * np.pi / segments)
    r = np.cos(q * t) + 2.0
    c = np.stack([r * np.cos(p * t), r * np.sin(p * t), -np.sin(q * t)], 1)
    dr = -q * np.sin(q * t)
    d1 = np.stack([dr * np.cos(p * t) - p * r * np.sin(p * t), dr * np.sin(p * t) + p * r * np.cos(p * t),
                   -q * np.cos(q * t)], 1)
    ddr = -q * q * np.cos(q * t)
    d2 = np.stack([ddr * np.cos(p * t) - 2 * p * dr * np.sin(p * t) - p * p * r * np.cos(p * t),
                   ddr * np.sin(p * t) + 2 * p * dr * np.cos(p * t) - p * p * r * np.sin(p * t),
                   q * q * np.sin(q * t)], 1)
    T = d1 / np.linalg.norm(d1, axis=1, keepdims=True)
    B = np.cross(d1, d2)  # a torus knot's curvature never vanishes: the Frenet frame is defined
    B /= np.linalg.norm(B, axis=1, keepdims=True)
    N = np.cross(B, T)
    th = np.arange(sides, dtype=np.float64) * (2.0 * np.pi / sides)
    ring = np.cos(th)[None, :, None] * N[:, None, :] + np.sin(th)[None, :, None] * B[:, None, :]
    centre = (c * scale)[:, None, :]
    base = centre + tube * ring
    noise = np.zeros(segments * sides)
    norm = 0.0
    pts = base.reshape(-1, 3) * 20.0
    for o in range(3):
        a = 0.5 ** o
        noise += a * value_noise(pts * (2 ** o), seed + 7919 * o)
        norm += a
    noise = 2.0 * (noise / norm) - 1.0
    v = centre + (tube * (1.0 + amplitude * noise.reshape(segments, sides)))[:, :, None] * ring
    v = v.reshape(-1, 3)
    i = np.arange(segments)[:, None]
    j = np.arange(sides)[None, :]
    a = i * sides + j
    b = ((i + 1) % segments) * sides + j
    cc = ((i + 1) % segments) * sides + (j + 1) % sides
    d = i * sides + (j + 1) % sides
    f = np.concatenate([np.stack([a, b, cc], -1).reshape(-1, 3), np.stack([a, cc, d], -1).reshape(-1, 3)])
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    n = np.cross(p2 - p1, p1 - p0)
    mid_ring = np.concatenate([np.repeat(c * scale, sides, axis=0)] * 2)
    inward = (n * ((p0 + p1 + p2) / 3.0 - mid_ring)).sum(1) < 0
    f[inward] = f[inward][:, ::-1]
    return v.astype(np.float32), f.astype(np.uint32)


def radiance_cache_scene(width: int = 1920, height: int = 1080, segments: int = 10627, sides: int = 41,
                         seed: int = 4):
    """The learned-cache workload: the closed box of cornell_box (walls and ceiling light,
    without its two inner boxes) around a displaced torus knot of 2·segments·sides
    triangles (871,414 by default) whose faces are, seeded per quad, one of two diffuse or
    two glossy (metal, fuzz 0.25 and 0.1) materials."""
    desc, camera = cornell_box(width, height)
    walls = desc["meshes"][0]
    desc["meshes"][0] = dict(vertices=walls["vertices"][:18], indices=walls["indices"][:6])  # floor, ceiling, back
    v, f = torus_knot(segments, sides, seed=seed)
    v = v + np.array([0.0, -0.02, -0.08], np.float32)
    rng = np.random.Generator(np.random.PCG64(seed))
    quad_mat = rng.integers(0, 4, segments * sides)
    base = len(desc["materials"])
    desc["materials"] += [dict(kind=0, color=(0.75, 0.45, 0.2)), dict(kind=0, color=(0.3, 0.5, 0.8)),
                          dict(kind=1, color=(0.9, 0.75, 0.4), fuzz=0.25), dict(kind=1, color=(0.8, 0.8, 0.85), fuzz=0.1)]
    fm = (base + np.concatenate([quad_mat, quad_mat])).astype(np.uint32)
    desc["meshes"].append(dict(vertices=v, indices=f, face_materials=fm))
    desc["objects"].append(dict(shape=0, mesh=len(desc["meshes"]) - 1, material=base, to_world=None, to_local=None))
    desc["bvh_bins"], desc["bvh_max_leaf"] = 16, 4
    return desc, camera


def batch_scenes(n: int = 64, seed: int = 3, width: int = 512, height: int = 512, max_depth: int = 8,
                 levels=(3, 9), spp=(4, 64)):
    """The batched-rendering workload: n independent scenes, each the closed box of
    cornell_box (walls and ceiling light, without its inner boxes) around a displaced
    icosphere (radius 0.3, value-noise amplitude 0.1·r) of level U{levels}, rendered at
    width x height with U{spp} samples per pixel and max depth max_depth. Scenes of the same
    level share one seeded mesh; each scene is still committed (and its BVH built) on its
    own. Returns [(description, camera, spp)] in scene order."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lv = rng.integers(levels[0], levels[1] + 1, n)
    sp = rng.integers(spp[0], spp[1] + 1, n)
    meshes = {}
    out = []
    for i in range(n):
        level = int(lv[i])
        if level not in meshes:
            v, f = displaced_icosphere(level, seed=seed * 1000 + level, radius=0.3, amplitude=0.1)
            meshes[level] = ((v + np.array([0.0, -0.18, -0.05], np.float32)).astype(np.float32), f)
        desc, cam = cornell_box(width, height)
        walls = desc["meshes"][0]
        desc["meshes"][0] = dict(vertices=walls["vertices"][:18], indices=walls["indices"][:6])
        v, f = meshes[level]
        desc["materials"].append(dict(kind=0, color=(0.4, 0.5, 0.8)))
        desc["meshes"].append(dict(vertices=v, indices=f))
        desc["objects"].append(dict(shape=0, mesh=len(desc["meshes"]) - 1, material=len(desc["materials"]) - 1,
                                    to_world=None, to_local=None))
        desc["bvh_bins"], desc["bvh_max_leaf"] = 16, 4
        desc["level"] = level
        out.append((desc, cam, int(sp[i])))
    return out
