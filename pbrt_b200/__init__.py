"""pbrt_b200 — a B200-native wavefront path tracer for nmichel/pbrt's hot path.

The Python layer mirrors the reference's Rust API for this path (src/scene.rs,
src/objects/, src/shapes/, src/materials/, src/lights/, src/renderers/) and lowers a scene to
the flat C description of include/pbrt_b200.h; everything it computes runs in
libpbrt_b200.so on the GPU. There is no CPU fallback: if the library or a GPU is missing,
calls raise.
"""
from __future__ import annotations

from ._capi import PBRT_MISS, PbrtError, load  # noqa: F401
from .scene import (  # noqa: F401
    AABox,
    AreaLight,
    BackgroundInfiniteLight,
    CheckerBoard,
    Compound,
    Context,
    Csg,
    Cylinder,
    Dielectric,
    DiffuseLight,
    Lambertian,
    Metal,
    Plane,
    PointLight,
    Rectangle,
    Scene,
    Simple,
    Sphere,
    Transform,
    Transformed,
    TriangleMesh,
    UniformInfiniteLight,
    default_context,
    film_to_png,
    film_to_rgba8,
    write_png,
)
from .stage import Stage, load_scene, read_ply  # noqa: F401

__all__ = [
    "PBRT_MISS", "PbrtError", "load", "Context", "default_context", "Scene", "TriangleMesh", "Sphere", "Cylinder",
    "Simple", "Transformed", "Transform", "Lambertian", "Metal", "Dielectric", "DiffuseLight", "PointLight",
    "UniformInfiniteLight", "BackgroundInfiniteLight", "AreaLight", "film_to_rgba8", "Rectangle", "AABox", "Plane",
    "CheckerBoard", "Compound", "Csg", "Stage", "load_scene", "read_ply", "write_png", "film_to_png",
]
