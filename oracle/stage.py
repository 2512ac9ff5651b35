"""Restatement of the reference's `.stage` scene loader — TEST INFRASTRUCTURE, not the product.

Follows, step for step:
  src/loader/parser/lexer.rs:123-360   tokens: keywords, numbers, strings, `#` comments
  src/loader/parser.rs:26-367          the grammar (camera, scene, object, shape, material,
                                       texture, transform)
  src/loader/visitors/scene_builder.rs the scene it builds: objects popped from a stack (so the
                                       scene and every compound hold their members in reverse
                                       file order); a transform block folded as
                                       identity * step_n * ... * step_1
  src/loader.rs:29-45                  the two lights it adds to every scene (a point light at
                                       (0, 2, 1) of intensity 15, a white-to-(0.5, 0.7, 1.0)
                                       background)
  src/config.rs:112-129                the camera settings a file does not hold (fov 90 degrees,
                                       near 1e-4, far 1000, 800 x 600)
  src/geom/matrix4.rs:44-66, 216-232   rotation matrices and the sequential 4x4 product
  src/geom/transform.rs:43-72, 119-127 translation / rotation inverses, Transform product

The result is the plain scene description the oracle and the product both take (see
oracle/__init__.py): meshes, materials, objects (one per Simple), the object tree (nodes,
roots), the loader's lights, and the camera dict.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Tuple

import numpy as np


class StageError(ValueError):
    """A scene file the reference's parser would reject (it panics)."""


KEYWORDS = {
    "aabox", "camera", "reverse", "checkerboard", "color", "csg", "compound", "cylinder", "dielectric",
    "diffuse_light", "elem", "file", "focal_length", "intersection", "lambertian", "look", "metal", "mesh",
    "object", "pos", "pin_hole", "plane", "radius", "rectangle", "rotate_x", "rotate_y", "rotate_z", "scene",
    "simple", "sphere", "substraction", "thin_lens", "transform", "transformed", "translate", "union", "up",
}
SPECIAL = {"{": "{", "}": "}", "[": "[", "]": "]", "(": "(", ")": ")"}


# ------------------------------------------------------------------------------------------
# Tokens (lexer.rs)
# ------------------------------------------------------------------------------------------
def tokenize(text: str) -> List[Tuple[str, object]]:
    """(kind, value) pairs: ("kw", name), ("id", name), ("num", float), ("str", s), ("sym", c).
    Stops where the reference's tokenizer answers None: the end of the text or a character that
    starts no token."""
    out = []
    i, n = 0, len(text)
    while True:
        while i < n and text[i].isspace():
            i += 1
        if i >= n:
            break
        c = text[i]
        if c == "#":  # a comment runs to the end of the line (lexer.rs:324-326)
            while i < n and text[i] != "\n":
                i += 1
            continue
        if c in SPECIAL:
            out.append(("sym", c))
            i += 1
            continue
        if c == '"':  # tokenize_string: up to the next quote; an empty string is no token
            j = i + 1
            while j < n and text[j] != '"':
                j += 1
            if j == i + 1:
                break
            out.append(("str", text[i + 1:j]))
            i = j + 1
            continue
        if c.isdigit() or c in "+-":  # tokenize_number: sign? digits (. digits*)?
            j = i
            state = "sign"
            while j < n:
                ch = text[j]
                if state == "sign":
                    if ch in "+-":
                        state = "first"
                    elif ch.isnumeric():
                        state = "int"
                    else:
                        break
                elif state == "first":
                    if ch.isnumeric():
                        state = "int"
                    else:
                        break
                elif state == "int":
                    if ch == ".":
                        state = "dot"
                    elif not ch.isnumeric():
                        break
                elif state == "dot":
                    if ch.isnumeric():
                        state = "dec"
                    else:
                        break
                else:
                    if not ch.isnumeric():
                        break
                j += 1
            try:
                out.append(("num", float(text[i:j])))
            except ValueError:
                raise StageError(f"bad number {text[i:j]!r}") from None
            i = j
            continue
        if c.isalpha():  # tokenize_identifier: alphanumerics and '_'
            j = i
            while j < n and (text[j].isalnum() or text[j] == "_"):
                j += 1
            w = text[i:j]
            out.append(("kw", w) if w in KEYWORDS else ("id", w))
            i = j
            continue
        break
    return out


# ------------------------------------------------------------------------------------------
# Transforms in float64 (matrix4.rs, transform.rs)
# ------------------------------------------------------------------------------------------
def _eye():
    return [[1.0 if i == j else 0.0 for j in range(4)] for i in range(4)]


def matmul4(a, b):
    """Matrix4 * Matrix4 (matrix4.rs:216-232): m[i][j] = 0, then += a[i][k] * b[k][j], k = 0..3."""
    m = [[0.0] * 4 for _ in range(4)]
    for i in range(4):
        for j in range(4):
            acc = 0.0
            for k in range(4):
                acc += a[i][k] * b[k][j]
            m[i][j] = acc
    return m


class Xf:
    """Transform {mat, inv_mat}."""

    def __init__(self, mat, inv):
        self.mat, self.inv = mat, inv

    @staticmethod
    def identity():
        return Xf(_eye(), _eye())

    @staticmethod
    def translation(x, y, z):
        m, i = _eye(), _eye()
        m[0][3], m[1][3], m[2][3] = x, y, z
        i[0][3], i[1][3], i[2][3] = -x, -y, -z
        return Xf(m, i)

    @staticmethod
    def rotation(axis: str, a: float):
        s, c = math.sin(a), math.cos(a)
        if axis == "x":
            m = [[1.0, 0.0, 0.0, 0.0], [0.0, c, -s, 0.0], [0.0, s, c, 0.0], [0.0, 0.0, 0.0, 1.0]]
        elif axis == "y":
            m = [[c, 0.0, s, 0.0], [0.0, 1.0, 0.0, 0.0], [-s, 0.0, c, 0.0], [0.0, 0.0, 0.0, 1.0]]
        else:
            m = [[c, -s, 0.0, 0.0], [s, c, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0], [0.0, 0.0, 0.0, 1.0]]
        return Xf(m, [[m[j][i] for j in range(4)] for i in range(4)])  # inverse = transpose

    def __mul__(self, o: "Xf") -> "Xf":  # transform.rs:119-127
        return Xf(matmul4(self.mat, o.mat), matmul4(o.inv, self.inv))

    def rows(self):
        """(to_world, to_local) as 12 float64 each (row-major 3x4)."""
        return (np.array(self.mat[:3], np.float64).reshape(-1), np.array(self.inv[:3], np.float64).reshape(-1))


# ------------------------------------------------------------------------------------------
# Parser + scene builder
# ------------------------------------------------------------------------------------------
SHAPE = dict(mesh=0, sphere=1, cylinder=2, rectangle=3, aabox=4, plane=5, csg=6)
CSG_OP = dict(union=0, intersection=1, substraction=2)
MAT = dict(lambertian=0, metal=1, dielectric=2, diffuse_light=3)


class _Parser:
    def __init__(self, text: str, load_mesh: Callable[[str, bool], Tuple[np.ndarray, np.ndarray]]):
        self.toks = tokenize(text)
        self.i = 0
        self.load_mesh = load_mesh
        self.meshes, self.mesh_ids = [], {}
        self.materials, self.objects, self.nodes = [], [], []

    # token helpers
    def next(self):
        if self.i >= len(self.toks):
            return None
        t = self.toks[self.i]
        self.i += 1
        return t

    def expect(self, kind, value=None, what=""):
        t = self.next()
        if t is None or t[0] != kind or (value is not None and t[1] != value):
            raise StageError(f"expected {what or value or kind}, got {t!r}")
        return t[1]

    def kw(self):
        t = self.next()
        return t[1] if t is not None and t[0] == "kw" else t

    def number(self):
        return self.expect("num", what="a number")

    def vector(self):
        return (self.number(), self.number(), self.number())

    # camera (parser.rs:34-83)
    def camera(self):
        self.expect("kw", "camera")
        kind = self.kw()
        if kind not in ("pin_hole", "thin_lens"):
            raise StageError("unknown camera type")
        self.expect("kw", "pos")
        pos = self.vector()
        self.expect("kw", "look")
        look = self.vector()
        self.expect("kw", "up")
        up = self.vector()
        cam = dict(kind=kind, position=pos, look_at=look, up=up)
        if kind == "thin_lens":
            self.expect("kw", "radius")
            cam["lens_radius"] = self.number()
            self.expect("kw", "focal_length")
            cam["focal_distance"] = self.number()
        return cam

    # objects (parser.rs:104-139, scene_builder.rs:95-116): returns a node index
    def object(self):
        k = self.kw()
        if k == "simple":
            shape = self.shape()
            mat = self.material()
            self.materials.append(mat)
            shape["material"] = len(self.materials) - 1
            self.objects.append(shape)
            self.nodes.append(dict(kind=0, object=len(self.objects) - 1))
            return len(self.nodes) - 1
        if k == "transformed":
            self.expect("kw", "object")
            child = self.object()
            xf = self.transform()
            w, l = xf.rows()
            self.nodes.append(dict(kind=1, children=[child], to_world=w, to_local=l))
            return len(self.nodes) - 1
        if k == "compound":
            self.expect("sym", "{")
            kids = []
            while True:
                t = self.next()
                if t == ("kw", "object"):
                    kids.append(self.object())
                elif t == ("sym", "}"):
                    break
                else:
                    raise StageError("expected } or object")
            self.nodes.append(dict(kind=2, children=kids[::-1]))  # popped: reverse order
            return len(self.nodes) - 1
        raise StageError("expected simple, transformed or compound")

    def shape(self):
        k = self.kw()
        if k == "aabox":
            return dict(shape=SHAPE["aabox"], extent=self.vector())
        if k == "sphere":
            return dict(shape=SHAPE["sphere"], radius=self.number())
        if k == "cylinder":
            r = self.number()
            return dict(shape=SHAPE["cylinder"], radius=r, height=self.number())
        if k == "rectangle":  # the two numbers become Rectangle::new(width, height)
            w = self.number()
            return dict(shape=SHAPE["rectangle"], radius=w, height=self.number())
        if k == "plane":
            return dict(shape=SHAPE["plane"])
        if k == "mesh":
            self.expect("kw", "file")
            name = self.expect("str", what="a file name")
            rev = False
            if self.i < len(self.toks) and self.toks[self.i] == ("kw", "reverse"):
                self.i += 1
                rev = True
            key = (name, rev)
            if key not in self.mesh_ids:
                v, idx = self.load_mesh(name, rev)
                self.mesh_ids[key] = len(self.meshes)
                self.meshes.append(dict(vertices=np.asarray(v, np.float32).reshape(-1, 3),
                                        indices=np.asarray(idx, np.uint32).reshape(-1, 3), file=name, reverse=rev))
            return dict(shape=SHAPE["mesh"], mesh=self.mesh_ids[key])
        if k == "csg":  # parser.rs:157-196, scene_builder.rs:118-143
            op = self.kw()
            if op not in CSG_OP:
                raise StageError("expected intersection, union or subtraction")
            self.expect("sym", "{")
            elems = []
            while True:
                t = self.next()
                if t == ("kw", "elem"):
                    e = self.shape()
                    if e["shape"] == SHAPE["csg"]:
                        raise StageError("a csg element is a plain shape")
                    w, l = self.transform().rows()
                    e.update(to_world=w, to_local=l)
                    elems.append(e)
                elif t == ("sym", "}"):
                    break
                else:
                    raise StageError("expected } or elem")
            return dict(shape=SHAPE["csg"], csg=dict(op=CSG_OP[op], elements=elems[::-1]))  # popped: reversed
        raise StageError("expected a shape")

    def material(self):
        k = self.kw()
        if k == "dielectric":
            ior = self.number()
            return dict(kind=MAT["dielectric"], ior=ior, **self.texture())
        if k == "metal":
            fuzz = self.number()
            return dict(kind=MAT["metal"], fuzz=fuzz, **self.texture())
        if k == "lambertian":
            return dict(kind=MAT["lambertian"], **self.texture())
        if k == "diffuse_light":
            return dict(kind=MAT["diffuse_light"], **self.texture())
        raise StageError("expected lambertian, dielectric, metal")

    def texture(self):
        k = self.kw()
        if k == "color":
            return dict(color=self.vector())
        if k == "checkerboard":
            c1, c2 = self.vector(), self.vector()
            return dict(texture=1, color=c1, color2=c2, scale=self.number())
        raise StageError("expected color, checkerboard")

    def transform(self):
        self.expect("kw", "transform")
        self.expect("sym", "{")
        steps = []
        while True:
            t = self.next()
            if t == ("kw", "translate"):
                steps.append(Xf.translation(*self.vector()))
            elif t in (("kw", "rotate_x"), ("kw", "rotate_y"), ("kw", "rotate_z")):
                steps.append(Xf.rotation(t[1][-1], self.number()))
            elif t == ("sym", "}"):
                break
            else:
                raise StageError("expected a transform step")
        res = Xf.identity()
        for st in reversed(steps):  # visit_transform: popped, folded from the identity
            res = res * st
        return res


def load_stage(text: str, load_mesh: Callable[[str, bool], Tuple[np.ndarray, np.ndarray]], width: int = 800,
               height: int = 600, fov_deg: float = 90.0, near: float = 0.0001, far: float = 1000.0,
               loader_lights: bool = True) -> dict:
    """Loader::load_scene(text, config): the scene description and its camera (under "camera").
    load_mesh(file, reverse) -> (vertices (n,3), indices (m,3)) stands for load_ply_mesh."""
    p = _Parser(text, load_mesh)
    cam = p.camera()
    p.expect("kw", "scene")
    top = []
    while True:
        t = p.next()
        if t is None:
            break
        if t != ("kw", "object"):
            raise StageError("expected object")
        top.append(p.object())
    lights = []
    if loader_lights:
        lights = [dict(kind=0, position=(0.0, 2.0, 1.0), radiance=(15.0, 15.0, 15.0)),
                  dict(kind=2, bottom=(1.0, 1.0, 1.0), top=(0.5, 0.7, 1.0))]
    cam.update(width=width, height=height, fov=fov_deg * math.pi / 180.0, near=near, far=far)
    return dict(meshes=p.meshes, materials=p.materials, objects=p.objects, nodes=p.nodes, roots=top[::-1],
                lights=lights, camera=cam, bvh_bins=8, bvh_max_leaf=1)
