// scene_device.cuh — the scene on the GPU: placed objects ("leaves"), compounds, the
// top-level BVH over the scene's primitives, the unbounded primitives, the analytic shapes,
// and the interaction (shading record) of a hit.
//
// Semantics follow the reference operation for operation (FP32, no FMA):
//   Scene::find_nearest + BVH::query      src/scene.rs:186-249, src/bvh.rs:153-230
//   Scene::any_hit + BVH::query_p         src/scene.rs:157-184, src/bvh.rs:239-275
//   Transformed::intersect / intersect_p  src/objects/transformed.rs:27-38, 62-65
//   Compound::intersect / intersect_p     src/objects/compound.rs:21-50
//   Simple::intersect (first listed hit)  src/objects/simple.rs:28-41
//   Sphere::intersect + details           src/shapes/sphere.rs:108-187
//   Cylinder::intersect + details         src/shapes/cylinder.rs:28-110, 324-344
//   Rectangle / Plane / AABox::intersect  src/shapes/rectangle.rs:25-60, plane.rs:19-45, aabox.rs:76-190
//   TriangleMesh::intersect post-hit      src/shapes/triangle_mesh/triangle_mesh.rs:73-132, 219-258
// A nested object tree is flattened on the host: each placed Simple is a leaf carrying the
// chain of transforms above it (applied in turn, each renormalising the direction as
// Ray::new does), and a Compound is a group of consecutive leaves.
#pragma once

#include <cfloat>

#include "device_math.cuh"
#include "scene_types.hpp"
#include "trace_mesh.cuh"

namespace pbrt {

struct MeshShade {  // original vertices/indices, for the post-hit shading record
  const float* v;
  const uint32_t* idx;
  const uint32_t* fmat;  // material per triangle, or NULL
};

struct SceneView {
  const float4* top;        // top-level BVH nodes (GPU numbering, 2 float4 per node); may be empty
  uint32_t top_node_count;
  const uint32_t* order;    // leaf slot -> primitive (leaf index, or kGroupBit | group)
  const uint32_t* unbounded;  // primitives kept out of the BVH, tested first
  uint32_t unbounded_count;
  const ObjRec* objects;    // leaves
  const XfRec* xforms;      // transform chains beyond each leaf's first
  const CsgRec* csg;        // constructive solids' elements
  const GroupRec* groups;   // compounds
  const MeshView* meshes;   // traversal views
  const MeshShade* shade;   // shading views
  const MatRec* materials;
  const LightRec* lights;
  uint32_t light_count;
  const float* light_tris;  // area lights: 9 floats per world-space triangle
  const float* light_cdf;   // running area per triangle
  uint32_t has_csg;         // some leaf is a constructive solid: only the kernels built with CSG may run it
  // A leaf the renderer's scene queries may leave out and answer in a pass of their own (the
  // scene's largest untransformed mesh placed directly in the top-level tree); kNoLeaf: none.
  uint32_t defer_leaf;
};
constexpr uint32_t kNoLeaf = 0xFFFFFFFFu;

struct Isect {
  F3 p, n, wo, dpdu;
  float d, u, v;
};

// Work counters of the scene-level queries (TraversalStats of Scene::intersect_instrumented).
struct SceneCount {
  uint32_t nodes, boxes, objects;
};

// ---- transforms (affine 3x4) -------------------------------------------------------------
PBRT_DEV F3 xf_point(const float* m, const F3& v) {
  return mk3(fa(fa(fa(fm(m[0], v.x), fm(m[1], v.y)), fm(m[2], v.z)), m[3]),
             fa(fa(fa(fm(m[4], v.x), fm(m[5], v.y)), fm(m[6], v.z)), m[7]),
             fa(fa(fa(fm(m[8], v.x), fm(m[9], v.y)), fm(m[10], v.z)), m[11]));
}
PBRT_DEV F3 xf_dir(const float* m, const F3& v) {
  return mk3(fa(fa(fm(m[0], v.x), fm(m[1], v.y)), fm(m[2], v.z)), fa(fa(fm(m[4], v.x), fm(m[5], v.y)), fm(m[6], v.z)),
             fa(fa(fm(m[8], v.x), fm(m[9], v.y)), fm(m[10], v.z)));
}
// transform_normal: multiplies by the transpose (src/geom/matrix4.rs:208-213)
PBRT_DEV F3 xf_normal(const float* m, const F3& v) {
  return mk3(fa(fa(fm(m[0], v.x), fm(m[4], v.y)), fm(m[8], v.z)), fa(fa(fm(m[1], v.x), fm(m[5], v.y)), fm(m[9], v.z)),
             fa(fa(fm(m[2], v.x), fm(m[6], v.y)), fm(m[10], v.z)));
}

// ---- analytic shapes ----------------------------------------------------------------------
PBRT_DEV bool sphere_hit(float radius, const F3& o, const F3& d, float near, float far, float& t_out) {
  const F3 l = mul3(o, -1.f);
  const float tca = dot3(l, d);
  if (tca < 0.f) return false;
  const float r2 = fm(radius, radius);
  const float d2 = fs(dot3(l, l), fm(tca, tca));
  if (d2 > r2) return false;
  const float thc = fsq(fs(r2, d2));
  const float t0 = fs(tca, thc), t1 = fa(tca, thc);
  const float tmin = fminf(t0, t1), tmax = fmaxf(t0, t1);
  if (tmax < near || tmin > far) return false;
  if (tmin > near) { t_out = tmin; return true; }
  if (tmax > near && tmax < far) { t_out = tmax; return true; }
  return false;
}

// piece: 0 wall, 1 bottom cap, 2 top cap; the nearest of the listed hits (sorted by d).
PBRT_DEV bool cylinder_hit(float radius, float hh, const F3& o, const F3& d, float near, float far, float& t_out,
                           int& piece) {
  const float a = fa(fm(d.x, d.x), fm(d.z, d.z));
  const float b = fm(2.f, fa(fm(o.x, d.x), fm(o.z, d.z)));
  const float c = fs(fa(fm(o.x, o.x), fm(o.z, o.z)), fm(radius, radius));
  const float disc = fs(fm(b, b), fm(fm(4.f, a), c));
  if (disc < 0.f) return false;
  const float rd = fsq(disc);
  const float q = b < 0.f ? fm(-0.5f, fs(b, rd)) : fm(-0.5f, fa(b, rd));
  const float t0 = fdv(q, a), t1 = fdv(c, q);
  const float tmin = fminf(t0, t1), tmax = fmaxf(t0, t1);
  if (tmax < near || tmin > far) return false;
  float best = 0.f;
  int bp = -1, n = 0;
  auto take = [&](float t, int p) {
    if (n == 0 || t < best) { best = t; bp = p; }
    ++n;
  };
  if (tmin > near) {
    const F3 p = add3(o, mul3(d, tmin));
    if (p.y > -hh && p.y < hh) take(tmin, 0);
  }
  if (tmax > near && tmax < far) {
    const F3 p = add3(o, mul3(d, tmax));
    if (p.y > -hh && p.y < hh) take(tmax, 0);
  }
  if (n < 2) {
    const float iy = frcp(d.y);
    const float c0 = fm(fs(-hh, o.y), iy);
    if (c0 > near && c0 < far) {
      const F3 p = add3(o, mul3(d, c0));
      if (fa(fm(p.x, p.x), fm(p.z, p.z)) <= fm(radius, radius)) take(c0, 1);
    }
    const float c1 = fm(fs(hh, o.y), iy);
    if (c1 > near && c1 < far) {
      const F3 p = add3(o, mul3(d, c1));
      if (fa(fm(p.x, p.x), fm(p.z, p.z)) <= fm(radius, radius)) take(c1, 2);
    }
  }
  if (n == 0) return false;
  t_out = best;
  piece = bp;
  return true;
}

// Rectangle::intersect: the y = 0 plane at d = (o.y * -1) / dir.y, within |x| <= hw, |z| <= hh
PBRT_DEV bool rectangle_hit(float hw, float hh, const F3& o, const F3& d, float near, float far, float& t_out) {
  if (d.y == 0.f) return false;
  const float t = fdv(fm(o.y, -1.f), d.y);
  if (t < near || t > far) return false;
  const F3 p = add3(o, mul3(d, t));
  if (fabsf(p.x) > hw || fabsf(p.z) > hh) return false;
  t_out = t;
  return true;
}

// Plane::intersect, its arithmetic as written: d = (o.y * -1) / (1 / dir.y)
PBRT_DEV bool plane_hit(const F3& o, const F3& d, float near, float far, float& t_out) {
  const float inv = frcp(d.y);
  const float t = fdv(fm(o.y, -1.f), inv);
  if (t < near || t > far) return false;
  t_out = t;
  return true;
}

// AABox::intersect over [-h, h] (min = 0 - h): the entry beyond near, else the exit before
// far. face: 0..5 = X_NEG, X_POS, Y_NEG, Y_POS, Z_NEG, Z_POS.
PBRT_DEV void aabox_axis(float o, float inv, float lo, float hi, int fneg, float& tmin, float& tmax, int& fmin,
                         int& fmax) {
  if (inv >= 0.f) {
    tmin = fm(fs(lo, o), inv);
    tmax = fm(fs(hi, o), inv);
    fmin = fneg;
    fmax = fneg + 1;
  } else {
    tmin = fm(fs(hi, o), inv);
    tmax = fm(fs(lo, o), inv);
    fmin = fneg + 1;
    fmax = fneg;
  }
}
PBRT_DEV bool aabox_hit(const float* h, const F3& o, const F3& d, float near, float far, float& t_out, int& face) {
  float tmin, tmax, tymin, tymax, tzmin, tzmax;
  int fmin, fmax, fymin, fymax, fzmin, fzmax;
  aabox_axis(o.x, frcp(d.x), fs(0.f, h[0]), h[0], 0, tmin, tmax, fmin, fmax);
  aabox_axis(o.y, frcp(d.y), fs(0.f, h[1]), h[1], 2, tymin, tymax, fymin, fymax);
  if ((tmin > tymax) || (tymin > tmax)) return false;
  if (tymin > tmin) { tmin = tymin; fmin = fymin; }
  if (tymax < tmax) { tmax = tymax; fmax = fymax; }
  aabox_axis(o.z, frcp(d.z), fs(0.f, h[2]), h[2], 4, tzmin, tzmax, fzmin, fzmax);
  if ((tmin > tzmax) || (tzmin > tmax)) return false;
  if (tzmin > tmin) { tmin = tzmin; fmin = fzmin; }
  if (tzmax < tmax) { tmax = tzmax; fmax = fzmax; }
  if (tmax < near || tmin > far) return false;
  if (tmin > near) { t_out = tmin; face = fmin; return true; }
  if (tmax < far) { t_out = tmax; face = fmax; return true; }
  return false;
}

// ---- constructive solids (src/shapes/csg/*.rs) ---------------------------------------------
// contain_point of a plain shape: sphere.rs:146-148, cylinder.rs:119-124, aabox.rs:192-199,
// plane.rs:47-52; a rectangle and a mesh enclose nothing
PBRT_DEV bool shape_contains(uint32_t shape, const float* p, const F3& q) {
  switch (shape) {
    case kShapeSphere: return dot3(q, q) <= fm(p[0], p[0]);
    case kShapeCylinder:
      return fa(fm(q.x, q.x), fm(q.z, q.z)) <= fm(p[0], p[0]) && q.y >= -p[1] && q.y <= p[1];
    case kShapeAABox: {
      const float lx = fs(0.f, p[0]), ly = fs(0.f, p[1]), lz = fs(0.f, p[2]);
      return q.x >= lx && q.x <= p[0] && q.y >= ly && q.y <= p[1] && q.z >= lz && q.z <= p[2];
    }
    case kShapePlane: return q.y <= 0.f;
    default: return false;
  }
}

// Every hit a plain shape lists (its IntersectionResult, in order): distances and pieces
PBRT_DEV int shape_hits(const SceneView& s, uint32_t shape, uint32_t mesh, const float* p, const F3& o, const F3& d,
                        float near, float far, float* ts, uint32_t* ps, uint32_t* err) {
  float t;
  switch (shape) {
    case kShapeMesh: {
      TraceCounters c;
      const uint32_t id = mesh_closest<false>(s.meshes[mesh], prepare_ray(o, d), near, far, &t, &c, err);
      if (id == 0xFFFFFFFFu) return 0;
      ts[0] = t;
      ps[0] = id;
      return 1;
    }
    case kShapeSphere: {  // sphere.rs:108-144: the entry beyond near, the exit inside (near, far)
      const F3 l = mul3(o, -1.f);
      const float tca = dot3(l, d);
      if (tca < 0.f) return 0;
      const float r2 = fm(p[0], p[0]);
      const float d2 = fs(dot3(l, l), fm(tca, tca));
      if (d2 > r2) return 0;
      const float thc = fsq(fs(r2, d2));
      const float t0 = fs(tca, thc), t1 = fa(tca, thc);
      const float tmin = fminf(t0, t1), tmax = fmaxf(t0, t1);
      if (tmax < near || tmin > far) return 0;
      int n = 0;
      if (tmin > near) { ts[n] = tmin; ps[n] = 0; ++n; }
      if (tmax > near && tmax < far) { ts[n] = tmax; ps[n] = 0; ++n; }
      return n;
    }
    case kShapeCylinder: {  // cylinder.rs:28-110, sorted by distance (stable)
      const float radius = p[0], hh = p[1];
      const float a = fa(fm(d.x, d.x), fm(d.z, d.z));
      const float b = fm(2.f, fa(fm(o.x, d.x), fm(o.z, d.z)));
      const float c = fs(fa(fm(o.x, o.x), fm(o.z, o.z)), fm(radius, radius));
      const float disc = fs(fm(b, b), fm(fm(4.f, a), c));
      if (disc < 0.f) return 0;
      const float rd = fsq(disc);
      const float q = b < 0.f ? fm(-0.5f, fs(b, rd)) : fm(-0.5f, fa(b, rd));
      const float q0 = fdv(q, a), q1 = fdv(c, q);
      const float tmin = fminf(q0, q1), tmax = fmaxf(q0, q1);
      if (tmax < near || tmin > far) return 0;
      int n = 0;
      if (tmin > near) {
        const F3 h = add3(o, mul3(d, tmin));
        if (h.y > -hh && h.y < hh) { ts[n] = tmin; ps[n] = 0; ++n; }
      }
      if (tmax > near && tmax < far) {
        const F3 h = add3(o, mul3(d, tmax));
        if (h.y > -hh && h.y < hh) { ts[n] = tmax; ps[n] = 0; ++n; }
      }
      if (n < 2) {
        const float iy = frcp(d.y);
        const float c0 = fm(fs(-hh, o.y), iy);
        if (c0 > near && c0 < far) {
          const F3 h = add3(o, mul3(d, c0));
          if (fa(fm(h.x, h.x), fm(h.z, h.z)) <= fm(radius, radius)) { ts[n] = c0; ps[n] = 1; ++n; }
        }
        const float c1 = fm(fs(hh, o.y), iy);
        if (c1 > near && c1 < far) {
          const F3 h = add3(o, mul3(d, c1));
          if (fa(fm(h.x, h.x), fm(h.z, h.z)) <= fm(radius, radius)) { ts[n] = c1; ps[n] = 2; ++n; }
        }
      }
      for (int i = 1; i < n; ++i)  // insertion sort: stable
        for (int j = i; j > 0 && ts[j] < ts[j - 1]; --j) {
          const float tt = ts[j]; ts[j] = ts[j - 1]; ts[j - 1] = tt;
          const uint32_t pp = ps[j]; ps[j] = ps[j - 1]; ps[j - 1] = pp;
        }
      return n;
    }
    case kShapeRectangle:
      if (!rectangle_hit(p[0], p[1], o, d, near, far, t)) return 0;
      ts[0] = t;
      ps[0] = 0;
      return 1;
    case kShapePlane:
      if (!plane_hit(o, d, near, far, t)) return 0;
      ts[0] = t;
      ps[0] = 0;
      return 1;
    default: {  // AABox: the entry beyond near, the exit before far (aabox.rs:76-190)
      float tmin, tmax, tymin, tymax, tzmin, tzmax;
      int fmin, fmax, fymin, fymax, fzmin, fzmax;
      aabox_axis(o.x, frcp(d.x), fs(0.f, p[0]), p[0], 0, tmin, tmax, fmin, fmax);
      aabox_axis(o.y, frcp(d.y), fs(0.f, p[1]), p[1], 2, tymin, tymax, fymin, fymax);
      if ((tmin > tymax) || (tymin > tmax)) return 0;
      if (tymin > tmin) { tmin = tymin; fmin = fymin; }
      if (tymax < tmax) { tmax = tymax; fmax = fymax; }
      aabox_axis(o.z, frcp(d.z), fs(0.f, p[2]), p[2], 4, tzmin, tzmax, fzmin, fzmax);
      if ((tmin > tzmax) || (tzmin > tmax)) return 0;
      if (tzmin > tmin) { tmin = tzmin; fmin = fzmin; }
      if (tzmax < tmax) { tmax = tzmax; fmax = fzmax; }
      if (tmax < near || tmin > far) return 0;
      int n = 0;
      if (tmin > near) { ts[n] = tmin; ps[n] = uint32_t(fmin); ++n; }
      if (tmax < far) { ts[n] = tmax; ps[n] = uint32_t(fmax); ++n; }
      return n;
    }
  }
}

PBRT_DEV bool csg_point_in(const CsgRec& e, const F3& q) {
  return shape_contains(e.shape, e.p, xf_point(e.to_local, q));
}

// Union / Intersection / Substraction::intersect: every element's listed hits, each moved out
// of its element (the hit point as the element's record places it: on y = 0 for the flat
// shapes), kept by the operation's inside tests; the nearest kept, the earliest listed on a
// tie (the results are sorted stably). prim = element << 24 | the element's piece.
PBRT_DEV bool csg_closest(const SceneView& s, const ObjRec& ob, const F3& o, const F3& d, float near, float far,
                          float& t_out, uint32_t& prim_out, uint32_t* err) {
  bool have = false;
  for (uint32_t e = 0; e < ob.csg_count; ++e) {
    const CsgRec& E = s.csg[ob.csg_first + e];
    const F3 lo = xf_point(E.to_local, o);
    const F3 ld = normalize3(xf_dir(E.to_local, d));
    float ts[4];
    uint32_t ps[4];
    const int n = shape_hits(s, E.shape, E.mesh, E.p, lo, ld, near, far, ts, ps, err);
    for (int k = 0; k < n; ++k) {
      if (have && !(ts[k] < t_out)) continue;
      F3 hp = add3(lo, mul3(ld, ts[k]));
      if (E.shape == kShapeRectangle || E.shape == kShapePlane) hp.y = 0.f;
      const F3 w = xf_point(E.to_world, hp);
      bool keep;
      if (ob.csg_op == kCsgUnion) {
        keep = true;
        for (uint32_t j = 0; j < ob.csg_count && keep; ++j)
          if (j != e && csg_point_in(s.csg[ob.csg_first + j], w)) keep = false;
      } else if (ob.csg_op == kCsgIntersection) {
        keep = true;
        for (uint32_t j = 0; j < ob.csg_count && keep; ++j)
          if (j != e && !csg_point_in(s.csg[ob.csg_first + j], w)) keep = false;
      } else {
        keep = e == 0 || csg_point_in(s.csg[ob.csg_first], w);
        for (uint32_t j = 1; j < ob.csg_count && keep; ++j)
          if (j != e && csg_point_in(s.csg[ob.csg_first + j], w)) keep = false;
      }
      if (!keep) continue;
      have = true;
      t_out = ts[k];
      prim_out = (e << 24) | ps[k];
    }
  }
  return have;
}

// ---- leaves --------------------------------------------------------------------------------
PBRT_DEV const float* leaf_to_local(const SceneView& s, const ObjRec& ob, uint32_t k) {
  return k == 0 ? ob.to_local : s.xforms[ob.xf_rest + k - 1].to_local;
}
PBRT_DEV const float* leaf_to_world(const SceneView& s, const ObjRec& ob, uint32_t k) {
  return k == 0 ? ob.to_world : s.xforms[ob.xf_rest + k - 1].to_world;
}

// The leaf's local ray: transform_ray_to_local at every level of its chain, outermost first;
// each renormalises (transform.rs:98-103, ray.rs:10-18).
PBRT_DEV void local_ray(const SceneView& s, const ObjRec& ob, const F3& o, const F3& d, F3& lo, F3& ld) {
  lo = o;
  ld = d;
  for (uint32_t k = 0; k < ob.xf_count; ++k) {
    const float* inv = leaf_to_local(s, ob, k);
    lo = xf_point(inv, lo);
    ld = normalize3(xf_dir(inv, ld));
  }
}

// Object::intersect distance of one leaf within [near, far]; prim = triangle index, cylinder
// piece or box face (0 for the other shapes).
template <bool kCsg = true>
PBRT_DEV bool leaf_closest(const SceneView& s, uint32_t li, const F3& o, const F3& d, float near, float far,
                           float& t, uint32_t& prim, uint32_t* err) {
  const ObjRec& ob = s.objects[li];
  F3 lo, ld;
  local_ray(s, ob, o, d, lo, ld);
  prim = 0;
  switch (ob.shape) {
    case kShapeMesh: {
      const PRay r = prepare_ray(lo, ld);
      TraceCounters c;
      const uint32_t id = mesh_closest<false>(s.meshes[ob.mesh], r, near, far, &t, &c, err);
      prim = id;
      return id != 0xFFFFFFFFu;
    }
    case kShapeSphere: return sphere_hit(ob.p[0], lo, ld, near, far, t);
    case kShapeCylinder: {
      int piece = 0;
      const bool hit = cylinder_hit(ob.p[0], ob.p[1], lo, ld, near, far, t, piece);
      prim = uint32_t(piece);
      return hit;
    }
    case kShapeRectangle: return rectangle_hit(ob.p[0], ob.p[1], lo, ld, near, far, t);
    case kShapeAABox: {
      int face = 0;
      const bool hit = aabox_hit(ob.p, lo, ld, near, far, t, face);
      prim = uint32_t(face);
      return hit;
    }
    case kShapeCsg:
      if (kCsg) return csg_closest(s, ob, lo, ld, near, far, t, prim, err);
      return false;
    default: return plane_hit(lo, ld, near, far, t);
  }
}

template <bool kCsg = true>
PBRT_DEV bool leaf_any(const SceneView& s, uint32_t li, const F3& o, const F3& d, float near, float far,
                       uint32_t* err) {
  const ObjRec& ob = s.objects[li];
  F3 lo, ld;
  local_ray(s, ob, o, d, lo, ld);
  float t;
  int k;
  switch (ob.shape) {
    case kShapeMesh: return mesh_any(s.meshes[ob.mesh], prepare_ray(lo, ld), near, far, err);
    case kShapeSphere: return sphere_hit(ob.p[0], lo, ld, near, far, t);
    case kShapeCylinder: return cylinder_hit(ob.p[0], ob.p[1], lo, ld, near, far, t, k);
    case kShapeRectangle: return rectangle_hit(ob.p[0], ob.p[1], lo, ld, near, far, t);
    case kShapeAABox: return aabox_hit(ob.p, lo, ld, near, far, t, k);
    case kShapeCsg: {  // the default intersect_p: any listed hit (intersectable.rs:48-50)
      if (!kCsg) return false;
      uint32_t prim;
      return csg_closest(s, ob, lo, ld, near, far, t, prim, err);
    }
    default: return plane_hit(lo, ld, near, far, t);
  }
}

// ---- primitives (a leaf or a compound) -----------------------------------------------------
// A compound asks every member over the same [near, far] and keeps the strictly nearest hit,
// the earlier member on a tie (compound.rs:21-38).
template <bool kCsg = true>
PBRT_DEV bool prim_closest(const SceneView& s, uint32_t ref, const F3& o, const F3& d, float near, float far,
                           float& t, uint32_t& leaf, uint32_t& prim, uint32_t* err) {
  if (!(ref & kGroupBit)) {
    leaf = ref;
    return leaf_closest<kCsg>(s, ref, o, d, near, far, t, prim, err);
  }
  const GroupRec g = s.groups[ref & ~kGroupBit];
  bool have = false;
  for (uint32_t k = 0; k < g.count; ++k) {
    float tk;
    uint32_t pk;
    if (leaf_closest<kCsg>(s, g.first + k, o, d, near, far, tk, pk, err) && (!have || tk < t)) {
      have = true;
      t = tk;
      leaf = g.first + k;
      prim = pk;
    }
  }
  return have;
}

template <bool kCsg = true>
PBRT_DEV bool prim_any(const SceneView& s, uint32_t ref, const F3& o, const F3& d, float near, float far,
                       uint32_t* err) {
  if (!(ref & kGroupBit)) return leaf_any<kCsg>(s, ref, o, d, near, far, err);
  const GroupRec g = s.groups[ref & ~kGroupBit];
  for (uint32_t k = 0; k < g.count; ++k)
    if (leaf_any<kCsg>(s, g.first + k, o, d, near, far, err)) return true;  // compound.rs:47-49
  return false;
}

// Scene::find_nearest: the unbounded primitives first, each over [near, far]; then the
// top-level query over [near, nearest so far], narrowing to every adopted hit and offering
// each primitive [near, min_t]; a candidate is adopted only when strictly nearer.
// `skip` (a leaf index, or kNoLeaf) is a primitive the query leaves out.
template <bool kCount, bool kCsg = true>
PBRT_DEV bool scene_closest_t(const SceneView& s, const F3& o, const F3& d, float near, float far, float& t_out,
                              uint32_t& leaf_out, uint32_t& prim_out, uint32_t* err, SceneCount* cnt,
                              uint32_t skip = kNoLeaf) {
  float min_t = far;
  bool have = false;
  for (uint32_t k = 0; k < s.unbounded_count; ++k) {  // nearest_among + closer (scene.rs:222-249)
    if (kCount) cnt->objects++;
    float t;
    uint32_t leaf, prim;
    if (prim_closest<kCsg>(s, __ldg(&s.unbounded[k]), o, d, near, far, t, leaf, prim, err) && (!have || t < min_t)) {
      have = true;
      min_t = t;
      leaf_out = leaf;
      prim_out = prim;
    }
  }
  if (s.top_node_count == 0) {
    if (have) t_out = min_t;
    return have;
  }
  const PRay r = prepare_ray(o, d);
  const float4 rlo = __ldg(&s.top[0]);
  const float4 rhi = __ldg(&s.top[1]);
  float entry;
  if (kCount) cnt->boxes++;
  if (!box_hit(r, rlo, rhi, near, min_t, entry)) {
    if (have) t_out = min_t;
    return have;
  }
  uint32_t stk_lf[kTraceStack], stk_cnt[kTraceStack];
  float stk_e[kTraceStack];
  int sp = 0;
  uint32_t lf = __float_as_uint(rlo.w), count = __float_as_uint(rhi.w);
  float cur_e = entry;
  uint32_t budget = 2u * s.top_node_count + 2u;  // every node is pushed (and popped) at most once
  for (;;) {
    if (budget-- == 0) {
      atomicOr(err, kErrBudget);
      break;
    }
    bool pop = true;
    if (cur_e < min_t) {
      if (kCount) cnt->nodes++;
      if (count > 0) {
        for (uint32_t k = lf; k < lf + count; ++k) {
          if (kCount) cnt->objects++;
          const uint32_t ref = __ldg(&s.order[k]);
          if (ref == skip) continue;
          float t;
          uint32_t leaf, prim;
          if (prim_closest<kCsg>(s, ref, o, d, near, min_t, t, leaf, prim, err) && (!have || t < min_t)) {
            have = true;
            min_t = t;
            leaf_out = leaf;
            prim_out = prim;
          }
        }
      } else {
        float4 l0, l1, r0, r1;
        load_node(&s.top[2 * lf], l0, l1);
        load_node(&s.top[2 * lf + 2], r0, r1);
        float dl, dr;
        if (kCount) cnt->boxes += 2;
        const bool hl = box_hit(r, l0, l1, near, min_t, dl);
        const bool hr = box_hit(r, r0, r1, near, min_t, dr);
        const bool swap = hl && hr && dr < dl;
        const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
        const float dn = swap ? dr : dl, df = swap ? dl : dr;
        if (hf) {
          if (sp >= kTraceStack) {
            atomicOr(err, kErrStack);
            break;
          }
          stk_lf[sp] = __float_as_uint(swap ? l0.w : r0.w);
          stk_cnt[sp] = __float_as_uint(swap ? l1.w : r1.w);
          stk_e[sp] = df;
          ++sp;
        }
        if (hn) {
          lf = __float_as_uint(swap ? r0.w : l0.w);
          count = __float_as_uint(swap ? r1.w : l1.w);
          cur_e = dn;
          pop = false;
        }
      }
    }
    if (pop) {
      if (sp == 0) break;
      --sp;
      lf = stk_lf[sp];
      count = stk_cnt[sp];
      cur_e = stk_e[sp];
    }
  }
  if (have) t_out = min_t;  // the adopted hit's distance (min_t = c.d)
  return have;
}

template <bool kCsg = true>
PBRT_DEV bool scene_closest(const SceneView& s, const F3& o, const F3& d, float near, float far, float& t_out,
                            uint32_t& leaf_out, uint32_t& prim_out, uint32_t* err, uint32_t skip = kNoLeaf) {
  return scene_closest_t<false, kCsg>(s, o, d, near, far, t_out, leaf_out, prim_out, err, nullptr, skip);
}

// Scene::any_hit: the unbounded primitives first; then unordered, the box tested at pop,
// right pushed before left (bvh.rs:269-270).
template <bool kCount, bool kCsg = true>
PBRT_DEV bool scene_any_t(const SceneView& s, const F3& o, const F3& d, float near, float far, uint32_t* err,
                          SceneCount* cnt, uint32_t skip = kNoLeaf) {
  for (uint32_t k = 0; k < s.unbounded_count; ++k) {  // any_blocks (scene.rs:170-184)
    if (kCount) cnt->objects++;
    if (prim_any<kCsg>(s, __ldg(&s.unbounded[k]), o, d, near, far, err)) return true;
  }
  if (s.top_node_count == 0) return false;
  const PRay r = prepare_ray(o, d);
  uint32_t stk[kTraceStack];
  int sp = 0;
  stk[sp++] = 0;
  uint32_t budget = 2u * s.top_node_count + 2u;
  while (sp > 0) {
    if (budget-- == 0) {
      atomicOr(err, kErrBudget);
      return false;
    }
    const uint32_t ni = stk[--sp];
    const float4 lo = __ldg(&s.top[2 * ni]), hi = __ldg(&s.top[2 * ni + 1]);
    float e;
    if (kCount) cnt->boxes++;
    if (!box_hit(r, lo, hi, near, far, e)) continue;
    if (kCount) cnt->nodes++;
    const uint32_t lf = __float_as_uint(lo.w), count = __float_as_uint(hi.w);
    if (count > 0) {
      for (uint32_t k = lf; k < lf + count; ++k) {
        if (kCount) cnt->objects++;
        const uint32_t ref = __ldg(&s.order[k]);
        if (ref != skip && prim_any<kCsg>(s, ref, o, d, near, far, err)) return true;
      }
    } else {
      if (sp + 2 > kTraceStack) {
        atomicOr(err, kErrStack);
        return false;
      }
      stk[sp++] = lf + 1;
      stk[sp++] = lf;
    }
  }
  return false;
}

template <bool kCsg = true>
PBRT_DEV bool scene_any(const SceneView& s, const F3& o, const F3& d, float near, float far, uint32_t* err,
                        uint32_t skip = kNoLeaf) {
  return scene_any_t<false, kCsg>(s, o, d, near, far, err, nullptr, skip);
}

// ---- the interaction of an adopted hit -----------------------------------------------------
PBRT_DEV F3 vtx(const MeshShade& m, uint32_t i) { return mk3(m.v[3 * i], m.v[3 * i + 1], m.v[3 * i + 2]); }

// The material of a hit: the triangle's own when its mesh carries per-face materials.
PBRT_DEV uint32_t material_index(const SceneView& s, uint32_t li, uint32_t prim) {
  const ObjRec& ob = s.objects[li];
  if (ob.shape == kShapeMesh) {
    const uint32_t* fm = s.shade[ob.mesh].fmat;
    if (fm) return fm[prim];
  }
  return ob.material;
}

// AABox face frames (aabox.rs:29-63): normal, du, dv
static __constant__ float kBoxFace[6][9] = {
    {-1.f, 0.f, 0.f, 0.f, 0.f, -1.f, 0.f, 1.f, 0.f}, {1.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f, 1.f, 0.f},
    {0.f, -1.f, 0.f, -1.f, 0.f, 0.f, 0.f, 0.f, 1.f}, {0.f, 1.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 1.f},
    {0.f, 0.f, -1.f, 0.f, -1.f, 0.f, 1.f, 0.f, 0.f}, {0.f, 0.f, 1.f, 0.f, 1.f, 0.f, 1.f, 0.f, 0.f}};

// World-space shading record of leaf `li` hit at distance t (recomputed from the same local
// ray and the same arithmetic as the hit itself). With uv = false the texture coordinates of
// mesh and sphere hits are left 0 (only textured materials read them).
// The record of a hit on a plain shape, in its own frame (the shape's details functions:
// triangle_mesh.rs:73-132, 219-258; sphere.rs:152-187; cylinder.rs:266-344; aabox.rs:165-190;
// rectangle.rs:46-55; plane.rs:31-40).
PBRT_DEV Isect shape_isect(const SceneView& s, uint32_t shape, uint32_t mesh, const float* pr, uint32_t prim,
                           const F3& lo, const F3& ld, float t, bool uv) {
  Isect h;
  h.d = t;
  h.u = 0.f;
  h.v = 0.f;
  h.wo = mul3(ld, -1.f);
  F3 dpdv;
  const float kTwoPi = fm(2.f, 3.14159265358979323846f);
  switch (shape) {
    case kShapeMesh: {
      const MeshShade& m = s.shade[mesh];
      const F3 p0 = vtx(m, m.idx[3 * prim]), p1 = vtx(m, m.idx[3 * prim + 1]), p2 = vtx(m, m.idx[3 * prim + 2]);
      h.p = add3(lo, mul3(ld, t));
      // compute_texture_derivatives with the default uvs (0,0), (1,0), (1,1)
      const float d02x = fs(0.f, 1.f), d02y = fs(0.f, 1.f), d12x = fs(1.f, 1.f), d12y = fs(0.f, 1.f);
      const F3 dp02 = sub3(p0, p2), dp12 = sub3(p1, p2);
      const float det = fs(fm(d12x, d02y), fm(d12y, d02x));
      const float inv = frcp(det);
      h.dpdu = mul3(sub3(mul3(dp12, d02y), mul3(dp02, d12y)), inv);
      dpdv = mul3(sub3(mul3(dp02, d12x), mul3(dp12, d02x)), inv);
      h.n = normalize3(cross3(dpdv, h.dpdu));
      if (uv) {  // interpolate_texture_coords (triangle_mesh.rs:219-224) from Möller–Trumbore's u, v
        const F3 e1 = sub3(p1, p0), e2 = sub3(p2, p0);
        const F3 pv = cross3(ld, e2);
        const float idet = frcp(dot3(e1, pv));
        const F3 sv = sub3(lo, p0);
        const float bu = fm(idet, dot3(sv, pv));
        const float bv = fm(idet, dot3(ld, cross3(sv, e1)));
        const float bw = fs(fs(1.f, bu), bv);
        h.u = fa(fa(fm(bw, 0.f), fm(bu, 1.f)), fm(bv, 1.f));
        h.v = fa(fa(fm(bw, 0.f), fm(bu, 0.f)), fm(bv, 1.f));
      }
      break;
    }
    case kShapeSphere: {
      const F3 hit = add3(lo, mul3(ld, t));
      h.p = hit;
      h.n = normalize3(hit);
      h.dpdu = mul3(mk3(-hit.y, hit.x, 0.f), kTwoPi);
      dpdv = mk3(0.f, 0.f, 0.f);  // not used by the shading frame
      if (uv) {  // compute_intersection_details (sphere.rs:152-172)
        float phi = atan2f(hit.y, hit.x);
        if (phi < 0.f) phi = fa(phi, kTwoPi);
        h.u = fdv(phi, kTwoPi);
        const float theta = acosf(fminf(fmaxf(fdv(hit.z, pr[0]), -1.f), 1.f));
        h.v = fdv(theta, 3.14159265358979323846f);
      }
      break;
    }
    case kShapeCylinder: {
      const F3 p = add3(lo, mul3(ld, t));
      h.p = p;
      dpdv = mk3(0.f, 1.f, 0.f);
      const uint32_t piece = prim;  // the piece: 0 wall, 1 bottom cap, 2 top cap
      if (piece == 0) {
        h.n = normalize3(mk3(p.x, 0.f, p.z));
        h.dpdu = mul3(mk3(-p.z, 0.f, p.x), kTwoPi);
        if (uv) {
          float phi = atan2f(p.z, p.x);
          if (phi < 0.f) phi = fa(phi, kTwoPi);
          h.u = fdv(phi, kTwoPi);
          h.v = p.y;
        }
      } else {
        const bool top = piece == 2;
        h.n = mk3(0.f, top ? 1.f : -1.f, 0.f);
        h.dpdu = mk3(top ? 1.f : -1.f, 0.f, 0.f);
        h.u = p.x;
        h.v = p.z;
      }
      break;
    }
    case kShapeAABox: {
      const float* f = kBoxFace[prim < 6 ? prim : 0];
      const F3 p = add3(lo, mul3(ld, t));
      h.p = p;
      h.n = mk3(f[0], f[1], f[2]);
      h.dpdu = mk3(f[3], f[4], f[5]);
      dpdv = mk3(f[6], f[7], f[8]);
      h.u = dot3(p, h.dpdu);
      h.v = dot3(p, dpdv);
      break;
    }
    default: {  // rectangle, plane: p on y = 0, n = +y, u = p.x, v = p.z
      F3 p = add3(lo, mul3(ld, t));
      p.y = 0.f;
      h.p = p;
      h.n = mk3(0.f, 1.f, 0.f);
      h.dpdu = mk3(1.f, 0.f, 0.f);
      dpdv = mk3(0.f, 0.f, 1.f);
      h.u = p.x;
      h.v = p.z;
      break;
    }
  }
  (void)dpdv;
  return h;
}

// World-space shading record of leaf `li` hit at distance t (recomputed from the same local
// ray and the same arithmetic as the hit itself). With uv = false the texture coordinates of
// mesh and sphere hits are left 0 (only textured materials read them).
PBRT_DEV Isect interaction(const SceneView& s, uint32_t li, uint32_t prim, const F3& o, const F3& d, float t,
                           bool uv = false) {
  const ObjRec& ob = s.objects[li];
  F3 lo, ld;
  local_ray(s, ob, o, d, lo, ld);
  Isect h;
  if (ob.shape == kShapeCsg) {  // the element's record, moved out of the element (csg/*.rs)
    const uint32_t e = prim >> 24;
    const CsgRec& E = s.csg[ob.csg_first + e];
    const F3 elo = xf_point(E.to_local, lo);
    const F3 eld = normalize3(xf_dir(E.to_local, ld));
    h = shape_isect(s, E.shape, E.mesh, E.p, prim & 0xFFFFFFu, elo, eld, t, uv);
    h.n = xf_normal(E.to_local, h.n);
    h.p = xf_point(E.to_world, h.p);
    h.wo = xf_dir(E.to_world, h.wo);
    h.dpdu = xf_dir(E.to_world, h.dpdu);
    if (ob.csg_op == kCsgSubtraction && e > 0) h.n = mul3(h.n, -1.f);  // substraction.rs:73-76
  } else {
    h = shape_isect(s, ob.shape, ob.mesh, ob.p, prim, lo, ld, t, uv);
  }
  // transform_interaction_to_world (transform.rs:105-116), innermost level first
  for (uint32_t k = ob.xf_count; k-- > 0;) {
    const float* w = leaf_to_world(s, ob, k);
    h.n = xf_normal(leaf_to_local(s, ob, k), h.n);
    h.p = xf_point(w, h.p);
    h.wo = xf_dir(w, h.wo);
    h.dpdu = xf_dir(w, h.dpdu);
  }
  return h;
}

// Texture::shade at a hit: PlainColor, or CheckerBoard::shade (checker_board.rs:17-28) on the
// record's u, v (`%` is fmod, exact; signum(+-0) = +-1).
PBRT_DEV F3 texel(const MatRec& m, const Isect& it) {
  if (m.texture == kTexColor) return mk3(m.color[0], m.color[1], m.color[2]);
  const float su = fmodf(fm(fabsf(it.u), m.scale), 1.f);
  const float sv = fmodf(fm(fabsf(it.v), m.scale), 1.f);
  const bool use_color = (su < 0.5f && sv < 0.5f) || (su >= 0.5f && sv >= 0.5f);
  const bool positive = !isnan(it.u) && !isnan(it.v) && fm(copysignf(1.f, it.u), copysignf(1.f, it.v)) >= 0.f;
  return (use_color != positive) ? mk3(m.color[0], m.color[1], m.color[2]) : mk3(m.color2[0], m.color2[1], m.color2[2]);
}

// Shading frame: ss = normalize(dpdu), ts = n x ss, ns = n (intersectable.rs:92-144)
PBRT_DEV F3 to_local(const Isect& it, const F3& w) {
  const F3 ss = normalize3(it.dpdu);
  const F3 ts = cross3(it.n, ss);
  return mk3(dot3(ss, w), dot3(ts, w), dot3(it.n, w));
}
PBRT_DEV F3 to_world(const Isect& it, const F3& l) {
  const F3 ss = normalize3(it.dpdu);
  const F3 ts = cross3(it.n, ss);
  return mk3(fa(fa(fm(ss.x, l.x), fm(ts.x, l.y)), fm(it.n.x, l.z)), fa(fa(fm(ss.y, l.x), fm(ts.y, l.y)), fm(it.n.y, l.z)),
             fa(fa(fm(ss.z, l.x), fm(ts.z, l.y)), fm(it.n.z, l.z)));
}

}  // namespace pbrt
