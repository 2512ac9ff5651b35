// scene_device.cuh — the scene on the GPU: objects, the top-level BVH over them, the
// analytic shapes, and the interaction (shading record) of a hit.
//
// Semantics follow the reference operation for operation (FP32, no FMA):
//   Scene::find_nearest + BVH::query      src/scene.rs:186-220, src/bvh.rs:153-230
//   Scene::any_hit + BVH::query_p         src/scene.rs:157-168, src/bvh.rs:239-275
//   Transformed::intersect / intersect_p  src/objects/transformed.rs:27-38, 62-65
//   Simple::intersect (first listed hit)  src/objects/simple.rs:28-41
//   Sphere::intersect + details           src/shapes/sphere.rs:108-187
//   Cylinder::intersect + details         src/shapes/cylinder.rs:28-110, 324-344
//   TriangleMesh::intersect post-hit      src/shapes/triangle_mesh/triangle_mesh.rs:73-132, 219-258
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
  const float4* top;        // top-level BVH nodes (GPU numbering, 2 float4 per node)
  uint32_t top_node_count;
  const uint32_t* order;    // leaf slot -> object index
  const ObjRec* objects;
  const MeshView* meshes;   // traversal views
  const MeshShade* shade;   // shading views
  const MatRec* materials;
  const LightRec* lights;
  uint32_t light_count;
  const float* light_tris;  // area lights: 9 floats per world-space triangle
  const float* light_cdf;   // running area per triangle
};

struct Isect {
  F3 p, n, wo, dpdu;
  float d;
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

// The object's local ray: transform_ray_to_local renormalises (transform.rs:98-103, ray.rs:10-18).
PBRT_DEV void local_ray(const ObjRec& ob, const F3& o, const F3& d, F3& lo, F3& ld) {
  if (ob.transformed) {
    lo = xf_point(ob.to_local, o);
    ld = normalize3(xf_dir(ob.to_local, d));
  } else {
    lo = o;
    ld = d;
  }
}

// Object::intersect distance within [near, far]; prim = triangle index (0 for analytic).
PBRT_DEV bool object_closest(const SceneView& s, uint32_t oi, const F3& o, const F3& d, float near, float far,
                             float& t, uint32_t& prim, uint32_t* err) {
  const ObjRec& ob = s.objects[oi];
  F3 lo, ld;
  local_ray(ob, o, d, lo, ld);
  if (ob.shape == kShapeMesh) {
    const PRay r = prepare_ray(lo, ld);
    TraceCounters c;
    const uint32_t id = mesh_closest<false>(s.meshes[ob.mesh], r, near, far, &t, &c, err);
    prim = id;
    return id != 0xFFFFFFFFu;
  }
  prim = 0;
  if (ob.shape == kShapeSphere) return sphere_hit(ob.radius, lo, ld, near, far, t);
  int piece = 0;
  const bool hit = cylinder_hit(ob.radius, ob.half_height, lo, ld, near, far, t, piece);
  prim = uint32_t(piece);  // cylinders report which piece was hit: 0 wall, 1 bottom cap, 2 top cap
  return hit;
}

PBRT_DEV bool object_any(const SceneView& s, uint32_t oi, const F3& o, const F3& d, float near, float far,
                         uint32_t* err) {
  const ObjRec& ob = s.objects[oi];
  F3 lo, ld;
  local_ray(ob, o, d, lo, ld);
  if (ob.shape == kShapeMesh) return mesh_any(s.meshes[ob.mesh], prepare_ray(lo, ld), near, far, err);
  float t;
  if (ob.shape == kShapeSphere) return sphere_hit(ob.radius, lo, ld, near, far, t);
  int piece;
  return cylinder_hit(ob.radius, ob.half_height, lo, ld, near, far, t, piece);
}

// Scene::find_nearest: the top-level query narrows its interval to every adopted hit and
// offers each object [near, min_t]; a candidate is adopted only when strictly nearer.
PBRT_DEV bool scene_closest(const SceneView& s, const F3& o, const F3& d, float near, float far, float& t_out,
                            uint32_t& obj_out, uint32_t& prim_out, uint32_t* err) {
  const PRay r = prepare_ray(o, d);
  float min_t = far;
  bool have = false;
  const float4 rlo = __ldg(&s.top[0]);
  const float4 rhi = __ldg(&s.top[1]);
  float entry;
  if (!box_hit(r, rlo, rhi, near, min_t, entry)) return false;
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
      if (count > 0) {
        for (uint32_t k = lf; k < lf + count; ++k) {
          const uint32_t oi = __ldg(&s.order[k]);
          float t;
          uint32_t prim;
          if (object_closest(s, oi, o, d, near, min_t, t, prim, err) && (!have || t < min_t)) {
            have = true;
            min_t = t;
            obj_out = oi;
            prim_out = prim;
          }
        }
      } else {
        const float4 l0 = __ldg(&s.top[2 * lf]), l1 = __ldg(&s.top[2 * lf + 1]);
        const float4 r0 = __ldg(&s.top[2 * lf + 2]), r1 = __ldg(&s.top[2 * lf + 3]);
        float dl, dr;
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

// Scene::any_hit: unordered, the box tested at pop, right pushed before left (bvh.rs:269-270).
PBRT_DEV bool scene_any(const SceneView& s, const F3& o, const F3& d, float near, float far, uint32_t* err) {
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
    if (!box_hit(r, lo, hi, near, far, e)) continue;
    const uint32_t lf = __float_as_uint(lo.w), count = __float_as_uint(hi.w);
    if (count > 0) {
      for (uint32_t k = lf; k < lf + count; ++k)
        if (object_any(s, __ldg(&s.order[k]), o, d, near, far, err)) return true;
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

// ---- the interaction of an adopted hit -----------------------------------------------------
PBRT_DEV F3 vtx(const MeshShade& m, uint32_t i) { return mk3(m.v[3 * i], m.v[3 * i + 1], m.v[3 * i + 2]); }

// World-space shading record of object `oi` hit at distance t (recomputed from the same
// local ray and the same arithmetic as the hit itself).
// The material of a hit: the triangle's own when its mesh carries per-face materials.
PBRT_DEV uint32_t material_index(const SceneView& s, uint32_t oi, uint32_t prim) {
  const ObjRec& ob = s.objects[oi];
  if (ob.shape == kShapeMesh) {
    const uint32_t* fm = s.shade[ob.mesh].fmat;
    if (fm) return fm[prim];
  }
  return ob.material;
}

PBRT_DEV Isect interaction(const SceneView& s, uint32_t oi, uint32_t prim, const F3& o, const F3& d, float t) {
  const ObjRec& ob = s.objects[oi];
  F3 lo, ld;
  local_ray(ob, o, d, lo, ld);
  Isect h;
  h.d = t;
  F3 dpdv;
  if (ob.shape == kShapeMesh) {
    const MeshShade& m = s.shade[ob.mesh];
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
    h.wo = mul3(ld, -1.f);
  } else if (ob.shape == kShapeSphere) {
    const F3 hit = add3(lo, mul3(ld, t));
    h.p = hit;
    h.n = normalize3(hit);
    h.dpdu = mul3(mk3(-hit.y, hit.x, 0.f), fm(2.f, 3.14159265358979323846f));
    dpdv = mk3(0.f, 0.f, 0.f);  // not used by the shading frame
    h.wo = mul3(ld, -1.f);
  } else {
    const F3 p = add3(lo, mul3(ld, t));
    h.p = p;
    h.wo = mul3(ld, -1.f);
    dpdv = mk3(0.f, 1.f, 0.f);
    const uint32_t piece = prim;  // object_closest reports the piece in prim
    if (piece == 0) {
      h.n = normalize3(mk3(p.x, 0.f, p.z));
      h.dpdu = mul3(mk3(-p.z, 0.f, p.x), fm(2.f, 3.14159265358979323846f));
    } else {
      const bool top = piece == 2;
      h.n = mk3(0.f, top ? 1.f : -1.f, 0.f);
      h.dpdu = mk3(top ? 1.f : -1.f, 0.f, 0.f);
    }
  }
  if (ob.transformed) {  // transform_interaction_to_world (transform.rs:105-116)
    h.n = xf_normal(ob.to_local, h.n);
    h.p = xf_point(ob.to_world, h.p);
    h.wo = xf_dir(ob.to_world, h.wo);
    h.dpdu = xf_dir(ob.to_world, h.dpdu);
  }
  return h;
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
