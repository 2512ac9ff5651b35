// pbrt_oracle_pt.hpp — TEST INFRASTRUCTURE, NOT THE PRODUCT.
//
// The scene-level half of the CPU oracle: objects (Simple / Transformed), analytic shapes,
// the scene BVH, materials, lights, the sampler and the path integrator, restated from
// nmichel/pbrt in the reference's operation order (citations are path:line there).
//
// Extensions the reference plans but does not implement, written from its own notes:
//   - AreaLight NEE (ideas/area_light.md §2-§6): uniform area sampling, p(ω) = p(A)·d²/|cosθ_l|,
//     zero pdf → no sample; emission is two-sided, as DiffuseLight::emit is
//     (src/materials/diffuse_light.rs:18-22); the shadow ray stops at (1 - 1e-4)·d so the
//     sampled point's own surface does not occlude it. The specular guard of path.rs:58 is kept.
//   - Russian roulette in the commented form of path.rs:92-101, from bounce `rr_start`, with
//     q clamped to 1 (without the clamp a path with max(β) > 1 would be scaled down, a bias).
//   - A seeded sampler (ideas/rng_graine.md §7-§8): PCG32, one stream per pixel, re-keyed per
//     (pixel, sample); a uniform draw is the top 24 bits of one output times 2^-24.
//   - The naive estimator (src/integrators/naive.rs:29-52) with the scene's infinite lights as
//     its background instead of the hard-coded sky, so naive and path integrate the same scene
//     (the cross-check ideas/area_light.md:131-136 asks for).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <memory>
#include <stdexcept>
#include <vector>

#include "pbrt_oracle.hpp"

namespace oracle {

// ---------------------------------------------------------------------------------------
// Sampler
// ---------------------------------------------------------------------------------------
struct Pcg32 {
  uint64_t state = 0, inc = 1;
  uint32_t next() {
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = uint32_t(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  void seed(uint64_t initstate, uint64_t initseq) {
    state = 0;
    inc = (initseq << 1u) | 1u;
    next();
    state += initstate;
    next();
  }
  float uniform() { return float(next() >> 8) * (1.0f / 16777216.0f); }
};

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// One stream per pixel, re-keyed per (pixel, sample).
inline Pcg32 path_rng(uint64_t seed, uint32_t pixel, uint32_t sample) {
  Pcg32 r;
  r.seed(splitmix64(seed ^ splitmix64((uint64_t(pixel) << 32) | sample)), pixel);
  return r;
}

template <class R> struct Consts {
  static R pi() { return R(3.141592653589793238462643383279502884L); }
};

// ---------------------------------------------------------------------------------------
// Intersection record — src/geom/intersectable.rs:8-28, 92-144
// ---------------------------------------------------------------------------------------
template <class R>
struct Isect {
  V3<R> p, n, wo, dpdu, dpdv;
  R d, u, v;
  // world_to_local / local_to_world: ss = normalize(dpdu), ts = n x ss, ns = n
  V3<R> to_local(const V3<R>& w) const {
    V3<R> ss = normalized(dpdu);
    V3<R> ts = cross(n, ss);
    return V3<R>{dot(ss, w), dot(ts, w), dot(n, w)};
  }
  V3<R> to_world(const V3<R>& l) const {
    V3<R> ss = normalized(dpdu);
    V3<R> ts = cross(n, ss);
    return V3<R>{ss.x * l.x + ts.x * l.y + n.x * l.z, ss.y * l.x + ts.y * l.y + n.y * l.z,
                 ss.z * l.x + ts.z * l.y + n.z * l.z};
  }
};

// 3x4 affine matrix (the bottom row of every Transform on the path is 0 0 0 1, so the
// `w != 1` division of Matrix4::transform_point never triggers).
template <class R>
struct Affine {
  R m[3][4];
  V3<R> point(const V3<R>& v) const {
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z + m[0][3], m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z + m[1][3],
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z + m[2][3]};
  }
  V3<R> direction(const V3<R>& v) const {
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
  }
  // transform_normal multiplies by the transpose (matrix4.rs:208-213)
  V3<R> normal(const V3<R>& v) const {
    return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
            m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
  }
};

// ---------------------------------------------------------------------------------------
// Scene description (the oracle's own POD; tests lower one scene into it and into the
// product's C description)
// ---------------------------------------------------------------------------------------
enum { O_SHAPE_MESH = 0, O_SHAPE_SPHERE = 1, O_SHAPE_CYLINDER = 2, O_SHAPE_RECTANGLE = 3, O_SHAPE_AABOX = 4,
       O_SHAPE_PLANE = 5, O_SHAPE_CSG = 6 };
enum { O_CSG_UNION = 0, O_CSG_INTERSECTION = 1, O_CSG_SUBTRACTION = 2 };
enum { O_MAT_LAMBERTIAN = 0, O_MAT_METAL = 1, O_MAT_DIELECTRIC = 2, O_MAT_DIFFUSE_LIGHT = 3 };
enum { O_LIGHT_POINT = 0, O_LIGHT_UNIFORM = 1, O_LIGHT_BACKGROUND = 2, O_LIGHT_AREA = 3 };
enum { O_TEX_PLAIN = 0, O_TEX_CHECKERBOARD = 1 };
enum { O_NODE_SIMPLE = 0, O_NODE_TRANSFORMED = 1, O_NODE_COMPOUND = 2 };

struct OMeshDesc {
  const float* vertices;
  uint32_t vertex_count;
  const uint32_t* indices;
  uint32_t triangle_count;
  const uint32_t* face_materials;  // optional per-triangle material (an extension of the reference)
};
struct OMaterialDesc {
  uint32_t kind;
  float color[3];
  float fuzz, ior;
  uint32_t texture;  // O_TEX_*: PlainColor(color) or CheckerBoard(color, color2, scale)
  float color2[3];
  float scale;
};
// A Simple(shape, material) object, optionally wrapped in one Transformed. Sizes are the
// reference's constructor arguments: sphere radius; cylinder radius, height; rectangle
// width, height; aabox extent (full sizes; the shapes halve them).
struct OObjectDesc {
  uint32_t shape, mesh;
  double radius, height;
  double extent[3];
  uint32_t material, transformed;
  double to_world[12], to_local[12];
  uint32_t csg_op, csg_first, csg_count;  // O_SHAPE_CSG: csg_elems[csg_first .. + csg_count)
};
// One element of a constructive solid (csg::Elem, src/shapes/csg.rs:7-10): a shape (any but
// O_SHAPE_CSG) placed by its transform.
struct OCsgElemDesc {
  uint32_t shape, mesh;
  double radius, height;
  double extent[3];
  double to_world[12], to_local[12];
};
// Object tree of a scene file (src/objects/*.rs): SIMPLE names an object; TRANSFORMED wraps
// children[first]; COMPOUND holds children[first .. first + count).
struct ONodeDesc {
  uint32_t kind, object, first, count;
  double to_world[12], to_local[12];
};
struct OLightDesc {
  uint32_t kind;
  float position[3], radiance[3], bottom[3], top[3];
  uint32_t object;
};
struct OSceneDesc {
  const OMeshDesc* meshes;
  uint32_t mesh_count;
  const OMaterialDesc* materials;
  uint32_t material_count;
  const OObjectDesc* objects;
  uint32_t object_count;
  const OLightDesc* lights;
  uint32_t light_count;
  uint32_t bvh_bins, bvh_max_leaf;
  // Optional tree (nodes == NULL: every object is one primitive of the scene, in order).
  const ONodeDesc* nodes;
  uint32_t node_count;
  const uint32_t* children;
  uint32_t child_count;
  const uint32_t* roots;  // the scene's primitives in Scene::add_object order
  uint32_t root_count;
  const OCsgElemDesc* csg_elems;
  uint32_t csg_elem_count;
};
struct OCameraDesc {
  uint32_t width, height;
  double fov, near, far;
  double position[3], look_at[3], up[3];
  uint32_t thin_lens;  // 1: ThinLensCamera with the two values below
  double lens_radius, focal_distance;
};
struct ORenderParams {
  OCameraDesc camera;
  uint32_t spp, max_depth, rr_start, sample_offset;
  uint64_t seed;
  uint32_t integrator;  // 0 path, 1 naive
};

// Ends paths into a radiance cache: at hit number >= term_hit on a Lambertian or metal
// surface the path takes no light sample, adds beta * max(query(record), 0) and stops. The
// record is 16 floats: p, roughness (fuzz; 1 for Lambertian), wo, 0, the normal turned to
// face wo, 0, albedo, 0.
struct CacheHook {
  uint32_t term_hit;
  float max_radiance;  // answers are clamped to [0, max_radiance]
  std::function<void(const float* rec, float* rgb)> query;
};

// ---------------------------------------------------------------------------------------
// Scene
// ---------------------------------------------------------------------------------------
// Work counters of a scene query (TraversalStats as Scene::intersect_instrumented and
// Scene::intersect_p_instrumented fill them: src/scene.rs:124-153, src/bvh.rs:153-275).
struct SceneStats {
  uint64_t nodes_visited = 0, box_tests = 0, object_tests = 0;
};

// The work of a render, summed over its scene queries (for the render path's algorithmic
// bytes): rays and shadow rays traced, top-level box tests and objects tested, the meshes'
// own box and triangle tests, and analytic shape tests (spheres, cylinders, rectangles,
// boxes, planes, solids). A render thread points work_tally at its own tally.
struct WorkTally {
  uint64_t rays = 0, shadow_rays = 0, top_boxes = 0, objects = 0, mesh_boxes = 0, triangles = 0, shapes = 0;
  void add(const WorkTally& o) {
    rays += o.rays; shadow_rays += o.shadow_rays; top_boxes += o.top_boxes; objects += o.objects;
    mesh_boxes += o.mesh_boxes; triangles += o.triangles; shapes += o.shapes;
  }
};
inline thread_local WorkTally* work_tally = nullptr;

template <class R>
class OScene {
 public:
  struct Mesh {
    std::unique_ptr<MeshBVH<R>> bvh;
    std::vector<R> v;
    std::vector<uint32_t> idx;
    std::vector<uint32_t> fmat;  // empty: the object's material
  };
  struct Object {
    uint32_t shape, mesh, material;
    R radius, height, half_height;  // sphere, cylinder
    R half_w, half_h;               // rectangle (Rectangle::new halves width and height)
    V3<R> amin, amax;               // aabox (AABox::new: min = 0 - extent/2, max = extent/2)
    bool transformed;
    Affine<R> mat, inv;
    uint32_t csg_op = 0, csg_first = 0, csg_count = 0;
  };
  struct Material {
    uint32_t kind;
    V3<R> color;
    R fuzz, ior;
    uint32_t texture;
    V3<R> color2;
    R scale;
  };
  struct Light {
    uint32_t kind;
    V3<R> pos, rad, bottom, top;
    uint32_t object;
    // area lights: world-space triangles (mesh) and their area CDF, or the sphere's centre/radius
    std::vector<V3<R>> tp;  // 3 per triangle
    std::vector<R> cdf;     // running sum of areas
    R area = R(0);
  };
  struct Node {
    uint32_t kind, object;
    std::vector<uint32_t> kids;
    Affine<R> mat, inv;
  };
  struct BNode {
    AABB<R> box;
    uint32_t left_first, count;
  };

  static Affine<R> affine(const double* m) {
    Affine<R> a;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) a.m[r][c] = R(m[4 * r + c]);
    return a;
  }

  explicit OScene(const OSceneDesc& d) {
    for (uint32_t i = 0; i < d.mesh_count; ++i) {
      const OMeshDesc& md = d.meshes[i];
      Mesh m;
      m.v.assign(md.vertices, md.vertices + 3 * size_t(md.vertex_count));
      m.idx.assign(md.indices, md.indices + 3 * size_t(md.triangle_count));
      if (md.face_materials) m.fmat.assign(md.face_materials, md.face_materials + md.triangle_count);
      m.bvh.reset(new MeshBVH<R>(m.v.data(), md.vertex_count, m.idx.data(), md.triangle_count,
                                 d.bvh_bins ? int(d.bvh_bins) : 8, d.bvh_max_leaf ? d.bvh_max_leaf : 1));
      meshes.push_back(std::move(m));
    }
    for (uint32_t i = 0; i < d.material_count; ++i) {
      const OMaterialDesc& m = d.materials[i];
      Material mm{m.kind, V3<R>{R(m.color[0]), R(m.color[1]), R(m.color[2])}, R(m.fuzz), R(m.ior), m.texture,
                  V3<R>{R(m.color2[0]), R(m.color2[1]), R(m.color2[2])}, R(m.scale)};
      if (m.texture > O_TEX_CHECKERBOARD) throw std::invalid_argument("unknown texture");
      materials.push_back(mm);
      if (m.kind == O_MAT_DIFFUSE_LIGHT)
        for (int c = 0; c < 3; ++c) {
          max_radiance = std::max(max_radiance, m.color[c]);
          if (m.texture == O_TEX_CHECKERBOARD) max_radiance = std::max(max_radiance, m.color2[c]);
        }
    }
    for (uint32_t i = 0; i < d.csg_elem_count; ++i) {
      const OCsgElemDesc& e = d.csg_elems[i];
      Object ob = shape_object(e.shape, e.mesh, e.radius, e.height, e.extent);
      ob.transformed = true;
      ob.mat = affine(e.to_world);
      ob.inv = affine(e.to_local);
      if (ob.shape > O_SHAPE_PLANE) throw std::invalid_argument("a csg element is a plain shape");
      celems.push_back(ob);
    }
    for (uint32_t i = 0; i < d.object_count; ++i) {
      const OObjectDesc& o = d.objects[i];
      Object ob = shape_object(o.shape, o.mesh, o.radius, o.height, o.extent);
      ob.material = o.material;
      ob.transformed = o.transformed != 0;
      ob.mat = affine(o.to_world);
      ob.inv = affine(o.to_local);
      ob.csg_op = o.csg_op;
      ob.csg_first = o.csg_first;
      ob.csg_count = o.csg_count;
      if (ob.shape > O_SHAPE_CSG) throw std::invalid_argument("unknown shape");
      if (ob.shape == O_SHAPE_CSG &&
          (o.csg_op > O_CSG_SUBTRACTION || uint64_t(o.csg_first) + o.csg_count > celems.size()))
        throw std::invalid_argument("bad csg object");
      if (ob.material >= materials.size()) throw std::invalid_argument("bad material index");
      objects.push_back(ob);
    }
    if (d.nodes) {
      for (uint32_t i = 0; i < d.node_count; ++i) {
        const ONodeDesc& nd = d.nodes[i];
        Node n{};
        n.kind = nd.kind;
        n.object = nd.object;
        if (nd.kind == O_NODE_SIMPLE) {
          if (nd.object >= objects.size()) throw std::invalid_argument("node names no object");
        } else if (nd.kind == O_NODE_TRANSFORMED || nd.kind == O_NODE_COMPOUND) {
          const uint32_t cnt = nd.kind == O_NODE_TRANSFORMED ? 1u : nd.count;
          if (uint64_t(nd.first) + cnt > d.child_count) throw std::invalid_argument("node children out of range");
          for (uint32_t k = 0; k < cnt; ++k) {
            if (d.children[nd.first + k] >= d.node_count) throw std::invalid_argument("bad child node");
            n.kids.push_back(d.children[nd.first + k]);
          }
          n.mat = affine(nd.to_world);
          n.inv = affine(nd.to_local);
        } else {
          throw std::invalid_argument("unknown node kind");
        }
        nodes.push_back(std::move(n));
      }
      for (uint32_t i = 0; i < d.root_count; ++i) {
        if (d.roots[i] >= nodes.size()) throw std::invalid_argument("bad root node");
        roots.push_back(d.roots[i]);
      }
      check_acyclic();
    } else {
      for (uint32_t i = 0; i < objects.size(); ++i) {
        Node n{};
        n.kind = O_NODE_SIMPLE;
        n.object = i;
        nodes.push_back(n);
        roots.push_back(i);
      }
    }
    for (uint32_t i = 0; i < d.light_count; ++i) {
      const OLightDesc& l = d.lights[i];
      Light L;
      L.kind = l.kind;
      L.pos = {R(l.position[0]), R(l.position[1]), R(l.position[2])};
      L.rad = {R(l.radiance[0]), R(l.radiance[1]), R(l.radiance[2])};
      L.bottom = {R(l.bottom[0]), R(l.bottom[1]), R(l.bottom[2])};
      L.top = {R(l.top[0]), R(l.top[1]), R(l.top[2])};
      L.object = l.object;
      if (L.kind == O_LIGHT_AREA) setup_area(L);
      lights.push_back(L);
      if (l.kind == O_LIGHT_POINT) max_radiance = std::numeric_limits<float>::infinity();
      for (int c = 0; c < 3; ++c) {
        if (l.kind == O_LIGHT_UNIFORM) max_radiance = std::max(max_radiance, l.radiance[c]);
        if (l.kind == O_LIGHT_BACKGROUND) max_radiance = std::max(max_radiance, std::max(l.bottom[c], l.top[c]));
      }
    }
    commit();
  }

  Object shape_object(uint32_t shape, uint32_t mesh, double radius, double height, const double* extent) const {
    Object ob{};
    ob.shape = shape;
    ob.mesh = mesh;
    ob.radius = R(radius);
    ob.height = R(height);
    ob.half_height = R(height) / R(2);  // Cylinder::new (cylinder.rs:12-19)
    ob.half_w = R(radius) / R(2);       // Rectangle::new(width, height) (rectangle.rs:15-20)
    ob.half_h = R(height) / R(2);
    const V3<R> half = V3<R>{R(extent[0]), R(extent[1]), R(extent[2])} * R(0.5);  // AABox::new
    ob.amin = V3<R>{R(0), R(0), R(0)} - half;
    ob.amax = half;
    if (shape == O_SHAPE_MESH && mesh >= meshes.size()) throw std::invalid_argument("bad mesh index");
    return ob;
  }

  // A node may be shared (the reference holds objects in Arc), but the tree may not loop.
  void check_acyclic() const {
    std::vector<int> state(nodes.size(), 0);
    std::function<void(uint32_t)> walk = [&](uint32_t n) {
      if (state[n] == 1) throw std::invalid_argument("object tree has a cycle");
      if (state[n] == 2) return;
      state[n] = 1;
      for (uint32_t k : nodes[n].kids) walk(k);
      state[n] = 2;
    };
    for (uint32_t r : roots) walk(r);
  }

  // ---- bounds (src/geom/aabound.rs, the AABound impls of src/shapes and src/objects) -----
  // AABoundingBox::transform (aabound.rs:437-468): the eight corners; unbounded stays unbounded
  static AABB<R> transform_box(const AABB<R>& b, const Affine<R>& m) {
    if (!b.is_bounded()) {
      const R inf = std::numeric_limits<R>::infinity();
      return AABB<R>{{-inf, -inf, -inf}, {inf, inf, inf}};
    }
    const V3<R> mn = b.bmin, mx = b.bmax;
    const V3<R> c[8] = {{mn.x, mn.y, mn.z}, {mn.x, mn.y, mx.z}, {mn.x, mx.y, mn.z}, {mn.x, mx.y, mx.z},
                        {mx.x, mx.y, mx.z}, {mx.x, mx.y, mn.z}, {mx.x, mn.y, mx.z}, {mx.x, mn.y, mn.z}};
    AABB<R> t = AABB<R>::empty();
    for (int k = 0; k < 8; ++k) {
      const V3<R> p = m.point(c[k]);
      t.bmin = {rmin(t.bmin.x, p.x), rmin(t.bmin.y, p.y), rmin(t.bmin.z, p.z)};
      t.bmax = {rmax(t.bmax.x, p.x), rmax(t.bmax.y, p.y), rmax(t.bmax.z, p.z)};
    }
    return t;
  }

  AABB<R> shape_box(const Object& o) const {
    const R inf = std::numeric_limits<R>::infinity();
    switch (o.shape) {
      case O_SHAPE_MESH: return meshes[o.mesh].bvh->vertex_bounds();
      case O_SHAPE_SPHERE: return AABB<R>{{-o.radius, -o.radius, -o.radius}, {o.radius, o.radius, o.radius}};
      case O_SHAPE_CYLINDER:
        return AABB<R>{{-o.radius, -o.half_height, -o.radius}, {o.radius, o.half_height, o.radius}};
      case O_SHAPE_RECTANGLE: return AABB<R>{{-o.half_w, R(0), -o.half_h}, {o.half_w, R(0), o.half_h}};
      case O_SHAPE_AABOX: return AABB<R>{o.amin, o.amax};
      case O_SHAPE_CSG: return csg_box(o);
      default: return AABB<R>{{-inf, -inf, -inf}, {inf, R(0), inf}};  // Plane (plane.rs:89-93)
    }
  }

  // get_bounding_box of a constructive solid: Union the union of its elements' boxes
  // (union.rs:56-70), Intersection their intersection (intersection.rs:57-71), Subtraction the
  // first element's (substraction.rs:97-108); no element: the point box at the origin
  AABB<R> csg_box(const Object& o) const {
    if (o.csg_count == 0) return AABB<R>{{R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
    const Object& e0 = celems[o.csg_first];
    AABB<R> b = transform_box(shape_box(e0), e0.mat);
    if (o.csg_op == O_CSG_SUBTRACTION) return b;
    for (uint32_t k = 1; k < o.csg_count; ++k) {
      const Object& e = celems[o.csg_first + k];
      const AABB<R> x = transform_box(shape_box(e), e.mat);
      if (o.csg_op == O_CSG_UNION) {
        b.combine(x);
      } else {  // intersect_with (aabound.rs:397-401): maximize the mins, minimize the maxes
        b.bmin = {rmax(b.bmin.x, x.bmin.x), rmax(b.bmin.y, x.bmin.y), rmax(b.bmin.z, x.bmin.z)};
        b.bmax = {rmin(b.bmax.x, x.bmax.x), rmin(b.bmax.y, x.bmax.y), rmin(b.bmax.z, x.bmax.z)};
      }
    }
    return b;
  }

  // contain_point of a plain shape: sphere.rs:146-148, cylinder.rs:119-124, aabox.rs:192-199,
  // plane.rs:47-52; a rectangle and a mesh enclose nothing
  static bool contains(const Object& s, const V3<R>& p) {
    switch (s.shape) {
      case O_SHAPE_SPHERE: return dot(p, p) <= s.radius * s.radius;
      case O_SHAPE_CYLINDER:
        return p.x * p.x + p.z * p.z <= s.radius * s.radius && p.y >= -s.half_height && p.y <= s.half_height;
      case O_SHAPE_AABOX:
        return p.x >= s.amin.x && p.x <= s.amax.x && p.y >= s.amin.y && p.y <= s.amax.y && p.z >= s.amin.z &&
               p.z <= s.amax.z;
      case O_SHAPE_PLANE: return p.y <= R(0);
      default: return false;
    }
  }

  // Every hit a plain shape lists (its IntersectionResult, in order): distances and pieces
  // (triangle, cylinder piece, box face)
  int shape_hits(const Object& s, const Ray<R>& r, R near, R far, R* ts, uint32_t* ps) const {
    R t;
    int piece;
    switch (s.shape) {
      case O_SHAPE_MESH: {
        TriHit<R> th;
        uint32_t tri;
        TraversalStats st;
        if (!meshes[s.mesh].bvh->traverse(r, near, far, &th, &tri, &st)) return 0;
        ts[0] = th.t;
        ps[0] = tri;
        return 1;
      }
      case O_SHAPE_SPHERE: {  // sphere.rs:108-144: the entry beyond near, the exit inside (near, far)
        const V3<R> l = r.o * R(-1);
        const R tca = dot(l, r.d);
        if (tca < R(0)) return 0;
        const R r2 = s.radius * s.radius;
        const R d2 = dot(l, l) - tca * tca;
        if (d2 > r2) return 0;
        const R thc = std::sqrt(r2 - d2);
        const R t0 = tca - thc, t1 = tca + thc;
        const R tmin = rmin(t0, t1), tmax = rmax(t0, t1);
        if (tmax < near || tmin > far) return 0;
        int n = 0;
        if (tmin > near) { ts[n] = tmin; ps[n] = 0; ++n; }
        if (tmax > near && tmax < far) { ts[n] = tmax; ps[n] = 0; ++n; }
        return n;
      }
      case O_SHAPE_CYLINDER: {  // cylinder.rs:28-110, the list sorted by distance (stable)
        const V3<R>& org = r.o;
        const V3<R>& dir = r.d;
        const R a = dir.x * dir.x + dir.z * dir.z;
        const R b = R(2) * (org.x * dir.x + org.z * dir.z);
        const R c = org.x * org.x + org.z * org.z - s.radius * s.radius;
        const R disc = b * b - R(4) * a * c;
        if (disc < R(0)) return 0;
        const R rd = std::sqrt(disc);
        const R q = b < R(0) ? R(-0.5) * (b - rd) : R(-0.5) * (b + rd);
        const R q0 = q / a, q1 = c / q;
        const R tmin = rmin(q0, q1), tmax = rmax(q0, q1);
        if (tmax < near || tmin > far) return 0;
        int n = 0;
        if (tmin > near) {
          const V3<R> p = org + dir * tmin;
          if (p.y > -s.half_height && p.y < s.half_height) { ts[n] = tmin; ps[n] = 0; n++; }
        }
        if (tmax > near && tmax < far) {
          const V3<R> p = org + dir * tmax;
          if (p.y > -s.half_height && p.y < s.half_height) { ts[n] = tmax; ps[n] = 0; n++; }
        }
        if (n < 2) {
          const R iy = R(1) / dir.y;
          const R c0 = (-s.half_height - org.y) * iy;
          if (c0 > near && c0 < far) {
            const V3<R> p = org + dir * c0;
            if (p.x * p.x + p.z * p.z <= s.radius * s.radius) { ts[n] = c0; ps[n] = 1; n++; }
          }
          const R c1 = (s.half_height - org.y) * iy;
          if (c1 > near && c1 < far) {
            const V3<R> p = org + dir * c1;
            if (p.x * p.x + p.z * p.z <= s.radius * s.radius) { ts[n] = c1; ps[n] = 2; n++; }
          }
        }
        for (int i = 1; i < n; ++i)  // insertion sort: stable
          for (int j = i; j > 0 && ts[j] < ts[j - 1]; --j) {
            std::swap(ts[j], ts[j - 1]);
            std::swap(ps[j], ps[j - 1]);
          }
        return n;
      }
      case O_SHAPE_RECTANGLE:
        if (!rectangle_hit(s, r, near, far, &t)) return 0;
        ts[0] = t;
        ps[0] = 0;
        return 1;
      case O_SHAPE_PLANE:
        if (!plane_hit(r, near, far, &t)) return 0;
        ts[0] = t;
        ps[0] = 0;
        return 1;
      default: {  // AABox (aabox.rs:76-190): the entry beyond near, the exit before far
        (void)piece;
        R tmin, tmax;
        int fmin, fmax;
        if (!aabox_span(s, r, &tmin, &tmax, &fmin, &fmax)) return 0;
        if (tmax < near || tmin > far) return 0;
        int n = 0;
        if (tmin > near) { ts[n] = tmin; ps[n] = uint32_t(fmin); ++n; }
        if (tmax < far) { ts[n] = tmax; ps[n] = uint32_t(fmax); ++n; }
        return n;
      }
    }
  }

  // The record of one listed hit of a plain shape, in the shape's frame.
  Isect<R> shape_details(const Object& s, const Ray<R>& r, R t, uint32_t piece) const {
    Isect<R> h{};
    switch (s.shape) {
      case O_SHAPE_MESH: {
        const Mesh& m = meshes[s.mesh];
        const uint32_t i0 = m.idx[3 * size_t(piece)], i1 = m.idx[3 * size_t(piece) + 1],
                       i2 = m.idx[3 * size_t(piece) + 2];
        const V3<R> p0{m.v[3 * size_t(i0)], m.v[3 * size_t(i0) + 1], m.v[3 * size_t(i0) + 2]};
        const V3<R> p1{m.v[3 * size_t(i1)], m.v[3 * size_t(i1) + 1], m.v[3 * size_t(i1) + 2]};
        const V3<R> p2{m.v[3 * size_t(i2)], m.v[3 * size_t(i2) + 1], m.v[3 * size_t(i2) + 2]};
        TriHit<R> th;
        intersect_ray(r, p0, p1, p2, &th);
        th.t = t;
        mesh_details(m, piece, r, th, &h);
        break;
      }
      case O_SHAPE_SPHERE: sphere_details(s, r, t, &h); break;
      case O_SHAPE_CYLINDER: cylinder_details(s, r, t, int(piece), &h); break;
      case O_SHAPE_AABOX: aabox_details(r, t, int(piece), &h); break;
      default: flat_details(r, t, &h); break;
    }
    return h;
  }

  // Union / Intersection / Substraction::intersect (src/shapes/csg/*.rs): every element's
  // hits, moved out of the element's frame, kept by the operation's inside tests, sorted by
  // distance (stable); Simple keeps the first. prim = element << 24 | piece.
  bool csg_closest(const Object& o, const Ray<R>& ray, R near, R far, Isect<R>* out, uint32_t* prim) const {
    bool have = false;
    for (uint32_t e = 0; e < o.csg_count; ++e) {
      const Object& E = celems[o.csg_first + e];
      const Ray<R> lr = make_ray(E.inv.point(ray.o), E.inv.direction(ray.d));
      R ts[4];
      uint32_t ps[4];
      const int n = shape_hits(E, lr, near, far, ts, ps);
      for (int k = 0; k < n; ++k) {
        if (have && !(ts[k] < out->d)) continue;
        Isect<R> w = to_world_isect(shape_details(E, lr, ts[k], ps[k]), E.mat, E.inv);
        bool keep;
        if (o.csg_op == O_CSG_UNION) {  // outside every other element (union.rs:76-93)
          keep = true;
          for (uint32_t j = 0; j < o.csg_count && keep; ++j)
            if (j != e && contains(celems[o.csg_first + j], celems[o.csg_first + j].inv.point(w.p))) keep = false;
        } else if (o.csg_op == O_CSG_INTERSECTION) {  // inside every other (intersection.rs:74-91)
          keep = true;
          for (uint32_t j = 0; j < o.csg_count && keep; ++j)
            if (j != e && !contains(celems[o.csg_first + j], celems[o.csg_first + j].inv.point(w.p))) keep = false;
        } else {  // the base outside the subtracted; a subtracted one inside the base, outside the others
          keep = e == 0 || contains(celems[o.csg_first], celems[o.csg_first].inv.point(w.p));
          for (uint32_t j = 1; j < o.csg_count && keep; ++j)
            if (j != e && contains(celems[o.csg_first + j], celems[o.csg_first + j].inv.point(w.p))) keep = false;
          if (e > 0) w.n = w.n * R(-1);
        }
        if (!keep) continue;
        have = true;
        *out = w;
        *prim = (e << 24) | ps[k];
      }
    }
    return have;
  }

  AABB<R> object_box(const Object& o) const {
    const AABB<R> b = shape_box(o);
    return o.transformed ? transform_box(b, o.mat) : b;
  }

  // get_bounding_box of a node: Simple = its shape's; Transformed = the child's through the
  // transform (transformed.rs:70-74); Compound = the union (compound.rs:57-64)
  AABB<R> node_box(uint32_t n) const {
    const Node& nd = nodes[n];
    if (nd.kind == O_NODE_SIMPLE) return object_box(objects[nd.object]);
    if (nd.kind == O_NODE_TRANSFORMED) return transform_box(node_box(nd.kids[0]), nd.mat);
    AABB<R> u = AABB<R>::empty();
    for (uint32_t k : nd.kids) u.combine(node_box(k));
    return u;
  }

  // ---- the analytic shapes ------------------------------------------------------------------
  // Sphere::intersect (sphere.rs:108-144) — first listed hit, as Simple::intersect keeps
  bool sphere_hit(const Object& o, const Ray<R>& ray, R near, R far, R* t_out) const {
    const V3<R> l = ray.o * R(-1);
    const R tca = dot(l, ray.d);
    if (tca < R(0)) return false;
    const R r2 = o.radius * o.radius;
    const R d2 = dot(l, l) - tca * tca;
    if (d2 > r2) return false;
    const R thc = std::sqrt(r2 - d2);
    const R t0 = tca - thc, t1 = tca + thc;
    const R tmin = rmin(t0, t1), tmax = rmax(t0, t1);
    if (tmax < near || tmin > far) return false;
    if (tmin > near) { *t_out = tmin; return true; }
    if (tmax > near && tmax < far) { *t_out = tmax; return true; }
    return false;
  }

  // Cylinder::intersect (cylinder.rs:28-110): all hits, sorted; first kept. Returns the
  // index of the piece (0 wall, 1 bottom cap, 2 top cap) through *piece.
  bool cylinder_hit(const Object& o, const Ray<R>& ray, R near, R far, R* t_out, int* piece) const {
    const V3<R>& org = ray.o;
    const V3<R>& dir = ray.d;
    const R a = dir.x * dir.x + dir.z * dir.z;
    const R b = R(2) * (org.x * dir.x + org.z * dir.z);
    const R c = org.x * org.x + org.z * org.z - o.radius * o.radius;
    const R disc = b * b - R(4) * a * c;
    if (disc < R(0)) return false;
    const R rd = std::sqrt(disc);
    const R q = b < R(0) ? R(-0.5) * (b - rd) : R(-0.5) * (b + rd);
    const R t0 = q / a, t1 = c / q;
    const R tmin = rmin(t0, t1), tmax = rmax(t0, t1);
    if (tmax < near || tmin > far) return false;
    R ts[4];
    int ps[4];
    int n = 0;
    if (tmin > near) {
      const V3<R> p = org + dir * tmin;
      if (p.y > -o.half_height && p.y < o.half_height) { ts[n] = tmin; ps[n] = 0; n++; }
    }
    if (tmax > near && tmax < far) {
      const V3<R> p = org + dir * tmax;
      if (p.y > -o.half_height && p.y < o.half_height) { ts[n] = tmax; ps[n] = 0; n++; }
    }
    if (n < 2) {
      const R inv_dir_y = R(1) / dir.y;
      const R c0 = (-o.half_height - org.y) * inv_dir_y;
      if (c0 > near && c0 < far) {
        const V3<R> p = org + dir * c0;
        if (p.x * p.x + p.z * p.z <= o.radius * o.radius) { ts[n] = c0; ps[n] = 1; n++; }
      }
      const R c1 = (o.half_height - org.y) * inv_dir_y;
      if (c1 > near && c1 < far) {
        const V3<R> p = org + dir * c1;
        if (p.x * p.x + p.z * p.z <= o.radius * o.radius) { ts[n] = c1; ps[n] = 2; n++; }
      }
    }
    if (n == 0) return false;
    // sort_by partial_cmp (stable): the smallest d, first among equals
    int best = 0;
    for (int k = 1; k < n; ++k)
      if (ts[k] < ts[best]) best = k;
    *t_out = ts[best];
    *piece = ps[best];
    return true;
  }

  // Rectangle::intersect (rectangle.rs:25-60): the y = 0 plane within |x| <= hw, |z| <= hh
  bool rectangle_hit(const Object& o, const Ray<R>& ray, R near, R far, R* t_out) const {
    if (ray.d.y == R(0)) return false;
    const R d = (ray.o.y * R(-1)) / ray.d.y;
    if (d < near || d > far) return false;
    V3<R> p = ray.o + ray.d * d;
    p.y = R(0);
    if (std::fabs(p.x) > o.half_w || std::fabs(p.z) > o.half_h) return false;
    *t_out = d;
    return true;
  }

  // Plane::intersect (plane.rs:19-45), its arithmetic as written: d = (o.y * -1) / (1 / dir.y)
  static bool plane_hit(const Ray<R>& ray, R near, R far, R* t_out) {
    const R inv_dir = R(1) / ray.d.y;
    const R d = (ray.o.y * R(-1)) / inv_dir;
    if (d < near || d > far) return false;
    *t_out = d;
    return true;
  }

  // The slab span of AABox::intersect (aabox.rs:76-160) with its entering / leaving faces;
  // false when the slabs do not overlap.
  static bool aabox_span(const Object& o, const Ray<R>& ray, R* tmin_out, R* tmax_out, int* fmin_out, int* fmax_out) {
    const V3<R> inv{R(1) / ray.d.x, R(1) / ray.d.y, R(1) / ray.d.z};
    R tmin, tmax;
    int fmin, fmax;
    if (inv.x >= R(0)) { tmin = (o.amin.x - ray.o.x) * inv.x; tmax = (o.amax.x - ray.o.x) * inv.x; fmin = 0; fmax = 1; }
    else { tmin = (o.amax.x - ray.o.x) * inv.x; tmax = (o.amin.x - ray.o.x) * inv.x; fmin = 1; fmax = 0; }
    R tymin, tymax;
    int fymin, fymax;
    if (inv.y >= R(0)) { tymin = (o.amin.y - ray.o.y) * inv.y; tymax = (o.amax.y - ray.o.y) * inv.y; fymin = 2; fymax = 3; }
    else { tymin = (o.amax.y - ray.o.y) * inv.y; tymax = (o.amin.y - ray.o.y) * inv.y; fymin = 3; fymax = 2; }
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) { tmin = tymin; fmin = fymin; }
    if (tymax < tmax) { tmax = tymax; fmax = fymax; }
    R tzmin, tzmax;
    int fzmin, fzmax;
    if (inv.z >= R(0)) { tzmin = (o.amin.z - ray.o.z) * inv.z; tzmax = (o.amax.z - ray.o.z) * inv.z; fzmin = 4; fzmax = 5; }
    else { tzmin = (o.amax.z - ray.o.z) * inv.z; tzmax = (o.amin.z - ray.o.z) * inv.z; fzmin = 5; fzmax = 4; }
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) { tmin = tzmin; fmin = fzmin; }
    if (tzmax < tmax) { tmax = tzmax; fmax = fzmax; }
    *tmin_out = tmin;
    *tmax_out = tmax;
    *fmin_out = fmin;
    *fmax_out = fmax;
    return true;
  }

  // AABox::intersect (aabox.rs:76-190): slabs with the entering/leaving face tracked; the
  // first listed hit is the entry when it lies beyond near, else the exit. face: 0..5 for
  // X_NEG, X_POS, Y_NEG, Y_POS, Z_NEG, Z_POS.
  static bool aabox_hit(const Object& o, const Ray<R>& ray, R near, R far, R* t_out, int* face) {
    const V3<R> inv{R(1) / ray.d.x, R(1) / ray.d.y, R(1) / ray.d.z};
    R tmin, tmax;
    int fmin, fmax;
    if (inv.x >= R(0)) { tmin = (o.amin.x - ray.o.x) * inv.x; tmax = (o.amax.x - ray.o.x) * inv.x; fmin = 0; fmax = 1; }
    else { tmin = (o.amax.x - ray.o.x) * inv.x; tmax = (o.amin.x - ray.o.x) * inv.x; fmin = 1; fmax = 0; }
    R tymin, tymax;
    int fymin, fymax;
    if (inv.y >= R(0)) { tymin = (o.amin.y - ray.o.y) * inv.y; tymax = (o.amax.y - ray.o.y) * inv.y; fymin = 2; fymax = 3; }
    else { tymin = (o.amax.y - ray.o.y) * inv.y; tymax = (o.amin.y - ray.o.y) * inv.y; fymin = 3; fymax = 2; }
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) { tmin = tymin; fmin = fymin; }
    if (tymax < tmax) { tmax = tymax; fmax = fymax; }
    R tzmin, tzmax;
    int fzmin, fzmax;
    if (inv.z >= R(0)) { tzmin = (o.amin.z - ray.o.z) * inv.z; tzmax = (o.amax.z - ray.o.z) * inv.z; fzmin = 4; fzmax = 5; }
    else { tzmin = (o.amax.z - ray.o.z) * inv.z; tzmax = (o.amin.z - ray.o.z) * inv.z; fzmin = 5; fzmax = 4; }
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) { tmin = tzmin; fmin = fzmin; }
    if (tzmax < tmax) { tmax = tzmax; fmax = fzmax; }
    if (tmax < near || tmin > far) return false;
    if (tmin > near) { *t_out = tmin; *face = fmin; return true; }
    if (tmax < far) { *t_out = tmax; *face = fmax; return true; }
    return false;
  }

  Ray<R> local_ray(const Object& o, const Ray<R>& ray) const {
    if (!o.transformed) return ray;
    return make_ray(o.inv.point(ray.o), o.inv.direction(ray.d));  // transform_ray_to_local (transform.rs:98-103)
  }

  // transform_interaction_to_world (transform.rs:105-116): d, u, v are kept
  static Isect<R> to_world_isect(const Isect<R>& h, const Affine<R>& mat, const Affine<R>& inv) {
    Isect<R> w = h;
    w.n = inv.normal(h.n);
    w.p = mat.point(h.p);
    w.wo = mat.direction(h.wo);
    w.dpdu = mat.direction(h.dpdu);
    w.dpdv = mat.direction(h.dpdv);
    return w;
  }

  // Simple::intersect (simple.rs:28-41) of one object, through its own transform if any;
  // prim = triangle index, cylinder piece or aabox face (0 otherwise)
  bool intersect_object(uint32_t oi, const Ray<R>& ray, R near, R far, Isect<R>* out, uint32_t* prim) const {
    const Object& o = objects[oi];
    const Ray<R> lr = local_ray(o, ray);
    Isect<R> h;
    R t;
    if (work_tally && o.shape != O_SHAPE_MESH) work_tally->shapes++;
    if (o.shape == O_SHAPE_MESH) {
      const Mesh& m = meshes[o.mesh];
      TriHit<R> th;
      uint32_t tri;
      TraversalStats st;
      const bool hit = m.bvh->traverse(lr, near, far, &th, &tri, &st);
      if (work_tally) {
        work_tally->mesh_boxes += st.box_tests;
        work_tally->triangles += st.triangle_tests;
      }
      if (!hit) return false;
      mesh_details(m, tri, lr, th, &h);
      *prim = tri;
    } else if (o.shape == O_SHAPE_SPHERE) {
      if (!sphere_hit(o, lr, near, far, &t)) return false;
      sphere_details(o, lr, t, &h);
      *prim = 0;
    } else if (o.shape == O_SHAPE_CYLINDER) {
      int piece;
      if (!cylinder_hit(o, lr, near, far, &t, &piece)) return false;
      cylinder_details(o, lr, t, piece, &h);
      *prim = uint32_t(piece);  // 0 wall, 1 bottom cap, 2 top cap
    } else if (o.shape == O_SHAPE_RECTANGLE || o.shape == O_SHAPE_PLANE) {
      if (o.shape == O_SHAPE_RECTANGLE ? !rectangle_hit(o, lr, near, far, &t) : !plane_hit(lr, near, far, &t))
        return false;
      flat_details(lr, t, &h);
      *prim = 0;
    } else if (o.shape == O_SHAPE_AABOX) {
      int face;
      if (!aabox_hit(o, lr, near, far, &t, &face)) return false;
      aabox_details(lr, t, face, &h);
      *prim = uint32_t(face);
    } else {
      if (!csg_closest(o, lr, near, far, &h, prim)) return false;
    }
    *out = o.transformed ? to_world_isect(h, o.mat, o.inv) : h;
    return true;
  }

  // Intersectable::intersect_p through Simple (simple.rs:54-56): the shape's default
  // `!intersect().is_empty()` (intersectable.rs:48-50), the mesh's own BVH any-hit
  bool occluded_object(uint32_t oi, const Ray<R>& ray, R near, R far) const {
    const Object& o = objects[oi];
    const Ray<R> lr = local_ray(o, ray);
    R t;
    int piece;
    if (work_tally && o.shape != O_SHAPE_MESH) work_tally->shapes++;
    switch (o.shape) {
      case O_SHAPE_MESH: {
        TraversalStats st;
        const bool hit = meshes[o.mesh].bvh->intersect_p(lr, near, far, work_tally ? &st : nullptr);
        if (work_tally) {
          work_tally->mesh_boxes += st.box_tests;
          work_tally->triangles += st.triangle_tests;
        }
        return hit;
      }
      case O_SHAPE_SPHERE: return sphere_hit(o, lr, near, far, &t);
      case O_SHAPE_CYLINDER: return cylinder_hit(o, lr, near, far, &t, &piece);
      case O_SHAPE_RECTANGLE: return rectangle_hit(o, lr, near, far, &t);
      case O_SHAPE_AABOX: return aabox_hit(o, lr, near, far, &t, &piece);
      case O_SHAPE_CSG: {  // the default intersect_p: any hit listed (intersectable.rs:48-50)
        Isect<R> h;
        uint32_t prim;
        return csg_closest(o, lr, near, far, &h, &prim);
      }
      default: return plane_hit(lr, near, far, &t);
    }
  }

  // Object::intersect of a tree node: Transformed (transformed.rs:27-38) moves the ray in
  // and the interaction out; Compound (compound.rs:21-38) keeps the strictly nearest, the
  // earlier member on a tie.
  bool intersect_node(uint32_t n, const Ray<R>& ray, R near, R far, Isect<R>* out, uint32_t* obj,
                      uint32_t* prim) const {
    const Node& nd = nodes[n];
    if (nd.kind == O_NODE_SIMPLE) {
      if (!intersect_object(nd.object, ray, near, far, out, prim)) return false;
      *obj = nd.object;
      return true;
    }
    if (nd.kind == O_NODE_TRANSFORMED) {
      const Ray<R> lr = make_ray(nd.inv.point(ray.o), nd.inv.direction(ray.d));
      Isect<R> h;
      if (!intersect_node(nd.kids[0], lr, near, far, &h, obj, prim)) return false;
      *out = to_world_isect(h, nd.mat, nd.inv);
      return true;
    }
    bool have = false;
    for (uint32_t k : nd.kids) {
      Isect<R> c;
      uint32_t co, cp;
      if (!intersect_node(k, ray, near, far, &c, &co, &cp)) continue;
      if (have && !(c.d < out->d)) continue;
      have = true;
      *out = c;
      *obj = co;
      *prim = cp;
    }
    return have;
  }

  bool occluded_node(uint32_t n, const Ray<R>& ray, R near, R far) const {
    const Node& nd = nodes[n];
    if (nd.kind == O_NODE_SIMPLE) return occluded_object(nd.object, ray, near, far);
    if (nd.kind == O_NODE_TRANSFORMED)
      return occluded_node(nd.kids[0], make_ray(nd.inv.point(ray.o), nd.inv.direction(ray.d)), near, far);
    for (uint32_t k : nd.kids)
      if (occluded_node(k, ray, near, far)) return true;  // compound.rs:47-49
    return false;
  }

  // TriangleMesh::intersect post-hit (triangle_mesh.rs:73-132, 219-258) with default uvs
  void mesh_details(const Mesh& m, uint32_t tri, const Ray<R>& ray, const TriHit<R>& th, Isect<R>* h) const {
    const uint32_t i0 = m.idx[3 * size_t(tri)], i1 = m.idx[3 * size_t(tri) + 1], i2 = m.idx[3 * size_t(tri) + 2];
    const V3<R> p0{m.v[3 * size_t(i0)], m.v[3 * size_t(i0) + 1], m.v[3 * size_t(i0) + 2]};
    const V3<R> p1{m.v[3 * size_t(i1)], m.v[3 * size_t(i1) + 1], m.v[3 * size_t(i1) + 2]};
    const V3<R> p2{m.v[3 * size_t(i2)], m.v[3 * size_t(i2) + 1], m.v[3 * size_t(i2) + 2]};
    h->p = ray.o + ray.d * th.t;
    h->d = th.t;
    const R uv0x = R(0), uv0y = R(0), uv1x = R(1), uv1y = R(0), uv2x = R(1), uv2y = R(1);
    h->u = th.w * uv0x + th.u * uv1x + th.v * uv2x;
    h->v = th.w * uv0y + th.u * uv1y + th.v * uv2y;
    const R d02x = uv0x - uv2x, d02y = uv0y - uv2y, d12x = uv1x - uv2x, d12y = uv1y - uv2y;
    const V3<R> dp02 = p0 - p2, dp12 = p1 - p2;
    const R det = d12x * d02y - d12y * d02x;
    if (std::fabs(det) < R(1e-8)) {
      const V3<R> nn = cross(dp12, dp02);
      const V3<R> tg = std::fabs(nn.x) < R(0.9) ? cross(V3<R>{R(1), R(0), R(0)}, nn) : cross(V3<R>{R(0), R(1), R(0)}, nn);
      h->dpdu = tg;
      h->dpdv = cross(nn, tg);
    } else {
      const R inv = R(1) / det;
      h->dpdu = (dp12 * d02y - dp02 * d12y) * inv;
      h->dpdv = (dp02 * d12x - dp12 * d02x) * inv;
    }
    h->n = normalized(cross(h->dpdv, h->dpdu));
    h->wo = ray.d * R(-1);
  }

  // compute_intersection_details (sphere.rs:152-187)
  void sphere_details(const Object& o, const Ray<R>& ray, R t, Isect<R>* h) const {
    const R PI = Consts<R>::pi();
    const V3<R> hit = ray.o + ray.d * t;
    h->p = hit;
    h->n = normalized(hit);
    R phi = std::atan2(hit.y, hit.x);
    if (phi < R(0)) phi += R(2) * PI;
    h->u = phi / (R(2) * PI);
    const R theta = std::acos(std::min(std::max(hit.z / o.radius, R(-1)), R(1)));
    h->v = theta / PI;
    const R zr = std::sqrt(hit.x * hit.x + hit.y * hit.y);
    const R izr = R(1) / zr;
    const R cphi = hit.x * izr, sphi = hit.y * izr;
    h->dpdu = V3<R>{-hit.y, hit.x, R(0)} * (R(2) * PI);
    h->dpdv = V3<R>{hit.z * cphi, hit.z * sphi, -o.radius * std::sin(theta)} * PI;
    h->d = t;
    h->wo = ray.d * R(-1);
  }

  // compute_cynlinder_intersection_details (cylinder.rs:324-344) and the caps (:266-300)
  void cylinder_details(const Object& o, const Ray<R>& ray, R t, int piece, Isect<R>* h) const {
    const R PI = Consts<R>::pi();
    const V3<R> p = ray.o + ray.d * t;
    h->p = p;
    h->d = t;
    h->wo = ray.d * R(-1);
    if (piece == 0) {
      h->n = normalized(V3<R>{p.x, R(0), p.z});
      R phi = std::atan2(p.z, p.x);
      if (phi < R(0)) phi += R(2) * PI;
      h->u = phi / (R(2) * PI);
      h->v = p.y;
      h->dpdu = V3<R>{-p.z, R(0), p.x} * (R(2) * PI);
      h->dpdv = V3<R>{R(0), R(1), R(0)};
    } else {
      const bool top = piece == 2;
      h->n = V3<R>{R(0), top ? R(1) : R(-1), R(0)};
      h->u = p.x;
      h->v = p.z;
      h->dpdu = V3<R>{top ? R(1) : R(-1), R(0), R(0)};
      h->dpdv = V3<R>{R(0), R(0), R(1)};
    }
  }

  // Rectangle and Plane records (rectangle.rs:46-55, plane.rs:31-40): p on y = 0, n = +y,
  // u = p.x, v = p.z, dpdu = +x, dpdv = +z
  static void flat_details(const Ray<R>& ray, R t, Isect<R>* h) {
    V3<R> p = ray.o + ray.d * t;
    p.y = R(0);
    h->p = p;
    h->d = t;
    h->n = V3<R>{R(0), R(1), R(0)};
    h->wo = ray.d * R(-1);
    h->u = p.x;
    h->v = p.z;
    h->dpdu = V3<R>{R(1), R(0), R(0)};
    h->dpdv = V3<R>{R(0), R(0), R(1)};
  }

  // AABox face records (aabox.rs:29-63, 165-190): u = p·du, v = p·dv
  static void aabox_details(const Ray<R>& ray, R t, int face, Isect<R>* h) {
    static const R F[6][9] = {
        {-1, 0, 0, 0, 0, -1, 0, 1, 0}, {1, 0, 0, 0, 0, 1, 0, 1, 0},  {0, -1, 0, -1, 0, 0, 0, 0, 1},
        {0, 1, 0, 1, 0, 0, 0, 0, 1},   {0, 0, -1, 0, -1, 0, 1, 0, 0}, {0, 0, 1, 0, 1, 0, 1, 0, 0}};
    const R* f = F[face];
    const V3<R> p = ray.o + ray.d * t;
    h->p = p;
    h->d = t;
    h->n = V3<R>{f[0], f[1], f[2]};
    h->wo = ray.d * R(-1);
    h->dpdu = V3<R>{f[3], f[4], f[5]};
    h->dpdv = V3<R>{f[6], f[7], f[8]};
    h->u = dot(p, h->dpdu);
    h->v = dot(p, h->dpdv);
  }

  // ---- the scene: Scene::commit + BVH::new (scene.rs:101-115, bvh.rs:109-132, 291-357) ----
  void commit() {
    order.clear();
    bnodes.clear();
    boxes.clear();
    unbounded.clear();
    std::vector<uint32_t> bounded;
    for (uint32_t r : roots) {
      const AABB<R> b = node_box(r);
      if (b.is_bounded()) {
        bounded.push_back(r);
        boxes.push_back(b);
      } else {
        unbounded.push_back(r);
      }
    }
    if (bounded.empty()) return;
    // order[k] indexes `boxes`/`bounded`; prim_root maps it to the root node
    prim_root = bounded;
    for (uint32_t i = 0; i < bounded.size(); ++i) order.push_back(i);
    bnodes.push_back(BNode{AABB<R>::empty(), 0, uint32_t(bounded.size())});
    subdivide(0);
  }

  AABB<R> subdivide(uint32_t ni) {
    const uint32_t first = bnodes[ni].left_first, count = bnodes[ni].count;
    if (count == 1) {
      bnodes[ni].box = boxes[order[first]];
      return bnodes[ni].box;
    }
    // widest_centroid_axis (bvh.rs:358-378)
    R mn[3] = {Limits<R>::max(), Limits<R>::max(), Limits<R>::max()};
    R mx[3] = {Limits<R>::lowest(), Limits<R>::lowest(), Limits<R>::lowest()};
    for (uint32_t k = first; k < first + count; ++k) {
      const V3<R> c = boxes[order[k]].centroid();
      for (int a = 0; a < 3; ++a) { mn[a] = rmin(mn[a], c[a]); mx[a] = rmax(mx[a], c[a]); }
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (mx[a] - mn[a] > mx[axis] - mn[axis]) axis = a;
    std::stable_sort(order.begin() + first, order.begin() + first + count,
                     [&](uint32_t a, uint32_t b) { return boxes[a].centroid()[axis] < boxes[b].centroid()[axis]; });
    const uint32_t lc = count / 2;
    const uint32_t li = uint32_t(bnodes.size());
    bnodes.push_back(BNode{AABB<R>::empty(), first, lc});
    bnodes.push_back(BNode{AABB<R>::empty(), first + lc, count - lc});
    bnodes[ni].left_first = li;
    bnodes[ni].count = 0;
    const AABB<R> lb = subdivide(li);
    const AABB<R> rb = subdivide(li + 1);
    AABB<R> u = AABB<R>::empty();
    u.combine(lb);
    u.combine(rb);
    bnodes[ni].box = u;
    return u;
  }

  bool hit_box(const BNode& nd, const Ray<R>& ray, R near, R far, R* e, SceneStats* st) const {
    if (st) st->box_tests++;
    return box_hit(nd.box, ray, near, far, e);
  }

  // Scene::find_nearest (scene.rs:186-235): the unbounded primitives first, then BVH::query
  // (bvh.rs:153-230) over [near, nearest so far], adopting only strictly nearer hits.
  bool intersect(const Ray<R>& ray, R near, R far, Isect<R>* out, uint32_t* obj_out, uint32_t* prim_out,
                 SceneStats* st = nullptr) const {
    if (work_tally && !st) {  // count this query into the render's tally
      SceneStats local;
      const bool h = intersect(ray, near, far, out, obj_out, prim_out, &local);
      work_tally->rays++;
      work_tally->top_boxes += local.box_tests;
      work_tally->objects += local.object_tests;
      return h;
    }
    bool have = false;
    Isect<R> nearest{};
    for (uint32_t r : unbounded) {  // nearest_among + closer (scene.rs:222-249)
      if (st) st->object_tests++;
      Isect<R> c;
      uint32_t o, p;
      if (!intersect_node(r, ray, near, far, &c, &o, &p)) continue;
      if (have && !(c.d < nearest.d)) continue;
      have = true;
      nearest = c;
      *obj_out = o;
      *prim_out = p;
    }
    if (!bnodes.empty()) {
      R min_t = have ? nearest.d : far;
      R e;
      if (hit_box(bnodes[0], ray, near, min_t, &e, st)) {
        struct Ent { uint32_t n; R e; };
        std::vector<Ent> stack;
        stack.reserve(64);
        stack.push_back(Ent{0, e});
        while (!stack.empty()) {
          const Ent en = stack.back();
          stack.pop_back();
          if (en.e >= min_t) continue;
          if (st) st->nodes_visited++;
          const BNode& nd = bnodes[en.n];
          if (nd.count > 0) {
            for (uint32_t k = nd.left_first; k < nd.left_first + nd.count; ++k) {
              if (st) st->object_tests++;
              Isect<R> c;
              uint32_t o, p;
              if (!intersect_node(prim_root[order[k]], ray, near, min_t, &c, &o, &p)) continue;
              if (have && !(c.d < nearest.d)) continue;  // strictly nearer (scene.rs:206-210)
              have = true;
              nearest = c;
              *obj_out = o;
              *prim_out = p;
              min_t = c.d;
            }
          } else {
            R dl = R(0), dr = R(0);
            const bool hl = hit_box(bnodes[nd.left_first], ray, near, min_t, &dl, st);
            const bool hr = hit_box(bnodes[nd.left_first + 1], ray, near, min_t, &dr, st);
            uint32_t nn = nd.left_first, ff = nd.left_first + 1;
            bool hn = hl, hf = hr;
            R dn = dl, df = dr;
            if (hl && hr && dr < dl) { nn = nd.left_first + 1; ff = nd.left_first; hn = hr; hf = hl; dn = dr; df = dl; }
            if (hf) stack.push_back(Ent{ff, df});
            if (hn) stack.push_back(Ent{nn, dn});
          }
        }
      }
    }
    if (have) *out = nearest;
    return have;
  }

  // Scene::any_hit (scene.rs:157-184): the unbounded primitives first, then BVH::query_p
  // (bvh.rs:239-275): unordered, the box tested at pop, left popped first.
  bool occluded(const Ray<R>& ray, R near, R far, SceneStats* st = nullptr) const {
    if (work_tally && !st) {
      SceneStats local;
      const bool h = occluded(ray, near, far, &local);
      work_tally->shadow_rays++;
      work_tally->top_boxes += local.box_tests;
      work_tally->objects += local.object_tests;
      return h;
    }
    for (uint32_t r : unbounded) {
      if (st) st->object_tests++;
      if (occluded_node(r, ray, near, far)) return true;
    }
    if (bnodes.empty()) return false;
    std::vector<uint32_t> stack;
    stack.reserve(64);
    stack.push_back(0);
    while (!stack.empty()) {
      const BNode& nd = bnodes[stack.back()];
      stack.pop_back();
      R e;
      if (!hit_box(nd, ray, near, far, &e, st)) continue;
      if (st) st->nodes_visited++;
      if (nd.count > 0) {
        for (uint32_t k = nd.left_first; k < nd.left_first + nd.count; ++k) {
          if (st) st->object_tests++;
          if (occluded_node(prim_root[order[k]], ray, near, far)) return true;
        }
      } else {
        stack.push_back(nd.left_first + 1);
        stack.push_back(nd.left_first);
      }
    }
    return false;
  }

  // ---- lights -------------------------------------------------------------------------------
  void setup_area(Light& L) {
    if (L.object >= objects.size()) throw std::invalid_argument("area light object out of range");
    // the emitter must be one primitive of the scene (a root Simple node), so that its own
    // transform is its whole placement
    uint32_t refs = 0, root_refs = 0;
    for (const Node& n : nodes) refs += n.kind == O_NODE_SIMPLE && n.object == L.object;
    for (uint32_t r : roots) root_refs += nodes[r].kind == O_NODE_SIMPLE && nodes[r].object == L.object;
    if (refs != 1 || root_refs != 1)
      throw std::invalid_argument("an area light's object must be placed once, as a primitive of the scene");
    const Object& o = objects[L.object];
    if (materials[o.material].texture != O_TEX_PLAIN)
      throw std::invalid_argument("an area light's emission must be a plain color");
    if (o.shape == O_SHAPE_MESH) {
      const Mesh& m = meshes[o.mesh];
      const size_t nt = m.idx.size() / 3;
      R run = R(0);
      for (size_t t = 0; t < nt; ++t) {
        V3<R> p[3];
        for (int k = 0; k < 3; ++k) {
          const uint32_t vi = m.idx[3 * t + k];
          V3<R> v{m.v[3 * size_t(vi)], m.v[3 * size_t(vi) + 1], m.v[3 * size_t(vi) + 2]};
          p[k] = o.transformed ? o.mat.point(v) : v;
          L.tp.push_back(p[k]);
        }
        const R a = R(0.5) * length(cross(p[1] - p[0], p[2] - p[0]));
        run = run + a;
        L.cdf.push_back(run);
      }
      L.area = run;
    } else if (o.shape == O_SHAPE_SPHERE) {
      L.area = R(4) * Consts<R>::pi() * o.radius * o.radius;
    } else {
      throw std::invalid_argument("area lights are triangle meshes or spheres");
    }
  }

  struct LiSample {
    V3<R> spectrum, wi;
    R pdf;
    Ray<R> ray;
    R dist;
  };

  // SpherePdf::generate (pdfs/sphere.rs:10-23)
  static V3<R> sphere_dir(Pcg32& rng) {
    const R two_pi = R(2) * Consts<R>::pi();
    const R phi = two_pi * R(rng.uniform());
    const R ct = R(1) - R(2) * R(rng.uniform());
    const R st = std::sqrt(R(1) - ct * ct);
    return V3<R>{std::cos(phi) * st, std::sin(phi) * st, ct};
  }

  V3<R> gradient(const Light& L, const V3<R>& dir) const {
    const R f = R(0.5) * (dir.y + R(1));
    return L.bottom * (R(1) - f) + L.top * f;
  }

  // Light::le for infinite lights (background_infinite_light.rs:33-37, uniform_infinite_light.rs:23-25)
  V3<R> background(const V3<R>& dir) const {
    V3<R> res{R(0), R(0), R(0)};
    for (const Light& L : lights) {
      if (L.kind == O_LIGHT_BACKGROUND) res = res + gradient(L, normalized(dir));
      else if (L.kind == O_LIGHT_UNIFORM) res = res + L.rad;
    }
    return res;
  }

  bool sample_li(const Light& L, const Isect<R>& it, Pcg32& rng, LiSample* s) const {
    if (L.kind == O_LIGHT_POINT) {  // point_light.rs:23-35
      const V3<R> wi = L.pos - it.p;
      const R sl = dot(wi, wi);
      s->spectrum = V3<R>{L.rad.x / sl, L.rad.y / sl, L.rad.z / sl};
      s->wi = normalized(wi);
      s->pdf = R(1);
      s->ray = spawn_from_through(it.p, L.pos);  // VisibilityTester::between (lights.rs:40-47)
      s->dist = length(L.pos - it.p);
      return true;
    }
    if (L.kind == O_LIGHT_BACKGROUND || L.kind == O_LIGHT_UNIFORM) {  // background_infinite_light.rs:39-51
      const V3<R> wi = sphere_dir(rng);
      s->pdf = R(1) / (R(4) * Consts<R>::pi());
      s->spectrum = L.kind == O_LIGHT_BACKGROUND ? gradient(L, wi) : L.rad;
      s->wi = wi;
      s->ray = make_ray(it.p, wi);  // towards_infinity (lights.rs:55-60)
      s->dist = Limits<R>::max();
      return true;
    }
    // area light (ideas/area_light.md §3)
    const Object& o = objects[L.object];
    V3<R> pl, nl;
    if (o.shape == O_SHAPE_MESH) {
      const R u0 = R(rng.uniform()) * L.area;
      size_t t = size_t(std::upper_bound(L.cdf.begin(), L.cdf.end(), u0) - L.cdf.begin());
      if (t >= L.cdf.size()) t = L.cdf.size() - 1;
      const R su = std::sqrt(R(rng.uniform()));
      const R u2 = R(rng.uniform());
      const R b0 = R(1) - su, b1 = u2 * su;
      const V3<R> p0 = L.tp[3 * t], p1 = L.tp[3 * t + 1], p2 = L.tp[3 * t + 2];
      pl = p0 * b0 + p1 * b1 + p2 * (R(1) - b0 - b1);
      // the mesh's own normal convention: normalize(dpdv x dpdu) = normalize((p2-p1) x (p1-p0))
      nl = normalized(cross(p2 - p1, p1 - p0));
    } else {
      const V3<R> dir = sphere_dir(rng);
      const V3<R> lp = dir * o.radius;
      pl = o.transformed ? o.mat.point(lp) : lp;
      nl = o.transformed ? normalized(o.inv.normal(dir)) : dir;
    }
    const V3<R> w = pl - it.p;
    const R d2 = dot(w, w);
    const R dist = std::sqrt(d2);
    const V3<R> wi = normalized(w);
    const R cosl = std::fabs(dot(nl, wi));
    const R pdf = (R(1) / L.area) * d2 / cosl;
    if (!(pdf > R(0)) || !std::isfinite(pdf)) return false;
    s->spectrum = materials[o.material].color;  // DiffuseLight emission, two-sided
    s->wi = wi;
    s->pdf = pdf;
    s->ray = make_ray(it.p, wi);
    s->dist = dist * (R(1) - R(1e-4));
    return true;
  }

  // ---- materials ----------------------------------------------------------------------------
  // Texture::shade at the interaction: PlainColor, or CheckerBoard::shade
  // (textures/checker_board.rs:17-28) on the record's u, v (`%` is fmod; signum(±0) = ±1)
  static V3<R> texel(const Material& m, const Isect<R>& it) {
    if (m.texture == O_TEX_PLAIN) return m.color;
    const R su = std::fmod(std::fabs(it.u) * m.scale, R(1));
    const R sv = std::fmod(std::fabs(it.v) * m.scale, R(1));
    const bool use_color = (su < R(0.5) && sv < R(0.5)) || (su >= R(0.5) && sv >= R(0.5));
    const bool positive = !std::isnan(it.u) && !std::isnan(it.v) &&
                          std::copysign(R(1), it.u) * std::copysign(R(1), it.v) >= R(0);
    return (use_color != positive) ? m.color : m.color2;
  }

  // Material::f (materials.rs:32-34, lambertian.rs:40-52)
  V3<R> bsdf_f(const Material& m, const V3<R>& wo, const V3<R>& wi, const Isect<R>& it) const {
    if (m.kind != O_MAT_LAMBERTIAN) return V3<R>{R(0), R(0), R(0)};
    const V3<R> lwi = it.to_local(wi), lwo = it.to_local(wo);
    const V3<R> c = texel(m, it);
    if (lwo.z * lwi.z > R(0)) return V3<R>{c.x / Consts<R>::pi(), c.y / Consts<R>::pi(), c.z / Consts<R>::pi()};
    return V3<R>{R(0), R(0), R(0)};
  }

  struct Scatter {
    V3<R> att;
    Ray<R> ray;
    R pdf;
  };

  // random_in_unit_sphere (utils.rs:24-32); bounded at 64 draws (p(more) ≈ 1e-21)
  static V3<R> in_unit_sphere(Pcg32& rng) {
    V3<R> p{R(0), R(0), R(0)};
    for (int k = 0; k < 64; ++k) {
      const R x = R(rng.uniform()), y = R(rng.uniform()), z = R(rng.uniform());
      p = V3<R>{x * R(2) - R(1), y * R(2) - R(1), z * R(2) - R(1)};
      if (dot(p, p) < R(1)) return p;
    }
    return p * R(0.5);
  }

  bool scatter(const Material& m, const Isect<R>& it, Pcg32& rng, Scatter* s) const {
    const R PI = Consts<R>::pi();
    const V3<R> col = texel(m, it);
    if (m.kind == O_MAT_LAMBERTIAN) {  // lambertian.rs:24-38, pdfs/cosine.rs:10-24
      const R two_pi = R(2) * PI;
      const R phi = two_pi * R(rng.uniform());
      const R r2 = R(rng.uniform());
      const R r2s = std::sqrt(r2);
      const R ct = std::sqrt(R(1) - r2);
      const V3<R> lwi{std::cos(phi) * r2s, std::sin(phi) * r2s, ct};
      const V3<R> wi = it.to_world(lwi);
      s->ray = make_ray(it.p + it.n * R(0.001), wi);
      s->att = V3<R>{col.x / PI, col.y / PI, col.z / PI};
      s->pdf = std::fabs(lwi.z / PI);
      return true;
    }
    if (m.kind == O_MAT_METAL) {  // metal.rs:22-59
      const V3<R> lwo = normalized(it.to_local(it.wo));
      const V3<R> refl{-lwo.x, -lwo.y, lwo.z};
      const V3<R> tgt = normalized(refl + in_unit_sphere(rng) * m.fuzz);
      if (!(tgt.z > R(0))) return false;
      const V3<R> w = it.to_world(tgt);
      s->ray = make_ray(it.p + it.n * R(0.001), w);
      const R ac = std::fabs(tgt.z);
      s->att = V3<R>{col.x / ac, col.y / ac, col.z / ac};
      s->pdf = R(1);
      return true;
    }
    if (m.kind == O_MAT_DIELECTRIC) {  // dielectric.rs:32-182
      const V3<R> lwo = normalized(it.to_local(it.wo));
      const V3<R> refl{-lwo.x, -lwo.y, lwo.z};
      V3<R> ln, wn;
      R ni, nt;
      if (lwo.z <= R(0)) { ln = V3<R>{R(0), R(0), R(-1)}; wn = it.n * R(-1); ni = m.ior; nt = R(1); }
      else { ln = V3<R>{R(0), R(0), R(1)}; wn = it.n; ni = R(1); nt = m.ior; }
      const R nint = ni / nt;
      // refract (dielectric.rs:129-157)
      const R ci = dot(lwo, ln);
      const R s2i = R(1) - ci * ci;
      const R s2t = nint * nint * s2i;
      const R disc = R(1) - s2t;
      V3<R> ldir;
      V3<R> origin;
      if (disc > R(0)) {
        const R ctt = std::sqrt(disc);
        const V3<R> wi = lwo * R(-1);
        const V3<R> refr = normalized(wi * nint + ln * (nint * ci - ctt));
        // fresnel (dielectric.rs:168-182)
        const R n12 = ni / nt;
        const R cti = lwo.z * ln.z;
        const R ctf = std::sqrt(R(1) - n12 * n12 * (R(1) - cti * cti));
        const R ro = (ni * cti - nt * ctf) / (ni * cti + nt * ctf);
        const R rp = (nt * cti - ni * ctf) / (nt * cti + ni * ctf);
        const R refl_p = (ro * ro + rp * rp) * R(0.5);
        if (R(rng.uniform()) < refl_p) { ldir = refl; origin = it.p + wn * R(0.001); }
        else { ldir = refr; origin = it.p + wn * R(-0.001); }
      } else {
        ldir = refl;
        origin = it.p + wn * R(0.001);
      }
      s->ray = make_ray(origin, it.to_world(ldir));
      const R ac = std::fabs(ldir.z);
      s->att = V3<R>{col.x / ac, col.y / ac, col.z / ac};
      s->pdf = R(1);
      return true;
    }
    return false;  // DiffuseLight scatters nothing
  }

  uint32_t material_of(uint32_t obj, uint32_t prim) const {
    const Object& o = objects[obj];
    if (o.shape == O_SHAPE_MESH && !meshes[o.mesh].fmat.empty()) return meshes[o.mesh].fmat[prim];
    return o.material;
  }

  // ---- integrators --------------------------------------------------------------------------
  // PathIntegrator::li (path.rs:48-115) with area-light NEE and Russian roulette
  V3<R> li_path(Ray<R> ray, R near, R far, uint32_t max_depth, uint32_t rr_start, Pcg32& rng,
                const CacheHook* cache = nullptr) const {
    V3<R> beta{R(1), R(1), R(1)}, L{R(0), R(0), R(0)};
    bool specular = true;
    uint32_t bounce = 0;
    const R SHADOW_EPS = R(0.00001);
    for (;;) {
      Isect<R> it;
      uint32_t obj, prim;
      if (!intersect(ray, near, far, &it, &obj, &prim)) {
        if (specular) {
          const V3<R> bg = background(ray.d);
          L = L + V3<R>{bg.x * beta.x, bg.y * beta.y, bg.z * beta.z};
        }
        break;
      }
      const Material& m = materials[material_of(obj, prim)];
      if (specular && m.kind == O_MAT_DIFFUSE_LIGHT) {  // DiffuseLight::emit (diffuse_light.rs:18-22)
        const V3<R> e = texel(m, it);
        L = L + V3<R>{e.x * beta.x, e.y * beta.y, e.z * beta.z};
      }
      bounce++;
      if (bounce == max_depth) break;
      if (cache && bounce >= cache->term_hit && (m.kind == O_MAT_LAMBERTIAN || m.kind == O_MAT_METAL)) {
        const V3<R> wo = ray.d * R(-1);
        const V3<R> n = dot(it.n, wo) < R(0) ? it.n * R(-1) : it.n;
        const V3<R> alb = texel(m, it);
        const float rec[16] = {float(it.p.x), float(it.p.y), float(it.p.z),
                               m.kind == O_MAT_METAL ? float(m.fuzz) : 1.0f,
                               float(wo.x), float(wo.y), float(wo.z), 0.f,
                               float(n.x), float(n.y), float(n.z), 0.f,
                               float(alb.x), float(alb.y), float(alb.z), 0.f};
        float o[3];
        cache->query(rec, o);
        const float mx = cache->max_radiance;
        L = L + V3<R>{beta.x * R(std::fmin(std::fmax(o[0], 0.f), mx)), beta.y * R(std::fmin(std::fmax(o[1], 0.f), mx)),
                      beta.z * R(std::fmin(std::fmax(o[2], 0.f), mx))};
        break;
      }
      if (!lights.empty()) {  // sample_light (path.rs:31-44)
        const R cnt = R(lights.size());
        const R pick = std::min(R(rng.uniform()) * cnt, cnt - R(1));
        const uint32_t li = uint32_t(pick);
        const R pl = R(1) / cnt;
        LiSample s;
        if (sample_li(lights[li], it, rng, &s)) {
          const V3<R> f0 = bsdf_f(m, ray.d * R(-1), s.wi, it);
          const R ac = std::fabs(dot(s.wi, it.n));
          const V3<R> f{f0.x * ac, f0.y * ac, f0.z * ac};
          if (f.x != R(0) || f.y != R(0) || f.z != R(0)) {  // zero contributions skip the shadow ray
            if (!occluded(s.ray, SHADOW_EPS, s.dist)) {
              const R den = pl * s.pdf;
              const V3<R> c{((s.spectrum.x * f.x) * beta.x) / den, ((s.spectrum.y * f.y) * beta.y) / den,
                            ((s.spectrum.z * f.z) * beta.z) / den};
              L = L + c;
            }
          }
        }
      }
      Scatter sc;
      if (!scatter(m, it, rng, &sc)) break;
      const R ac = std::fabs(dot(sc.ray.d, it.n));
      const V3<R> k{(sc.att.x * ac) / sc.pdf, (sc.att.y * ac) / sc.pdf, (sc.att.z * ac) / sc.pdf};
      beta = V3<R>{beta.x * k.x, beta.y * k.y, beta.z * k.z};
      ray = sc.ray;
      specular = m.kind == O_MAT_METAL || m.kind == O_MAT_DIELECTRIC;
      if (rr_start && bounce >= rr_start) {
        const R q = std::min(R(1), rmax(rmax(beta.x, beta.y), beta.z));
        if (R(rng.uniform()) > q) break;
        const R iq = R(1) / q;
        beta = beta * iq;
      }
    }
    return L;
  }

  // NormalIntegrator::li (normal.rs:17-27): (n + (1, 1, 1)) * 0.5 at the first hit; a miss is
  // black (the trait's default background, integrators.rs:9-11)
  V3<R> li_normal(const Ray<R>& ray, R near, R far) const {
    Isect<R> it;
    uint32_t obj, prim;
    if (!intersect(ray, near, far, &it, &obj, &prim)) return V3<R>{R(0), R(0), R(0)};
    return (it.n + V3<R>{R(1), R(1), R(1)}) * R(0.5);
  }

  // NaiveIntegrator::li (naive.rs:29-52), written as a loop, background = infinite lights
  V3<R> li_naive(Ray<R> ray, R near, R far, uint32_t max_depth, Pcg32& rng) const {
    V3<R> beta{R(1), R(1), R(1)}, L{R(0), R(0), R(0)};
    for (uint32_t depth = max_depth; depth > 0; --depth) {
      Isect<R> it;
      uint32_t obj, prim;
      if (!intersect(ray, near, far, &it, &obj, &prim)) {
        const V3<R> bg = background(ray.d);
        L = L + V3<R>{bg.x * beta.x, bg.y * beta.y, bg.z * beta.z};
        break;
      }
      const Material& m = materials[material_of(obj, prim)];
      if (m.kind == O_MAT_DIFFUSE_LIGHT) {
        const V3<R> e = texel(m, it);
        L = L + V3<R>{e.x * beta.x, e.y * beta.y, e.z * beta.z};
      }
      Scatter sc;
      if (!scatter(m, it, rng, &sc)) break;
      const R ac = std::fabs(dot(sc.ray.d, it.n));
      const V3<R> k{(sc.att.x * ac) / sc.pdf, (sc.att.y * ac) / sc.pdf, (sc.att.z * ac) / sc.pdf};
      beta = V3<R>{beta.x * k.x, beta.y * k.y, beta.z * k.z};
      ray = sc.ray;
    }
    return L;
  }

  float max_radiance = 0.f;  // the largest emitted radiance (+inf with a point light)
  std::vector<Mesh> meshes;
  std::vector<Object> objects;
  std::vector<Material> materials;
  std::vector<Light> lights;
  std::vector<Object> celems;       // constructive solids' elements
  std::vector<Node> nodes;
  std::vector<uint32_t> roots;      // the scene's primitives (tree nodes), in add order
  std::vector<uint32_t> unbounded;  // roots kept out of the BVH (Scene::commit)
  std::vector<uint32_t> prim_root;  // BVH primitive -> root node
  std::vector<AABB<R>> boxes;       // BVH primitive boxes
  std::vector<uint32_t> order;      // leaf slot -> BVH primitive
  std::vector<BNode> bnodes;
};

// PinHoleCamera, or ThinLensCamera::get_ray (thin_lens.rs:60-75): the lens sample
// (random_in_unit_disk, utils.rs:9-17, bounded at 64 draws) is drawn after the pixel jitter.
template <class R>
struct Camera {
  PinHoleCamera<R> pin;
  bool thin = false;
  R lens_radius = R(0), focal_distance = R(0);
  Ray<R> get_ray(R px, R py, Pcg32& rng) const {
    if (!thin) return pin.get_ray(px, py);
    const V3<R> cv = normalized(pin.raster_to_screen.point(V3<R>{px, py, R(0)}));
    const Ray<R> ray = make_ray(V3<R>{R(0), R(0), R(0)}, cv);
    R x = R(0), y = R(0);
    for (int k = 0; k < 64; ++k) {
      x = R(rng.uniform()) * R(2) - R(1);
      y = R(rng.uniform()) * R(2) - R(1);
      if (x * x + y * y < R(1)) break;
      if (k == 63) { x = x * R(0.5); y = y * R(0.5); }
    }
    const V3<R> lens{x * lens_radius, y * lens_radius, R(0)};
    const R ft = focal_distance / cv.z;
    const V3<R> dir = normalized((ray.o + ray.d * ft) - lens);
    return make_ray(pin.cam_to_world.point(lens), pin.cam_to_world.direction(dir));
  }
};

template <class R>
Camera<R> make_camera(const OCameraDesc& c) {
  const V3<R> pos{R(c.position[0]), R(c.position[1]), R(c.position[2])};
  const V3<R> look{R(c.look_at[0]), R(c.look_at[1]), R(c.look_at[2])};
  const V3<R> up{R(c.up[0]), R(c.up[1]), R(c.up[2])};
  Camera<R> cam{PinHoleCamera<R>(c.width, c.height, R(c.fov), R(c.near), R(c.far), M4<R>::look_at(pos, look, up))};
  cam.thin = c.thin_lens != 0;
  cam.lens_radius = R(c.lens_radius);
  cam.focal_distance = R(c.focal_distance);
  return cam;
}

}  // namespace oracle
