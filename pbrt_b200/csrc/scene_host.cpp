// scene_host.cpp — host-side scene build; see scene_host.hpp. Compiled with
// -ffp-contract=off so every FP32 expression rounds as the reference's does.
#include "scene_host.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <utility>

namespace pbrt {
namespace {

constexpr float kPi = 3.14159265358979323846f;

struct Box3 {
  float lo[3], hi[3];
  void set_empty() {
    for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
  }
  void grow(const Box3& b) {
    for (int a = 0; a < 3; ++a) { lo[a] = std::fmin(lo[a], b.lo[a]); hi[a] = std::fmax(hi[a], b.hi[a]); }
  }
  float centroid(int a) const { return (hi[a] + lo[a]) * 0.5f; }
};

struct V3f {
  float x, y, z;
};
V3f sub(V3f a, V3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3f scale(V3f a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dot(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3f cross(V3f u, V3f v) { return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x}; }
V3f normalized(V3f v) {
  const float inv = 1.0f / std::sqrt(dot(v, v));
  return scale(v, inv);
}

V3f xf_point(const float* m, V3f v) {
  return {m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3], m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7],
          m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11]};
}

// Matrix4 in FP32 (src/geom/matrix4.rs)
struct M4f {
  float m[4][4];
  static M4f zero() {
    M4f r;
    for (auto& row : r.m)
      for (float& x : row) x = 0.0f;
    return r;
  }
  static M4f identity() {
    M4f r = zero();
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
    return r;
  }
  static M4f translation(float x, float y, float z) {
    M4f r = identity();
    r.m[0][3] = x; r.m[1][3] = y; r.m[2][3] = z;
    return r;
  }
  static M4f scaling(float x, float y, float z) {
    M4f r = zero();
    r.m[0][0] = x; r.m[1][1] = y; r.m[2][2] = z; r.m[3][3] = 1.0f;
    return r;
  }
  static M4f perspective(float fov, float n, float f) {  // matrix4.rs:70-79
    const float s = 1.0f / std::tan(fov / 2.0f);
    M4f r = zero();
    r.m[0][0] = s; r.m[1][1] = s; r.m[2][2] = f / (f - n); r.m[2][3] = -f * n / (f - n); r.m[3][2] = 1.0f;
    return r;
  }
  static M4f look_at(V3f pos, V3f look, V3f up) {  // matrix4.rs:81-98
    const V3f dir = normalized(sub(look, pos));
    const V3f nu = normalized(up);
    const V3f right = normalized(cross(nu, dir));
    const V3f ru = cross(dir, right);
    M4f r = zero();
    r.m[0][0] = right.x; r.m[0][1] = ru.x; r.m[0][2] = dir.x; r.m[0][3] = pos.x;
    r.m[1][0] = right.y; r.m[1][1] = ru.y; r.m[1][2] = dir.y; r.m[1][3] = pos.y;
    r.m[2][0] = right.z; r.m[2][1] = ru.z; r.m[2][2] = dir.z; r.m[2][3] = pos.z;
    r.m[3][3] = 1.0f;
    return r;
  }
  M4f inverse() const {  // Gauss-Jordan with full pivoting (matrix4.rs:100-174)
    int indxc[4] = {0, 0, 0, 0}, indxr[4] = {0, 0, 0, 0}, ipiv[4] = {0, 0, 0, 0};
    float a[4][4];
    std::memcpy(a, m, sizeof(a));
    for (int i = 0; i < 4; ++i) {
      int irow = 0, icol = 0;
      float big = 0.0f;
      for (int j = 0; j < 4; ++j)
        if (ipiv[j] != 1)
          for (int k = 0; k < 4; ++k)
            if (ipiv[k] == 0 && std::fabs(a[j][k]) >= big) { big = std::fabs(a[j][k]); irow = j; icol = k; }
      ipiv[icol] += 1;
      if (irow != icol)
        for (int k = 0; k < 4; ++k) std::swap(a[irow][k], a[icol][k]);
      indxr[i] = irow;
      indxc[i] = icol;
      const float pivinv = 1.0f / a[icol][icol];
      a[icol][icol] = 1.0f;
      for (int j = 0; j < 4; ++j) a[icol][j] *= pivinv;
      for (int j = 0; j < 4; ++j)
        if (j != icol) {
          const float save = a[j][icol];
          a[j][icol] = 0.0f;
          for (int k = 0; k < 4; ++k) a[j][k] -= a[icol][k] * save;
        }
    }
    for (int j = 3; j >= 0; --j)
      if (indxr[j] != indxc[j])
        for (int k = 0; k < 4; ++k) std::swap(a[k][indxr[j]], a[k][indxc[j]]);
    M4f r;
    std::memcpy(r.m, a, sizeof(a));
    return r;
  }
  M4f operator*(const M4f& o) const {  // matrix4.rs:216-231
    M4f r = zero();
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 4; ++k) r.m[i][j] += m[i][k] * o.m[k][j];
    return r;
  }
};

class TopBuilder {
 public:
  TopBuilder(const std::vector<Box3>& boxes) : boxes_(boxes) {}

  void run(std::vector<GpuNode>* gpu, std::vector<uint32_t>* order, uint32_t* depth) {
    const uint32_t n = uint32_t(boxes_.size());
    order_.resize(n);
    for (uint32_t i = 0; i < n; ++i) order_[i] = i;
    nodes_.clear();
    nodes_.push_back(Node{Box3{}, 0, n, 1});
    subdivide(0);
    gpu->assign(nodes_.size() + 1, GpuNode{});
    *depth = 0;
    for (size_t k = 0; k < nodes_.size(); ++k) {
      const Node& r = nodes_[k];
      GpuNode& g = (*gpu)[k == 0 ? 0 : k + 1];
      for (int a = 0; a < 3; ++a) { g.bmin[a] = r.box.lo[a]; g.bmax[a] = r.box.hi[a]; }
      g.left_first = r.count > 0 ? r.left_first : r.left_first + 1;
      g.count = r.count;
      *depth = std::max(*depth, r.depth);
    }
    *order = order_;
  }

 private:
  struct Node {
    Box3 box;
    uint32_t left_first, count, depth;
  };

  // BVH::subdivide (bvh.rs:291-335), recursive as the reference is (depth ~ log2 n).
  Box3 subdivide(uint32_t ni) {
    const uint32_t first = nodes_[ni].left_first, count = nodes_[ni].count;
    if (count == 1) {
      nodes_[ni].box = boxes_[order_[first]];
      return nodes_[ni].box;
    }
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t k = first; k < first + count; ++k)
      for (int a = 0; a < 3; ++a) {
        const float c = boxes_[order_[k]].centroid(a);
        mn[a] = std::fmin(mn[a], c);
        mx[a] = std::fmax(mx[a], c);
      }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (mx[a] - mn[a] > mx[axis] - mn[axis]) axis = a;
    std::stable_sort(order_.begin() + first, order_.begin() + first + count, [&](uint32_t a, uint32_t b) {
      return boxes_[a].centroid(axis) < boxes_[b].centroid(axis);
    });
    const uint32_t lc = count / 2;
    const uint32_t li = uint32_t(nodes_.size());
    const uint32_t dep = nodes_[ni].depth + 1;
    nodes_.push_back(Node{Box3{}, first, lc, dep});
    nodes_.push_back(Node{Box3{}, first + lc, count - lc, dep});
    nodes_[ni].left_first = li;
    nodes_[ni].count = 0;
    const Box3 lb = subdivide(li);
    const Box3 rb = subdivide(li + 1);
    Box3 u;
    u.set_empty();
    u.grow(lb);
    u.grow(rb);
    nodes_[ni].box = u;
    return u;
  }

  const std::vector<Box3>& boxes_;
  std::vector<uint32_t> order_;
  std::vector<Node> nodes_;
};

}  // namespace

bool build_scene(const pbrt_scene_desc& d, FlatScene* out, std::string* err) {
  if (d.object_count == 0) { *err = "a scene needs at least one object"; return false; }
  if (!d.objects) { *err = "objects is NULL"; return false; }
  if (d.mesh_count && !d.meshes) { *err = "meshes is NULL"; return false; }
  if (d.material_count == 0 || !d.materials) { *err = "a scene needs at least one material"; return false; }
  if (d.light_count && !d.lights) { *err = "lights is NULL"; return false; }
  MeshBuildParams bp;
  bp.bins = d.bvh_bins ? int(d.bvh_bins) : 8;
  bp.max_leaf = d.bvh_max_leaf ? d.bvh_max_leaf : 1;

  out->meshes.resize(d.mesh_count);
  out->mesh_v.resize(d.mesh_count);
  out->mesh_idx.resize(d.mesh_count);
  out->mesh_fmat.resize(d.mesh_count);
  for (uint32_t i = 0; i < d.mesh_count; ++i) {
    const pbrt_mesh_desc& md = d.meshes[i];
    std::string e;
    if (!build_mesh_bvh(md.vertices, md.vertex_count, md.indices, md.triangle_count, bp, &out->meshes[i], &e)) {
      *err = "mesh " + std::to_string(i) + ": " + e;
      return false;
    }
    out->mesh_v[i].assign(md.vertices, md.vertices + 3 * size_t(md.vertex_count));
    out->mesh_idx[i].assign(md.indices, md.indices + 3 * size_t(md.triangle_count));
    if (md.face_materials) {
      for (uint32_t t = 0; t < md.triangle_count; ++t)
        if (md.face_materials[t] >= d.material_count) {
          *err = "mesh " + std::to_string(i) + ": triangle " + std::to_string(t) + " has a bad material";
          return false;
        }
      out->mesh_fmat[i].assign(md.face_materials, md.face_materials + md.triangle_count);
    }
  }

  for (uint32_t i = 0; i < d.material_count; ++i) {
    const pbrt_material_desc& m = d.materials[i];
    if (m.kind > PBRT_MAT_DIFFUSE_LIGHT) { *err = "material " + std::to_string(i) + ": unknown kind"; return false; }
    MatRec r{};
    r.kind = m.kind;
    r.fuzz = m.fuzz;
    r.ior = m.ior;
    for (int c = 0; c < 3; ++c) r.color[c] = m.color[c];
    out->materials.push_back(r);
    if (m.kind == PBRT_MAT_DIFFUSE_LIGHT)
      for (int c = 0; c < 3; ++c) out->max_radiance = std::max(out->max_radiance, m.color[c]);
    if (m.kind == PBRT_MAT_DIELECTRIC) out->has_dielectric = true;
  }

  std::vector<Box3> boxes(d.object_count);
  for (uint32_t i = 0; i < d.object_count; ++i) {
    const pbrt_object_desc& o = d.objects[i];
    ObjRec r{};
    r.shape = o.shape;
    r.mesh = o.mesh;
    r.material = o.material;
    r.transformed = o.transformed ? 1u : 0u;
    r.radius = o.radius;
    r.half_height = o.height / 2.0f;  // Cylinder::new (cylinder.rs:12-19)
    std::memcpy(r.to_world, o.to_world, sizeof(r.to_world));
    std::memcpy(r.to_local, o.to_local, sizeof(r.to_local));
    if (o.material >= d.material_count) { *err = "object " + std::to_string(i) + ": bad material"; return false; }
    Box3 b;
    if (o.shape == PBRT_SHAPE_MESH) {
      if (o.mesh >= d.mesh_count) { *err = "object " + std::to_string(i) + ": bad mesh"; return false; }
      const FlatMesh& fm = out->meshes[o.mesh];
      for (int a = 0; a < 3; ++a) { b.lo[a] = fm.bounds_min[a]; b.hi[a] = fm.bounds_max[a]; }
    } else if (o.shape == PBRT_SHAPE_SPHERE) {
      if (!(o.radius > 0.0f)) { *err = "object " + std::to_string(i) + ": sphere radius must be > 0"; return false; }
      for (int a = 0; a < 3; ++a) { b.lo[a] = -o.radius; b.hi[a] = o.radius; }
    } else if (o.shape == PBRT_SHAPE_CYLINDER) {
      if (!(o.radius > 0.0f) || !(o.height > 0.0f)) { *err = "object " + std::to_string(i) + ": bad cylinder"; return false; }
      b.lo[0] = -o.radius; b.lo[1] = -r.half_height; b.lo[2] = -o.radius;
      b.hi[0] = o.radius; b.hi[1] = r.half_height; b.hi[2] = o.radius;
    } else {
      *err = "object " + std::to_string(i) + ": unknown shape";
      return false;
    }
    if (o.transformed) {  // the eight corners (aabound.rs:437-468)
      const float* lo = b.lo;
      const float* hi = b.hi;
      const V3f c[8] = {{lo[0], lo[1], lo[2]}, {lo[0], lo[1], hi[2]}, {lo[0], hi[1], lo[2]}, {lo[0], hi[1], hi[2]},
                        {hi[0], hi[1], hi[2]}, {hi[0], hi[1], lo[2]}, {hi[0], lo[1], hi[2]}, {hi[0], lo[1], lo[2]}};
      Box3 t;
      t.set_empty();
      for (const V3f& p0 : c) {
        const V3f p = xf_point(o.to_world, p0);
        t.lo[0] = std::fmin(t.lo[0], p.x); t.lo[1] = std::fmin(t.lo[1], p.y); t.lo[2] = std::fmin(t.lo[2], p.z);
        t.hi[0] = std::fmax(t.hi[0], p.x); t.hi[1] = std::fmax(t.hi[1], p.y); t.hi[2] = std::fmax(t.hi[2], p.z);
      }
      b = t;
    }
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(b.lo[a]) || !std::isfinite(b.hi[a])) {
        *err = "object " + std::to_string(i) + ": unbounded objects are not supported";
        return false;
      }
    boxes[i] = b;
    out->objects.push_back(r);
  }
  TopBuilder(boxes).run(&out->top, &out->order, &out->top_depth);

  for (uint32_t i = 0; i < d.light_count; ++i) {
    const pbrt_light_desc& l = d.lights[i];
    LightRec r{};
    r.kind = l.kind;
    r.object = l.object;
    for (int c = 0; c < 3; ++c) {
      r.pos[c] = l.position[c];
      r.rad[c] = l.radiance[c];
      r.bottom[c] = l.bottom[c];
      r.top[c] = l.top[c];
    }
    if (l.kind > PBRT_LIGHT_AREA) { *err = "light " + std::to_string(i) + ": unknown kind"; return false; }
    if (l.kind == PBRT_LIGHT_AREA) {
      if (l.object >= d.object_count) { *err = "light " + std::to_string(i) + ": bad object"; return false; }
      const pbrt_object_desc& o = d.objects[l.object];
      if (d.materials[o.material].kind != PBRT_MAT_DIFFUSE_LIGHT) {
        *err = "light " + std::to_string(i) + ": an area light's object must have a diffuse-light material";
        return false;
      }
      if (o.shape == PBRT_SHAPE_MESH) {
        const std::vector<float>& v = out->mesh_v[o.mesh];
        const std::vector<uint32_t>& ix = out->mesh_idx[o.mesh];
        r.tri_first = uint32_t(out->light_cdf.size());
        r.tri_count = uint32_t(ix.size() / 3);
        float run = 0.0f;
        for (size_t t = 0; t < ix.size() / 3; ++t) {
          V3f p[3];
          for (int k = 0; k < 3; ++k) {
            const uint32_t vi = ix[3 * t + k];
            const V3f q{v[3 * size_t(vi)], v[3 * size_t(vi) + 1], v[3 * size_t(vi) + 2]};
            p[k] = o.transformed ? xf_point(o.to_world, q) : q;
            out->light_tris.push_back(p[k].x);
            out->light_tris.push_back(p[k].y);
            out->light_tris.push_back(p[k].z);
          }
          const V3f cr = cross(sub(p[1], p[0]), sub(p[2], p[0]));
          const float a = 0.5f * std::sqrt(dot(cr, cr));
          run = run + a;
          out->light_cdf.push_back(run);
        }
        r.area = run;
      } else if (o.shape == PBRT_SHAPE_SPHERE) {
        r.area = 4.0f * kPi * o.radius * o.radius;
      } else {
        *err = "light " + std::to_string(i) + ": area lights are triangle meshes or spheres";
        return false;
      }
      if (!(r.area > 0.0f)) { *err = "light " + std::to_string(i) + ": zero area"; return false; }
    }
    out->lights.push_back(r);
    if (l.kind == PBRT_LIGHT_POINT) out->max_radiance = INFINITY;
    for (int c = 0; c < 3; ++c) {
      if (l.kind == PBRT_LIGHT_UNIFORM_INFINITE) out->max_radiance = std::max(out->max_radiance, l.radiance[c]);
      if (l.kind == PBRT_LIGHT_BACKGROUND_INFINITE)
        out->max_radiance = std::max(out->max_radiance, std::max(l.bottom[c], l.top[c]));
    }
  }
  return true;
}

CameraRec build_camera(const pbrt_camera_desc& c) {
  CameraRec r{};
  const float aspect = float(c.width) / float(c.height);
  float xmin, xmax, ymin, ymax;
  if (aspect > 1.0f) { xmin = -aspect; xmax = aspect; ymin = -1.0f; ymax = 1.0f; }
  else { xmin = -1.0f; xmax = 1.0f; ymin = -1.0f / aspect; ymax = 1.0f / aspect; }
  const M4f rs = ((M4f::perspective(c.fov, c.near, c.far).inverse() * M4f::translation(xmin, ymax, 0.0f)) *
                  M4f::scaling(xmax - xmin, ymin - ymax, 1.0f)) *
                 M4f::scaling(1.0f / float(c.width), 1.0f / float(c.height), 1.0f);
  const M4f cw = M4f::look_at(V3f{c.position[0], c.position[1], c.position[2]},
                              V3f{c.look_at[0], c.look_at[1], c.look_at[2]}, V3f{c.up[0], c.up[1], c.up[2]});
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.raster_to_screen[4 * i + j] = rs.m[i][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) r.cam_to_world[4 * i + j] = cw.m[i][j];
  r.width = c.width;
  r.height = c.height;
  r.near = c.near;
  r.far = c.far;
  return r;
}

}  // namespace pbrt
