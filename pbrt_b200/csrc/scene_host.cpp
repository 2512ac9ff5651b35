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

namespace {

// aabound.rs:68-75: an empty box counts as bounded; otherwise every extent must be finite
bool is_bounded(const Box3& b) {
  for (int a = 0; a < 3; ++a)
    if (b.lo[a] > b.hi[a]) return true;
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(b.hi[a] - b.lo[a])) return false;
  return true;
}

// AABoundingBox::transform (aabound.rs:437-468)
Box3 transform_box(const Box3& b, const float* to_world) {
  Box3 t;
  if (!is_bounded(b)) {
    for (int a = 0; a < 3; ++a) { t.lo[a] = -INFINITY; t.hi[a] = INFINITY; }
    return t;
  }
  const float* lo = b.lo;
  const float* hi = b.hi;
  const V3f c[8] = {{lo[0], lo[1], lo[2]}, {lo[0], lo[1], hi[2]}, {lo[0], hi[1], lo[2]}, {lo[0], hi[1], hi[2]},
                    {hi[0], hi[1], hi[2]}, {hi[0], hi[1], lo[2]}, {hi[0], lo[1], hi[2]}, {hi[0], lo[1], lo[2]}};
  t.set_empty();
  for (const V3f& p0 : c) {
    const V3f p = xf_point(to_world, p0);
    t.lo[0] = std::fmin(t.lo[0], p.x); t.lo[1] = std::fmin(t.lo[1], p.y); t.lo[2] = std::fmin(t.lo[2], p.z);
    t.hi[0] = std::fmax(t.hi[0], p.x); t.hi[1] = std::fmax(t.hi[1], p.y); t.hi[2] = std::fmax(t.hi[2], p.z);
  }
  return t;
}

struct Xf {
  const float* to_world;
  const float* to_local;
};

// Flattens the object tree: every placed Simple becomes a leaf with its chain of transforms.
class Flattener {
 public:
  Flattener(const pbrt_scene_desc& d, const std::vector<Box3>& shape_boxes, FlatScene* out)
      : d_(d), shape_boxes_(shape_boxes), out_(out) {}

  // Acyclic, in range, of known kinds.
  bool check_tree(std::string* err) {
    if (!d_.nodes) return true;
    for (uint32_t i = 0; i < d_.node_count; ++i) {
      const pbrt_node_desc& n = d_.nodes[i];
      if (n.kind == PBRT_NODE_SIMPLE) {
        if (n.object >= d_.object_count) { *err = "node " + std::to_string(i) + ": bad object"; return false; }
      } else if (n.kind == PBRT_NODE_TRANSFORMED || n.kind == PBRT_NODE_COMPOUND) {
        const uint64_t cnt = n.kind == PBRT_NODE_TRANSFORMED ? 1 : n.count;
        if (uint64_t(n.first) + cnt > d_.child_count || (cnt && !d_.node_children)) {
          *err = "node " + std::to_string(i) + ": children out of range";
          return false;
        }
        for (uint64_t k = 0; k < cnt; ++k)
          if (d_.node_children[n.first + k] >= d_.node_count) {
            *err = "node " + std::to_string(i) + ": bad child";
            return false;
          }
      } else {
        *err = "node " + std::to_string(i) + ": unknown kind";
        return false;
      }
    }
    if (d_.root_count && !d_.roots) { *err = "roots is NULL"; return false; }
    for (uint32_t r = 0; r < d_.root_count; ++r)
      if (d_.roots[r] >= d_.node_count) { *err = "root " + std::to_string(r) + ": bad node"; return false; }
    std::vector<uint8_t> state(d_.node_count, 0);
    std::vector<std::pair<uint32_t, uint32_t>> stack;  // node, next child
    for (uint32_t r = 0; r < d_.root_count; ++r) {
      if (state[d_.roots[r]] == 2) continue;
      stack.push_back({d_.roots[r], 0});
      state[d_.roots[r]] = 1;
      while (!stack.empty()) {
        auto& top = stack.back();
        const pbrt_node_desc& n = d_.nodes[top.first];
        const uint32_t cnt = n.kind == PBRT_NODE_TRANSFORMED ? 1u : (n.kind == PBRT_NODE_COMPOUND ? n.count : 0u);
        if (top.second == cnt) {
          state[top.first] = 2;
          stack.pop_back();
          continue;
        }
        const uint32_t c = d_.node_children[n.first + top.second++];
        if (state[c] == 1) { *err = "the object tree has a cycle"; return false; }
        if (state[c] == 0) {
          state[c] = 1;
          stack.push_back({c, 0});
        }
      }
    }
    return true;
  }

  // The scene's primitives in order: (reference, box).
  bool run(std::vector<uint32_t>* refs, std::vector<Box3>* boxes, std::vector<uint8_t>* grouped, std::string* err) {
    grouped_ = grouped;
    const uint32_t n = d_.nodes ? d_.root_count : d_.object_count;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t first = uint32_t(out_->objects.size());
      std::vector<Xf> chain;
      Box3 box;
      if (d_.nodes) {
        if (!node(d_.roots[i], &chain, 0, err)) return false;
        box = node_box(d_.roots[i]);
      } else {
        if (!leaf(i, &chain, err)) return false;
        box = object_box(i);
      }
      const uint32_t count = uint32_t(out_->objects.size()) - first;
      if (count == 1) {
        refs->push_back(first);
      } else {
        refs->push_back(kGroupBit | uint32_t(out_->groups.size()));
        out_->groups.push_back(GroupRec{first, count});
        for (uint32_t k = first; k < first + count; ++k) (*grouped_)[k] = 1;
      }
      boxes->push_back(box);
    }
    return true;
  }

 private:
  Box3 object_box(uint32_t oi) const {
    const pbrt_object_desc& o = d_.objects[oi];
    return o.transformed ? transform_box(shape_boxes_[oi], o.to_world) : shape_boxes_[oi];
  }

  // get_bounding_box of a node (transformed.rs:70-74, compound.rs:57-64)
  Box3 node_box(uint32_t ni) const {
    const pbrt_node_desc& n = d_.nodes[ni];
    if (n.kind == PBRT_NODE_SIMPLE) return object_box(n.object);
    if (n.kind == PBRT_NODE_TRANSFORMED) return transform_box(node_box(d_.node_children[n.first]), n.to_world);
    Box3 u;
    u.set_empty();
    for (uint32_t k = 0; k < n.count; ++k) u.grow(node_box(d_.node_children[n.first + k]));
    return u;
  }

  bool node(uint32_t ni, std::vector<Xf>* chain, int depth, std::string* err) {
    if (depth > 64) { *err = "the object tree is deeper than 64 levels"; return false; }
    const pbrt_node_desc& n = d_.nodes[ni];
    if (n.kind == PBRT_NODE_SIMPLE) return leaf(n.object, chain, err);
    if (n.kind == PBRT_NODE_TRANSFORMED) {
      chain->push_back(Xf{n.to_world, n.to_local});
      const bool ok = node(d_.node_children[n.first], chain, depth + 1, err);
      chain->pop_back();
      return ok;
    }
    for (uint32_t k = 0; k < n.count; ++k)
      if (!node(d_.node_children[n.first + k], chain, depth + 1, err)) return false;
    return true;
  }

  bool leaf(uint32_t oi, std::vector<Xf>* chain, std::string* err) {
    const pbrt_object_desc& o = d_.objects[oi];
    if (out_->objects.size() >= (1u << 26)) { *err = "the object tree places more than 2^26 objects"; return false; }
    std::vector<Xf> c = *chain;
    if (o.transformed) c.push_back(Xf{o.to_world, o.to_local});
    ObjRec r{};
    r.shape = o.shape;
    r.mesh = o.mesh;
    r.material = o.material;
    r.desc_id = oi;
    r.xf_count = uint32_t(c.size());
    if (o.shape == PBRT_SHAPE_CSG) {
      r.csg_op = o.csg_op;
      r.csg_first = o.csg_first;
      r.csg_count = o.csg_count;
    }
    switch (o.shape) {
      case PBRT_SHAPE_SPHERE: r.p[0] = o.radius; break;
      case PBRT_SHAPE_CYLINDER: r.p[0] = o.radius; r.p[1] = o.height / 2.0f; break;  // Cylinder::new
      case PBRT_SHAPE_RECTANGLE: r.p[0] = o.radius / 2.0f; r.p[1] = o.height / 2.0f; break;  // Rectangle::new
      case PBRT_SHAPE_AABOX:
        for (int a = 0; a < 3; ++a) r.p[a] = o.extent[a] * 0.5f;  // AABox::new
        break;
      default: break;
    }
    if (!c.empty()) {
      std::memcpy(r.to_world, c[0].to_world, sizeof(r.to_world));
      std::memcpy(r.to_local, c[0].to_local, sizeof(r.to_local));
    }
    r.xf_rest = uint32_t(out_->xforms.size());
    for (size_t k = 1; k < c.size(); ++k) {
      XfRec x;
      std::memcpy(x.to_world, c[k].to_world, sizeof(x.to_world));
      std::memcpy(x.to_local, c[k].to_local, sizeof(x.to_local));
      out_->xforms.push_back(x);
    }
    out_->objects.push_back(r);
    grouped_->push_back(0);
    return true;
  }

  const pbrt_scene_desc& d_;
  const std::vector<Box3>& shape_boxes_;
  FlatScene* out_;
  std::vector<uint8_t>* grouped_ = nullptr;
};

// The box of a plain shape before any transform (its get_bounding_box), with its sizes checked.
bool plain_shape_box(const pbrt_object_desc& o, const pbrt_scene_desc& d, const FlatScene* out, const std::string& who,
                   Box3* bp, std::string* err) {
  Box3& b = *bp;
  switch (o.shape) {
    case PBRT_SHAPE_MESH: {
      if (o.mesh >= d.mesh_count) { *err = who + "bad mesh"; return false; }
      const FlatMesh& fm = out->meshes[o.mesh];
      for (int a = 0; a < 3; ++a) { b.lo[a] = fm.bounds_min[a]; b.hi[a] = fm.bounds_max[a]; }
      break;
    }
    case PBRT_SHAPE_SPHERE:
      if (!(o.radius > 0.0f) || !std::isfinite(o.radius)) { *err = who + "sphere radius must be > 0"; return false; }
      for (int a = 0; a < 3; ++a) { b.lo[a] = -o.radius; b.hi[a] = o.radius; }
      break;
    case PBRT_SHAPE_CYLINDER: {
      if (!(o.radius > 0.0f) || !(o.height > 0.0f)) { *err = who + "bad cylinder"; return false; }
      const float hh = o.height / 2.0f;
      b.lo[0] = -o.radius; b.lo[1] = -hh; b.lo[2] = -o.radius;
      b.hi[0] = o.radius; b.hi[1] = hh; b.hi[2] = o.radius;
      break;
    }
    case PBRT_SHAPE_RECTANGLE: {  // rectangle.rs:63-69: flat at y = 0
      if (!(o.radius >= 0.0f) || !(o.height >= 0.0f) || !std::isfinite(o.radius) || !std::isfinite(o.height)) {
        *err = who + "rectangle sides must be finite and >= 0";
        return false;
      }
      const float hw = o.radius / 2.0f, hh = o.height / 2.0f;
      b.lo[0] = -hw; b.lo[1] = 0.0f; b.lo[2] = -hh;
      b.hi[0] = hw; b.hi[1] = 0.0f; b.hi[2] = hh;
      break;
    }
    case PBRT_SHAPE_AABOX:
      for (int a = 0; a < 3; ++a) {
        if (!(o.extent[a] >= 0.0f) || !std::isfinite(o.extent[a])) {
          *err = who + "box extents must be finite and >= 0";
          return false;
        }
        const float h = o.extent[a] * 0.5f;
        b.lo[a] = 0.0f - h;
        b.hi[a] = h;
      }
      break;
    case PBRT_SHAPE_PLANE:  // plane.rs:89-93: the half-space below y = 0
      for (int a = 0; a < 3; ++a) { b.lo[a] = -INFINITY; b.hi[a] = INFINITY; }
      b.hi[1] = 0.0f;
      break;
    default: *err = who + "unknown shape"; return false;
    }
  return true;
}

}  // namespace

bool build_scene(const pbrt_scene_desc& d, FlatScene* out, std::string* err, const std::vector<MeshPrebuilt>* pre) {
  if (d.object_count == 0) { *err = "a scene needs at least one object"; return false; }
  if (!d.objects) { *err = "objects is NULL"; return false; }
  if (d.mesh_count && !d.meshes) { *err = "meshes is NULL"; return false; }
  if (d.material_count == 0 || !d.materials) { *err = "a scene needs at least one material"; return false; }
  if (d.light_count && !d.lights) { *err = "lights is NULL"; return false; }
  if (d.nodes && d.root_count == 0) { *err = "a scene with an object tree needs at least one root"; return false; }
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
    if (pre && i < pre->size() && (*pre)[i].used) {  // built on the GPU: its bounds and statistics
      const MeshPrebuilt& pb = (*pre)[i];
      for (int a = 0; a < 3; ++a) {
        out->meshes[i].bounds_min[a] = pb.bounds_min[a];
        out->meshes[i].bounds_max[a] = pb.bounds_max[a];
      }
      out->meshes[i].stats = pb.stats;
    } else if (!build_mesh_bvh(md.vertices, md.vertex_count, md.indices, md.triangle_count, bp, &out->meshes[i],
                               &e)) {
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
    if (m.texture > PBRT_TEXTURE_CHECKERBOARD) {
      *err = "material " + std::to_string(i) + ": unknown texture";
      return false;
    }
    MatRec r{};
    r.kind = m.kind;
    r.texture = m.texture;
    r.fuzz = m.fuzz;
    r.ior = m.ior;
    for (int c = 0; c < 3; ++c) {
      r.color[c] = m.color[c];
      r.color2[c] = m.color2[c];
    }
    r.scale = m.scale;
    out->materials.push_back(r);
    if (m.kind == PBRT_MAT_DIFFUSE_LIGHT)
      for (int c = 0; c < 3; ++c) {
        out->max_radiance = std::max(out->max_radiance, m.color[c]);
        if (m.texture == PBRT_TEXTURE_CHECKERBOARD) out->max_radiance = std::max(out->max_radiance, m.color2[c]);
      }
    if (m.kind == PBRT_MAT_DIELECTRIC) out->has_dielectric = true;
  }

  // the elements of the constructive solids: plain shapes placed by their transforms
  if (d.csg_elem_count && !d.csg_elems) { *err = "csg_elems is NULL"; return false; }
  std::vector<Box3> elem_boxes(d.csg_elem_count);
  for (uint32_t i = 0; i < d.csg_elem_count; ++i) {
    const pbrt_csg_elem_desc& e = d.csg_elems[i];
    pbrt_object_desc as{};
    as.shape = e.shape;
    as.mesh = e.mesh;
    as.radius = e.radius;
    as.height = e.height;
    for (int a = 0; a < 3; ++a) as.extent[a] = e.extent[a];
    const std::string who = "csg element " + std::to_string(i) + ": ";
    if (e.shape >= PBRT_SHAPE_CSG) { *err = who + "an element is a plain shape"; return false; }
    Box3 b;
    if (!plain_shape_box(as, d, out, who, &b, err)) return false;
    if (e.shape == PBRT_SHAPE_MESH && d.meshes[e.mesh].triangle_count > (1u << 24)) {
      *err = who + "a mesh inside a constructive solid has at most 2^24 triangles";
      return false;
    }
    elem_boxes[i] = transform_box(b, e.to_world);
    CsgRec r{};
    r.shape = e.shape;
    r.mesh = e.mesh;
    switch (e.shape) {
      case PBRT_SHAPE_SPHERE: r.p[0] = e.radius; break;
      case PBRT_SHAPE_CYLINDER: r.p[0] = e.radius; r.p[1] = e.height / 2.0f; break;
      case PBRT_SHAPE_RECTANGLE: r.p[0] = e.radius / 2.0f; r.p[1] = e.height / 2.0f; break;
      case PBRT_SHAPE_AABOX:
        for (int a = 0; a < 3; ++a) r.p[a] = e.extent[a] * 0.5f;
        break;
      default: break;
    }
    std::memcpy(r.to_world, e.to_world, sizeof(r.to_world));
    std::memcpy(r.to_local, e.to_local, sizeof(r.to_local));
    out->csg.push_back(r);
  }

  // every object's shape box, before any transform
  std::vector<Box3> shape_boxes(d.object_count);
  for (uint32_t i = 0; i < d.object_count; ++i) {
    const pbrt_object_desc& o = d.objects[i];
    const std::string who = "object " + std::to_string(i) + ": ";
    if (o.material >= d.material_count) { *err = who + "bad material"; return false; }
    Box3& b = shape_boxes[i];
    if (o.shape == PBRT_SHAPE_CSG) {  // Union / Intersection / Substraction::get_bounding_box
      if (o.csg_op > PBRT_CSG_SUBTRACTION || uint64_t(o.csg_first) + o.csg_count > d.csg_elem_count ||
          o.csg_count > 256) {
        *err = who + "bad constructive solid (operation, element range, at most 256 elements)";
        return false;
      }
      if (o.csg_count == 0) {
        for (int a = 0; a < 3; ++a) { b.lo[a] = 0.0f; b.hi[a] = 0.0f; }
        continue;
      }
      b = elem_boxes[o.csg_first];
      if (o.csg_op == PBRT_CSG_SUBTRACTION) continue;
      for (uint32_t k = 1; k < o.csg_count; ++k) {
        const Box3& x = elem_boxes[o.csg_first + k];
        if (o.csg_op == PBRT_CSG_UNION) {
          b.grow(x);
        } else {  // intersect_with (aabound.rs:397-401)
          for (int a = 0; a < 3; ++a) {
            b.lo[a] = std::fmax(b.lo[a], x.lo[a]);
            b.hi[a] = std::fmin(b.hi[a], x.hi[a]);
          }
        }
      }
      continue;
    }
    if (!plain_shape_box(o, d, out, who, &b, err)) return false;
  }

  Flattener fl(d, shape_boxes, out);
  if (!fl.check_tree(err)) return false;
  std::vector<uint32_t> refs;
  std::vector<Box3> boxes;
  std::vector<uint8_t> grouped;
  if (!fl.run(&refs, &boxes, &grouped, err)) return false;
  out->primitive_count = refs.size();
  // Scene::commit: the unbounded primitives stay out of the tree, in scene order
  std::vector<uint32_t> bounded_refs;
  std::vector<Box3> bounded_boxes;
  for (size_t i = 0; i < refs.size(); ++i) {
    if (is_bounded(boxes[i])) {
      bounded_refs.push_back(refs[i]);
      bounded_boxes.push_back(boxes[i]);
    } else {
      out->unbounded.push_back(refs[i]);
    }
  }
  if (!bounded_boxes.empty()) {
    std::vector<uint32_t> slot;
    TopBuilder(bounded_boxes).run(&out->top, &slot, &out->top_depth);
    out->order.resize(slot.size());
    for (size_t k = 0; k < slot.size(); ++k) out->order[k] = bounded_refs[slot[k]];
  }
  if (refs.size() == 1 && out->unbounded.empty() && !(refs[0] & kGroupBit)) {
    const ObjRec& r = out->objects[refs[0]];
    if (r.shape == PBRT_SHAPE_MESH && r.xf_count == 0) out->single_mesh = int(r.mesh);
  }

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
    const std::string who = "light " + std::to_string(i) + ": ";
    if (l.kind > PBRT_LIGHT_AREA) { *err = who + "unknown kind"; return false; }
    if (l.kind == PBRT_LIGHT_AREA) {
      if (l.object >= d.object_count) { *err = who + "bad object"; return false; }
      // the emitter: the one leaf placing the object, a primitive of its own under at most one transform
      uint32_t leaf = 0, found = 0;
      for (uint32_t k = 0; k < out->objects.size(); ++k)
        if (out->objects[k].desc_id == l.object) { leaf = k; ++found; }
      if (found != 1 || grouped[leaf] || out->objects[leaf].xf_count > 1) {
        *err = who + "an area light's object must be placed once, as a primitive of the scene under at most one "
                     "transform";
        return false;
      }
      const ObjRec& ob = out->objects[leaf];
      r.object = leaf;
      const pbrt_material_desc& em = d.materials[ob.material];
      if (em.kind != PBRT_MAT_DIFFUSE_LIGHT) {
        *err = who + "an area light's object must have a diffuse-light material";
        return false;
      }
      if (em.texture != PBRT_TEXTURE_COLOR) { *err = who + "an area light's emission must be a plain colour"; return false; }
      if (ob.shape == PBRT_SHAPE_MESH) {
        const std::vector<float>& v = out->mesh_v[ob.mesh];
        const std::vector<uint32_t>& ix = out->mesh_idx[ob.mesh];
        r.tri_first = uint32_t(out->light_cdf.size());
        r.tri_count = uint32_t(ix.size() / 3);
        float run = 0.0f;
        for (size_t t = 0; t < ix.size() / 3; ++t) {
          V3f p[3];
          for (int k = 0; k < 3; ++k) {
            const uint32_t vi = ix[3 * t + k];
            const V3f q{v[3 * size_t(vi)], v[3 * size_t(vi) + 1], v[3 * size_t(vi) + 2]};
            p[k] = ob.xf_count ? xf_point(ob.to_world, q) : q;
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
      } else if (ob.shape == PBRT_SHAPE_SPHERE) {
        r.area = 4.0f * kPi * ob.p[0] * ob.p[0];
      } else {
        *err = who + "area lights are triangle meshes or spheres";
        return false;
      }
      if (!(r.area > 0.0f)) { *err = who + "zero area"; return false; }
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
  r.thin_lens = c.thin_lens ? 1u : 0u;
  r.lens_radius = c.lens_radius;
  r.focal_distance = c.focal_distance;
  return r;
}

}  // namespace pbrt
