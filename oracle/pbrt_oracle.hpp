// pbrt_oracle.hpp — TEST INFRASTRUCTURE, NOT THE PRODUCT.
//
// A CPU restatement of nmichel/pbrt's data-parallel hot path (ray/BVH traversal,
// Möller–Trumbore, analytic sphere/cylinder, the path integrator), written to be the
// checker of the CUDA path in pbrt_b200/. Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load it.
//
// Every function follows the reference's operation order so that, instantiated with
// R = double, it traverses what the Rust reference traverses (pinned by the exact hit
// counts the reference publishes in docs/mesures_bvh.md:706-713), and instantiated with
// R = float it is the FP32 restatement the GPU path must match bit for bit.
//
// Build with -ffp-contract=off -fno-fast-math: no fused multiply-add may be formed, since
// the reference's arithmetic has none.
//
// Citations are path:line inside the reference project (nmichel/pbrt).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <utility>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------------------
// Vector3 — src/geom/vector3.rs
// ---------------------------------------------------------------------------------------
template <class R>
struct V3 {
  R x, y, z;
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

template <class R> inline V3<R> v3(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R> inline V3<R> operator+(const V3<R>& a, const V3<R>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(const V3<R>& a, const V3<R>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(const V3<R>& a, R s) { return {a.x * s, a.y * s, a.z * s}; }

// dot: u.x*v.x + u.y*v.y + u.z*v.z, left to right (vector3.rs:291-296)
template <class R> inline R dot(const V3<R>& u, const V3<R>& v) { return u.x * v.x + u.y * v.y + u.z * v.z; }

// cross (vector3.rs:298-307)
template <class R> inline V3<R> cross(const V3<R>& u, const V3<R>& v) {
  return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}

// normalize: inv = 1 / sqrt(|v|²), v *= inv (vector3.rs:69-74)
template <class R> inline V3<R> normalized(const V3<R>& v) {
  R norm = dot(v, v);
  R inv = R(1) / std::sqrt(norm);
  return v * inv;
}

template <class R> inline R length(const V3<R>& v) { return std::sqrt(dot(v, v)); }

// Rust f64::min / f64::max drop a NaN operand; fmin/fmax do the same.
template <class R> inline R rmin(R a, R b) { return std::fmin(a, b); }
template <class R> inline R rmax(R a, R b) { return std::fmax(a, b); }

// ---------------------------------------------------------------------------------------
// Ray — src/geom/ray.rs:10-18 (the direction is always normalised on construction)
// ---------------------------------------------------------------------------------------
template <class R>
struct Ray {
  V3<R> o, d;
};

template <class R> inline Ray<R> make_ray(const V3<R>& o, const V3<R>& d) { return Ray<R>{o, normalized(d)}; }

// Ray::spawn_from_through (ray.rs:20-24): normalises twice, as the reference does.
template <class R> inline Ray<R> spawn_from_through(const V3<R>& from, const V3<R>& through) {
  V3<R> dir = normalized(through - from);
  return make_ray(from, dir);
}

// ---------------------------------------------------------------------------------------
// Axis-aligned box — src/geom/aabound.rs
// ---------------------------------------------------------------------------------------
template <class R> struct Limits {
  static R max() { return std::numeric_limits<R>::max(); }
  static R lowest() { return std::numeric_limits<R>::lowest(); }
  // Unit roundoff u = eps/2 (aabound.rs:26), γ(3) = 3u/(1-3u) (:34), widening 2γ(3) (:39),
  // evaluated in R's own arithmetic.
  static R slab_widening() {
    const R u = std::numeric_limits<R>::epsilon() * R(0.5);
    const R g3 = (R(3) * u) / (R(1) - R(3) * u);
    return R(2) * g3;
  }
};

template <class R>
struct AABB {
  V3<R> bmin, bmax;
  static AABB empty() { return AABB{{Limits<R>::max(), Limits<R>::max(), Limits<R>::max()},
                                    {Limits<R>::lowest(), Limits<R>::lowest(), Limits<R>::lowest()}}; }
  bool is_empty() const { return bmin.x > bmax.x || bmin.y > bmax.y || bmin.z > bmax.z; }
  // aabound.rs:68-75
  bool is_bounded() const {
    if (is_empty()) return true;
    V3<R> d = bmax - bmin;
    return std::isfinite(d.x) && std::isfinite(d.y) && std::isfinite(d.z);
  }
  // combine_with: minimize_by / maximize_by (aabound.rs:369-373, vector3.rs:108-133)
  void combine(const AABB& o) {
    bmin.x = rmin(bmin.x, o.bmin.x); bmin.y = rmin(bmin.y, o.bmin.y); bmin.z = rmin(bmin.z, o.bmin.z);
    bmax.x = rmax(bmax.x, o.bmax.x); bmax.y = rmax(bmax.y, o.bmax.y); bmax.z = rmax(bmax.z, o.bmax.z);
  }
  // half_area (aabound.rs:123-130)
  R half_area() const {
    if (is_empty()) return R(0);
    V3<R> d = bmax - bmin;
    return d.x * d.y + d.y * d.z + d.z * d.x;
  }
  // centroid (aabound.rs:132-134)
  V3<R> centroid() const { return (bmax + bmin) * R(0.5); }
};

// AABoundingBox::hit — conservative slab test (aabound.rs:323-355). Returns the entry
// distance through *entry (clamped to tmin) or false on a miss.
template <class R>
inline bool box_hit(const AABB<R>& b, const Ray<R>& ray, R tmin, R tmax, R* entry) {
  const R W = Limits<R>::slab_widening();
  for (int i = 0; i < 3; ++i) {
    const R d = ray.d[i];
    const R o = ray.o[i];
    if (d == R(0)) {
      if (o < b.bmin[i] || o > b.bmax[i]) return false;
      continue;
    }
    const R inv = R(1) / d;
    R t0 = (b.bmin[i] - o) * inv;
    R t1 = (b.bmax[i] - o) * inv;
    if (inv < R(0)) std::swap(t0, t1);
    t0 = t0 - std::fabs(t0) * W;
    t1 = t1 + std::fabs(t1) * W;
    tmin = rmax(t0, tmin);
    tmax = rmin(t1, tmax);
    if (tmax < tmin) return false;
  }
  *entry = tmin;
  return true;
}

// ---------------------------------------------------------------------------------------
// Möller–Trumbore — src/shapes/triangle_mesh/triangle_mesh.rs:183-217
// ---------------------------------------------------------------------------------------
template <class R>
struct TriHit {
  R t, u, v, w;
};

template <class R>
inline bool intersect_ray(const Ray<R>& ray, const V3<R>& p0, const V3<R>& p1, const V3<R>& p2, TriHit<R>* out) {
  const V3<R> edge1 = p1 - p0;
  const V3<R> edge2 = p2 - p0;
  const V3<R> pv = cross(ray.d, edge2);
  const R det = dot(edge1, pv);
  if (std::fabs(det) < R(1e-8)) return false;
  const R inv_det = R(1) / det;
  const V3<R> s = ray.o - p0;
  const R u = inv_det * dot(s, pv);
  if (u < R(0) || u > R(1)) return false;
  const V3<R> q = cross(s, edge1);
  const R v = inv_det * dot(ray.d, q);
  if (v < R(0) || u + v > R(1)) return false;
  const R t = inv_det * dot(edge2, q);
  out->t = t;
  out->u = u;
  out->v = v;
  out->w = R(1) - u - v;
  return true;
}

// ---------------------------------------------------------------------------------------
// Mesh BVH — src/shapes/triangle_mesh/bvh.rs
//
// The reference hard-codes 8 bins (bvh.rs:129) and keeps splitting while the binned SAH
// beats the leaf cost with t_trav = 0 (bvh.rs:248-254, 733-735), i.e. down to one triangle
// per leaf. `bins` and `max_leaf` generalise the two knobs: bins = 8, max_leaf = 1 is the
// reference; max_leaf = k stops splitting any node holding k triangles or fewer.
// ---------------------------------------------------------------------------------------
struct TraversalStats {
  uint64_t nodes_visited = 0, box_tests = 0, triangle_tests = 0;
};

struct BuildStats {
  uint64_t node_count = 0, leaf_count = 0, max_depth = 0, max_leaf_tri_count = 0, total_leaf_tri_count = 0;
};

template <class R>
class MeshBVH {
 public:
  struct Node {
    AABB<R> box;
    uint64_t left_first;
    uint64_t count;  // > 0: leaf (bvh.rs:102-106)
  };
  struct Tri {
    uint32_t v0, v1, v2;
    V3<R> centroid;
  };

  // BVHTree::new + build (bvh.rs:179-230)
  MeshBVH(const R* vertices, size_t vertex_count, const uint32_t* indices, size_t tri_count, int bins, uint32_t max_leaf)
      : verts_(vertices, vertices + vertex_count * 3), bins_(bins), max_leaf_(max_leaf ? max_leaf : 1) {
    if (tri_count == 0) throw std::invalid_argument("a TriangleMesh needs at least one triangle");
    if (bins < 2 || bins > 64) throw std::invalid_argument("bins must be in [2, 64]");
    tris_.reserve(tri_count);
    tri_idx_.reserve(tri_count);
    for (size_t i = 0; i < tri_count; ++i) {
      Tri t;
      t.v0 = indices[3 * i];
      t.v1 = indices[3 * i + 1];
      t.v2 = indices[3 * i + 2];
      if (t.v0 >= vertex_count || t.v1 >= vertex_count || t.v2 >= vertex_count)
        throw std::invalid_argument("vertex index out of range");
      // tri_centroid (bvh.rs:578-584): ((v0 + v1) + v2) * (1/3)
      V3<R> c = vertex(t.v0);
      c = c + vertex(t.v1);
      c = c + vertex(t.v2);
      c = c * (R(1) / R(3));
      t.centroid = c;
      tris_.push_back(t);
      tri_idx_.push_back(uint32_t(i));
    }
    nodes_.reserve(2 * tri_count);
    Node root{AABB<R>::empty(), 0, tri_count};
    update_bounds(root);
    nodes_.push_back(root);
    subdivide(0);
  }

  V3<R> vertex(uint32_t i) const { return V3<R>{verts_[3 * size_t(i)], verts_[3 * size_t(i) + 1], verts_[3 * size_t(i) + 2]}; }

  const std::vector<Node>& nodes() const { return nodes_; }
  const std::vector<uint32_t>& tri_idx() const { return tri_idx_; }
  const std::vector<Tri>& tris() const { return tris_; }

  // build_stats (bvh.rs:538-562)
  BuildStats build_stats() const {
    BuildStats s;
    collect(0, 1, s);
    return s;
  }

  // BVHTree::traverse (bvh.rs:450-526): ordered DFS, nearer child first, each box tested
  // once (the entry distance travels on the stack), pop skipped when entry >= min_t.
  bool traverse(const Ray<R>& ray, R near, R far, TriHit<R>* hit, uint32_t* hit_tri, TraversalStats* st) const {
    R min_t = Limits<R>::max();
    bool found = false;
    uint32_t cur_tri = 0;
    TriHit<R> cur{};
    R root_dist;
    st->box_tests++;
    if (!box_hit(nodes_[0].box, ray, near, far, &root_dist)) return false;
    struct Entry { uint64_t node; R dist; };
    Entry stack[256];
    int sp = 0;
    stack[sp++] = Entry{0, root_dist};
    while (sp > 0) {
      Entry e = stack[--sp];
      if (e.dist >= min_t) continue;
      st->nodes_visited++;
      const Node& n = nodes_[e.node];
      if (n.count > 0) {
        for (uint64_t i = 0; i < n.count; ++i) {
          const Tri& t = tris_[tri_idx_[n.left_first + i]];
          TriHit<R> h;
          st->triangle_tests++;
          if (intersect_ray(ray, vertex(t.v0), vertex(t.v1), vertex(t.v2), &h)) {
            if (h.t < min_t && h.t >= near && h.t <= far) {
              min_t = h.t;
              cur = h;
              found = true;
              cur_tri = tri_idx_[n.left_first + i];
            }
          }
        }
      } else {
        const uint64_t l = n.left_first, r = n.left_first + 1;
        R dl = R(0), dr = R(0);
        st->box_tests++;
        const bool hl = box_hit(nodes_[l].box, ray, near, far, &dl);
        st->box_tests++;
        const bool hr = box_hit(nodes_[r].box, ray, near, far, &dr);
        // nearer first; right only if strictly nearer (bvh.rs:503-506)
        uint64_t nearer = l, farther = r;
        bool hn = hl, hf = hr;
        R dn = dl, df = dr;
        if (hl && hr && dr < dl) {
          nearer = r; farther = l; hn = hr; hf = hl; dn = dr; df = dl;
        }
        if (hf && df < min_t) {
          if (sp >= 256) throw std::runtime_error("oracle stack overflow");
          stack[sp++] = Entry{farther, df};
        }
        if (hn && dn < min_t) {
          if (sp >= 256) throw std::runtime_error("oracle stack overflow");
          stack[sp++] = Entry{nearer, dn};
        }
      }
    }
    if (found) {
      *hit = cur;
      *hit_tri = cur_tri;
    }
    return found;
  }

  // BVHTree::intersect_p (bvh.rs:381-420): unordered, fixed interval, first hit wins.
  // `st` (optional) counts the work as traverse() does: nodes visited, box and triangle tests.
  bool intersect_p(const Ray<R>& ray, R near, R far, TraversalStats* st = nullptr) const {
    R dist;
    if (st) st->box_tests++;
    if (!box_hit(nodes_[0].box, ray, near, far, &dist)) return false;
    uint64_t stack[256];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const Node& n = nodes_[stack[--sp]];
      if (st) st->nodes_visited++;
      if (n.count > 0) {
        for (uint64_t i = 0; i < n.count; ++i) {
          const Tri& t = tris_[tri_idx_[n.left_first + i]];
          TriHit<R> h;
          if (st) st->triangle_tests++;
          if (intersect_ray(ray, vertex(t.v0), vertex(t.v1), vertex(t.v2), &h))
            if (h.t >= near && h.t <= far) return true;
        }
      } else {
        for (uint64_t c = n.left_first; c <= n.left_first + 1; ++c) {
          if (st) st->box_tests++;
          if (box_hit(nodes_[c].box, ray, near, far, &dist)) {
            if (sp >= 256) throw std::runtime_error("oracle stack overflow");
            stack[sp++] = c;
          }
        }
      }
    }
    return false;
  }

  // Brute force nearest over every triangle (test helper, bvh.rs:792-816).
  bool brute_force(const Ray<R>& ray, R near, R far, R* t_out, uint32_t* idx_out) const {
    bool found = false;
    R best = R(0);
    uint32_t bi = 0;
    for (size_t i = 0; i < tris_.size(); ++i) {
      const Tri& t = tris_[i];
      TriHit<R> h;
      if (!intersect_ray(ray, vertex(t.v0), vertex(t.v1), vertex(t.v2), &h)) continue;
      if (h.t < near || h.t > far) continue;
      if (!found || h.t < best) {
        found = true;
        best = h.t;
        bi = uint32_t(i);
      }
    }
    if (found) { *t_out = best; *idx_out = bi; }
    return found;
  }

  // get_bounding_box over vertices (triangle_mesh.rs:150-173)
  AABB<R> vertex_bounds() const {
    AABB<R> b{{Limits<R>::max(), Limits<R>::max(), Limits<R>::max()}, {Limits<R>::lowest(), Limits<R>::lowest(), Limits<R>::lowest()}};
    for (size_t i = 0; i + 2 < verts_.size(); i += 3) {
      b.bmin.x = rmin(verts_[i], b.bmin.x); b.bmin.y = rmin(verts_[i + 1], b.bmin.y); b.bmin.z = rmin(verts_[i + 2], b.bmin.z);
      b.bmax.x = rmax(verts_[i], b.bmax.x); b.bmax.y = rmax(verts_[i + 1], b.bmax.y); b.bmax.z = rmax(verts_[i + 2], b.bmax.z);
    }
    return b;
  }

  size_t triangle_count() const { return tris_.size(); }

 private:
  struct Bin { AABB<R> bounds; uint64_t count; };
  struct Split { int axis; int boundary; R cmin, width, cost; };

  // aabound_from_triangle (bvh.rs:564-572)
  AABB<R> tri_box(const Tri& t) const {
    V3<R> p1 = vertex(t.v0), p2 = vertex(t.v1), p3 = vertex(t.v2);
    AABB<R> b;
    b.bmin = {rmin(rmin(p1.x, p2.x), p3.x), rmin(rmin(p1.y, p2.y), p3.y), rmin(rmin(p1.z, p2.z), p3.z)};
    b.bmax = {rmax(rmax(p1.x, p2.x), p3.x), rmax(rmax(p1.y, p2.y), p3.y), rmax(rmax(p1.z, p2.z), p3.z)};
    return b;
  }

  // update_bounds (bvh.rs:232-238)
  void update_bounds(Node& n) const {
    for (uint64_t i = n.left_first; i < n.left_first + n.count; ++i) n.box.combine(tri_box(tris_[tri_idx_[i]]));
  }

  // bin_index (bvh.rs:173-176). Rust's `as usize` saturates (negative or NaN -> 0), then
  // clamps to the last bin.
  int bin_index(R pos, R cmin, R width) const {
    const R q = (pos - cmin) / width;
    const R f = std::floor(q);
    if (!(f >= R(0))) return 0;
    if (f >= R(bins_ - 1)) return bins_ - 1;
    return int(f);
  }

  // find_best_split_plane (bvh.rs:609-685)
  bool best_split(const Node& n, Split* best) const {
    bool have = false;
    for (int axis = 0; axis < 3; ++axis) {
      R cmin = Limits<R>::max(), cmax = Limits<R>::lowest();
      for (uint64_t i = n.left_first; i < n.left_first + n.count; ++i) {
        const R c = tris_[tri_idx_[i]].centroid[axis];
        cmin = rmin(cmin, c);
        cmax = rmax(cmax, c);
      }
      if (cmin == cmax) continue;
      const R width = (cmax - cmin) / R(bins_);
      std::vector<Bin> bins(bins_, Bin{AABB<R>::empty(), 0});
      for (uint64_t i = n.left_first; i < n.left_first + n.count; ++i) {
        const Tri& t = tris_[tri_idx_[i]];
        Bin& b = bins[bin_index(t.centroid[axis], cmin, width)];
        b.bounds.combine(tri_box(t));
        b.count++;
      }
      const int S = bins_ - 1;
      std::vector<R> la(S), ra(S);
      std::vector<uint64_t> lc(S), rc(S);
      AABB<R> lb = AABB<R>::empty(), rb = AABB<R>::empty();
      uint64_t ls = 0, rs = 0;
      for (int i = 0; i < S; ++i) {
        lb.combine(bins[i].bounds);
        ls += bins[i].count;
        la[i] = lb.half_area();
        lc[i] = ls;
        const int m = S - 1 - i;
        rb.combine(bins[m + 1].bounds);
        rs += bins[m + 1].count;
        ra[m] = rb.half_area();
        rc[m] = rs;
      }
      for (int b = 0; b < S; ++b) {
        if (lc[b] == 0 || rc[b] == 0) continue;
        const R cost = la[b] * R(lc[b]) + ra[b] * R(rc[b]);
        if (!have || cost < best->cost) {
          have = true;
          *best = Split{axis, b, cmin, width, cost};
        }
      }
    }
    return have;
  }

  // subdivide (bvh.rs:240-309)
  void subdivide(uint64_t idx) {
    const uint64_t first = nodes_[idx].left_first, count = nodes_[idx].count;
    if (count <= max_leaf_) return;
    const R leaf_cost = nodes_[idx].box.half_area() * R(count);
    Split s;
    if (!best_split(nodes_[idx], &s) || !(s.cost < leaf_cost)) return;
    uint64_t left_end = first;
    for (uint64_t i = first; i < first + count; ++i) {
      const R pos = tris_[tri_idx_[i]].centroid[s.axis];
      if (bin_index(pos, s.cmin, s.width) <= s.boundary) {
        std::swap(tri_idx_[i], tri_idx_[left_end]);
        left_end++;
      }
    }
    const uint64_t left_count = left_end - first;
    if (left_count == 0 || left_count == count) return;
    Node ln{AABB<R>::empty(), first, left_count};
    update_bounds(ln);
    Node rn{AABB<R>::empty(), left_end, count - left_count};
    update_bounds(rn);
    const uint64_t li = nodes_.size();
    nodes_.push_back(ln);
    nodes_.push_back(rn);
    nodes_[idx].left_first = li;
    nodes_[idx].count = 0;
    subdivide(li);
    subdivide(li + 1);
  }

  void collect(uint64_t idx, uint64_t depth, BuildStats& s) const {
    const Node& n = nodes_[idx];
    s.node_count++;
    s.max_depth = std::max(s.max_depth, depth);
    if (n.count > 0) {
      s.leaf_count++;
      s.total_leaf_tri_count += n.count;
      s.max_leaf_tri_count = std::max<uint64_t>(s.max_leaf_tri_count, n.count);
    } else {
      collect(n.left_first, depth + 1, s);
      collect(n.left_first + 1, depth + 1, s);
    }
  }

  std::vector<R> verts_;
  int bins_;
  uint64_t max_leaf_;
  std::vector<Tri> tris_;
  std::vector<uint32_t> tri_idx_;
  std::vector<Node> nodes_;
};

// ---------------------------------------------------------------------------------------
// Matrix4 — src/geom/matrix4.rs
// ---------------------------------------------------------------------------------------
template <class R>
struct M4 {
  R m[4][4];
  static M4 zero() { M4 r; std::memset(r.m, 0, sizeof(r.m)); for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) r.m[i][j] = R(0); return r; }
  static M4 identity() { M4 r = zero(); for (int i = 0; i < 4; ++i) r.m[i][i] = R(1); return r; }
  static M4 translation(R x, R y, R z) { M4 r = identity(); r.m[0][3] = x; r.m[1][3] = y; r.m[2][3] = z; return r; }
  static M4 scale(R x, R y, R z) { M4 r = zero(); r.m[0][0] = x; r.m[1][1] = y; r.m[2][2] = z; r.m[3][3] = R(1); return r; }
  // rotation_x/y/z (matrix4.rs:46-68)
  static M4 rotation_x(R th) { R s = std::sin(th), c = std::cos(th); M4 r = identity(); r.m[1][1] = c; r.m[1][2] = -s; r.m[2][1] = s; r.m[2][2] = c; return r; }
  static M4 rotation_y(R th) { R s = std::sin(th), c = std::cos(th); M4 r = identity(); r.m[0][0] = c; r.m[0][2] = s; r.m[2][0] = -s; r.m[2][2] = c; return r; }
  static M4 rotation_z(R th) { R s = std::sin(th), c = std::cos(th); M4 r = identity(); r.m[0][0] = c; r.m[0][1] = -s; r.m[1][0] = s; r.m[1][1] = c; return r; }
  // perspective (matrix4.rs:70-79)
  static M4 perspective(R fov, R n, R f) {
    R s = R(1) / std::tan(fov / R(2));
    M4 r = zero();
    r.m[0][0] = s; r.m[1][1] = s; r.m[2][2] = f / (f - n); r.m[2][3] = -f * n / (f - n); r.m[3][2] = R(1);
    return r;
  }
  // look_at (matrix4.rs:81-98)
  static M4 look_at(const V3<R>& pos, const V3<R>& look, const V3<R>& up) {
    V3<R> dir = normalized(look - pos);
    V3<R> nu = normalized(up);
    V3<R> right = normalized(cross(nu, dir));
    V3<R> ru = cross(dir, right);
    M4 r = zero();
    r.m[0][0] = right.x; r.m[0][1] = ru.x; r.m[0][2] = dir.x; r.m[0][3] = pos.x;
    r.m[1][0] = right.y; r.m[1][1] = ru.y; r.m[1][2] = dir.y; r.m[1][3] = pos.y;
    r.m[2][0] = right.z; r.m[2][1] = ru.z; r.m[2][2] = dir.z; r.m[2][3] = pos.z;
    r.m[3][3] = R(1);
    return r;
  }
  // inverse: Gauss-Jordan with full pivoting (matrix4.rs:100-174)
  M4 inverse() const {
    int indxc[4] = {0, 0, 0, 0}, indxr[4] = {0, 0, 0, 0}, ipiv[4] = {0, 0, 0, 0};
    R minv[4][4];
    std::memcpy(minv, m, sizeof(minv));
    for (int i = 0; i < 4; ++i) {
      int irow = 0, icol = 0;
      R big = R(0);
      for (int j = 0; j < 4; ++j) {
        if (ipiv[j] != 1) {
          for (int k = 0; k < 4; ++k) {
            if (ipiv[k] == 0) {
              if (std::fabs(minv[j][k]) >= big) { big = std::fabs(minv[j][k]); irow = j; icol = k; }
            }
          }
        }
      }
      ipiv[icol] += 1;
      if (irow != icol) for (int k = 0; k < 4; ++k) std::swap(minv[irow][k], minv[icol][k]);
      indxr[i] = irow;
      indxc[i] = icol;
      R pivinv = R(1) / minv[icol][icol];
      minv[icol][icol] = R(1);
      for (int j = 0; j < 4; ++j) minv[icol][j] *= pivinv;
      for (int j = 0; j < 4; ++j) {
        if (j != icol) {
          R save = minv[j][icol];
          minv[j][icol] = R(0);
          for (int k = 0; k < 4; ++k) minv[j][k] -= minv[icol][k] * save;
        }
      }
    }
    for (int j = 3; j >= 0; --j) {
      if (indxr[j] != indxc[j])
        for (int k = 0; k < 4; ++k) std::swap(minv[k][indxr[j]], minv[k][indxc[j]]);
    }
    M4 r;
    std::memcpy(r.m, minv, sizeof(minv));
    return r;
  }
  M4 transpose() const { M4 r; for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) r.m[i][j] = m[j][i]; return r; }
  // Mul (matrix4.rs:216-231): accumulate from zero, k in order
  M4 operator*(const M4& o) const {
    M4 r = zero();
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 4; ++k) r.m[i][j] += m[i][k] * o.m[k][j];
    return r;
  }
  // transform_point (matrix4.rs:187-199) — also `&Matrix4 * &Vector3f` (:243-258)
  V3<R> point(const V3<R>& v) const {
    R x = m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z + m[0][3];
    R y = m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z + m[1][3];
    R z = m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z + m[2][3];
    R w = m[3][0] * v.x + m[3][1] * v.y + m[3][2] * v.z + m[3][3];
    V3<R> res{x, y, z};
    if (w != R(1)) return res * (R(1) / w);
    return res;
  }
  // transform_direction (matrix4.rs:201-206)
  V3<R> direction(const V3<R>& v) const {
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
  }
  // transform_normal (matrix4.rs:208-213): multiplies by the transpose
  V3<R> normal(const V3<R>& v) const {
    return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
            m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
  }
};

// ---------------------------------------------------------------------------------------
// PinHoleCamera — src/cameras/pin_hole.rs:17-50
// ---------------------------------------------------------------------------------------
template <class R>
struct PinHoleCamera {
  M4<R> raster_to_screen, cam_to_world;
  PinHoleCamera(uint32_t w, uint32_t h, R fov, R near, R far, const M4<R>& c2w) : cam_to_world(c2w) {
    const R aspect = R(w) / R(h);
    R xmin, xmax, ymin, ymax;
    if (aspect > R(1)) { xmin = -aspect; xmax = aspect; ymin = R(-1); ymax = R(1); }
    else { xmin = R(-1); xmax = R(1); ymin = R(-1) / aspect; ymax = R(1) / aspect; }
    raster_to_screen = ((M4<R>::perspective(fov, near, far).inverse() * M4<R>::translation(xmin, ymax, R(0))) *
                        M4<R>::scale(xmax - xmin, ymin - ymax, R(1))) *
                       M4<R>::scale(R(1) / R(w), R(1) / R(h), R(1));
  }
  Ray<R> get_ray(R px, R py) const {
    V3<R> cv = normalized(raster_to_screen.point(V3<R>{px, py, R(0)}));
    return make_ray(cam_to_world.point(V3<R>{R(0), R(0), R(0)}), cam_to_world.direction(cv));
  }
};

// Orbit camera of the traversal benchmark (src/bin/bvh_stats.rs:385-401, constants :96-116).
template <class R>
inline PinHoleCamera<R> orbit_camera(int view, const V3<R>& center, R distance) {
  const R PI = R(3.141592653589793238462643383279502884L);
  const R elev = R(20) * PI / R(180);
  const R fov = R(40) * PI / R(180);
  const R az = R(2) * PI * R(view) / R(6);
  V3<R> dir{std::cos(elev) * std::cos(az), std::sin(elev), std::cos(elev) * std::sin(az)};
  V3<R> pos = center + dir * distance;
  return PinHoleCamera<R>(200, 200, fov, R(0.0001), R(1000), M4<R>::look_at(pos, center, V3<R>{R(0), R(1), R(0)}));
}

}  // namespace oracle
