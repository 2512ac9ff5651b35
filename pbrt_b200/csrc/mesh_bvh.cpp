// mesh_bvh.cpp — host BVH build for one triangle mesh; see mesh_bvh.hpp for the layout.
//
// Compiled with -ffp-contract=off: the split costs and centroids must round exactly as the
// reference's expressions do, or the tree (and with it the traversal order) would differ.
#include "mesh_bvh.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace pbrt {
namespace {

// min / max with the tie rule of the C library's fmin / fmax (the first argument wins a tie,
// which only matters for the sign of a zero); inputs are finite (checked before the build).
inline float mn(float x, float y) { return y < x ? y : x; }
inline float mx(float x, float y) { return x < y ? y : x; }
// Stored boxes hold +0 for a zero bound: the sign of a zero bound depends on the order the
// triangles were met in, and no slab test can tell the two apart (near > 0), so both
// builders (this one and the GPU's) store the same canonical value.
inline float canon(float x) { return x == 0.0f ? 0.0f : x; }

struct Box {
  float lo[3], hi[3];
  void set_empty() {
    for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
  }
  void grow(const float* l, const float* h) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = mn(lo[a], l[a]);
      hi[a] = mx(hi[a], h[a]);
    }
  }
  void grow(const Box& b) { grow(b.lo, b.hi); }
  bool empty() const { return lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]; }
  // AABoundingBox::half_area (src/geom/aabound.rs:123-130)
  float half_area() const {
    if (empty()) return 0.0f;
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
  }
};

struct RefNode {
  Box box;
  uint32_t left_first;
  uint32_t count;
  uint32_t depth;
};

// One triangle as the build sees it. The records themselves are permuted by the partition
// (the same permutation the reference applies to its index list), so every pass over a
// node's triangles reads memory in order.
struct TriRef {
  float c[3];          // centroid
  float lo[3], hi[3];  // bounds
  uint32_t id;
};

class Builder {
 public:
  Builder(const float* v, const uint32_t* idx, uint32_t n, const MeshBuildParams& p) : v_(v), idx_(idx), n_(n), p_(p) {}

  void run(std::vector<RefNode>* nodes_out, std::vector<uint32_t>* order_out) {
    refs_.resize(n_);
    const float third = 1.0f / 3.0f;
    for (uint32_t i = 0; i < n_; ++i) {
      const float* p0 = v_ + 3 * size_t(idx_[3 * size_t(i)]);
      const float* p1 = v_ + 3 * size_t(idx_[3 * size_t(i) + 1]);
      const float* p2 = v_ + 3 * size_t(idx_[3 * size_t(i) + 2]);
      TriRef& r = refs_[i];
      for (int a = 0; a < 3; ++a) {
        // aabound_from_triangle (bvh.rs:564-572)
        r.lo[a] = mn(mn(p0[a], p1[a]), p2[a]);
        r.hi[a] = mx(mx(p0[a], p1[a]), p2[a]);
        // tri_centroid (bvh.rs:578-584)
        float c = p0[a];
        c = c + p1[a];
        c = c + p2[a];
        r.c[a] = c * third;
      }
      r.id = i;
    }

    nodes_.clear();
    nodes_.reserve(size_t(2) * n_ / std::max<uint32_t>(1, p_.max_leaf) + 2);
    RefNode root;
    root.left_first = 0;
    root.count = n_;
    root.depth = 1;
    bounds(0, n_, &root.box);
    nodes_.push_back(root);

    // Depth-first, left child first: the same node numbering as the reference's recursion.
    const int B = p_.bins, S = B - 1;
    std::vector<uint32_t> stack;
    stack.push_back(0);
    std::vector<Box> bin_box(size_t(3) * B);
    std::vector<uint32_t> bin_cnt(size_t(3) * B);
    std::vector<float> la(B), ra(B);
    std::vector<uint32_t> lc(B), rc(B);
    while (!stack.empty()) {
      const uint32_t ni = stack.back();
      stack.pop_back();
      const uint32_t first = nodes_[ni].left_first, count = nodes_[ni].count;
      if (count <= p_.max_leaf) continue;
      const float leaf_cost = nodes_[ni].box.half_area() * float(count);
      const TriRef* rr = refs_.data() + first;

      // centroid extent of every axis in one pass
      float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      for (uint32_t k = 0; k < count; ++k)
        for (int a = 0; a < 3; ++a) {
          cmin[a] = mn(cmin[a], rr[k].c[a]);
          cmax[a] = mx(cmax[a], rr[k].c[a]);
        }
      bool use[3];
      float width[3];
      for (int a = 0; a < 3; ++a) {
        use[a] = !(cmin[a] == cmax[a]);
        width[a] = (cmax[a] - cmin[a]) / float(B);
        for (int b = 0; b < B; ++b) {
          bin_box[a * B + b].set_empty();
          bin_cnt[a * B + b] = 0;
        }
      }
      // the bins of every splittable axis in one pass
      for (uint32_t k = 0; k < count; ++k)
        for (int a = 0; a < 3; ++a) {
          if (!use[a]) continue;
          const int b = a * B + bin_of(rr[k].c[a], cmin[a], width[a]);
          bin_box[b].grow(rr[k].lo, rr[k].hi);
          bin_cnt[b]++;
        }

      bool have = false;
      int best_axis = 0, best_boundary = 0;
      float best_cost = 0;
      for (int a = 0; a < 3; ++a) {
        if (!use[a]) continue;
        Box lb, rb;
        lb.set_empty();
        rb.set_empty();
        uint32_t ls = 0, rs = 0;
        for (int i = 0; i < S; ++i) {
          lb.grow(bin_box[a * B + i]);
          ls += bin_cnt[a * B + i];
          la[i] = lb.half_area();
          lc[i] = ls;
          const int m = S - 1 - i;
          rb.grow(bin_box[a * B + m + 1]);
          rs += bin_cnt[a * B + m + 1];
          ra[m] = rb.half_area();
          rc[m] = rs;
        }
        for (int b = 0; b < S; ++b) {
          if (lc[b] == 0 || rc[b] == 0) continue;
          const float cost = la[b] * float(lc[b]) + ra[b] * float(rc[b]);
          if (!have || cost < best_cost) {
            have = true;
            best_axis = a;
            best_boundary = b;
            best_cost = cost;
          }
        }
      }
      if (!have || !(best_cost < leaf_cost)) continue;

      // Forward-swap partition by bin index (bvh.rs:260-267), children's boxes on the way.
      TriRef* w = refs_.data();
      const float bmin = cmin[best_axis], bw = width[best_axis];
      uint32_t left_end = first;
      for (uint32_t k = first; k < first + count; ++k) {
        if (bin_of(w[k].c[best_axis], bmin, bw) <= best_boundary) {
          std::swap(w[k], w[left_end]);
          left_end++;
        }
      }
      const uint32_t left_count = left_end - first;
      if (left_count == 0 || left_count == count) continue;

      RefNode l, r;
      l.left_first = first;
      l.count = left_count;
      l.depth = nodes_[ni].depth + 1;
      bounds(first, left_count, &l.box);
      r.left_first = left_end;
      r.count = count - left_count;
      r.depth = l.depth;
      bounds(left_end, count - left_count, &r.box);
      const uint32_t li = uint32_t(nodes_.size());
      nodes_.push_back(l);
      nodes_.push_back(r);
      nodes_[ni].left_first = li;
      nodes_[ni].count = 0;
      stack.push_back(li + 1);
      stack.push_back(li);
    }
    nodes_out->swap(nodes_);
    order_out->resize(n_);
    for (uint32_t k = 0; k < n_; ++k) (*order_out)[k] = refs_[k].id;
  }

 private:
  // bin_index (bvh.rs:173-176): floor, then Rust's saturating float-to-usize cast. For
  // 0 <= q < bins - 1 the floor is the truncation; q < 0 and NaN give 0, q >= bins - 1 the
  // last bin (floor(q) >= bins - 1 exactly when q >= bins - 1, bins - 1 being an integer).
  int bin_of(float pos, float cmin, float width) const {
    const float q = (pos - cmin) / width;
    if (!(q >= 0.0f)) return 0;
    if (q >= float(p_.bins - 1)) return p_.bins - 1;
    return int(q);
  }

  void bounds(uint32_t first, uint32_t count, Box* out) const {
    out->set_empty();
    for (uint32_t k = first; k < first + count; ++k) out->grow(refs_[k].lo, refs_[k].hi);
  }

  const float* v_;
  const uint32_t* idx_;
  uint32_t n_;
  MeshBuildParams p_;
  std::vector<TriRef> refs_;
  std::vector<RefNode> nodes_;
};

}  // namespace

bool build_mesh_bvh(const float* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t tri_count,
                    const MeshBuildParams& params, FlatMesh* out, std::string* err) {
  if (tri_count == 0) { *err = "a TriangleMesh needs at least one triangle"; return false; }
  if (!vertices || !indices) { *err = "mesh arrays must not be NULL"; return false; }
  if (params.bins < 2 || params.bins > 64) { *err = "bvh_bins must be in [2, 64]"; return false; }
  for (uint64_t k = 0; k < uint64_t(tri_count) * 3; ++k)
    if (indices[k] >= vertex_count) { *err = "triangle vertex index out of range"; return false; }
  for (uint64_t k = 0; k < uint64_t(vertex_count) * 3; ++k)
    if (!std::isfinite(vertices[k])) { *err = "non-finite vertex coordinate"; return false; }

  std::vector<RefNode> ref;
  std::vector<uint32_t> order;
  Builder(vertices, indices, tri_count, params).run(&ref, &order);

  // Flatten: GPU index g(0) = 0, g(k) = k + 1 (slot 1 pads sibling pairs to 64 bytes).
  out->nodes.assign(ref.size() + 1, GpuNode{});
  MeshBuildStats st;
  st.node_count = ref.size();
  for (size_t k = 0; k < ref.size(); ++k) {
    const RefNode& r = ref[k];
    GpuNode& g = out->nodes[k == 0 ? 0 : k + 1];
    for (int a = 0; a < 3; ++a) { g.bmin[a] = canon(r.box.lo[a]); g.bmax[a] = canon(r.box.hi[a]); }
    if (r.count > 0) {
      g.left_first = r.left_first;
      g.count = r.count;
      st.leaf_count++;
      st.max_leaf_tris = std::max(st.max_leaf_tris, r.count);
    } else {
      g.left_first = r.left_first + 1;
      g.count = 0;
    }
    st.max_depth = std::max(st.max_depth, r.depth);
  }
  out->stats = st;

  out->tri_a.resize(size_t(tri_count) * 4);
  out->tri_b.resize(size_t(tri_count) * 4);
  out->tri_c.resize(size_t(tri_count) * 2);
  out->tri_index = order;
  for (uint32_t k = 0; k < tri_count; ++k) {
    const uint32_t t = order[k];
    const float* p0 = vertices + 3 * size_t(indices[3 * size_t(t)]);
    const float* p1 = vertices + 3 * size_t(indices[3 * size_t(t) + 1]);
    const float* p2 = vertices + 3 * size_t(indices[3 * size_t(t) + 2]);
    const float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    float* a = &out->tri_a[size_t(k) * 4];
    float* b = &out->tri_b[size_t(k) * 4];
    float* c = &out->tri_c[size_t(k) * 2];
    a[0] = p0[0]; a[1] = p0[1]; a[2] = p0[2]; a[3] = e1[0];
    b[0] = e1[1]; b[1] = e1[2]; b[2] = e2[0]; b[3] = e2[1];
    c[0] = e2[2];
    std::memcpy(&c[1], &t, sizeof(float));
  }
  for (int a = 0; a < 3; ++a) { out->bounds_min[a] = FLT_MAX; out->bounds_max[a] = -FLT_MAX; }
  for (uint32_t i = 0; i < vertex_count; ++i)
    for (int a = 0; a < 3; ++a) {
      out->bounds_min[a] = std::fmin(vertices[3 * size_t(i) + a], out->bounds_min[a]);
      out->bounds_max[a] = std::fmax(vertices[3 * size_t(i) + a], out->bounds_max[a]);
    }
  for (int a = 0; a < 3; ++a) {
    out->bounds_min[a] = canon(out->bounds_min[a]);
    out->bounds_max[a] = canon(out->bounds_max[a]);
  }
  return true;
}

}  // namespace pbrt
