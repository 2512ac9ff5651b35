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

struct Box {
  float lo[3], hi[3];
  void set_empty() {
    for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
  }
  void grow(const Box& b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::fmin(lo[a], b.lo[a]);
      hi[a] = std::fmax(hi[a], b.hi[a]);
    }
  }
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

class Builder {
 public:
  Builder(const float* v, const uint32_t* idx, uint32_t n, const MeshBuildParams& p) : v_(v), idx_(idx), n_(n), p_(p) {}

  void run(std::vector<RefNode>* nodes_out, std::vector<uint32_t>* order_out) {
    tri_box_.resize(n_);
    for (int a = 0; a < 3; ++a) cen_[a].resize(n_);
    const float third = 1.0f / 3.0f;
    for (uint32_t i = 0; i < n_; ++i) {
      const float* p0 = v_ + 3 * size_t(idx_[3 * size_t(i)]);
      const float* p1 = v_ + 3 * size_t(idx_[3 * size_t(i) + 1]);
      const float* p2 = v_ + 3 * size_t(idx_[3 * size_t(i) + 2]);
      Box& b = tri_box_[i];
      for (int a = 0; a < 3; ++a) {
        // aabound_from_triangle (bvh.rs:564-572)
        b.lo[a] = std::fmin(std::fmin(p0[a], p1[a]), p2[a]);
        b.hi[a] = std::fmax(std::fmax(p0[a], p1[a]), p2[a]);
        // tri_centroid (bvh.rs:578-584)
        float c = p0[a];
        c = c + p1[a];
        c = c + p2[a];
        cen_[a][i] = c * third;
      }
    }
    order_.resize(n_);
    for (uint32_t i = 0; i < n_; ++i) order_[i] = i;

    nodes_.clear();
    nodes_.reserve(size_t(2) * n_);
    RefNode root;
    root.left_first = 0;
    root.count = n_;
    root.depth = 1;
    bounds(0, n_, &root.box);
    nodes_.push_back(root);

    // Depth-first, left child first: the same node numbering as the reference's recursion.
    std::vector<uint32_t> stack;
    stack.push_back(0);
    std::vector<Box> bin_box(p_.bins);
    std::vector<uint32_t> bin_cnt(p_.bins);
    std::vector<float> la(p_.bins), ra(p_.bins);
    std::vector<uint32_t> lc(p_.bins), rc(p_.bins);
    while (!stack.empty()) {
      const uint32_t ni = stack.back();
      stack.pop_back();
      const uint32_t first = nodes_[ni].left_first, count = nodes_[ni].count;
      if (count <= p_.max_leaf) continue;
      const float leaf_cost = nodes_[ni].box.half_area() * float(count);

      bool have = false;
      int best_axis = 0, best_boundary = 0;
      float best_cmin = 0, best_width = 0, best_cost = 0;
      for (int a = 0; a < 3; ++a) {
        const std::vector<float>& c = cen_[a];
        float cmin = FLT_MAX, cmax = -FLT_MAX;
        for (uint32_t k = first; k < first + count; ++k) {
          const float x = c[order_[k]];
          cmin = std::fmin(cmin, x);
          cmax = std::fmax(cmax, x);
        }
        if (cmin == cmax) continue;
        const float width = (cmax - cmin) / float(p_.bins);
        for (int b = 0; b < p_.bins; ++b) { bin_box[b].set_empty(); bin_cnt[b] = 0; }
        for (uint32_t k = first; k < first + count; ++k) {
          const uint32_t t = order_[k];
          const int b = bin_of(c[t], cmin, width);
          bin_box[b].grow(tri_box_[t]);
          bin_cnt[b]++;
        }
        const int S = p_.bins - 1;
        Box lb, rb;
        lb.set_empty();
        rb.set_empty();
        uint32_t ls = 0, rs = 0;
        for (int i = 0; i < S; ++i) {
          lb.grow(bin_box[i]);
          ls += bin_cnt[i];
          la[i] = lb.half_area();
          lc[i] = ls;
          const int m = S - 1 - i;
          rb.grow(bin_box[m + 1]);
          rs += bin_cnt[m + 1];
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
            best_cmin = cmin;
            best_width = width;
            best_cost = cost;
          }
        }
      }
      if (!have || !(best_cost < leaf_cost)) continue;

      // Forward-swap partition by bin index (bvh.rs:260-267).
      const std::vector<float>& c = cen_[best_axis];
      uint32_t left_end = first;
      for (uint32_t k = first; k < first + count; ++k) {
        if (bin_of(c[order_[k]], best_cmin, best_width) <= best_boundary) {
          std::swap(order_[k], order_[left_end]);
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
    order_out->swap(order_);
  }

 private:
  // bin_index (bvh.rs:173-176) with Rust's saturating float-to-usize cast.
  int bin_of(float pos, float cmin, float width) const {
    const float q = (pos - cmin) / width;
    const float f = std::floor(q);
    if (!(f >= 0.0f)) return 0;
    if (f >= float(p_.bins - 1)) return p_.bins - 1;
    return int(f);
  }

  void bounds(uint32_t first, uint32_t count, Box* out) const {
    out->set_empty();
    for (uint32_t k = first; k < first + count; ++k) out->grow(tri_box_[order_[k]]);
  }

  const float* v_;
  const uint32_t* idx_;
  uint32_t n_;
  MeshBuildParams p_;
  std::vector<Box> tri_box_;
  std::vector<float> cen_[3];
  std::vector<uint32_t> order_;
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
    for (int a = 0; a < 3; ++a) { g.bmin[a] = r.box.lo[a]; g.bmax[a] = r.box.hi[a]; }
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
  return true;
}

}  // namespace pbrt
