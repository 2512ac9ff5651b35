// mesh_bvh.hpp — host-side build of a triangle mesh's BVH, flattened for the GPU.
//
// The tree is the one src/shapes/triangle_mesh/bvh.rs builds (binned SAH over triangle
// centroids, leaf cost A·N against split cost A_L·N_L + A_R·N_R, in-place forward-swap
// partition by bin index, child boxes recomputed from their triangles), computed in FP32.
// Two knobs generalise the reference's constants: the number of bins (bvh.rs:129 fixes 8)
// and a leaf size below which a node is not split (the reference splits down to one
// triangle whenever the SAH allows, bvh.rs:248-254).
//
// GPU layout (what the traversal kernels read):
//   nodes: 32-byte records {float bmin[3]; uint32 left_first; float bmax[3]; uint32 count},
//          read as two float4. count > 0 marks a leaf whose triangles are the `count`
//          records starting at left_first; an interior node's children are left_first and
//          left_first + 1. Index 0 is the root and index 1 is padding, so every sibling pair
//          starts at an even index and the pair is one aligned 64-byte read.
//   triangles, in leaf order, as three streams (SoA):
//          tri_a[k] = {v0.x, v0.y, v0.z, e1.x}
//          tri_b[k] = {e1.y, e1.z, e2.x, e2.y}
//          tri_c[k] = {e2.z, bits(original triangle index)}
//          with e1 = v1 - v0 and e2 = v2 - v0 rounded to FP32 exactly as the reference's
//          intersect_ray forms them (triangle_mesh.rs:190-191), so precomputing them
//          changes no bit of the intersection arithmetic.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pbrt {

struct GpuNode {
  float bmin[3];
  uint32_t left_first;
  float bmax[3];
  uint32_t count;
};
static_assert(sizeof(GpuNode) == 32, "GpuNode must be 32 bytes");

struct MeshBuildParams {
  int bins = 8;           // the reference's BIN_COUNT
  uint32_t max_leaf = 1;  // nodes with <= max_leaf triangles are not split
};

struct MeshBuildStats {
  uint64_t node_count = 0;  // reference numbering, no padding slot
  uint64_t leaf_count = 0;
  uint32_t max_depth = 0;   // root = 1
  uint32_t max_leaf_tris = 0;
};

struct FlatMesh {
  std::vector<GpuNode> nodes;      // GPU numbering (root 0, padding 1)
  std::vector<float> tri_a;        // 4 floats per triangle
  std::vector<float> tri_b;        // 4 floats per triangle
  std::vector<float> tri_c;        // 2 floats per triangle
  std::vector<uint32_t> tri_index; // leaf order -> original triangle index
  float bounds_min[3], bounds_max[3];  // vertex bounds (TriangleMesh::get_bounding_box)
  MeshBuildStats stats;
};

// Builds and flattens. Returns false with `err` set on invalid input (no triangle, an index
// out of range, a non-finite vertex).
bool build_mesh_bvh(const float* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t tri_count,
                    const MeshBuildParams& params, FlatMesh* out, std::string* err);

}  // namespace pbrt
