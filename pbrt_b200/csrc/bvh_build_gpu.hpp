// bvh_build_gpu.hpp — a triangle mesh's BVH built on the GPU (bvh_build_gpu.cu): the same tree,
// triangle order and flattened layout as build_mesh_bvh (mesh_bvh.hpp), left in device memory.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "mesh_bvh.hpp"

namespace pbrt {

struct DeviceMeshBuild {
  GpuNode* nodes = nullptr;     // node_slots records, GPU numbering (root 0, padding 1)
  uint64_t node_slots = 0;
  float4* tri_a = nullptr;      // the triangle streams of mesh_bvh.hpp, in leaf order
  float4* tri_b = nullptr;
  float2* tri_c = nullptr;
  uint32_t* tri_index = nullptr;  // leaf order -> original triangle index
  MeshBuildStats stats;
  float bounds_min[3] = {0, 0, 0}, bounds_max[3] = {0, 0, 0};  // vertex bounds
};

// vertices (3 floats each) and indices (3 per triangle) in device memory of the current
// device; runs on `st` and returns when the build is complete. On failure returns false with
// `err` set (bad input is reported, not read out of range).
bool build_mesh_bvh_device(const float* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t tri_count,
                           const MeshBuildParams& params, cudaStream_t st, int sm_count, DeviceMeshBuild* out,
                           std::string* err);
void free_device_mesh_build(DeviceMeshBuild* build);

}  // namespace pbrt
