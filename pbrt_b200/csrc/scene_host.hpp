// scene_host.hpp — host-side build of a whole scene for the GPU (no device code here).
//
// The top-level BVH is the reference's scene accelerator (src/bvh.rs:109-132, 291-388):
// median split on the widest centroid axis after a stable sort, one object per leaf, boxes
// combined bottom-up; object boxes are the shape's box, transformed corner by corner for
// Transformed objects (src/geom/aabound.rs:437-468). Everything is FP32, compiled with
// -ffp-contract=off, in the reference's operation order.
#pragma once

#include <string>
#include <vector>

#include "../../include/pbrt_b200.h"
#include "mesh_bvh.hpp"
#include "scene_types.hpp"

namespace pbrt {

struct FlatScene {
  std::vector<FlatMesh> meshes;
  std::vector<std::vector<float>> mesh_v;       // original vertices (shading)
  std::vector<std::vector<uint32_t>> mesh_idx;  // original indices (shading)
  std::vector<std::vector<uint32_t>> mesh_fmat; // per-triangle material, empty when absent
  std::vector<ObjRec> objects;
  std::vector<GpuNode> top;                     // GPU numbering (root 0, padding 1)
  std::vector<uint32_t> order;                  // leaf slot -> object
  uint32_t top_depth = 0;
  std::vector<MatRec> materials;
  std::vector<LightRec> lights;
  std::vector<float> light_tris;                // 9 floats per area-light triangle (world space)
  std::vector<float> light_cdf;                 // running area per area-light triangle
  // The largest radiance any emitter gives off (diffuse-light materials, infinite lights);
  // +inf with a point light. With energy-conserving materials no surface reflects more.
  float max_radiance = 0.f;
  bool has_dielectric = false;  // a dielectric lets paths go on past a cache hit
};

bool build_scene(const pbrt_scene_desc& d, FlatScene* out, std::string* err);

// PinHoleCamera::new + Matrix4::look_at in FP32 (src/cameras/pin_hole.rs:17-38,
// src/geom/matrix4.rs:70-175).
CameraRec build_camera(const pbrt_camera_desc& c);

}  // namespace pbrt
