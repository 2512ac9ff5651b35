// scene_host.hpp — host-side build of a whole scene for the GPU (no device code here).
//
// The scene's primitives are its objects, or the roots of its object tree (Simple,
// Transformed, Compound nodes: src/objects/*.rs). Scene::commit (src/scene.rs:101-115) keeps
// the unbounded ones (a Plane's box is infinite) in a list and builds the top-level BVH over
// the rest, as the reference's scene accelerator does (src/bvh.rs:109-132, 291-388): median
// split on the widest centroid axis after a stable sort, one primitive per leaf, boxes
// combined bottom-up. A primitive's box is its get_bounding_box: the shape's box, transformed
// corner by corner under every Transformed (src/geom/aabound.rs:437-468), the union over a
// Compound's members. Everything is FP32, compiled with -ffp-contract=off, in the
// reference's operation order. The tree is flattened for the GPU into leaves (a placed
// Simple with the chain of transforms above it) and groups (a Compound's leaves).
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
  std::vector<ObjRec> objects;                  // leaves: placed Simple objects
  std::vector<XfRec> xforms;                    // transform chains beyond each leaf's first
  std::vector<CsgRec> csg;                      // constructive solids' elements
  std::vector<GroupRec> groups;                 // compounds (consecutive leaves)
  std::vector<uint32_t> unbounded;              // primitives kept out of the BVH, in scene order
  std::vector<GpuNode> top;                     // GPU numbering (root 0, padding 1); empty when no
                                                // primitive is bounded
  std::vector<uint32_t> order;                  // leaf slot -> primitive (leaf, or kGroupBit | group)
  uint32_t top_depth = 0;
  uint64_t primitive_count = 0;                 // bounded + unbounded
  int single_mesh = -1;                         // the mesh, when the scene is one untransformed mesh
  std::vector<MatRec> materials;
  std::vector<LightRec> lights;
  std::vector<float> light_tris;                // 9 floats per area-light triangle (world space)
  std::vector<float> light_cdf;                 // running area per area-light triangle
  // The largest radiance any emitter gives off (diffuse-light materials, infinite lights);
  // +inf with a point light. With energy-conserving materials no surface reflects more.
  float max_radiance = 0.f;
  bool has_dielectric = false;  // a dielectric lets paths go on past a cache hit
};

// A mesh whose BVH was built elsewhere (on the GPU): the scene build takes its bounds and
// statistics instead of building it.
struct MeshPrebuilt {
  bool used = false;
  float bounds_min[3] = {0, 0, 0}, bounds_max[3] = {0, 0, 0};
  MeshBuildStats stats;
};

bool build_scene(const pbrt_scene_desc& d, FlatScene* out, std::string* err,
                 const std::vector<MeshPrebuilt>* prebuilt = nullptr);

// PinHoleCamera::new + Matrix4::look_at in FP32 (src/cameras/pin_hole.rs:17-38,
// src/geom/matrix4.rs:70-175).
CameraRec build_camera(const pbrt_camera_desc& c);

}  // namespace pbrt
