// scene_types.hpp — record layouts shared by the host scene builder and the device code.
#pragma once

#include <cstdint>

namespace pbrt {

enum : uint32_t { kShapeMesh = 0, kShapeSphere = 1, kShapeCylinder = 2 };
enum : uint32_t { kMatLambertian = 0, kMatMetal = 1, kMatDielectric = 2, kMatDiffuseLight = 3 };
enum : uint32_t { kLightPoint = 0, kLightUniform = 1, kLightBackground = 2, kLightArea = 3 };

// One object (Simple or Transformed(Simple)): 128 bytes, read as eight float4.
struct alignas(16) ObjRec {
  uint32_t shape, mesh, material, transformed;
  float radius, half_height, pad0, pad1;
  float to_world[12];  // row-major 3x4 of Transform::mat
  float to_local[12];  // row-major 3x4 of Transform::inv_mat
};
static_assert(sizeof(ObjRec) == 128, "ObjRec is 128 bytes");

struct alignas(16) MatRec {
  uint32_t kind, pad;
  float fuzz, ior;
  float color[4];
};
static_assert(sizeof(MatRec) == 32, "MatRec is 32 bytes");

struct alignas(16) LightRec {
  uint32_t kind, object, tri_first, tri_count;
  float pos[4], rad[4], bottom[4], top[4];
  float area, pad[3];
};
static_assert(sizeof(LightRec) == 96, "LightRec is 96 bytes");

// PinHoleCamera (src/cameras/pin_hole.rs:17-50), evaluated on the host in FP32.
struct CameraRec {
  float raster_to_screen[16];  // row-major 4x4 (the inverse perspective makes w != 1)
  float cam_to_world[12];      // row-major 3x4
  uint32_t width, height;
  float near, far;
};

}  // namespace pbrt
