// scene_types.hpp — record layouts shared by the host scene builder and the device code.
#pragma once

#include <cstdint>

namespace pbrt {

enum : uint32_t { kShapeMesh = 0, kShapeSphere = 1, kShapeCylinder = 2, kShapeRectangle = 3, kShapeAABox = 4,
                  kShapePlane = 5, kShapeCsg = 6 };
enum : uint32_t { kCsgUnion = 0, kCsgIntersection = 1, kCsgSubtraction = 2 };
enum : uint32_t { kMatLambertian = 0, kMatMetal = 1, kMatDielectric = 2, kMatDiffuseLight = 3 };
enum : uint32_t { kLightPoint = 0, kLightUniform = 1, kLightBackground = 2, kLightArea = 3 };
enum : uint32_t { kTexColor = 0, kTexChecker = 1 };

// A scene primitive, as the top-level BVH's leaves and the unbounded list name it: one
// placed object (a leaf index), or with kGroupBit set a group of leaves (a Compound).
constexpr uint32_t kGroupBit = 0x80000000u;

// One placed Simple object (a "leaf"): its shape and material, and the chain of transforms
// between it and the world (xf_count of them, outermost first: the first inline here, the
// rest at xforms[xf_rest ..]). 144 bytes.
struct alignas(16) ObjRec {
  uint32_t shape, mesh, material, xf_count;
  float p[3];        // sphere: r; cylinder: r, h/2; rectangle: w/2, h/2; aabox: extent/2 (x, y, z)
  uint32_t desc_id;  // the object's index in the caller's description (reported as object_id)
  uint32_t xf_rest;
  uint32_t csg_op, csg_first, csg_count;  // a constructive solid: its elements in the CsgRec array
  float to_world[12];  // row-major 3x4 of Transform::mat (outermost transform)
  float to_local[12];  // row-major 3x4 of Transform::inv_mat
};
static_assert(sizeof(ObjRec) == 144, "ObjRec is 144 bytes");

struct alignas(16) XfRec {
  float to_world[12], to_local[12];
};
static_assert(sizeof(XfRec) == 96, "XfRec is 96 bytes");

// One element of a constructive solid: a plain shape (sizes as ObjRec::p) and its transform.
struct alignas(16) CsgRec {
  uint32_t shape, mesh, pad0, pad1;
  float p[4];
  float to_world[12], to_local[12];
};
static_assert(sizeof(CsgRec) == 128, "CsgRec is 128 bytes");

// A Compound's members: leaves [first, first + count), in member order.
struct GroupRec {
  uint32_t first, count;
};

struct alignas(16) MatRec {
  uint32_t kind, texture;
  float fuzz, ior;
  float color[4];
  float color2[3];
  float scale;
};
static_assert(sizeof(MatRec) == 48, "MatRec is 48 bytes");

struct alignas(16) LightRec {
  uint32_t kind, object, tri_first, tri_count;
  float pos[4], rad[4], bottom[4], top[4];
  float area, pad[3];
};
static_assert(sizeof(LightRec) == 96, "LightRec is 96 bytes");

// PinHoleCamera (src/cameras/pin_hole.rs:17-50) or ThinLensCamera (src/cameras/thin_lens.rs),
// evaluated on the host in FP32.
struct CameraRec {
  float raster_to_screen[16];  // row-major 4x4 (the inverse perspective makes w != 1)
  float cam_to_world[12];      // row-major 3x4
  uint32_t width, height;
  float near, far;
  uint32_t thin_lens;
  float lens_radius, focal_distance;
};

}  // namespace pbrt
