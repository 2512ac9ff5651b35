// device_math.cuh — FP32 arithmetic that rounds exactly as the reference's expressions.
//
// The hot path must produce, for identical rays, the nearest-hit triangle bit-exactly and
// t within 2 ulp of the FP32 restatement of the reference (whose arithmetic has no fused
// multiply-add). Every product and sum below therefore goes through the explicit
// round-to-nearest intrinsics, which the compiler never contracts into an FMA, and
// division, reciprocal and square root use the correctly rounded forms.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define PBRT_DEV __device__ __forceinline__

namespace pbrt {

PBRT_DEV float fa(float a, float b) { return __fadd_rn(a, b); }
PBRT_DEV float fs(float a, float b) { return __fsub_rn(a, b); }
PBRT_DEV float fm(float a, float b) { return __fmul_rn(a, b); }
PBRT_DEV float fdv(float a, float b) { return __fdiv_rn(a, b); }
PBRT_DEV float frcp(float a) { return __frcp_rn(a); }  // == 1.0f / a, correctly rounded
PBRT_DEV float fsq(float a) { return __fsqrt_rn(a); }

struct F3 {
  float x, y, z;
};

PBRT_DEV F3 mk3(float x, float y, float z) { return F3{x, y, z}; }
PBRT_DEV F3 add3(const F3& a, const F3& b) { return F3{fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)}; }
PBRT_DEV F3 sub3(const F3& a, const F3& b) { return F3{fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)}; }
PBRT_DEV F3 mul3(const F3& a, float s) { return F3{fm(a.x, s), fm(a.y, s), fm(a.z, s)}; }
// dot: (u.x*v.x + u.y*v.y) + u.z*v.z  (src/geom/vector3.rs:291-296)
PBRT_DEV float dot3(const F3& u, const F3& v) { return fa(fa(fm(u.x, v.x), fm(u.y, v.y)), fm(u.z, v.z)); }
// cross (src/geom/vector3.rs:298-307)
PBRT_DEV F3 cross3(const F3& u, const F3& v) {
  return F3{fs(fm(u.y, v.z), fm(u.z, v.y)), fs(fm(u.z, v.x), fm(u.x, v.z)), fs(fm(u.x, v.y), fm(u.y, v.x))};
}
// normalize: v * (1 / sqrt(|v|^2))  (src/geom/vector3.rs:69-74)
PBRT_DEV F3 normalize3(const F3& v) {
  const float inv = frcp(fsq(dot3(v, v)));
  return mul3(v, inv);
}
PBRT_DEV float length3(const F3& v) { return fsq(dot3(v, v)); }

// 2·γ(3) with u = 2^-24, evaluated in FP32 (src/geom/aabound.rs:26-39):
// u = 2^-24, 3u / (1 - 3u) rounds to 0x34400002, doubled to 0x34C00002.
#define PBRT_SLAB_WIDENING_F32 (__uint_as_float(0x34C00002u))

}  // namespace pbrt
