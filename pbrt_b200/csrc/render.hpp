// render.hpp — host-visible declarations of the wavefront renderer and the general-scene
// ray-cast launchers (device code lives in kernels_render.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "scene_types.hpp"

namespace pbrt {

struct SceneView;

// SoA state of one wave of paths (capacity = the wave size) and its queues.
struct WaveBuffers {
  float *ox, *oy, *oz, *dx, *dy, *dz;  // current ray
  float *br, *bg, *bb;                 // path throughput (beta)
  float *lr, *lg, *lb;                 // radiance gathered so far (FP32 per sample)
  unsigned long long* rng;             // PCG32 state (the increment derives from the pixel)
  uint32_t* pixel;
  uint32_t* flags;                     // bounce count (low 16 bits) | last-bounce-specular (bit 31)
  float* ht;                           // nearest hit of the current ray
  uint32_t *hobj, *hprim;
  uint32_t *qa, *qb;                   // ping-pong queues of path indices
  uint32_t* s_path;                    // shadow queue
  float *s_ox, *s_oy, *s_oz, *s_dx, *s_dy, *s_dz, *s_tmax, *s_cr, *s_cg, *s_cb;
  uint32_t* counts;                    // [0] qa length, [1] qb length, [2] shadow queue length
};

struct RenderSettings {
  uint32_t max_depth, rr_start, sample_offset, naive;
  unsigned long long seed;
};

// One wave: generate, max_depth x (extend, shade, shadow), accumulate into `film` (sums).
cudaError_t render_wave(const SceneView& s, const WaveBuffers& w, const CameraRec& cam, uint64_t wave_base,
                        uint32_t n, uint32_t npix, const RenderSettings& rs, double* film, uint32_t* err, int sm_count,
                        cudaStream_t st);
cudaError_t scale_film(double* film, size_t n, double s, int sm_count, cudaStream_t st);

cudaError_t launch_scene_closest(const SceneView& s, const float* rays, uint64_t stride, uint64_t n, uint32_t* prim,
                                 float* t, uint32_t* obj, uint32_t* err, int sm_count, cudaStream_t st);
cudaError_t launch_scene_any(const SceneView& s, const float* rays, uint64_t stride, uint64_t n, uint8_t* occ,
                             uint32_t* err, int sm_count, cudaStream_t st);

}  // namespace pbrt
