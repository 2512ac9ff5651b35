// render.hpp — host-visible declarations of the wavefront renderer and the general-scene
// ray-cast launchers (device code lives in kernels_render.cu).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "scene_device.cuh"
#include "scene_types.hpp"

namespace pbrt {

// SoA state of one wave of paths (capacity = the wave size) and its queues.
struct WaveBuffers {
  float *ox, *oy, *oz, *dx, *dy, *dz;  // current ray
  float *br, *bg, *bb;                 // path throughput (beta)
  float *lr, *lg, *lb;                 // radiance gathered so far (FP32 per sample)
  unsigned long long* rng;             // PCG32 state (the increment derives from the pixel)
  uint32_t* pixel;
  uint32_t* scene;                     // batched renders: the path's scene (index into the batch table)
  uint32_t* flags;                     // bounce count (low 16 bits) | last-bounce-specular (bit 31)
  float* ht;                           // nearest hit of the current ray
  uint32_t *hobj, *hprim;
  uint32_t *qa, *qb;                   // ping-pong queues of path indices
  uint32_t* s_path;                    // shadow queue
  float *s_ox, *s_oy, *s_oz, *s_dx, *s_dy, *s_dz, *s_tmax, *s_cr, *s_cg, *s_cb;
  uint32_t* counts;                    // [0] qa length, [1] qb length, [2] shadow queue length
};

// The radiance cache's side of a wave. Query mode: a path that reaches hit `term_hit` on a
// Lambertian or metal surface stops there, and its query record (position, roughness,
// outgoing direction, normal facing it, albedo) joins the query list; after the wave the
// network's answer times the path's throughput is added to its radiance. Record mode
// (training paths): the same, with `term_hit` further along the path, and before that
// every Lambertian or metal vertex stores its record, the radiance gathered before it and
// the throughput at it, so that once the path (and its tail query) is done,
// (L_end - L_vertex) / beta_vertex is the radiance sample the vertex is trained towards.
enum : uint32_t { kCacheOff = 0, kCacheQuery = 1, kCacheRecord = 2 };
constexpr uint32_t kCacheRecordFloats = 16;

struct CacheWave {
  float* qrec;       // query records, 16 floats each (capacity qcap)
  uint32_t* qpath;   // path of each query
  float* qout;       // network output, 3 floats per query
  float* trec;       // training vertex records, 16 floats each (capacity tcap)
  float* tstate;     // per training vertex: radiance before it (rgb), throughput at it (rgb)
  uint32_t* tpath;   // path of each training vertex
  uint32_t qcap, tcap;
  uint32_t* counts;  // [0] queries, [1] training vertices offered (may exceed tcap), [2] batch valid
};

// Launch shape of the wavefront kernels: threads per block and the resident-block target per
// SM of the grid-stride traversal kernels (extend, shadow) and of the shading kernel.
struct LaunchShape {
  uint32_t trace_threads = 128, trace_blocks_per_sm = 16;
  uint32_t shade_threads = 128, shade_blocks_per_sm = 16;
};

struct RenderSettings {
  uint32_t max_depth, rr_start, sample_offset;
  uint32_t integrator;  // pbrt_integrator: 0 path, 1 naive, 2 normal
  unsigned long long seed;
  uint32_t cache_mode = kCacheOff;
  uint32_t term_hit = 0;       // the hit at which paths end into the cache
  uint32_t random_pixels = 0;  // training paths: each path draws its pixel
  uint32_t loop_depth = 0;     // bounce iterations the host launches (0: max_depth); no path
                               // may still be alive after them
  uint32_t stride = 1;         // film pixel (i, j) is image pixel (stride*i, stride*j)
  unsigned long long* stats = nullptr;  // when set: += rays traced, shadow rays, paths
  uint32_t film_w = 0;         // film columns (0: the image width)
  LaunchShape shape;
};

// One scene of a batched render (device table entry). Global path index g belongs to the
// scene with begin <= g < begin + npix * spp; its local index l = g - begin renders film
// pixel l % npix, sample sample_offset + frame * spp + l / npix.
struct BatchScene {
  SceneView view;
  CameraRec cam;
  double* film;       // sums; scaled by 1 / spp at the end
  unsigned long long begin, seed;
  uint32_t npix, spp, max_depth, rr_start, sample_offset, integrator, stride, film_w;
};

// One wave of a batched frame: global paths [base, base + n), run on concurrent branch
// `branch` (its own wave buffers and stream).
struct BatchWave {
  unsigned long long base;
  uint32_t n, branch;
};

// The waves of a batched frame (scenes in table order, waves of at most `wave` paths along
// scene boundaries) spread over `branches` concurrent branches: the waves that share a scene
// stay on one branch (a scene's film and completion belong to one stream), and each group of
// them goes to the branch with the least work so far (paths x max depth), in table order.
std::vector<BatchWave> batch_plan(const BatchScene* host_table, uint32_t nscenes, uint32_t wave, uint32_t branches);

// A batched frame: the planned waves, each on its branch's stream with its branch's wave
// buffers (bw[k], bst[k]; bst[0] is `st`). The films are cleared on `st` before the branches
// fork from it (event `fork`) and scaled after they join it again (events joins[1..]). The
// kernels read the frame number from `frame` (device memory), so a captured graph of these
// launches renders any frame. `done[s]`, when given, is recorded (as an external event, so it
// survives stream capture) on scene s's branch right after the wave that completes it.
cudaError_t render_batch(const BatchScene* table, const BatchScene* host_table, uint32_t nscenes,
                         const std::vector<BatchWave>& plan, const WaveBuffers* bw, const cudaStream_t* bst,
                         uint32_t nbranch, const uint32_t* frame, uint32_t max_depth, bool any_path_integrator,
                         const LaunchShape& shape, unsigned long long* stats, uint32_t* err, int sm_count,
                         cudaStream_t st, cudaEvent_t fork, const cudaEvent_t* joins, cudaEvent_t* done);

// A batched frame as one persistent launch: every path of every scene run to its end by
// persistent warps (between the films' zeroing and scaling). `scratch`: 2 + 2 * nscenes
// 64-bit words; words 1 and 2 + nscenes + s hold the frame's start and scene s's completion
// on the GPU clock (ns) afterwards.
cudaError_t render_batch_persistent(const BatchScene* table, const BatchScene* host_table, uint32_t nscenes,
                                    const uint32_t* frame, unsigned long long* scratch, unsigned long long* stats,
                                    uint32_t* err, int sm_count, cudaStream_t st);

// One wave: generate, max_depth x (extend, shade, shadow), accumulate into `film` (sums).
// `npix` is the number of film pixels (the image's, or the strided subset's).
cudaError_t render_wave(const SceneView& s, const WaveBuffers& w, const CameraRec& cam, uint64_t wave_base,
                        uint32_t n, uint32_t npix, const RenderSettings& rs, double* film, uint32_t* err, int sm_count,
                        cudaStream_t st);
// The same without the accumulation, with the cache's side (cw unused when cache_mode is off).
cudaError_t trace_wave(const SceneView& s, const WaveBuffers& w, const CacheWave& cw, const CameraRec& cam,
                       uint64_t wave_base, uint32_t n, uint32_t npix, const RenderSettings& rs, uint32_t* err,
                       int sm_count, cudaStream_t st);
cudaError_t accumulate_wave(const WaveBuffers& w, uint32_t n, double* film, uint32_t image_w, const RenderSettings& rs,
                            int sm_count, cudaStream_t st);
// radiance[path] += beta[path] * clamp(network output, 0, max_l) for every query of a wave of
// n paths (queries beyond qcap were never written; path indices >= n are skipped).
cudaError_t apply_cache(const WaveBuffers& w, const CacheWave& cw, uint32_t n, float max_l, int sm_count,
                        cudaStream_t st);
// A training batch of `batch` samples drawn with replacement from the m = min(counts[1],
// tcap) recorded vertices (m read on the device): their records and targets
// clamp((L_end - L_vertex) / beta_vertex, 0, max_l) (0 where beta is 0). Sets counts[2] to
// 1 when m > 0, else 0 (and the batch is all zeros).
cudaError_t train_batch(const WaveBuffers& w, const CacheWave& cw, uint32_t batch, uint32_t step,
                        unsigned long long seed, float max_l, float* rec, float* tgt, int sm_count, cudaStream_t st);
cudaError_t scale_film(double* film, size_t n, double s, int sm_count, cudaStream_t st);

// Scene-level ray casts; cnt (3 counters: nodes, boxes, objects) may be NULL.
cudaError_t launch_scene_closest(const SceneView& s, const float* rays, uint64_t stride, uint64_t n, uint32_t* prim,
                                 float* t, uint32_t* obj, unsigned long long* cnt, uint32_t* err, int sm_count,
                                 cudaStream_t st);
cudaError_t launch_scene_any(const SceneView& s, const float* rays, uint64_t stride, uint64_t n, uint8_t* occ,
                             unsigned long long* cnt, uint32_t* err, int sm_count, cudaStream_t st);

}  // namespace pbrt
