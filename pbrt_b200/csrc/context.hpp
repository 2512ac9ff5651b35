// context.hpp — the library's internal state behind the C ABI's opaque handles (host
// code only): the context with its streams, staging slots and error word, the scene with
// its device arrays, and the helpers every entry point shares.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pbrt_b200.h"
#include "kernels.hpp"
#include "render.hpp"
#include "scene_device.cuh"
#include "trace_mesh.cuh"

namespace pbrt {
namespace api {

constexpr uint64_t kSlotRays = uint64_t(1) << 20;  // rays per pipelined chunk (32 MiB of rays)
constexpr int kSlots = 3;
constexpr uint64_t kDevChunk = uint64_t(1) << 24;  // rays per launch pair on device buffers
// Concurrent branches of a wavefront batch frame (pbrt_ctx_set_batch_branches).
constexpr uint32_t kMaxBatchBranches = 8;
constexpr uint32_t kDefaultBatchBranches = 2;
// Concurrent branches of one render (pbrt_render, pbrt_render_cached); PBRT_RENDER_BRANCHES
// overrides it for measurements.
constexpr uint32_t kDefaultRenderBranches = 2;

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

enum class MemKind { Host, Device, Null };

inline MemKind mem_kind(const void* p) {
  if (!p) return MemKind::Null;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return MemKind::Host;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return MemKind::Device;
  return MemKind::Host;
}

struct Slot {
  cudaStream_t s = nullptr;
  float* rays = nullptr;     // 8 planes of kSlotRays
  uint32_t* prim = nullptr;
  float* t = nullptr;
  uint32_t* obj = nullptr;
  uint8_t* occ = nullptr;
  uint32_t* queue = nullptr;            // survivor queue of the two-stage nearest-hit pass
  float4* rec = nullptr;                // the survivors' ray records (32 bytes each)
  pbrt::DenseScratch dense;             // dense results: per-slot (id, t), survivor bitmask, chunk bases
  unsigned long long* fetch = nullptr;  // [queue length, fetch position] of that pass
};

// The wave's SoA state, grown on demand (one per context for pbrt_render / pbrt_render_cached,
// one per batch).
struct WaveAlloc {
  void* block = nullptr;
  uint32_t capacity = 0;
  WaveBuffers w{};
};

}  // namespace api
}  // namespace pbrt

struct pbrt_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;  // internal stream
  cudaStream_t user = nullptr;    // caller's stream (asynchronous device-buffer calls)
  std::string err;
  uint32_t* d_err = nullptr;
  unsigned long long* d_counters = nullptr;  // [0..2] traversal counters, [4..5] queue length / fetch position,
                                             // [8..10] rays / shadow rays / paths of the last render
  uint32_t* queue = nullptr;                  // survivor queue for device-buffer calls (kDevChunk entries)
  float4* queue_rec = nullptr;                // and their ray records (kDevChunk x 32 bytes)
  pbrt::DenseScratch queue_dense;             // and the dense-result scratch for kDevChunk rays
  bool persistent = true;                     // persistent dynamic-fetch traversal (default)
  uint32_t* noalloc_scratch = nullptr;        // device address of pbrt_trace_closest_noalloc's static
                                              // scratch array on this device, looked up at creation
  pbrt::api::Slot slots[pbrt::api::kSlots];
  bool slots_ready = false;
  std::vector<void*> allocs;
  pbrt::LaunchShape shape;          // wavefront launch shape (pbrt_ctx_set_tuning)
  uint32_t wave_paths = 1u << 26;   // paths per wave (136 bytes of path state each, allocated on demand)
  int batch_kernel = 0;             // batches created afterwards: PBRT_BATCH_WAVEFRONT / _PERSISTENT
  uint32_t batch_branches = pbrt::api::kDefaultBatchBranches;  // concurrent branches of a wavefront batch frame
  // a cached render's training rounds beside its frame: their stream, the fork and join
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // the path state of pbrt_render / pbrt_render_cached (grown on demand), and of a cached
  // render's training paths; per context, so contexts on one device may render at once
  pbrt::api::WaveAlloc waves, train_waves;
  // concurrent branches of one pbrt_render (branch k >= 1: its stream, wave buffers and join)
  pbrt::api::WaveAlloc branch_waves[pbrt::api::kMaxBatchBranches - 1];
  cudaStream_t branch_st[pbrt::api::kMaxBatchBranches] = {};
  cudaEvent_t branch_fork = nullptr, branch_join[pbrt::api::kMaxBatchBranches] = {};

  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PBRT_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PBRT_ERR_OUT_OF_MEMORY : PBRT_ERR_CUDA;
  }
  cudaStream_t work_stream() const { return user ? user : stream; }
};

struct DeviceMesh {
  void* nodes = nullptr;
  void* tri_a = nullptr;
  void* tri_b = nullptr;
  void* tri_c = nullptr;
  pbrt::MeshView view{};
  uint64_t bytes = 0;
};

struct pbrt_scene {
  pbrt_ctx* ctx = nullptr;
  std::vector<DeviceMesh> meshes;
  std::vector<void*> allocs;  // every other device array of the scene
  uint64_t extra_bytes = 0;
  pbrt::SceneView view{};
  pbrt_scene_info info{};
  int single_mesh = -1;  // index of the only (untransformed) mesh object, or -1
  float bounds[6] = {0, 0, 0, 0, 0, 0};  // world box of every object (min xyz, max xyz)
  float max_radiance = 0.f;              // bound of reflected radiance (see FlatScene)
  bool has_dielectric = false;

  int upload(void** dst, const void* src, size_t bytes) {
    if (bytes == 0) return PBRT_OK;
    int rc = ctx->cuda(cudaMalloc(dst, bytes), "cudaMalloc(scene)");
    if (rc != PBRT_OK) return rc;
    allocs.push_back(*dst);
    extra_bytes += bytes;
    // ordered on the context's stream (see upload in api.cu); scene creation synchronises it
    return ctx->cuda(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream), "cudaMemcpy(scene)");
  }
};

#define PBRT_TRY(expr)              \
  do {                              \
    int _rc = (expr);               \
    if (_rc != PBRT_OK) return _rc; \
  } while (0)

namespace pbrt {
namespace api {

// Reads and clears the device error word after the work that may have raised it.
inline int check_device_error(pbrt_ctx* c, cudaStream_t s) {
  PBRT_TRY(c->cuda(cudaStreamSynchronize(s), "kernel execution"));
  uint32_t h = 0;
  PBRT_TRY(c->cuda(cudaMemcpy(&h, c->d_err, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy(error word)"));
  if (h == 0) return PBRT_OK;
  PBRT_TRY(c->cuda(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), s), "cudaMemset(error word)"));
  PBRT_TRY(c->cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize"));
  if (h & kErrStack) return c->fail(PBRT_ERR_CAPACITY, "traversal stack capacity exceeded");
  if (h & 4u) return c->fail(PBRT_ERR_DEVICE_BUDGET, "a tensor-core completion wait ran out of its budget");
  if (h & kErrCopy) return c->fail(PBRT_ERR_DEVICE_BUDGET, "a wait for a bulk copy into shared memory ran out of its budget");
  return c->fail(PBRT_ERR_DEVICE_BUDGET, "a traversal exceeded its iteration budget (malformed tree)");
}

}  // namespace api
}  // namespace pbrt

namespace pbrt {
namespace api {
int ensure_wave(pbrt_ctx* c, WaveAlloc* wa, uint32_t cap);
// Validation of render parameters shared by every render entry point.
int check_render_params(pbrt_ctx* c, const pbrt_render_params* p, bool allow_no_samples);
// The kernels' settings for these parameters on this context (tuning, counters).
RenderSettings settings_of(pbrt_ctx* c, const pbrt_render_params* p);
// Film pixels of a render: the image's, or the strided subset's.
uint64_t film_pixels(const pbrt_render_params* p, const RenderSettings& rs);
}  // namespace api
}  // namespace pbrt

