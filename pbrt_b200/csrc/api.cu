// api.cu — implementation of the C ABI declared in include/pbrt_b200.h.
//
// Host responsibilities: validate descriptions, build acceleration structures, own device
// memory, pick the host- or device-buffer path, and turn device-side error flags into
// status codes. No computation of the hot path happens on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pbrt_b200.h"
#include "kernels.hpp"
#include "mesh_bvh.hpp"
#include "trace_mesh.cuh"

using namespace pbrt;

namespace {

constexpr uint64_t kSlotRays = uint64_t(1) << 21;  // rays per pipelined chunk (64 MiB of rays)
constexpr int kSlots = 3;
constexpr uint64_t kDevChunk = uint64_t(1) << 24;  // rays per launch pair on device buffers

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

MemKind mem_kind(const void* p) {
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
  unsigned long long* fetch = nullptr;  // [queue length, fetch position] of that pass
};

}  // namespace

struct pbrt_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;  // internal stream
  cudaStream_t user = nullptr;    // caller's stream (asynchronous device-buffer calls)
  std::string err;
  uint32_t* d_err = nullptr;
  unsigned long long* d_counters = nullptr;  // [0..2] traversal counters, [4..5] queue length / fetch position
  uint32_t* queue = nullptr;                  // survivor queue for device-buffer calls (kDevChunk entries)
  bool persistent = true;                     // persistent dynamic-fetch traversal (default)
  Slot slots[kSlots];
  bool slots_ready = false;
  std::vector<void*> allocs;

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
  MeshView view{};
  uint64_t bytes = 0;
};

struct pbrt_scene {
  pbrt_ctx* ctx = nullptr;
  std::vector<DeviceMesh> meshes;
  pbrt_scene_info info{};
  int single_mesh = -1;  // index of the only (untransformed) mesh object, or -1
};

#define PBRT_TRY(expr)              \
  do {                              \
    int _rc = (expr);               \
    if (_rc != PBRT_OK) return _rc; \
  } while (0)

namespace {

int ensure_slots(pbrt_ctx* c) {
  if (c->slots_ready) return PBRT_OK;
  for (Slot& s : c->slots) {
    PBRT_TRY(c->cuda(cudaStreamCreateWithFlags(&s.s, cudaStreamNonBlocking), "cudaStreamCreate"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.rays, sizeof(float) * 8 * kSlotRays), "cudaMalloc(staging rays)"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.prim, sizeof(uint32_t) * kSlotRays), "cudaMalloc(staging)"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.t, sizeof(float) * kSlotRays), "cudaMalloc(staging)"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.obj, sizeof(uint32_t) * kSlotRays), "cudaMalloc(staging)"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.occ, kSlotRays), "cudaMalloc(staging)"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.queue, sizeof(uint32_t) * kSlotRays), "cudaMalloc(staging)"));
    PBRT_TRY(c->cuda(cudaMalloc(&s.fetch, 2 * sizeof(unsigned long long)), "cudaMalloc(staging)"));
  }
  c->slots_ready = true;
  return PBRT_OK;
}

int ensure_queue(pbrt_ctx* c) {
  if (c->queue) return PBRT_OK;
  return c->cuda(cudaMalloc(&c->queue, sizeof(uint32_t) * kDevChunk), "cudaMalloc(survivor queue)");
}

// Reads and clears the device error word after the work that may have raised it.
int check_device_error(pbrt_ctx* c, cudaStream_t s) {
  PBRT_TRY(c->cuda(cudaStreamSynchronize(s), "kernel execution"));
  uint32_t h = 0;
  PBRT_TRY(c->cuda(cudaMemcpy(&h, c->d_err, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy(error word)"));
  if (h == 0) return PBRT_OK;
  PBRT_TRY(c->cuda(cudaMemset(c->d_err, 0, sizeof(uint32_t)), "cudaMemset(error word)"));
  if (h & kErrStack) return c->fail(PBRT_ERR_CAPACITY, "traversal stack capacity exceeded");
  return c->fail(PBRT_ERR_DEVICE_BUDGET, "a traversal exceeded its iteration budget (malformed tree)");
}

int upload(pbrt_ctx* c, void** dst, const void* src, size_t bytes, uint64_t* total) {
  PBRT_TRY(c->cuda(cudaMalloc(dst, bytes), "cudaMalloc(scene)"));
  *total += bytes;
  return c->cuda(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(scene)");
}

void free_mesh(DeviceMesh& m) {
  cudaFree(m.nodes);
  cudaFree(m.tri_a);
  cudaFree(m.tri_b);
  cudaFree(m.tri_c);
  m = DeviceMesh{};
}

}  // namespace

extern "C" {

int pbrt_ctx_create(int device, pbrt_ctx** out) {
  if (!out) return PBRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return PBRT_ERR_INVALID_ARGUMENT;
  }
  std::unique_ptr<pbrt_ctx> c(new pbrt_ctx);
  c->device = device;
  DeviceGuard g(device);
  cudaDeviceProp prop;
  if (c->cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties") != PBRT_OK) return PBRT_ERR_CUDA;
  if (prop.major < 10) return PBRT_ERR_UNSUPPORTED;  // built for sm_100a only
  c->sm_count = prop.multiProcessorCount;
  // PBRT_TRACE_KERNEL=simple selects the one-thread-per-ray kernel (same results) for A/B runs.
  if (const char* k = std::getenv("PBRT_TRACE_KERNEL")) c->persistent = std::strcmp(k, "simple") != 0;
  if (c->cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate") != PBRT_OK)
    return PBRT_ERR_CUDA;
  if (c->cuda(cudaMalloc(&c->d_err, sizeof(uint32_t)), "cudaMalloc") != PBRT_OK) return PBRT_ERR_OUT_OF_MEMORY;
  if (c->cuda(cudaMemset(c->d_err, 0, sizeof(uint32_t)), "cudaMemset") != PBRT_OK) return PBRT_ERR_CUDA;
  if (c->cuda(cudaMalloc(&c->d_counters, 8 * sizeof(unsigned long long)), "cudaMalloc") != PBRT_OK)
    return PBRT_ERR_OUT_OF_MEMORY;
  *out = c.release();
  return PBRT_OK;
}

void pbrt_ctx_destroy(pbrt_ctx* c) {
  if (!c) return;
  DeviceGuard g(c->device);
  cudaStreamSynchronize(c->stream);
  for (Slot& s : c->slots) {
    if (s.s) cudaStreamSynchronize(s.s);
    cudaFree(s.rays);
    cudaFree(s.prim);
    cudaFree(s.t);
    cudaFree(s.obj);
    cudaFree(s.occ);
    cudaFree(s.queue);
    cudaFree(s.fetch);
    if (s.s) cudaStreamDestroy(s.s);
  }
  cudaFree(c->d_err);
  cudaFree(c->d_counters);
  cudaFree(c->queue);
  cudaStreamDestroy(c->stream);
  delete c;
}

const char* pbrt_last_error(const pbrt_ctx* c) { return c ? c->err.c_str() : "null context"; }

int pbrt_ctx_set_stream(pbrt_ctx* c, void* stream) {
  if (!c) return PBRT_ERR_INVALID_ARGUMENT;
  c->user = (cudaStream_t)stream;
  return PBRT_OK;
}

int pbrt_ctx_sync(pbrt_ctx* c) {
  if (!c) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(c->device);
  return check_device_error(c, c->work_stream());
}

int pbrt_scene_create(pbrt_ctx* c, const pbrt_scene_desc* d, pbrt_scene** out) {
  if (!c || !d || !out) return PBRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  DeviceGuard g(c->device);
  if (d->object_count == 0) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "a scene needs at least one object");
  if (d->mesh_count && !d->meshes) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "meshes is NULL");
  if (!d->objects) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "objects is NULL");
  MeshBuildParams bp;
  bp.bins = d->bvh_bins ? int(d->bvh_bins) : 8;
  bp.max_leaf = d->bvh_max_leaf ? d->bvh_max_leaf : 1;

  std::unique_ptr<pbrt_scene> s(new pbrt_scene);
  s->ctx = c;
  for (uint32_t i = 0; i < d->object_count; ++i) {
    const pbrt_object_desc& o = d->objects[i];
    if (o.shape == PBRT_SHAPE_MESH && o.mesh >= d->mesh_count)
      return c->fail(PBRT_ERR_INVALID_ARGUMENT, "object references a mesh that does not exist");
  }
  if (!(d->object_count == 1 && d->objects[0].shape == PBRT_SHAPE_MESH && !d->objects[0].transformed))
    return c->fail(PBRT_ERR_UNSUPPORTED, "this build traces scenes made of one untransformed mesh");

  s->meshes.resize(d->mesh_count);
  for (uint32_t i = 0; i < d->mesh_count; ++i) {
    const pbrt_mesh_desc& md = d->meshes[i];
    FlatMesh fm;
    std::string e;
    if (!build_mesh_bvh(md.vertices, md.vertex_count, md.indices, md.triangle_count, bp, &fm, &e)) {
      for (auto& m : s->meshes) free_mesh(m);
      return c->fail(PBRT_ERR_INVALID_ARGUMENT, "mesh " + std::to_string(i) + ": " + e);
    }
    if (fm.stats.max_depth >= uint32_t(kTraceStack)) {
      for (auto& m : s->meshes) free_mesh(m);
      return c->fail(PBRT_ERR_CAPACITY, "mesh " + std::to_string(i) + ": BVH depth " +
                                             std::to_string(fm.stats.max_depth) + " exceeds the traversal stack");
    }
    DeviceMesh& dm = s->meshes[i];
    int rc = upload(c, &dm.nodes, fm.nodes.data(), fm.nodes.size() * sizeof(GpuNode), &dm.bytes);
    if (rc == PBRT_OK) rc = upload(c, &dm.tri_a, fm.tri_a.data(), fm.tri_a.size() * sizeof(float), &dm.bytes);
    if (rc == PBRT_OK) rc = upload(c, &dm.tri_b, fm.tri_b.data(), fm.tri_b.size() * sizeof(float), &dm.bytes);
    if (rc == PBRT_OK) rc = upload(c, &dm.tri_c, fm.tri_c.data(), fm.tri_c.size() * sizeof(float), &dm.bytes);
    if (rc != PBRT_OK) {
      for (auto& m : s->meshes) free_mesh(m);
      return rc;
    }
    dm.view.nodes = (const float4*)dm.nodes;
    dm.view.tri_a = (const float4*)dm.tri_a;
    dm.view.tri_b = (const float4*)dm.tri_b;
    dm.view.tri_c = (const float2*)dm.tri_c;
    dm.view.node_count = uint32_t(fm.nodes.size());
    s->info.triangle_count += md.triangle_count;
    s->info.mesh_node_count += fm.stats.node_count;
    s->info.mesh_leaf_count += fm.stats.leaf_count;
    s->info.mesh_max_depth = std::max(s->info.mesh_max_depth, fm.stats.max_depth);
    s->info.mesh_max_leaf_tris = std::max(s->info.mesh_max_leaf_tris, fm.stats.max_leaf_tris);
    s->info.device_bytes += dm.bytes;
  }
  s->info.object_count = d->object_count;
  s->single_mesh = int(d->objects[0].mesh);
  *out = s.release();
  return PBRT_OK;
}

void pbrt_scene_destroy(pbrt_scene* s) {
  if (!s) return;
  DeviceGuard g(s->ctx->device);
  cudaStreamSynchronize(s->ctx->work_stream());
  for (auto& m : s->meshes) free_mesh(m);
  delete s;
}

int pbrt_mesh_bvh_build_host(const pbrt_mesh_desc* md, uint32_t bins, uint32_t max_leaf, void* nodes,
                             uint64_t node_capacity, uint32_t* tri_order, uint64_t* node_count) {
  if (!md || !node_count) return PBRT_ERR_INVALID_ARGUMENT;
  MeshBuildParams bp;
  bp.bins = bins ? int(bins) : 8;
  bp.max_leaf = max_leaf ? max_leaf : 1;
  FlatMesh fm;
  std::string e;
  if (!build_mesh_bvh(md->vertices, md->vertex_count, md->indices, md->triangle_count, bp, &fm, &e))
    return PBRT_ERR_INVALID_ARGUMENT;
  *node_count = fm.nodes.size();
  if (!nodes) return PBRT_OK;
  if (node_capacity < fm.nodes.size()) return PBRT_ERR_CAPACITY;
  std::memcpy(nodes, fm.nodes.data(), fm.nodes.size() * sizeof(GpuNode));
  if (tri_order) std::memcpy(tri_order, fm.tri_index.data(), fm.tri_index.size() * sizeof(uint32_t));
  return PBRT_OK;
}

int pbrt_scene_get_info(const pbrt_scene* s, pbrt_scene_info* info) {
  if (!s || !info) return PBRT_ERR_INVALID_ARGUMENT;
  *info = s->info;
  return PBRT_OK;
}

}  // extern "C"

namespace {

// Runs the nearest-hit (or, with occ != NULL, any-hit) kernel over host or device buffers.
int trace_impl(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim, float* t, uint32_t* obj, uint8_t* occ,
               uint64_t* stats) {
  if (!s) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = s->ctx;
  DeviceGuard g(c->device);
  if (n == 0) return PBRT_OK;
  if (!rays || (!occ && (!prim || !t))) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "ray or result buffer is NULL");
  const MeshView& mv = s->meshes[s->single_mesh].view;

  const MemKind kr = mem_kind(rays);
  const MemKind ko = occ ? mem_kind(occ) : mem_kind(prim);
  const MemKind kt = occ ? ko : mem_kind(t);
  const MemKind kb = obj ? mem_kind(obj) : ko;
  if (kr != ko || ko != kt || kt != kb)
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "ray and result buffers must all be host memory or all device memory");

  unsigned long long* counters = nullptr;
  if (stats) {
    counters = c->d_counters;
    PBRT_TRY(c->cuda(cudaMemsetAsync(counters, 0, 3 * sizeof(unsigned long long), c->work_stream()), "cudaMemset"));
  }

  if (kr == MemKind::Device) {
    cudaStream_t st = c->work_stream();
    if (occ) {
      PBRT_TRY(c->cuda(launch_mesh_any(mv, rays, n, n, occ, c->d_err, c->sm_count, st), "kernel launch"));
    } else if (c->persistent && !counters) {
      // Chunks of at most kDevChunk rays bound the survivor queue (scratch) to 64 MiB.
      PBRT_TRY(ensure_queue(c));
      for (uint64_t base = 0; base < n; base += kDevChunk) {
        const uint64_t m = std::min<uint64_t>(kDevChunk, n - base);
        PBRT_TRY(c->cuda(launch_mesh_closest_persistent(mv, rays + base, n, m, prim + base, t + base,
                                                        obj ? obj + base : nullptr, c->queue, c->d_counters + 4,
                                                        c->d_err, c->sm_count, st),
                         "kernel launch"));
      }
    } else {
      PBRT_TRY(c->cuda(launch_mesh_closest(mv, rays, n, n, prim, t, obj, counters, c->d_err, c->sm_count, st),
                       "kernel launch"));
    }
    if (stats) {
      unsigned long long h[3];
      PBRT_TRY(c->cuda(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st), "cudaMemcpy"));
      PBRT_TRY(check_device_error(c, st));
      for (int k = 0; k < 3; ++k) stats[k] = h[k];
      return PBRT_OK;
    }
    if (c->user) return PBRT_OK;  // ordered on the caller's stream; errors surface at pbrt_ctx_sync
    return check_device_error(c, st);
  }

  // Host buffers: pipeline chunks through three staging slots, each on its own stream, so
  // the copy engines and the SMs overlap (H2D of chunk k+1 and D2H of k-1 run under the
  // kernel of chunk k).
  PBRT_TRY(ensure_slots(c));
  if (c->user) PBRT_TRY(c->cuda(cudaStreamSynchronize(c->user), "cudaStreamSynchronize"));
  if (stats)
    PBRT_TRY(c->cuda(cudaStreamSynchronize(c->work_stream()), "cudaStreamSynchronize"));
  uint64_t chunk = 0;
  for (uint64_t base = 0; base < n; base += kSlotRays, ++chunk) {
    Slot& sl = c->slots[chunk % kSlots];
    const uint64_t m = std::min<uint64_t>(kSlotRays, n - base);
    for (int p = 0; p < 8; ++p)
      PBRT_TRY(c->cuda(cudaMemcpyAsync(sl.rays + p * kSlotRays, rays + p * n + base, m * sizeof(float),
                                       cudaMemcpyHostToDevice, sl.s),
                       "cudaMemcpyAsync(rays)"));
    cudaError_t e;
    if (occ)
      e = launch_mesh_any(mv, sl.rays, kSlotRays, m, sl.occ, c->d_err, c->sm_count, sl.s);
    else if (c->persistent && !counters)
      e = launch_mesh_closest_persistent(mv, sl.rays, kSlotRays, m, sl.prim, sl.t, obj ? sl.obj : nullptr, sl.queue,
                                         sl.fetch, c->d_err, c->sm_count, sl.s);
    else
      e = launch_mesh_closest(mv, sl.rays, kSlotRays, m, sl.prim, sl.t, obj ? sl.obj : nullptr, counters, c->d_err,
                              c->sm_count, sl.s);
    PBRT_TRY(c->cuda(e, "kernel launch"));
    if (occ) {
      PBRT_TRY(c->cuda(cudaMemcpyAsync(occ + base, sl.occ, m, cudaMemcpyDeviceToHost, sl.s), "cudaMemcpyAsync"));
    } else {
      PBRT_TRY(c->cuda(cudaMemcpyAsync(prim + base, sl.prim, m * 4, cudaMemcpyDeviceToHost, sl.s), "cudaMemcpyAsync"));
      PBRT_TRY(c->cuda(cudaMemcpyAsync(t + base, sl.t, m * 4, cudaMemcpyDeviceToHost, sl.s), "cudaMemcpyAsync"));
      if (obj)
        PBRT_TRY(c->cuda(cudaMemcpyAsync(obj + base, sl.obj, m * 4, cudaMemcpyDeviceToHost, sl.s), "cudaMemcpyAsync"));
    }
  }
  int rc = PBRT_OK;
  for (Slot& sl : c->slots) {
    int r = c->cuda(cudaStreamSynchronize(sl.s), "kernel execution");
    if (rc == PBRT_OK) rc = r;
  }
  PBRT_TRY(rc);
  if (stats) {
    unsigned long long h[3];
    PBRT_TRY(c->cuda(cudaMemcpy(h, counters, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy"));
    for (int k = 0; k < 3; ++k) stats[k] = h[k];
  }
  return check_device_error(c, c->stream);
}

}  // namespace

extern "C" {

int pbrt_trace_closest(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim_id, float* t, uint32_t* object_id) {
  return trace_impl(s, rays, n, prim_id, t, object_id, nullptr, nullptr);
}

int pbrt_trace_closest_instrumented(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim_id, float* t,
                                    uint64_t* stats) {
  if (!stats) return PBRT_ERR_INVALID_ARGUMENT;
  return trace_impl(s, rays, n, prim_id, t, nullptr, nullptr, stats);
}

static_assert(kNoAllocMaxRays == PBRT_NOALLOC_MAX_RAYS, "header and kernels disagree on the no-alloc capacity");

// For callers that cannot call cudaMalloc (see the header): the same two kernels as the
// device-buffer path of pbrt_trace_closest, with their scratch in a static __device__ array.
int pbrt_trace_closest_noalloc(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim_id, float* t) {
  if (!s) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = s->ctx;
  DeviceGuard g(c->device);
  if (n > kNoAllocMaxRays)
    return c->fail(PBRT_ERR_CAPACITY, "pbrt_trace_closest_noalloc: n = " + std::to_string(n) +
                                          " exceeds its fixed scratch capacity of " + std::to_string(kNoAllocMaxRays) +
                                          " rays; split the batch or use pbrt_trace_closest");
  if (n > 0) {
    if (!rays || !prim_id || !t) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "ray or result buffer is NULL");
    if (mem_kind(rays) != MemKind::Device || mem_kind(prim_id) != MemKind::Device || mem_kind(t) != MemKind::Device)
      return c->fail(PBRT_ERR_INVALID_ARGUMENT,
                     "pbrt_trace_closest_noalloc takes device buffers only (host buffers need staging memory)");
  }
  const MeshView& mv = s->meshes[s->single_mesh].view;
  cudaStream_t st = c->work_stream();
  uint32_t* scratch = nullptr;
  PBRT_TRY(c->cuda(launch_mesh_closest_noalloc(mv, rays, n, prim_id, t, c->device, c->sm_count, st, &scratch),
                   "pbrt_trace_closest_noalloc"));
  if (n == 0) return PBRT_OK;
  PBRT_TRY(c->cuda(cudaStreamSynchronize(st), "kernel execution"));
  uint32_t h = 0;
  PBRT_TRY(c->cuda(cudaMemcpy(&h, scratch + 4, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy(error word)"));
  if (h & kErrStack) return c->fail(PBRT_ERR_CAPACITY, "traversal stack capacity exceeded");
  if (h) return c->fail(PBRT_ERR_DEVICE_BUDGET, "a traversal exceeded its iteration budget (malformed tree)");
  return PBRT_OK;
}

int pbrt_trace_any(pbrt_scene* s, const float* rays, uint64_t n, uint8_t* occluded) {
  if (!occluded) return s ? s->ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "occluded is NULL") : PBRT_ERR_INVALID_ARGUMENT;
  return trace_impl(s, rays, n, nullptr, nullptr, nullptr, occluded, nullptr);
}

}  // extern "C"
