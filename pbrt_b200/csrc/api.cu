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
#include <atomic>
#include <thread>

#include "../../include/pbrt_b200.h"
#include "cache.hpp"
#include "kernels.hpp"
#include "mesh_bvh.hpp"
#include "render.hpp"
#include "scene_device.cuh"
#include "bvh_build_gpu.hpp"
#include "scene_host.hpp"
#include "trace_mesh.cuh"
#include "context.hpp"

using namespace pbrt;
using namespace pbrt::api;

namespace {

// The dense-result scratch for `cap` rays: a (id, t) pair per queue slot, one mask bit per
// ray, one queue base per 1,024-ray chunk.
int alloc_dense(pbrt_ctx* c, DenseScratch* d, uint64_t cap) {
  if (!d->res) PBRT_TRY(c->cuda(cudaMalloc(&d->res, sizeof(uint2) * cap), "cudaMalloc(dense results)"));
  const uint64_t chunks = (cap + kDenseChunk - 1) / kDenseChunk;
  if (!d->mask) PBRT_TRY(c->cuda(cudaMalloc(&d->mask, sizeof(uint32_t) * 32 * chunks), "cudaMalloc(dense mask)"));
  if (!d->bases) PBRT_TRY(c->cuda(cudaMalloc(&d->bases, sizeof(uint32_t) * chunks), "cudaMalloc(dense bases)"));
  return PBRT_OK;
}

void free_dense(DenseScratch* d) {
  cudaFree(d->res);
  cudaFree(d->mask);
  cudaFree(d->bases);
  *d = DenseScratch{};
}

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
    PBRT_TRY(c->cuda(cudaMalloc(&s.rec, sizeof(float4) * 2 * kSlotRays), "cudaMalloc(staging)"));
    PBRT_TRY(alloc_dense(c, &s.dense, kSlotRays));
    PBRT_TRY(c->cuda(cudaMalloc(&s.fetch, 2 * sizeof(unsigned long long)), "cudaMalloc(staging)"));
  }
  c->slots_ready = true;
  return PBRT_OK;
}

int ensure_queue(pbrt_ctx* c) {
  if (c->queue && c->queue_rec && c->queue_dense.bases) return PBRT_OK;
  if (!c->queue) PBRT_TRY(c->cuda(cudaMalloc(&c->queue, sizeof(uint32_t) * kDevChunk), "cudaMalloc(survivor queue)"));
  if (!c->queue_rec)
    PBRT_TRY(c->cuda(cudaMalloc(&c->queue_rec, sizeof(float4) * 2 * kDevChunk), "cudaMalloc(survivor records)"));
  return alloc_dense(c, &c->queue_dense, kDevChunk);
}

// Host-to-device copies go on the context's own stream: a plain cudaMemcpy from pageable
// memory may return before its DMA lands, and kernels on a non-blocking stream would not wait
// for it. Scene creation synchronises that stream once all copies are queued.
int upload(pbrt_ctx* c, void** dst, const void* src, size_t bytes, uint64_t* total) {
  PBRT_TRY(c->cuda(cudaMalloc(dst, bytes), "cudaMalloc(scene)"));
  *total += bytes;
  return c->cuda(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, c->stream), "cudaMemcpy(scene)");
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
  if (c->cuda(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), c->stream), "cudaMemset") != PBRT_OK)
    return PBRT_ERR_CUDA;
  if (c->cuda(cudaMalloc(&c->d_counters, 16 * sizeof(unsigned long long)), "cudaMalloc") != PBRT_OK)
    return PBRT_ERR_OUT_OF_MEMORY;
  if (c->cuda(cudaMemsetAsync(c->d_counters, 0, 16 * sizeof(unsigned long long), c->stream), "cudaMemset") !=
      PBRT_OK)
    return PBRT_ERR_CUDA;
  // The allocation-free trace's scratch array: its address on this device (which loads the
  // trace kernels' module now, under lazy loading, so its 4 MiB are committed here and not
  // inside a later call).
  if (c->cuda(noalloc_scratch_lookup(&c->noalloc_scratch), "cudaGetSymbolAddress") != PBRT_OK) return PBRT_ERR_CUDA;
  if (c->cuda(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize") != PBRT_OK) return PBRT_ERR_CUDA;
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
    cudaFree(s.rec);
    free_dense(&s.dense);
    if (s.s) cudaStreamDestroy(s.s);
  }
  if (c->side) {
    cudaStreamSynchronize(c->side);
    cudaStreamDestroy(c->side);
  }
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->join) cudaEventDestroy(c->join);
  cudaFree(c->waves.block);
  cudaFree(c->train_waves.block);
  for (uint32_t k = 0; k < kMaxBatchBranches; ++k) {
    if (c->branch_st[k]) {
      cudaStreamSynchronize(c->branch_st[k]);
      cudaStreamDestroy(c->branch_st[k]);
    }
    if (c->branch_join[k]) cudaEventDestroy(c->branch_join[k]);
    if (k + 1 < kMaxBatchBranches) cudaFree(c->branch_waves[k].block);
  }
  if (c->branch_fork) cudaEventDestroy(c->branch_fork);
  cudaFree(c->d_err);
  cudaFree(c->d_counters);
  cudaFree(c->queue);
  cudaFree(c->queue_rec);
  free_dense(&c->queue_dense);
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

}  // extern "C"

namespace {

constexpr uint64_t kDeferMinTriangles = 4096;

// The device half of scene creation: checks the built structure, uploads it, fills the view.
// Meshes listed in `dev` (non-null nodes) were built on the GPU: their arrays are taken over.
int upload_scene(pbrt_ctx* c, const pbrt_scene_desc* d, const FlatScene& fs, pbrt_scene** out,
                 std::vector<DeviceMeshBuild>* dev = nullptr) {
  for (uint32_t i = 0; i < fs.meshes.size(); ++i)
    if (fs.meshes[i].stats.max_depth >= uint32_t(kTraceStack))
      return c->fail(PBRT_ERR_CAPACITY, "mesh " + std::to_string(i) + ": BVH depth " +
                                             std::to_string(fs.meshes[i].stats.max_depth) +
                                             " exceeds the traversal stack");
  if (fs.top_depth >= uint32_t(kTraceStack))
    return c->fail(PBRT_ERR_CAPACITY, "scene BVH depth exceeds the traversal stack");

  std::unique_ptr<pbrt_scene> s(new pbrt_scene);
  s->ctx = c;
  s->meshes.resize(fs.meshes.size());
  std::vector<MeshView> views(fs.meshes.size());
  std::vector<MeshShade> shades(fs.meshes.size());
  int rc = PBRT_OK;
  for (uint32_t i = 0; i < fs.meshes.size() && rc == PBRT_OK; ++i) {
    const FlatMesh& fm = fs.meshes[i];
    DeviceMesh& dm = s->meshes[i];
    const uint64_t ntri = d->meshes[i].triangle_count;
    if (dev && i < dev->size() && (*dev)[i].nodes) {  // built on the GPU: take its arrays
      DeviceMeshBuild& b = (*dev)[i];
      dm.nodes = b.nodes;
      dm.tri_a = b.tri_a;
      dm.tri_b = b.tri_b;
      dm.tri_c = b.tri_c;
      dm.bytes = b.node_slots * sizeof(GpuNode) + ntri * 40;
      dm.view.node_count = uint32_t(b.node_slots);
      cudaFree(b.tri_index);
      b = DeviceMeshBuild{};
    } else {
      rc = upload(c, &dm.nodes, fm.nodes.data(), fm.nodes.size() * sizeof(GpuNode), &dm.bytes);
      if (rc == PBRT_OK) rc = upload(c, &dm.tri_a, fm.tri_a.data(), fm.tri_a.size() * sizeof(float), &dm.bytes);
      if (rc == PBRT_OK) rc = upload(c, &dm.tri_b, fm.tri_b.data(), fm.tri_b.size() * sizeof(float), &dm.bytes);
      if (rc == PBRT_OK) rc = upload(c, &dm.tri_c, fm.tri_c.data(), fm.tri_c.size() * sizeof(float), &dm.bytes);
      if (rc != PBRT_OK) break;
      dm.view.node_count = uint32_t(fm.nodes.size());
    }
    dm.view.nodes = (const float4*)dm.nodes;
    dm.view.tri_a = (const float4*)dm.tri_a;
    dm.view.tri_b = (const float4*)dm.tri_b;
    dm.view.tri_c = (const float2*)dm.tri_c;
    views[i] = dm.view;
    void* pv = nullptr;
    void* pi = nullptr;
    rc = s->upload(&pv, fs.mesh_v[i].data(), fs.mesh_v[i].size() * sizeof(float));
    if (rc == PBRT_OK) rc = s->upload(&pi, fs.mesh_idx[i].data(), fs.mesh_idx[i].size() * sizeof(uint32_t));
    void* pf = nullptr;
    if (rc == PBRT_OK && !fs.mesh_fmat[i].empty())
      rc = s->upload(&pf, fs.mesh_fmat[i].data(), fs.mesh_fmat[i].size() * sizeof(uint32_t));
    shades[i] = MeshShade{(const float*)pv, (const uint32_t*)pi, (const uint32_t*)pf};
    s->info.triangle_count += ntri;
    s->info.mesh_node_count += fm.stats.node_count;
    s->info.mesh_leaf_count += fm.stats.leaf_count;
    s->info.mesh_max_depth = std::max(s->info.mesh_max_depth, fm.stats.max_depth);
    s->info.mesh_max_leaf_tris = std::max(s->info.mesh_max_leaf_tris, fm.stats.max_leaf_tris);
    s->info.device_bytes += dm.bytes;
  }
  void *top = nullptr, *order = nullptr, *objs = nullptr, *mviews = nullptr, *mshades = nullptr, *mats = nullptr,
       *lights = nullptr, *ltris = nullptr, *lcdf = nullptr, *unb = nullptr, *xfs = nullptr, *grps = nullptr,
       *csgs = nullptr;
  if (rc == PBRT_OK && !fs.top.empty()) rc = s->upload(&top, fs.top.data(), fs.top.size() * sizeof(GpuNode));
  if (rc == PBRT_OK && !fs.order.empty()) rc = s->upload(&order, fs.order.data(), fs.order.size() * sizeof(uint32_t));
  if (rc == PBRT_OK) rc = s->upload(&objs, fs.objects.data(), fs.objects.size() * sizeof(ObjRec));
  if (rc == PBRT_OK && !fs.unbounded.empty())
    rc = s->upload(&unb, fs.unbounded.data(), fs.unbounded.size() * sizeof(uint32_t));
  if (rc == PBRT_OK && !fs.xforms.empty()) rc = s->upload(&xfs, fs.xforms.data(), fs.xforms.size() * sizeof(XfRec));
  if (rc == PBRT_OK && !fs.groups.empty()) rc = s->upload(&grps, fs.groups.data(), fs.groups.size() * sizeof(GroupRec));
  if (rc == PBRT_OK && !fs.csg.empty()) rc = s->upload(&csgs, fs.csg.data(), fs.csg.size() * sizeof(CsgRec));
  if (rc == PBRT_OK && !views.empty()) rc = s->upload(&mviews, views.data(), views.size() * sizeof(MeshView));
  if (rc == PBRT_OK && !shades.empty()) rc = s->upload(&mshades, shades.data(), shades.size() * sizeof(MeshShade));
  if (rc == PBRT_OK) rc = s->upload(&mats, fs.materials.data(), fs.materials.size() * sizeof(MatRec));
  if (rc == PBRT_OK && !fs.lights.empty()) rc = s->upload(&lights, fs.lights.data(), fs.lights.size() * sizeof(LightRec));
  if (rc == PBRT_OK && !fs.light_tris.empty())
    rc = s->upload(&ltris, fs.light_tris.data(), fs.light_tris.size() * sizeof(float));
  if (rc == PBRT_OK && !fs.light_cdf.empty())
    rc = s->upload(&lcdf, fs.light_cdf.data(), fs.light_cdf.size() * sizeof(float));
  if (rc != PBRT_OK) {
    pbrt_scene_destroy(s.release());
    return rc;
  }
  SceneView& v = s->view;
  v.top = (const float4*)top;
  v.top_node_count = uint32_t(fs.top.size());
  v.order = (const uint32_t*)order;
  v.unbounded = (const uint32_t*)unb;
  v.unbounded_count = uint32_t(fs.unbounded.size());
  v.objects = (const ObjRec*)objs;
  v.xforms = (const XfRec*)xfs;
  v.groups = (const GroupRec*)grps;
  v.csg = (const CsgRec*)csgs;
  v.meshes = (const MeshView*)mviews;
  v.shade = (const MeshShade*)mshades;
  v.materials = (const MatRec*)mats;
  v.lights = (const LightRec*)lights;
  v.light_count = uint32_t(fs.lights.size());
  v.light_tris = (const float*)ltris;
  v.light_cdf = (const float*)lcdf;
  v.has_csg = 0;
  for (const ObjRec& ob : fs.objects) v.has_csg |= ob.shape == kShapeCsg ? 1u : 0u;
  // The leaf the renderer answers in passes of its own: the largest untransformed mesh placed
  // directly in the top-level tree, of at least kDeferMinTriangles triangles.
  v.defer_leaf = kNoLeaf;
  uint64_t defer_tris = kDeferMinTriangles - 1;
  for (const uint32_t ref : fs.order) {
    if (ref & kGroupBit) continue;
    const ObjRec& ob = fs.objects[ref];
    if (ob.shape != kShapeMesh || ob.xf_count != 0) continue;
    const uint64_t nt = d->meshes[ob.mesh].triangle_count;
    if (nt > defer_tris) {
      defer_tris = nt;
      v.defer_leaf = ref;
    }
  }
  s->info.object_count = fs.primitive_count;
  s->info.device_bytes += s->extra_bytes;
  s->max_radiance = fs.max_radiance;
  s->has_dielectric = fs.has_dielectric;
  for (int a = 0; a < 3; ++a) {  // the bounded primitives' box (none: an empty box)
    s->bounds[a] = fs.top.empty() ? 0.0f : fs.top[0].bmin[a];
    s->bounds[3 + a] = fs.top.empty() ? 0.0f : fs.top[0].bmax[a];
  }
  s->single_mesh = fs.single_mesh;
  const int rc2 = c->cuda(cudaStreamSynchronize(c->stream), "scene upload");
  if (rc2 != PBRT_OK) {
    pbrt_scene_destroy(s.release());
    return rc2;
  }
  *out = s.release();
  return PBRT_OK;
}

// The meshes' BVHs built on the GPU (pbrt_scene_desc::device_build). Mesh arrays in device
// memory are copied to the host for the scene build's host part (validation of face
// materials, area-light triangles, the shading copies); `md` receives the description's
// meshes pointing at host memory.
int build_meshes_on_device(pbrt_ctx* c, const pbrt_scene_desc* d, std::vector<pbrt_mesh_desc>* md,
                           std::vector<std::vector<float>>* hv, std::vector<std::vector<uint32_t>>* hi,
                           std::vector<std::vector<uint32_t>>* hf, std::vector<MeshPrebuilt>* pre,
                           std::vector<DeviceMeshBuild>* builds) {
  const uint32_t n = d->mesh_count;
  md->assign(d->meshes, d->meshes + n);
  hv->resize(n);
  hi->resize(n);
  hf->resize(n);
  pre->resize(n);
  builds->resize(n);
  MeshBuildParams bp;
  bp.bins = d->bvh_bins ? int(d->bvh_bins) : 8;
  bp.max_leaf = d->bvh_max_leaf ? d->bvh_max_leaf : 1;
  cudaStream_t st = c->stream;
  for (uint32_t i = 0; i < n; ++i) {
    const pbrt_mesh_desc& m = d->meshes[i];
    if (!m.vertices || !m.indices || m.triangle_count == 0)
      return c->fail(PBRT_ERR_INVALID_ARGUMENT, "mesh " + std::to_string(i) + ": a TriangleMesh needs triangles");
    const size_t vb = size_t(m.vertex_count) * 3 * sizeof(float), ib = size_t(m.triangle_count) * 3 * sizeof(uint32_t);
    const bool vdev = mem_kind(m.vertices) == MemKind::Device, idev = mem_kind(m.indices) == MemKind::Device;
    float* dv = nullptr;
    uint32_t* di = nullptr;
    int rc = PBRT_OK;
    if (vdev) {
      dv = const_cast<float*>(m.vertices);
      (*hv)[i].resize(size_t(m.vertex_count) * 3);
      rc = c->cuda(cudaMemcpyAsync((*hv)[i].data(), m.vertices, vb, cudaMemcpyDeviceToHost, st), "cudaMemcpy(vertices)");
      (*md)[i].vertices = (*hv)[i].data();
    } else {
      rc = c->cuda(cudaMalloc(&dv, std::max<size_t>(vb, 4)), "cudaMalloc(build vertices)");
      if (rc == PBRT_OK) rc = c->cuda(cudaMemcpyAsync(dv, m.vertices, vb, cudaMemcpyHostToDevice, st), "cudaMemcpy");
    }
    if (rc == PBRT_OK && idev) {
      di = const_cast<uint32_t*>(m.indices);
      (*hi)[i].resize(size_t(m.triangle_count) * 3);
      rc = c->cuda(cudaMemcpyAsync((*hi)[i].data(), m.indices, ib, cudaMemcpyDeviceToHost, st), "cudaMemcpy(indices)");
      (*md)[i].indices = (*hi)[i].data();
    } else if (rc == PBRT_OK) {
      rc = c->cuda(cudaMalloc(&di, std::max<size_t>(ib, 4)), "cudaMalloc(build indices)");
      if (rc == PBRT_OK) rc = c->cuda(cudaMemcpyAsync(di, m.indices, ib, cudaMemcpyHostToDevice, st), "cudaMemcpy");
    }
    if (rc == PBRT_OK && m.face_materials && mem_kind(m.face_materials) == MemKind::Device) {
      (*hf)[i].resize(m.triangle_count);
      rc = c->cuda(cudaMemcpyAsync((*hf)[i].data(), m.face_materials, size_t(m.triangle_count) * 4,
                                   cudaMemcpyDeviceToHost, st),
                   "cudaMemcpy(face materials)");
      (*md)[i].face_materials = (*hf)[i].data();
    }
    std::string e;
    if (rc == PBRT_OK &&
        !build_mesh_bvh_device(dv, m.vertex_count, di, m.triangle_count, bp, st, c->sm_count, &(*builds)[i], &e))
      rc = c->fail(PBRT_ERR_INVALID_ARGUMENT, "mesh " + std::to_string(i) + ": " + e);
    if (!vdev) cudaFree(dv);
    if (!idev) cudaFree(di);
    if (rc != PBRT_OK) {
      for (DeviceMeshBuild& b : *builds) free_device_mesh_build(&b);
      return rc;
    }
    MeshPrebuilt& p = (*pre)[i];
    p.used = true;
    p.stats = (*builds)[i].stats;
    for (int a = 0; a < 3; ++a) {
      p.bounds_min[a] = (*builds)[i].bounds_min[a];
      p.bounds_max[a] = (*builds)[i].bounds_max[a];
    }
  }
  return c->cuda(cudaStreamSynchronize(st), "device BVH build");
}

int check_scene_desc(pbrt_ctx* c, const pbrt_scene_desc* d) {
  if (!d) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "scene description is NULL");
  if (d->object_count == 0) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "a scene needs at least one object");
  if (d->mesh_count && !d->meshes) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "meshes is NULL");
  if (!d->objects) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "objects is NULL");
  return PBRT_OK;
}

}  // namespace

extern "C" {

int pbrt_scene_create(pbrt_ctx* c, const pbrt_scene_desc* d, pbrt_scene** out) {
  if (!c || !d || !out) return PBRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  DeviceGuard g(c->device);
  PBRT_TRY(check_scene_desc(c, d));
  FlatScene fs;
  std::string e;
  if (d->device_build && d->mesh_count) {
    std::vector<pbrt_mesh_desc> md;
    std::vector<std::vector<float>> hv;
    std::vector<std::vector<uint32_t>> hi, hf;
    std::vector<MeshPrebuilt> pre;
    std::vector<DeviceMeshBuild> builds;
    PBRT_TRY(build_meshes_on_device(c, d, &md, &hv, &hi, &hf, &pre, &builds));
    pbrt_scene_desc d2 = *d;
    d2.meshes = md.data();
    int rc = PBRT_OK;
    if (!build_scene(d2, &fs, &e, &pre)) rc = c->fail(PBRT_ERR_INVALID_ARGUMENT, e);
    if (rc == PBRT_OK) rc = upload_scene(c, &d2, fs, out, &builds);
    for (DeviceMeshBuild& b : builds) free_device_mesh_build(&b);  // those not taken over
    return rc;
  }
  if (!build_scene(*d, &fs, &e)) return c->fail(PBRT_ERR_INVALID_ARGUMENT, e);
  return upload_scene(c, d, fs, out);
}

int pbrt_scene_create_many(pbrt_ctx* c, const pbrt_scene_desc* descs, uint32_t n, uint32_t threads,
                           pbrt_scene** out) {
  if (!c || !descs || !out) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(c->device);
  for (uint32_t i = 0; i < n; ++i) out[i] = nullptr;
  for (uint32_t i = 0; i < n; ++i) PBRT_TRY(check_scene_desc(c, descs + i));
  // GPU mesh builds first (device_build scenes), one scene after another on the context's stream
  struct DevParts {
    std::vector<pbrt_mesh_desc> md;
    std::vector<std::vector<float>> hv;
    std::vector<std::vector<uint32_t>> hi, hf;
    std::vector<MeshPrebuilt> pre;
    std::vector<DeviceMeshBuild> builds;
  };
  std::vector<DevParts> parts(n);
  std::vector<pbrt_scene_desc> d2(descs, descs + n);
  auto free_builds = [&]() {
    for (DevParts& p : parts)
      for (DeviceMeshBuild& b : p.builds) free_device_mesh_build(&b);
  };
  for (uint32_t i = 0; i < n; ++i) {
    if (!descs[i].device_build || !descs[i].mesh_count) continue;
    DevParts& p = parts[i];
    const int rc = build_meshes_on_device(c, descs + i, &p.md, &p.hv, &p.hi, &p.hf, &p.pre, &p.builds);
    if (rc != PBRT_OK) {
      free_builds();
      return rc;
    }
    d2[i].meshes = p.md.data();
  }
  // host builds on a pool of threads (no device calls), then uploads in order
  std::vector<FlatScene> flat(n);
  std::vector<std::string> errs(n);
  std::vector<char> ok(n, 0);
  std::atomic<uint32_t> next{0};
  unsigned T = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
  T = std::min<unsigned>(T, n);
  auto work = [&]() {
    for (uint32_t i = next++; i < n; i = next++)
      ok[i] = build_scene(d2[i], &flat[i], &errs[i], parts[i].pre.empty() ? nullptr : &parts[i].pre) ? 1 : 0;
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < T; ++t) pool.emplace_back(work);
  work();
  for (std::thread& t : pool) t.join();
  for (uint32_t i = 0; i < n; ++i)
    if (!ok[i]) {
      free_builds();
      return c->fail(PBRT_ERR_INVALID_ARGUMENT, "scene " + std::to_string(i) + ": " + errs[i]);
    }
  for (uint32_t i = 0; i < n; ++i) {
    const int rc = upload_scene(c, &d2[i], flat[i], out + i, parts[i].builds.empty() ? nullptr : &parts[i].builds);
    if (rc != PBRT_OK) {
      for (uint32_t j = 0; j < i; ++j) {
        pbrt_scene_destroy(out[j]);
        out[j] = nullptr;
      }
      free_builds();
      return rc;
    }
    FlatScene().meshes.swap(flat[i].meshes);  // release host copies as we go
  }
  free_builds();  // anything not taken over
  return PBRT_OK;
}

void pbrt_scene_destroy(pbrt_scene* s) {
  if (!s) return;
  DeviceGuard g(s->ctx->device);
  cudaStreamSynchronize(s->ctx->work_stream());
  for (auto& m : s->meshes) free_mesh(m);
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

int pbrt_mesh_bvh_build_device(pbrt_ctx* c, const pbrt_mesh_desc* md, uint32_t bins, uint32_t max_leaf, void* nodes,
                               uint64_t node_capacity, uint32_t* tri_order, uint64_t* node_count, float* build_ms) {
  if (!c || !md || !node_count) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(c->device);
  pbrt_scene_desc d{};
  d.meshes = md;
  d.mesh_count = 1;
  d.bvh_bins = bins;
  d.bvh_max_leaf = max_leaf;
  std::vector<pbrt_mesh_desc> m2;
  std::vector<std::vector<float>> hv;
  std::vector<std::vector<uint32_t>> hi, hf;
  std::vector<MeshPrebuilt> pre;
  std::vector<DeviceMeshBuild> b;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (build_ms) {
    PBRT_TRY(c->cuda(cudaEventCreate(&e0), "cudaEventCreate"));
    PBRT_TRY(c->cuda(cudaEventCreate(&e1), "cudaEventCreate"));
    PBRT_TRY(c->cuda(cudaEventRecord(e0, c->stream), "cudaEventRecord"));
  }
  int rc = build_meshes_on_device(c, &d, &m2, &hv, &hi, &hf, &pre, &b);
  if (rc == PBRT_OK && build_ms) {
    rc = c->cuda(cudaEventRecord(e1, c->stream), "cudaEventRecord");
    if (rc == PBRT_OK) rc = c->cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
    if (rc == PBRT_OK) rc = c->cuda(cudaEventElapsedTime(build_ms, e0, e1), "cudaEventElapsedTime");
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc != PBRT_OK) return rc;
  DeviceMeshBuild& r = b[0];
  *node_count = r.node_slots;  // 32-byte records, the padding slot included (as the host variant)
  if (nodes && node_capacity < r.node_slots) rc = PBRT_ERR_CAPACITY;
  if (rc == PBRT_OK && nodes)
    rc = c->cuda(cudaMemcpy(nodes, r.nodes, r.node_slots * sizeof(GpuNode), cudaMemcpyDeviceToHost), "cudaMemcpy(nodes)");
  if (rc == PBRT_OK && nodes && tri_order)
    rc = c->cuda(cudaMemcpy(tri_order, r.tri_index, size_t(md->triangle_count) * 4, cudaMemcpyDeviceToHost),
                 "cudaMemcpy(order)");
  free_device_mesh_build(&r);
  return rc;
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

// Loader::load_scene (src/loader.rs:29-45): the scene file parsed, then built like any scene.
int pbrt_scene_load(pbrt_ctx* c, const char* text, const pbrt_stage_options* options, pbrt_scene** scene,
                    pbrt_camera_desc* camera) {
  if (!c || !scene) return PBRT_ERR_INVALID_ARGUMENT;
  *scene = nullptr;
  char err[512];
  pbrt_stage* st = nullptr;
  const int rc = pbrt_stage_parse(text, options, &st, err, sizeof(err));
  if (rc != PBRT_OK) return c->fail(rc, std::string("scene file: ") + err);
  pbrt_scene_desc d;
  pbrt_stage_describe(st, &d, camera, nullptr);
  const int rc2 = pbrt_scene_create(c, &d, scene);
  pbrt_stage_destroy(st);
  return rc2;
}

int pbrt_scene_get_info(const pbrt_scene* s, pbrt_scene_info* info) {
  if (!s || !info) return PBRT_ERR_INVALID_ARGUMENT;
  *info = s->info;
  return PBRT_OK;
}

}  // extern "C"

namespace {

// Runs the nearest-hit (or, with occ != NULL, any-hit) kernel over host or device buffers.
// stats with scene_stats: the scene accelerator's counters (any scene); stats alone: the
// mesh traversal's (scenes of one untransformed mesh).
int trace_impl(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim, float* t, uint32_t* obj, uint8_t* occ,
               uint64_t* stats, bool scene_stats = false) {
  if (!s) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = s->ctx;
  DeviceGuard g(c->device);
  if (n == 0) return PBRT_OK;
  if (!rays || (!occ && (!prim || !t))) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "ray or result buffer is NULL");
  if (stats && !scene_stats && s->single_mesh < 0)
    return c->fail(PBRT_ERR_UNSUPPORTED, "work counters are reported for scenes made of one untransformed mesh");
  const bool one_mesh = s->single_mesh >= 0 && !scene_stats;
  const MeshView mv = one_mesh ? s->meshes[s->single_mesh].view : MeshView{};
  // Nearest hit / any hit of one chunk of `m` rays (planes `stride` apart) on `st`.
  auto launch = [&](const float* r, uint64_t stride, uint64_t m, uint32_t* p, float* tt, uint32_t* ob, uint8_t* oc,
                    unsigned long long* cnt, uint32_t* queue, unsigned long long* qc, float4* rec,
                    cudaStream_t st, const DenseScratch* dense = nullptr) -> cudaError_t {
    if (!one_mesh)
      return oc ? launch_scene_any(s->view, r, stride, m, oc, cnt, c->d_err, c->sm_count, st)
                : launch_scene_closest(s->view, r, stride, m, p, tt, ob, cnt, c->d_err, c->sm_count, st);
    if (oc) return launch_mesh_any(mv, r, stride, m, oc, c->d_err, c->sm_count, st);
    if (c->persistent && !cnt)
      return launch_mesh_closest_persistent(mv, r, stride, m, p, tt, ob, queue, qc, c->d_err, c->sm_count, st, rec,
                                            dense);
    return launch_mesh_closest(mv, r, stride, m, p, tt, ob, cnt, c->d_err, c->sm_count, st);
  };

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
    if (one_mesh && !occ && c->persistent && !counters) {
      // Chunks of at most kDevChunk rays bound the survivor queue (scratch) to 64 MiB.
      PBRT_TRY(ensure_queue(c));
      for (uint64_t base = 0; base < n; base += kDevChunk) {
        const uint64_t m = std::min<uint64_t>(kDevChunk, n - base);
        PBRT_TRY(c->cuda(launch(rays + base, n, m, prim + base, t + base, obj ? obj + base : nullptr, nullptr, nullptr,
                                c->queue, c->d_counters + 4, c->queue_rec, st, &c->queue_dense),
                         "kernel launch"));
      }
    } else {
      PBRT_TRY(c->cuda(launch(rays, n, n, prim, t, obj, occ, counters, nullptr, nullptr, nullptr, st), "kernel launch"));
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
  // kernel of chunk k). With 1M-ray chunks and one 2D copy per chunk a 16M-ray call takes the
  // time of its bare copies (512 MiB in, 128 MiB out concurrently: 10.3 ms on PCIe 5).
  PBRT_TRY(ensure_slots(c));
  if (c->user) PBRT_TRY(c->cuda(cudaStreamSynchronize(c->user), "cudaStreamSynchronize"));
  if (stats)
    PBRT_TRY(c->cuda(cudaStreamSynchronize(c->work_stream()), "cudaStreamSynchronize"));
  uint64_t chunk = 0;
  for (uint64_t base = 0; base < n; base += kSlotRays, ++chunk) {
    Slot& sl = c->slots[chunk % kSlots];
    const uint64_t m = std::min<uint64_t>(kSlotRays, n - base);
    // the chunk's eight planes as one 2D copy (rows = planes): one DMA job instead of eight
    PBRT_TRY(c->cuda(cudaMemcpy2DAsync(sl.rays, kSlotRays * sizeof(float), rays + base, n * sizeof(float),
                                       m * sizeof(float), 8, cudaMemcpyHostToDevice, sl.s),
                     "cudaMemcpy2DAsync(rays)"));
    PBRT_TRY(c->cuda(launch(sl.rays, kSlotRays, m, sl.prim, sl.t, obj ? sl.obj : nullptr, occ ? sl.occ : nullptr,
                            counters, sl.queue, sl.fetch, sl.rec, sl.s, &sl.dense),
                     "kernel launch"));
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
// device-buffer path of pbrt_trace_closest, with their scratch in a static __device__ array
// whose address the context looked up when it was created.
int pbrt_trace_closest_noalloc(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim_id, float* t) {
  if (!s) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = s->ctx;
  if (n == 0) return PBRT_OK;  // as pbrt_trace_closest: nothing to do, whatever the scene
  DeviceGuard g(c->device);
  if (n > kNoAllocMaxRays)
    return c->fail(PBRT_ERR_CAPACITY, "pbrt_trace_closest_noalloc: n = " + std::to_string(n) +
                                          " exceeds its fixed scratch capacity of " + std::to_string(kNoAllocMaxRays) +
                                          " rays; split the batch or use pbrt_trace_closest");
  cudaStream_t st = c->work_stream();
  // The call waits for its results (it reads the error word back), which a stream under
  // capture cannot do: refuse before any other CUDA call, so the caller's capture survives.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PBRT_TRY(c->cuda(cudaStreamIsCapturing(st, &cap), "cudaStreamIsCapturing"));
  if (cap != cudaStreamCaptureStatusNone)
    return c->fail(PBRT_ERR_UNSUPPORTED,
                   "pbrt_trace_closest_noalloc waits for its results and cannot run on a stream being captured");
  if (!rays || !prim_id || !t) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "ray or result buffer is NULL");
  if (mem_kind(rays) != MemKind::Device || mem_kind(prim_id) != MemKind::Device || mem_kind(t) != MemKind::Device)
    return c->fail(PBRT_ERR_INVALID_ARGUMENT,
                   "pbrt_trace_closest_noalloc takes device buffers only (host buffers need staging memory)");
  if (s->single_mesh < 0)
    return c->fail(PBRT_ERR_UNSUPPORTED, "pbrt_trace_closest_noalloc traces scenes made of one untransformed mesh");
  const MeshView& mv = s->meshes[s->single_mesh].view;
  uint32_t* scratch = c->noalloc_scratch;
  PBRT_TRY(c->cuda(launch_mesh_closest_noalloc(mv, rays, n, prim_id, t, scratch, c->sm_count, st),
                   "pbrt_trace_closest_noalloc"));
  uint32_t h = 0;  // the error word, read back on the same stream (no legacy-stream wait)
  PBRT_TRY(c->cuda(cudaMemcpyAsync(&h, scratch + 4, sizeof(h), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync"));
  PBRT_TRY(c->cuda(cudaStreamSynchronize(st), "kernel execution"));
  if (h & kErrStack) return c->fail(PBRT_ERR_CAPACITY, "traversal stack capacity exceeded");
  if (h) return c->fail(PBRT_ERR_DEVICE_BUDGET, "a traversal exceeded its iteration budget (malformed tree)");
  return PBRT_OK;
}

int pbrt_trace_any(pbrt_scene* s, const float* rays, uint64_t n, uint8_t* occluded) {
  if (!occluded) return s ? s->ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "occluded is NULL") : PBRT_ERR_INVALID_ARGUMENT;
  return trace_impl(s, rays, n, nullptr, nullptr, nullptr, occluded, nullptr);
}

int pbrt_trace_closest_counted(pbrt_scene* s, const float* rays, uint64_t n, uint32_t* prim_id, float* t,
                               uint32_t* object_id, uint64_t* stats) {
  if (!stats) return s ? s->ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "stats is NULL") : PBRT_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 3; ++k) stats[k] = 0;
  return trace_impl(s, rays, n, prim_id, t, object_id, nullptr, stats, true);
}

int pbrt_trace_any_counted(pbrt_scene* s, const float* rays, uint64_t n, uint8_t* occluded, uint64_t* stats) {
  if (!occluded || !stats)
    return s ? s->ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "occluded or stats is NULL") : PBRT_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 3; ++k) stats[k] = 0;
  return trace_impl(s, rays, n, nullptr, nullptr, nullptr, occluded, stats, true);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Rendering
// ---------------------------------------------------------------------------------------
int pbrt::api::ensure_wave(pbrt_ctx* c, WaveAlloc* wa, uint32_t cap) {
  if (wa->capacity >= cap) return PBRT_OK;
  cudaFree(wa->block);
  wa->block = nullptr;
  wa->capacity = 0;
  const size_t n = cap;
  // 4-byte arrays: 6 ray + 3 beta + 3 L + pixel + scene + flags + ht + hobj + hprim + qa + qb + 11 shadow
  // = 32 words, plus the 8-byte rng state, plus 4 counters.
  const size_t bytes = n * (32 * 4 + 8) + 64;
  PBRT_TRY(c->cuda(cudaMalloc(&wa->block, bytes), "cudaMalloc(wave state)"));
  char* p = static_cast<char*>(wa->block);
  auto f32 = [&]() { float* r = reinterpret_cast<float*>(p); p += n * 4; return r; };
  auto u32 = [&]() { uint32_t* r = reinterpret_cast<uint32_t*>(p); p += n * 4; return r; };
  WaveBuffers& w = wa->w;
  w.rng = reinterpret_cast<unsigned long long*>(p);
  p += n * 8;
  w.ox = f32(); w.oy = f32(); w.oz = f32(); w.dx = f32(); w.dy = f32(); w.dz = f32();
  w.br = f32(); w.bg = f32(); w.bb = f32(); w.lr = f32(); w.lg = f32(); w.lb = f32();
  w.pixel = u32(); w.scene = u32(); w.flags = u32(); w.ht = f32(); w.hobj = u32(); w.hprim = u32(); w.qa = u32(); w.qb = u32();
  w.s_path = u32(); w.s_ox = f32(); w.s_oy = f32(); w.s_oz = f32(); w.s_dx = f32(); w.s_dy = f32(); w.s_dz = f32();
  w.s_tmax = f32(); w.s_cr = f32(); w.s_cg = f32(); w.s_cb = f32();
  w.counts = reinterpret_cast<uint32_t*>(p);
  wa->capacity = cap;
  return PBRT_OK;
}

int pbrt::api::check_render_params(pbrt_ctx* c, const pbrt_render_params* p, bool allow_no_samples) {
  const pbrt_camera_desc& cd = p->camera;
  if (cd.width == 0 || cd.height == 0) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "empty image");
  if (p->spp == 0 && !allow_no_samples) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "spp must be >= 1");
  if (p->max_depth == 0 || p->max_depth > 0xFFFF)
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "max_depth must be in [1, 65535]");
  if (p->integrator > PBRT_INTEGRATOR_NORMAL) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "unknown integrator");
  if (!(cd.fov > 0.f) || !(cd.fov < 3.14159265f) || !(cd.far > cd.near))
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "bad camera");
  if (cd.thin_lens && (!(cd.lens_radius >= 0.f) || !std::isfinite(cd.lens_radius) || !std::isfinite(cd.focal_distance)))
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "bad thin lens");
  if (uint64_t(cd.width) * cd.height > 0xFFFFFFFFull) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "image too large");
  if (p->pixel_stride > cd.width || p->pixel_stride > cd.height)
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "pixel_stride exceeds the image");
  return PBRT_OK;
}

RenderSettings pbrt::api::settings_of(pbrt_ctx* c, const pbrt_render_params* p) {
  RenderSettings rs;
  rs.stats = c->d_counters + 8;
  rs.shape = c->shape;
  rs.max_depth = p->max_depth;
  rs.rr_start = p->integrator == PBRT_INTEGRATOR_PATH ? p->rr_start : 0u;
  rs.sample_offset = p->sample_offset;
  rs.integrator = p->integrator;
  rs.seed = p->seed;
  rs.stride = p->pixel_stride > 1 ? p->pixel_stride : 1u;
  rs.film_w = (p->camera.width + rs.stride - 1) / rs.stride;
  return rs;
}

// Film pixels of a render: the image's, or the strided subset's.
uint64_t pbrt::api::film_pixels(const pbrt_render_params* p, const RenderSettings& rs) {
  return uint64_t(rs.film_w) * ((p->camera.height + rs.stride - 1) / rs.stride);
}

namespace {

// Training paths of the cached render go this many hits past the render's cache hit before
// they end into the cache themselves.
constexpr uint32_t kTrainTail = 3;

// Concurrent branches of one pbrt_render: the frame's paths split into this many contiguous
// parts, each a chain of waves on its own stream with its own wave buffers, so that one
// part's per-bounce kernel tails overlap another part's work. PBRT_RENDER_BRANCHES (1..8)
// overrides it for measurements; films do not depend on it.
static_assert(pbrt_cache::kBranchSlots + 1 >= kMaxBatchBranches, "a cached frame's branches need query buffers");

uint32_t render_branches(uint64_t total) {
  static const uint32_t v = [] {
    const char* e = std::getenv("PBRT_RENDER_BRANCHES");
    const int k = e ? std::atoi(e) : int(kDefaultRenderBranches);
    return uint32_t(k >= 1 && k <= int(kMaxBatchBranches) ? k : kDefaultRenderBranches);
  }();
  return uint32_t(std::min<uint64_t>(v, std::max<uint64_t>(1, total / 1024)));
}

unsigned long long host_mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

}  // namespace

extern "C" {

int pbrt_render(pbrt_scene* s, const pbrt_render_params* p, double* film) {
  if (!s) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = s->ctx;
  DeviceGuard g(c->device);
  if (!p || !film) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "params or film is NULL");
  PBRT_TRY(check_render_params(c, p, false));
  const pbrt_camera_desc& cd = p->camera;
  const CameraRec cam = build_camera(cd);
  const RenderSettings rs = settings_of(c, p);
  const uint64_t npix = film_pixels(p, rs);
  const uint64_t total = npix * p->spp;

  // the paths in `nb` contiguous parts [j * part, (j + 1) * part), part j on branch j
  const uint32_t nb = render_branches(total);
  const uint64_t part = (total + nb - 1) / nb;
  const uint32_t wave = uint32_t(std::min<uint64_t>(part, c->wave_paths));
  PBRT_TRY(ensure_wave(c, &c->waves, wave));
  for (uint32_t j = 1; j < nb; ++j) {
    PBRT_TRY(ensure_wave(c, &c->branch_waves[j - 1], wave));
    if (!c->branch_st[j])
      PBRT_TRY(c->cuda(cudaStreamCreateWithFlags(&c->branch_st[j], cudaStreamNonBlocking), "cudaStreamCreate"));
    if (!c->branch_join[j])
      PBRT_TRY(c->cuda(cudaEventCreateWithFlags(&c->branch_join[j], cudaEventDisableTiming), "cudaEventCreate"));
  }
  if (nb > 1 && !c->branch_fork)
    PBRT_TRY(c->cuda(cudaEventCreateWithFlags(&c->branch_fork, cudaEventDisableTiming), "cudaEventCreate"));
  cudaStream_t st = c->work_stream();
  const size_t film_n = size_t(npix) * 3;
  double* dfilm = film;
  const bool host_film = mem_kind(film) != MemKind::Device;
  if (host_film) PBRT_TRY(c->cuda(cudaMalloc(&dfilm, film_n * sizeof(double)), "cudaMalloc(film)"));
  int rc = c->cuda(cudaMemsetAsync(dfilm, 0, film_n * sizeof(double), st), "cudaMemset(film)");
  if (rc == PBRT_OK) rc = c->cuda(cudaMemsetAsync(rs.stats, 0, 3 * sizeof(unsigned long long), st), "cudaMemset");
  if (rc == PBRT_OK && nb > 1) rc = c->cuda(cudaEventRecord(c->branch_fork, st), "cudaEventRecord");
  for (uint32_t j = 1; j < nb && rc == PBRT_OK; ++j)
    rc = c->cuda(cudaStreamWaitEvent(c->branch_st[j], c->branch_fork, 0), "cudaStreamWaitEvent");
  for (uint32_t j = 0; j < nb && rc == PBRT_OK; ++j) {
    cudaStream_t bs = j ? c->branch_st[j] : st;
    const WaveBuffers& bw = j ? c->branch_waves[j - 1].w : c->waves.w;
    const uint64_t end = std::min<uint64_t>(total, (j + 1) * part);
    for (uint64_t base = j * part; base < end && rc == PBRT_OK; base += wave) {
      const uint32_t n = uint32_t(std::min<uint64_t>(wave, end - base));
      rc = c->cuda(render_wave(s->view, bw, cam, base, n, uint32_t(npix), rs, dfilm, c->d_err, c->sm_count, bs),
                   "render");
    }
  }
  // the branches join `st` again (also after a failed launch, so that no branch is left behind)
  for (uint32_t j = 1; j < nb; ++j) {
    const int jr = c->cuda(cudaEventRecord(c->branch_join[j], c->branch_st[j]), "cudaEventRecord");
    if (jr == PBRT_OK) cudaStreamWaitEvent(st, c->branch_join[j], 0);
    if (rc == PBRT_OK) rc = jr;
  }
  if (rc == PBRT_OK) rc = c->cuda(scale_film(dfilm, film_n, 1.0 / double(p->spp), c->sm_count, st), "render");
  if (host_film) {
    if (rc == PBRT_OK)
      rc = c->cuda(cudaMemcpyAsync(film, dfilm, film_n * sizeof(double), cudaMemcpyDeviceToHost, st), "cudaMemcpy(film)");
    if (rc == PBRT_OK) rc = check_device_error(c, st);
    cudaStreamSynchronize(st);
    cudaFree(dfilm);
    return rc;
  }
  PBRT_TRY(rc);
  if (c->user) return PBRT_OK;
  return check_device_error(c, st);
}

int pbrt_render_cached(pbrt_scene* s, pbrt_cache* k, const pbrt_render_params* p, uint32_t train_rounds,
                       double* film) {
  if (!s || !k) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = s->ctx;
  DeviceGuard g(c->device);
  if (k->ctx != c) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "the cache belongs to another context");
  if (!p) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "params is NULL");
  PBRT_TRY(check_render_params(c, p, true));
  if (p->spp && !film) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "film is NULL");
  if (p->integrator != PBRT_INTEGRATOR_PATH)
    return c->fail(PBRT_ERR_UNSUPPORTED, "the radiance cache ends path-integrator paths only");
  pbrt_cache_params& cp = k->params;
  if (cp.scene_min[0] == cp.scene_max[0] && cp.scene_min[1] == cp.scene_max[1] && cp.scene_min[2] == cp.scene_max[2])
    for (int a = 0; a < 3; ++a) {
      cp.scene_min[a] = s->bounds[a];
      cp.scene_max[a] = s->bounds[3 + a];
    }
  const pbrt_camera_desc& cd = p->camera;
  const CameraRec cam = build_camera(cd);
  const RenderSettings rs = settings_of(c, p);
  const uint64_t npix = film_pixels(p, rs);
  const uint64_t total = npix * p->spp;
  const uint32_t train_paths = std::max(128u, cp.train_samples / 4);
  const uint32_t steps = cp.train_steps;
  const uint32_t batch = std::max(128u, cp.train_samples / steps);
  const uint32_t wave = uint32_t(std::min<uint64_t>(total, c->wave_paths));

  WaveAlloc& wa = c->waves;
  PBRT_TRY(ensure_wave(c, &wa, std::max(wave, train_paths)));
  // one query per path at most: the render wave's and the training paths'
  PBRT_TRY(k->ensure_render_buffers(std::max(wave, train_paths), cp.train_samples, batch));
  cudaStream_t st = c->work_stream();
  const CacheWave& cw = k->cw;
  PBRT_TRY(c->cuda(cudaMemsetAsync(rs.stats, 0, 3 * sizeof(unsigned long long), st), "cudaMemset"));

  // A call that trains and renders runs its rounds beside the frame: the rounds on the
  // context's side stream with their own wave, the frame on `st` with its own query buffers,
  // reading a snapshot of the weights the call started with. The rounds' few thousand paths
  // leave most of the GPU idle; this way the frame's work fills it.
  const bool beside = train_rounds > 0 && p->spp > 0;
  cudaStream_t ts = st;            // the training rounds' stream
  WaveAlloc* twa = &wa;            // and their wave
  mlp::Net fnet{k->wfwd, k->wbwd};  // the weights the frame reads
  const CacheWave* fcw = &cw;      // and its query buffers
  if (beside) {
    if (!c->side) PBRT_TRY(c->cuda(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking), "cudaStreamCreate"));
    if (!c->fork) PBRT_TRY(c->cuda(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming), "cudaEventCreate"));
    if (!c->join) PBRT_TRY(c->cuda(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming), "cudaEventCreate"));
    twa = &c->train_waves;
    PBRT_TRY(ensure_wave(c, twa, train_paths));
    PBRT_TRY(k->ensure_frame_buffers(wave));
    PBRT_TRY(c->cuda(cudaMemcpyAsync(k->wsnap, k->wfwd, mlp::kParams * 2, cudaMemcpyDeviceToDevice, st),
                     "cudaMemcpy(weight snapshot)"));
    PBRT_TRY(c->cuda(cudaEventRecord(c->fork, st), "cudaEventRecord"));
    PBRT_TRY(c->cuda(cudaStreamWaitEvent(c->side, c->fork, 0), "cudaStreamWaitEvent"));
    ts = c->side;
    fnet.wpk_fwd = k->wsnap;
    fcw = &k->fcw;
  }

  // Online training. Training paths start at random pixels, go kTrainTail hits past the
  // render's cache hit and end into the cache there; their earlier Lambertian and metal
  // vertices become training samples. No host synchronisation: counts stay on the device.
  const uint32_t term_hit = cp.terminate_bounce + 1;
  const uint32_t tail_hit = term_hit + kTrainTail;
  const mlp::Net net{k->wfwd, k->wbwd};
  const mlp::Bounds nb = k->bounds();
  int trc = PBRT_OK;
  {
    auto train = [&]() -> int {
      for (uint32_t r = 0; r < train_rounds; ++r) {
        RenderSettings tr = rs;
        tr.cache_mode = kCacheRecord;
        tr.term_hit = tail_hit;
        tr.random_pixels = 1;
        tr.sample_offset = 0;
        tr.seed = host_mix64(p->seed ^ host_mix64(0x747261696e696e67ULL + k->rounds));
        if (!s->has_dielectric) tr.loop_depth = std::min(rs.max_depth, tail_hit);
        PBRT_TRY(c->cuda(cudaMemsetAsync(cw.counts, 0, 3 * sizeof(uint32_t), ts), "cudaMemset(cache counts)"));
        PBRT_TRY(c->cuda(trace_wave(s->view, twa->w, cw, cam, 0, train_paths, uint32_t(npix), tr, c->d_err, c->sm_count, ts),
                         "cache training paths"));
        PBRT_TRY(c->cuda(mlp::launch_infer_dev(net, nb, cw.qrec, cw.counts, train_paths, cw.qout, c->d_err, c->sm_count,
                                               ts),
                         "cache training tails"));
        PBRT_TRY(c->cuda(apply_cache(twa->w, cw, train_paths, s->max_radiance, c->sm_count, ts), "cache training tails"));
        for (uint32_t step = 0; step < steps; ++step) {
          PBRT_TRY(c->cuda(train_batch(twa->w, cw, batch, step, tr.seed, s->max_radiance, k->brec, k->btgt, c->sm_count, ts),
                           "cache training batch"));
          PBRT_TRY(k->gradient_device(k->brec, k->btgt, batch, ts));
          PBRT_TRY(k->adam_device(ts, cw.counts + 2));
        }
        ++k->rounds;
      }
      return PBRT_OK;
    };
    trc = train();
  }
  if (beside) {  // the call ends when its rounds have: `st` waits for them at the end
    const int jr = c->cuda(cudaEventRecord(c->join, c->side), "cudaEventRecord");
    if (trc == PBRT_OK) trc = jr;
  }
  if (trc != PBRT_OK) {
    if (beside) cudaStreamWaitEvent(st, c->join, 0);
    return trc;
  }
  if (p->spp == 0) {
    if (c->user) return PBRT_OK;
    return check_device_error(c, st);
  }

  // rendering: paths end into the cache at hit terminate_bounce + 1
  RenderSettings qr = rs;
  qr.cache_mode = kCacheQuery;
  qr.term_hit = term_hit;
  if (!s->has_dielectric) qr.loop_depth = std::min(rs.max_depth, term_hit);
  const size_t film_n = size_t(npix) * 3;
  double* dfilm = film;
  const bool host_film = mem_kind(film) != MemKind::Device;
  if (host_film) PBRT_TRY(c->cuda(cudaMalloc(&dfilm, film_n * sizeof(double)), "cudaMalloc(film)"));
  // the frame's paths in `nbr` contiguous parts on concurrent branches, as pbrt_render's;
  // branch j >= 1 has its own wave buffers and query buffers
  const uint32_t nbr = render_branches(total);
  const uint64_t part = (total + nbr - 1) / nbr;
  const uint32_t fwave = uint32_t(std::min<uint64_t>(part, wave));
  int rc = PBRT_OK;
  for (uint32_t j = 1; j < nbr && rc == PBRT_OK; ++j) {
    rc = ensure_wave(c, &c->branch_waves[j - 1], fwave);
    if (rc == PBRT_OK) rc = k->ensure_branch_buffers(j - 1, fwave);
    if (rc == PBRT_OK && !c->branch_st[j])
      rc = c->cuda(cudaStreamCreateWithFlags(&c->branch_st[j], cudaStreamNonBlocking), "cudaStreamCreate");
    if (rc == PBRT_OK && !c->branch_join[j])
      rc = c->cuda(cudaEventCreateWithFlags(&c->branch_join[j], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (rc == PBRT_OK && nbr > 1 && !c->branch_fork)
    rc = c->cuda(cudaEventCreateWithFlags(&c->branch_fork, cudaEventDisableTiming), "cudaEventCreate");
  if (rc != PBRT_OK) {
    if (beside) cudaStreamWaitEvent(st, c->join, 0);
    if (host_film) cudaFree(dfilm);
    return rc;
  }
  rc = c->cuda(cudaMemsetAsync(dfilm, 0, film_n * sizeof(double), st), "cudaMemset(film)");
  if (rc == PBRT_OK && nbr > 1) rc = c->cuda(cudaEventRecord(c->branch_fork, st), "cudaEventRecord");
  for (uint32_t j = 1; j < nbr && rc == PBRT_OK; ++j)
    rc = c->cuda(cudaStreamWaitEvent(c->branch_st[j], c->branch_fork, 0), "cudaStreamWaitEvent");
  for (uint32_t j = 0; j < nbr && rc == PBRT_OK; ++j) {
    cudaStream_t bs = j ? c->branch_st[j] : st;
    const WaveBuffers& bw = j ? c->branch_waves[j - 1].w : wa.w;
    const CacheWave& q = j ? k->bcw[j - 1] : *fcw;
    const uint64_t end = std::min<uint64_t>(total, (j + 1) * part);
    for (uint64_t base = j * part; base < end && rc == PBRT_OK; base += fwave) {
      const uint32_t n = uint32_t(std::min<uint64_t>(fwave, end - base));
      rc = c->cuda(cudaMemsetAsync(q.counts, 0, sizeof(uint32_t), bs), "cudaMemset(cache counts)");
      if (rc == PBRT_OK)
        rc = c->cuda(trace_wave(s->view, bw, q, cam, base, n, uint32_t(npix), qr, c->d_err, c->sm_count, bs),
                     "cached render");
      if (rc == PBRT_OK)
        rc = c->cuda(mlp::launch_infer_dev(fnet, nb, q.qrec, q.counts, n, q.qout, c->d_err, c->sm_count, bs),
                     "cache query");
      if (rc == PBRT_OK) rc = c->cuda(apply_cache(bw, q, n, s->max_radiance, c->sm_count, bs), "cache apply");
      if (rc == PBRT_OK) rc = c->cuda(accumulate_wave(bw, n, dfilm, cd.width, qr, c->sm_count, bs), "cached render");
    }
  }
  for (uint32_t j = 1; j < nbr; ++j) {  // the branches join `st` again
    const int jr = c->cuda(cudaEventRecord(c->branch_join[j], c->branch_st[j]), "cudaEventRecord");
    if (jr == PBRT_OK) cudaStreamWaitEvent(st, c->branch_join[j], 0);
    if (rc == PBRT_OK) rc = jr;
  }
  if (rc == PBRT_OK) rc = c->cuda(scale_film(dfilm, film_n, 1.0 / double(p->spp), c->sm_count, st), "render");
  if (beside) {
    const int jr = c->cuda(cudaStreamWaitEvent(st, c->join, 0), "cudaStreamWaitEvent");
    if (rc == PBRT_OK) rc = jr;
  }
  if (host_film) {
    if (rc == PBRT_OK)
      rc = c->cuda(cudaMemcpyAsync(film, dfilm, film_n * sizeof(double), cudaMemcpyDeviceToHost, st), "cudaMemcpy(film)");
    if (rc == PBRT_OK) rc = check_device_error(c, st);
    cudaStreamSynchronize(st);
    cudaFree(dfilm);
    return rc;
  }
  PBRT_TRY(rc);
  if (c->user) return PBRT_OK;
  return check_device_error(c, st);
}

int pbrt_ctx_set_tuning(pbrt_ctx* c, const pbrt_tuning* t) {
  if (!c) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_tuning d{};
  if (t) d = *t;
  LaunchShape sh;
  const uint32_t wave = d.wave_paths ? d.wave_paths : (1u << 26);
  if (d.trace_threads) sh.trace_threads = d.trace_threads;
  if (d.trace_blocks_per_sm) sh.trace_blocks_per_sm = d.trace_blocks_per_sm;
  if (d.shade_threads) sh.shade_threads = d.shade_threads;
  if (d.shade_blocks_per_sm) sh.shade_blocks_per_sm = d.shade_blocks_per_sm;
  auto bad_threads = [](uint32_t x) { return x < 32 || x > 256 || x % 32 != 0; };
  auto bad_blocks = [](uint32_t x) { return x < 1 || x > 64; };
  if (bad_threads(sh.trace_threads) || bad_threads(sh.shade_threads))
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "threads per block must be a multiple of 32 in [32, 256]");
  if (bad_blocks(sh.trace_blocks_per_sm) || bad_blocks(sh.shade_blocks_per_sm))
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "blocks per SM must be in [1, 64]");
  if (wave < 1024 || wave > (1u << 26)) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "wave_paths must be in [1024, 2^26]");
  c->shape = sh;
  c->wave_paths = wave;
  return PBRT_OK;
}

int pbrt_ctx_get_tuning(pbrt_ctx* c, pbrt_tuning* t) {
  if (!c || !t) return PBRT_ERR_INVALID_ARGUMENT;
  t->wave_paths = c->wave_paths;
  t->trace_threads = c->shape.trace_threads;
  t->trace_blocks_per_sm = c->shape.trace_blocks_per_sm;
  t->shade_threads = c->shape.shade_threads;
  t->shade_blocks_per_sm = c->shape.shade_blocks_per_sm;
  return PBRT_OK;
}

int pbrt_ctx_render_stats(pbrt_ctx* c, uint64_t* stats) {
  if (!c || !stats) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(c->device);
  PBRT_TRY(c->cuda(cudaStreamSynchronize(c->work_stream()), "sync"));
  unsigned long long h[3];
  PBRT_TRY(c->cuda(cudaMemcpy(h, c->d_counters + 8, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy(render stats)"));
  for (int i = 0; i < 3; ++i) stats[i] = h[i];
  return PBRT_OK;
}

int pbrt_film_to_rgba8(const double* film, uint32_t w, uint32_t h, uint8_t* rgba) {
  if (!film || !rgba) return PBRT_ERR_INVALID_ARGUMENT;
  for (size_t i = 0; i < size_t(w) * h; ++i) {
    for (int ch = 0; ch < 3; ++ch) {
      const double v = std::sqrt(film[3 * i + ch]);           // gamma_correct (spectrum.rs:19-23)
      const double b = std::fmin(1.0, std::fmax(0.0, v));      // in_bound (spectrum.rs:134-136)
      rgba[4 * i + ch] = uint8_t(b * 255.0);                   // `as u8` truncates (spectrum.rs:13-17)
    }
    rgba[4 * i + 3] = 255;
  }
  return PBRT_OK;
}

}  // extern "C"
