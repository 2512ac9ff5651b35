// batch.cu — many scenes rendered together, one frame's launches recorded once in a CUDA graph
// (pbrt_batch_* in include/pbrt_b200.h): by one wavefront over the batch table (the wavefront
// kernels of kernels_render.cu), or by one persistent launch that runs every path to its end
// (k_batch_paths). Host code.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pbrt_b200.h"
#include "context.hpp"
#include "render.hpp"
#include "scene_host.hpp"

using namespace pbrt;
using namespace pbrt::api;

struct pbrt_batch {
  pbrt_ctx* ctx = nullptr;
  std::vector<BatchScene> table;  // host copy (film pointers are the batch's device films)
  std::vector<size_t> film_n;     // doubles per film
  std::vector<uint32_t> slot;     // the table position of the caller's scene i (cheapest first)
  BatchScene* d_table = nullptr;
  uint32_t* d_frame = nullptr;
  uint32_t frame_host = 0;
  std::vector<double*> films;
  WaveAlloc wave;
  uint32_t wave_paths = 0, max_depth = 0;
  bool any_path = false;
  bool persistent = false;                 // one persistent launch instead of the wavefront
  unsigned long long* d_scratch = nullptr;  // its fetch position, clock stamps, completion counters
  std::vector<unsigned long long> h_stamps;
  LaunchShape shape;
  // concurrent branches of a wavefront frame: branch 0 runs on `cap`, branch k >= 1 on
  // branch_st[k] with its own wave buffers extra[k - 1]
  std::vector<BatchWave> plan;
  uint32_t branches = 1;
  std::vector<WaveAlloc> extra;
  std::vector<cudaStream_t> branch_st;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t start = nullptr;
  std::vector<cudaEvent_t> done;

  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap) cudaStreamDestroy(cap);
    for (size_t k = 1; k < branch_st.size(); ++k)
      if (branch_st[k]) cudaStreamDestroy(branch_st[k]);
    if (fork) cudaEventDestroy(fork);
    for (cudaEvent_t e : joins)
      if (e) cudaEventDestroy(e);
    for (WaveAlloc& w : extra) cudaFree(w.block);
    if (start) cudaEventDestroy(start);
    for (cudaEvent_t e : done) cudaEventDestroy(e);
    for (double* f : films) cudaFree(f);
    cudaFree(d_table);
    cudaFree(d_frame);
    cudaFree(d_scratch);
    cudaFree(wave.block);
  }
};

namespace {

// Records one frame's launches (all waves of all scenes) into b->graph and instantiates it.
int capture(pbrt_batch* b) {
  pbrt_ctx* c = b->ctx;
  PBRT_TRY(c->cuda(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "cudaStreamCreate"));
  std::vector<WaveBuffers> bw(b->branches);
  b->branch_st.assign(b->branches, nullptr);
  b->joins.assign(b->branches, nullptr);
  b->branch_st[0] = b->cap;
  bw[0] = b->wave.w;
  for (uint32_t k = 1; k < b->branches; ++k) {
    PBRT_TRY(c->cuda(cudaStreamCreateWithFlags(&b->branch_st[k], cudaStreamNonBlocking), "cudaStreamCreate"));
    PBRT_TRY(c->cuda(cudaEventCreateWithFlags(&b->joins[k], cudaEventDisableTiming), "cudaEventCreate"));
    bw[k] = b->extra[k - 1].w;
  }
  if (b->branches > 1) PBRT_TRY(c->cuda(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate"));
  PBRT_TRY(c->cuda(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture"));
  cudaError_t e = cudaMemsetAsync(c->d_counters + 8, 0, 3 * sizeof(unsigned long long), b->cap);
  if (e == cudaSuccess && b->persistent)
    e = render_batch_persistent(b->d_table, b->table.data(), uint32_t(b->table.size()), b->d_frame, b->d_scratch,
                                c->d_counters + 8, c->d_err, c->sm_count, b->cap);
  else if (e == cudaSuccess)
    e = render_batch(b->d_table, b->table.data(), uint32_t(b->table.size()), b->plan, bw.data(), b->branch_st.data(),
                     b->branches, b->d_frame, b->max_depth, b->any_path, b->shape, c->d_counters + 8, c->d_err,
                     c->sm_count, b->cap, b->fork, b->joins.data(), b->done.data());
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(b->cap, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return c->cuda(e != cudaSuccess ? e : e2, "batch graph capture");
  }
  b->graph = g;
  return c->cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
}

}  // namespace

extern "C" {

int pbrt_batch_create(pbrt_ctx* c, pbrt_scene* const* scenes, const pbrt_render_params* params, uint32_t n,
                      pbrt_batch** out) {
  if (!c || !out) return PBRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  DeviceGuard g(c->device);
  if (n == 0 || !scenes || !params) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "empty batch");
  std::unique_ptr<pbrt_batch> b(new pbrt_batch);
  b->ctx = c;
  b->shape = c->shape;
  // Scenes run cheapest first (pixels x spp x max depth; ties keep the given order), which
  // minimises the mean completion time of a frame; films and times stay per caller index.
  std::vector<uint32_t> order(n);
  std::vector<unsigned long long> cost(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    order[i] = i;
    const pbrt_render_params* p = params + i;
    const unsigned long long px = (unsigned long long)p->camera.width * p->camera.height;
    cost[i] = px * p->spp * std::max<uint32_t>(1u, p->max_depth);
  }
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b2) { return cost[a] < cost[b2]; });
  b->slot.assign(n, 0);
  unsigned long long begin = 0;
  for (uint32_t pos = 0; pos < n; ++pos) {
    const uint32_t i = order[pos];
    b->slot[i] = pos;
    const pbrt_scene* s = scenes[i];
    const pbrt_render_params* p = params + i;
    if (!s || s->ctx != c) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "scene " + std::to_string(i) + " is NULL or "
                                                                     "belongs to another context");
    PBRT_TRY(check_render_params(c, p, false));
    const RenderSettings rs = settings_of(c, p);
    BatchScene e{};
    e.view = s->view;
    e.cam = build_camera(p->camera);
    e.begin = begin;
    e.seed = p->seed;
    e.npix = uint32_t(film_pixels(p, rs));
    e.spp = p->spp;
    e.max_depth = rs.max_depth;
    e.rr_start = rs.rr_start;
    e.sample_offset = p->sample_offset;
    e.integrator = rs.integrator;
    e.stride = rs.stride;
    e.film_w = rs.film_w;
    const unsigned long long paths = (unsigned long long)e.npix * e.spp;
    if (begin + paths < begin || begin + paths > (1ull << 62))
      return c->fail(PBRT_ERR_INVALID_ARGUMENT, "too many paths in the batch");
    begin += paths;
    b->table.push_back(e);
    b->film_n.push_back(size_t(e.npix) * 3);
    b->max_depth = std::max(b->max_depth, e.max_depth);
    b->any_path = b->any_path || !e.integrator;
  }
  int rc = PBRT_OK;
  for (uint32_t i = 0; i < n && rc == PBRT_OK; ++i) {
    double* f = nullptr;
    rc = c->cuda(cudaMalloc(&f, b->film_n[i] * sizeof(double)), "cudaMalloc(batch film)");
    if (rc == PBRT_OK) {
      b->films.push_back(f);
      b->table[i].film = f;
    }
  }
  if (rc == PBRT_OK) rc = c->cuda(cudaMalloc(&b->d_table, n * sizeof(BatchScene)), "cudaMalloc(batch table)");
  if (rc == PBRT_OK)
    rc = c->cuda(cudaMemcpyAsync(b->d_table, b->table.data(), n * sizeof(BatchScene), cudaMemcpyHostToDevice,
                                 c->stream),
                 "cudaMemcpy(batch table)");
  if (rc == PBRT_OK) rc = c->cuda(cudaMalloc(&b->d_frame, sizeof(uint32_t)), "cudaMalloc(batch frame)");
  if (rc == PBRT_OK) rc = c->cuda(cudaMemsetAsync(b->d_frame, 0, sizeof(uint32_t), c->stream), "cudaMemset(batch frame)");
  if (rc == PBRT_OK) rc = c->cuda(cudaStreamSynchronize(c->stream), "batch upload");
  b->wave_paths = uint32_t(std::min<unsigned long long>(begin, c->wave_paths));
  b->persistent = c->batch_kernel == PBRT_BATCH_PERSISTENT;
  if (b->persistent) {
    b->h_stamps.assign(2 + 2 * size_t(n), 0);
    if (rc == PBRT_OK)
      rc = c->cuda(cudaMalloc(&b->d_scratch, b->h_stamps.size() * sizeof(unsigned long long)),
                   "cudaMalloc(batch counters)");
  } else if (rc == PBRT_OK) {
    // each branch's wave buffers hold its largest wave
    b->plan = batch_plan(b->table.data(), n, b->wave_paths, std::max<uint32_t>(1u, c->batch_branches));
    std::vector<uint32_t> cap(1, 0);
    for (const BatchWave& wv : b->plan) {
      if (wv.branch >= cap.size()) cap.resize(wv.branch + 1, 0);
      cap[wv.branch] = std::max(cap[wv.branch], wv.n);
    }
    b->branches = uint32_t(cap.size());
    b->extra.resize(b->branches - 1);
    rc = ensure_wave(c, &b->wave, cap[0]);
    for (uint32_t k = 1; k < b->branches && rc == PBRT_OK; ++k) rc = ensure_wave(c, &b->extra[k - 1], cap[k]);
  }
  if (rc == PBRT_OK) rc = c->cuda(cudaEventCreate(&b->start), "cudaEventCreate");
  b->done.assign(n, nullptr);
  for (uint32_t i = 0; i < n && rc == PBRT_OK; ++i) rc = c->cuda(cudaEventCreate(&b->done[i]), "cudaEventCreate");
  if (rc == PBRT_OK) rc = capture(b.get());
  if (rc != PBRT_OK) {
    b->release();
    return rc;
  }
  *out = b.release();
  return PBRT_OK;
}

int pbrt_batch_render(pbrt_batch* b, uint32_t frame, double* const* films, float* scene_ms) {
  if (!b) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = b->ctx;
  DeviceGuard g(c->device);
  cudaStream_t st = c->work_stream();
  b->frame_host = frame;
  PBRT_TRY(c->cuda(cudaMemcpyAsync(b->d_frame, &b->frame_host, sizeof(uint32_t), cudaMemcpyHostToDevice, st),
                   "cudaMemcpy(batch frame)"));
  PBRT_TRY(c->cuda(cudaEventRecord(b->start, st), "cudaEventRecord"));
  PBRT_TRY(c->cuda(cudaGraphLaunch(b->exec, st), "cudaGraphLaunch"));
  if (films)
    for (size_t i = 0; i < b->slot.size(); ++i)
      if (films[i]) {
        const uint32_t k = b->slot[i];
        PBRT_TRY(c->cuda(cudaMemcpyAsync(films[i], b->films[k], b->film_n[k] * sizeof(double), cudaMemcpyDefault, st),
                         "cudaMemcpy(batch film)"));
      }
  if (scene_ms && b->persistent)  // the kernel's clock stamps: frame start, each scene's completion
    PBRT_TRY(c->cuda(cudaMemcpyAsync(b->h_stamps.data(), b->d_scratch, b->h_stamps.size() * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, st),
                     "cudaMemcpy(batch clock)"));
  PBRT_TRY(check_device_error(c, st));
  if (scene_ms && b->persistent) {
    const size_t n = b->slot.size();
    for (size_t i = 0; i < n; ++i) {
      const unsigned long long t0 = b->h_stamps[1], t1 = b->h_stamps[2 + n + b->slot[i]];
      scene_ms[i] = t1 >= t0 ? float(double(t1 - t0) * 1e-6) : 0.f;
    }
  } else if (scene_ms) {
    for (size_t i = 0; i < b->slot.size(); ++i)
      PBRT_TRY(c->cuda(cudaEventElapsedTime(scene_ms + i, b->start, b->done[b->slot[i]]), "cudaEventElapsedTime"));
  }
  return PBRT_OK;
}

void pbrt_batch_destroy(pbrt_batch* b) {
  if (!b) return;
  DeviceGuard g(b->ctx->device);
  cudaStreamSynchronize(b->ctx->work_stream());
  b->release();
  delete b;
}

int pbrt_ctx_set_batch_kernel(pbrt_ctx* c, int kind) {
  if (!c) return PBRT_ERR_INVALID_ARGUMENT;
  if (kind != PBRT_BATCH_WAVEFRONT && kind != PBRT_BATCH_PERSISTENT)
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "unknown batch kernel " + std::to_string(kind));
  c->batch_kernel = kind;
  return PBRT_OK;
}

int pbrt_ctx_set_batch_branches(pbrt_ctx* c, uint32_t branches) {
  if (!c) return PBRT_ERR_INVALID_ARGUMENT;
  if (branches < 1 || branches > kMaxBatchBranches)
    return c->fail(PBRT_ERR_INVALID_ARGUMENT, "batch branches must be in [1, " + std::to_string(kMaxBatchBranches) +
                                                  "], not " + std::to_string(branches));
  c->batch_branches = branches;
  return PBRT_OK;
}

int pbrt_render_batch(pbrt_scene* const* scenes, const pbrt_render_params* params, uint32_t n, double* const* films) {
  if (!scenes || n == 0 || !scenes[0]) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_batch* b = nullptr;
  PBRT_TRY(pbrt_batch_create(scenes[0]->ctx, scenes, params, n, &b));
  const int rc = pbrt_batch_render(b, 0, films, nullptr);
  pbrt_batch_destroy(b);
  return rc;
}

}  // extern "C"
