// cache.cu — the learned radiance cache: network state on the device and its C ABI
// (create, query, gradient, Adam step, checkpoint). The cached render itself is in
// kernels_render.cu / api.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "cache.hpp"
#include "context.hpp"

using namespace pbrt;
using namespace pbrt::api;

namespace {

uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// He-uniform initial weights (U(-sqrt(6/fan_in), +sqrt(6/fan_in))); the padded input
// columns of the first layer and the padded output rows of the last stay zero.
std::vector<float> initial_weights(uint64_t seed) {
  std::vector<float> w(mlp::kParams, 0.f);
  uint64_t s = mix64(seed);
  for (int l = 0; l < mlp::kLayers; ++l) {
    const int K = mlp::layer_k(l), N = mlp::layer_n(l);
    const int fan_in = l == 0 ? mlp::kIn : K;
    const int outs = l == mlp::kLayers - 1 ? mlp::kOut : N;
    const float bound = std::sqrt(6.0f / float(fan_in));
    for (int o = 0; o < outs; ++o)
      for (int i = 0; i < fan_in; ++i) {
        s = mix64(s);
        const float u = float(s >> 40) * (1.0f / 16777216.0f);
        w[mlp::layer_off(l) + o * K + i] = (2.0f * u - 1.0f) * bound;
      }
  }
  return w;
}

}  // namespace

int pbrt_cache::device_arrays() {
  const size_t P = mlp::kParams;
  PBRT_TRY(ctx->cuda(cudaMalloc(&w, P * 4), "cudaMalloc(cache)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&m, P * 4), "cudaMalloc(cache)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&v, P * 4), "cudaMalloc(cache)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&grad, P * 4), "cudaMalloc(cache)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&wfwd, P * 2), "cudaMalloc(cache)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&wbwd, P * 2), "cudaMalloc(cache)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&loss, 4), "cudaMalloc(cache)"));
  return PBRT_OK;
}

int pbrt_cache::ensure_tiles(uint32_t tiles) {
  if (tiles <= tile_cap) return PBRT_OK;
  cudaFree(partials);
  cudaFree(tile_loss);
  partials = nullptr;
  tile_loss = nullptr;
  PBRT_TRY(ctx->cuda(cudaMalloc(&partials, size_t(tiles) * mlp::kParams * 4), "cudaMalloc(cache gradients)"));
  PBRT_TRY(ctx->cuda(cudaMalloc(&tile_loss, size_t(tiles) * 4), "cudaMalloc(cache gradients)"));
  tile_cap = tiles;
  return PBRT_OK;
}

mlp::Bounds pbrt_cache::bounds() const {
  mlp::Bounds b;
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = params.scene_min[a];
    const float ext = params.scene_max[a] - params.scene_min[a];
    b.inv_extent[a] = ext > 0.f ? 1.0f / ext : 1.0f;
  }
  return b;
}

int pbrt_cache::reset() {
  const std::vector<float> w0 = initial_weights(params.seed);
  cudaStream_t s = ctx->work_stream();
  PBRT_TRY(ctx->cuda(cudaMemcpyAsync(w, w0.data(), w0.size() * 4, cudaMemcpyHostToDevice, s), "cudaMemcpy(cache)"));
  PBRT_TRY(ctx->cuda(cudaMemsetAsync(m, 0, mlp::kParams * 4, s), "cudaMemset(cache)"));
  PBRT_TRY(ctx->cuda(cudaMemsetAsync(v, 0, mlp::kParams * 4, s), "cudaMemset(cache)"));
  PBRT_TRY(ctx->cuda(cudaMemsetAsync(wfwd, 0, mlp::kParams * 2, s), "cudaMemset(cache)"));
  PBRT_TRY(ctx->cuda(cudaMemsetAsync(wbwd, 0, mlp::kParams * 2, s), "cudaMemset(cache)"));
  PBRT_TRY(ctx->cuda(mlp::launch_pack(w, wfwd, wbwd, s), "cache pack"));
  step = 0;
  return ctx->cuda(cudaStreamSynchronize(s), "cache reset");
}

// Gradient of the mean relative-L2 loss over n device-resident samples into `grad` (and the
// summed loss into `loss`), without a host synchronisation.
int pbrt_cache::gradient_device(const float* records, const float* targets, uint64_t n, cudaStream_t s) {
  const uint32_t tiles = uint32_t((n + mlp::kTile - 1) / mlp::kTile);
  PBRT_TRY(ensure_tiles(tiles));
  const mlp::Net net{wfwd, wbwd};
  const float scale = 1.0f / (float(n) * float(mlp::kOut));
  PBRT_TRY(ctx->cuda(mlp::launch_grad_tiles(net, bounds(), records, targets, n, scale, partials, tile_loss,
                                            ctx->d_err, s),
                     "cache gradient"));
  return ctx->cuda(mlp::launch_reduce(partials, tile_loss, tiles, grad, loss, s), "cache gradient");
}

int pbrt_cache::adam_device(cudaStream_t s, const uint32_t* active) {
  ++step;
  return ctx->cuda(mlp::launch_adam(w, m, v, grad, step, params.learning_rate, params.beta1, params.beta2,
                                    params.epsilon, wfwd, wbwd, s, active),
                   "cache adam");
}

int pbrt_cache::query_device(const float* records, uint64_t n, float* rgb, cudaStream_t s) {
  const mlp::Net net{wfwd, wbwd};
  return ctx->cuda(mlp::launch_infer(net, bounds(), records, n, rgb, ctx->d_err, ctx->sm_count, s), "cache query");
}

int pbrt_cache::ensure_render_buffers(uint32_t queries, uint32_t train_vertices, uint32_t batch) {
  if (render_block && qcap >= queries && cw.tcap >= train_vertices && bcap >= batch) return PBRT_OK;
  queries = std::max(queries, qcap);
  train_vertices = std::max(train_vertices, cw.tcap);
  batch = std::max(batch, bcap);
  cudaFree(render_block);
  render_block = nullptr;
  qcap = bcap = 0;
  cw = pbrt::CacheWave{};
  const size_t R = pbrt::kCacheRecordFloats * 4;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t bytes = up(64) + up(size_t(queries) * R) + up(size_t(queries) * 12) + up(size_t(queries) * 4) +
                       up(size_t(train_vertices) * R) + up(size_t(train_vertices) * 24) +
                       up(size_t(train_vertices) * 4) + up(size_t(batch) * R) + up(size_t(batch) * 12);
  PBRT_TRY(ctx->cuda(cudaMalloc(&render_block, bytes), "cudaMalloc(cache render buffers)"));
  char* p = static_cast<char*>(render_block);
  auto take = [&](size_t b) { char* r = p; p += up(b); return r; };
  cw.counts = reinterpret_cast<uint32_t*>(take(64));
  cw.qrec = reinterpret_cast<float*>(take(size_t(queries) * R));
  cw.qout = reinterpret_cast<float*>(take(size_t(queries) * 12));
  cw.qpath = reinterpret_cast<uint32_t*>(take(size_t(queries) * 4));
  cw.trec = reinterpret_cast<float*>(take(size_t(train_vertices) * R));
  cw.tstate = reinterpret_cast<float*>(take(size_t(train_vertices) * 24));
  cw.tpath = reinterpret_cast<uint32_t*>(take(size_t(train_vertices) * 4));
  cw.tcap = train_vertices;
  cw.qcap = queries;
  brec = reinterpret_cast<float*>(take(size_t(batch) * R));
  btgt = reinterpret_cast<float*>(take(size_t(batch) * 12));
  qcap = queries;
  bcap = batch;
  return PBRT_OK;
}

int pbrt_cache::ensure_frame_buffers(uint32_t queries) {
  if (frame_block && fqcap >= queries) return PBRT_OK;
  cudaFree(frame_block);
  frame_block = nullptr;
  fqcap = 0;
  fcw = pbrt::CacheWave{};
  const size_t R = pbrt::kCacheRecordFloats * 4;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t bytes =
      up(64) + up(size_t(queries) * R) + up(size_t(queries) * 12) + up(size_t(queries) * 4) + up(mlp::kParams * 2);
  PBRT_TRY(ctx->cuda(cudaMalloc(&frame_block, bytes), "cudaMalloc(cache frame buffers)"));
  char* p = static_cast<char*>(frame_block);
  auto take = [&](size_t b) { char* r = p; p += up(b); return r; };
  fcw.counts = reinterpret_cast<uint32_t*>(take(64));
  fcw.qrec = reinterpret_cast<float*>(take(size_t(queries) * R));
  fcw.qout = reinterpret_cast<float*>(take(size_t(queries) * 12));
  fcw.qpath = reinterpret_cast<uint32_t*>(take(size_t(queries) * 4));
  fcw.qcap = queries;  // no training vertices: the frame only queries
  wsnap = reinterpret_cast<uint16_t*>(take(mlp::kParams * 2));
  fqcap = queries;
  return PBRT_OK;
}

int pbrt_cache::ensure_branch_buffers(uint32_t slot, uint32_t queries) {
  if (slot >= kBranchSlots) return ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "no such frame branch");
  if (branch_block[slot] && branch_qcap[slot] >= queries) return PBRT_OK;
  cudaFree(branch_block[slot]);
  branch_block[slot] = nullptr;
  branch_qcap[slot] = 0;
  pbrt::CacheWave& q = bcw[slot];
  q = pbrt::CacheWave{};
  const size_t R = pbrt::kCacheRecordFloats * 4;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t bytes = up(64) + up(size_t(queries) * R) + up(size_t(queries) * 12) + up(size_t(queries) * 4);
  PBRT_TRY(ctx->cuda(cudaMalloc(&branch_block[slot], bytes), "cudaMalloc(cache branch buffers)"));
  char* p = static_cast<char*>(branch_block[slot]);
  auto take = [&](size_t b) { char* r = p; p += up(b); return r; };
  q.counts = reinterpret_cast<uint32_t*>(take(64));
  q.qrec = reinterpret_cast<float*>(take(size_t(queries) * R));
  q.qout = reinterpret_cast<float*>(take(size_t(queries) * 12));
  q.qpath = reinterpret_cast<uint32_t*>(take(size_t(queries) * 4));
  q.qcap = queries;  // queries only, like the frame's own buffers
  branch_qcap[slot] = queries;
  return PBRT_OK;
}

void pbrt_cache::release() {
  for (void* p : {(void*)w, (void*)m, (void*)v, (void*)grad, (void*)wfwd, (void*)wbwd, (void*)loss, (void*)partials,
                  (void*)tile_loss, render_block, frame_block})
    cudaFree(p);
  for (void* p : branch_block) cudaFree(p);
}

namespace {

// Copies host arrays to temporary device buffers when needed (tests and host callers).
struct DeviceIn {
  const float* ptr = nullptr;
  float* owned = nullptr;
  ~DeviceIn() { cudaFree(owned); }
  int set(pbrt_ctx* c, const float* p, size_t count) {
    if (mem_kind(p) == MemKind::Device) {
      if (reinterpret_cast<uintptr_t>(p) % 16 != 0)
        return c->fail(PBRT_ERR_INVALID_ARGUMENT, "device records and targets must be 16-byte aligned");
      ptr = p;
      return PBRT_OK;
    }
    PBRT_TRY(c->cuda(cudaMalloc(&owned, std::max<size_t>(count, 1) * 4), "cudaMalloc(cache input)"));
    // on the stream the kernels that read it run on (a plain cudaMemcpy from pageable memory
    // may return before its DMA lands)
    PBRT_TRY(c->cuda(cudaMemcpyAsync(owned, p, count * 4, cudaMemcpyHostToDevice, c->work_stream()),
                     "cudaMemcpy(cache input)"));
    ptr = owned;
    return PBRT_OK;
  }
};

}  // namespace

extern "C" {

int pbrt_cache_create(pbrt_ctx* c, const pbrt_cache_params* p, pbrt_cache** out) {
  if (!c || !p || !out) return PBRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  DeviceGuard g(c->device);
  std::unique_ptr<pbrt_cache> k(new pbrt_cache);
  k->ctx = c;
  k->params = *p;
  if (!(k->params.learning_rate > 0.f)) k->params.learning_rate = 1e-2f;
  if (!(k->params.beta1 > 0.f)) k->params.beta1 = 0.9f;
  if (!(k->params.beta2 > 0.f)) k->params.beta2 = 0.99f;
  if (!(k->params.epsilon > 0.f)) k->params.epsilon = 1e-8f;
  if (k->params.terminate_bounce == 0) k->params.terminate_bounce = 2;
  if (k->params.train_samples == 0) k->params.train_samples = 1u << 16;
  if (k->params.train_steps == 0) k->params.train_steps = 4;
  if (k->device_arrays() != PBRT_OK) {
    k->release();
    return PBRT_ERR_OUT_OF_MEMORY;
  }
  const int rc = k->reset();
  if (rc != PBRT_OK) {
    k->release();
    return rc;
  }
  *out = k.release();
  return PBRT_OK;
}

void pbrt_cache_destroy(pbrt_cache* k) {
  if (!k) return;
  DeviceGuard g(k->ctx->device);
  cudaStreamSynchronize(k->ctx->work_stream());
  k->release();
  delete k;
}

int pbrt_cache_reset(pbrt_cache* k) {
  if (!k) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(k->ctx->device);
  return k->reset();
}

int pbrt_cache_get_weights(pbrt_cache* k, float* w) {
  if (!k || !w) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(k->ctx->device);
  PBRT_TRY(k->ctx->cuda(cudaStreamSynchronize(k->ctx->work_stream()), "sync"));
  return k->ctx->cuda(cudaMemcpy(w, k->w, mlp::kParams * 4, cudaMemcpyDefault), "cudaMemcpy(weights)");
}

int pbrt_cache_set_weights(pbrt_cache* k, const float* w) {
  if (!k || !w) return PBRT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(k->ctx->device);
  cudaStream_t s = k->ctx->work_stream();
  PBRT_TRY(k->ctx->cuda(cudaMemcpyAsync(k->w, w, mlp::kParams * 4, cudaMemcpyDefault, s), "cudaMemcpy(weights)"));
  PBRT_TRY(k->ctx->cuda(mlp::launch_pack(k->w, k->wfwd, k->wbwd, s), "cache pack"));
  return k->ctx->cuda(cudaStreamSynchronize(s), "cache pack");
}

int pbrt_cache_query(pbrt_cache* k, const float* records, uint64_t n, float* rgb) {
  if (!k) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = k->ctx;
  DeviceGuard g(c->device);
  if (n == 0) return PBRT_OK;
  if (!records || !rgb) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "records or rgb is NULL");
  DeviceIn in;
  PBRT_TRY(in.set(c, records, size_t(n) * mlp::kRecord));
  const bool host_out = mem_kind(rgb) != MemKind::Device;
  float* dout = rgb;
  if (host_out) PBRT_TRY(c->cuda(cudaMalloc(&dout, size_t(n) * 3 * 4), "cudaMalloc(cache output)"));
  cudaStream_t s = c->work_stream();
  int rc = k->query_device(in.ptr, n, dout, s);
  if (rc == PBRT_OK) rc = check_device_error(c, s);
  if (host_out) {
    if (rc == PBRT_OK) rc = c->cuda(cudaMemcpy(rgb, dout, size_t(n) * 3 * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    cudaFree(dout);
  }
  return rc;
}

int pbrt_cache_gradient(pbrt_cache* k, const float* records, const float* targets, uint64_t n, float* grad,
                        float* loss) {
  if (!k) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = k->ctx;
  DeviceGuard g(c->device);
  if (n == 0 || !records || !targets || !grad) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "empty batch or NULL buffer");
  DeviceIn rin, tin;
  PBRT_TRY(rin.set(c, records, size_t(n) * mlp::kRecord));
  PBRT_TRY(tin.set(c, targets, size_t(n) * 3));
  cudaStream_t s = c->work_stream();
  PBRT_TRY(k->gradient_device(rin.ptr, tin.ptr, n, s));
  PBRT_TRY(check_device_error(c, s));
  PBRT_TRY(c->cuda(cudaMemcpy(grad, k->grad, mlp::kParams * 4, cudaMemcpyDefault), "cudaMemcpy(gradient)"));
  if (loss) {
    float l = 0.f;
    PBRT_TRY(c->cuda(cudaMemcpy(&l, k->loss, 4, cudaMemcpyDeviceToHost), "cudaMemcpy(loss)"));
    *loss = l / (float(n) * float(mlp::kOut));
  }
  return PBRT_OK;
}

int pbrt_cache_train_step(pbrt_cache* k, const float* records, const float* targets, uint64_t n, float* loss) {
  if (!k) return PBRT_ERR_INVALID_ARGUMENT;
  pbrt_ctx* c = k->ctx;
  DeviceGuard g(c->device);
  if (n == 0 || !records || !targets) return c->fail(PBRT_ERR_INVALID_ARGUMENT, "empty batch or NULL buffer");
  DeviceIn rin, tin;
  PBRT_TRY(rin.set(c, records, size_t(n) * mlp::kRecord));
  PBRT_TRY(tin.set(c, targets, size_t(n) * 3));
  cudaStream_t s = c->work_stream();
  PBRT_TRY(k->gradient_device(rin.ptr, tin.ptr, n, s));
  PBRT_TRY(k->adam_device(s));
  PBRT_TRY(check_device_error(c, s));
  if (loss) {
    float l = 0.f;
    PBRT_TRY(c->cuda(cudaMemcpy(&l, k->loss, 4, cudaMemcpyDeviceToHost), "cudaMemcpy(loss)"));
    *loss = l / (float(n) * float(mlp::kOut));
  }
  return PBRT_OK;
}

int pbrt_cache_save(pbrt_cache* k, void* buf, uint64_t cap, uint64_t* size) {
  if (!k || !size) return PBRT_ERR_INVALID_ARGUMENT;
  const uint64_t need = 8 + 3ull * mlp::kParams * 4;
  *size = need;
  if (!buf) return PBRT_OK;
  if (cap < need) return PBRT_ERR_CAPACITY;
  DeviceGuard g(k->ctx->device);
  PBRT_TRY(k->ctx->cuda(cudaStreamSynchronize(k->ctx->work_stream()), "sync"));
  uint8_t* b = static_cast<uint8_t*>(buf);
  const uint32_t magic = 0x43524e50u, step = k->step;  // "PNRC"
  std::memcpy(b, &magic, 4);
  std::memcpy(b + 4, &step, 4);
  PBRT_TRY(k->ctx->cuda(cudaMemcpy(b + 8, k->w, mlp::kParams * 4, cudaMemcpyDeviceToHost), "cudaMemcpy"));
  PBRT_TRY(k->ctx->cuda(cudaMemcpy(b + 8 + mlp::kParams * 4, k->m, mlp::kParams * 4, cudaMemcpyDeviceToHost), "cudaMemcpy"));
  return k->ctx->cuda(cudaMemcpy(b + 8 + 2 * mlp::kParams * 4, k->v, mlp::kParams * 4, cudaMemcpyDeviceToHost),
                      "cudaMemcpy");
}

int pbrt_cache_load(pbrt_cache* k, const void* buf, uint64_t size) {
  if (!k || !buf) return PBRT_ERR_INVALID_ARGUMENT;
  if (size != 8 + 3ull * mlp::kParams * 4) return k->ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "not a cache checkpoint");
  const uint8_t* b = static_cast<const uint8_t*>(buf);
  uint32_t magic, step;
  std::memcpy(&magic, b, 4);
  std::memcpy(&step, b + 4, 4);
  if (magic != 0x43524e50u) return k->ctx->fail(PBRT_ERR_INVALID_ARGUMENT, "not a cache checkpoint");
  DeviceGuard g(k->ctx->device);
  cudaStream_t s = k->ctx->work_stream();
  PBRT_TRY(k->ctx->cuda(cudaMemcpyAsync(k->w, b + 8, mlp::kParams * 4, cudaMemcpyHostToDevice, s), "cudaMemcpy"));
  PBRT_TRY(k->ctx->cuda(cudaMemcpyAsync(k->m, b + 8 + mlp::kParams * 4, mlp::kParams * 4, cudaMemcpyHostToDevice, s),
                        "cudaMemcpy"));
  PBRT_TRY(k->ctx->cuda(
      cudaMemcpyAsync(k->v, b + 8 + 2 * mlp::kParams * 4, mlp::kParams * 4, cudaMemcpyHostToDevice, s), "cudaMemcpy"));
  k->step = step;
  PBRT_TRY(k->ctx->cuda(mlp::launch_pack(k->w, k->wfwd, k->wbwd, s), "cache pack"));
  return k->ctx->cuda(cudaStreamSynchronize(s), "cache pack");
}

}  // extern "C"
