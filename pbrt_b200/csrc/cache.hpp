// cache.hpp — the radiance cache object behind the C ABI's pbrt_cache handle (host code).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/pbrt_b200.h"
#include "mlp.hpp"
#include "render.hpp"

struct pbrt_cache {
  pbrt_ctx* ctx = nullptr;
  pbrt_cache_params params{};
  float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
  uint16_t *wfwd = nullptr, *wbwd = nullptr;
  float *partials = nullptr, *tile_loss = nullptr;
  uint32_t tile_cap = 0;
  uint32_t step = 0;
  uint64_t rounds = 0;  // training rounds run by cached renders (keys their path streams)

  // the cached render's buffers: queries, training vertices and one training batch
  void* render_block = nullptr;
  uint32_t qcap = 0, bcap = 0;
  pbrt::CacheWave cw{};
  float *brec = nullptr, *btgt = nullptr;
  int ensure_render_buffers(uint32_t queries, uint32_t train_vertices, uint32_t batch);

  // A call that trains and renders: the frame's own query buffers and the snapshot of the
  // forward weights it reads, while the training rounds (with `cw`) update the weights.
  void* frame_block = nullptr;
  uint32_t fqcap = 0;
  pbrt::CacheWave fcw{};
  uint16_t* wsnap = nullptr;
  int ensure_frame_buffers(uint32_t queries);

  // The query buffers of a frame's concurrent branches 1.. (branch 0 takes fcw or cw).
  static constexpr uint32_t kBranchSlots = 7;
  void* branch_block[kBranchSlots] = {};
  uint32_t branch_qcap[kBranchSlots] = {};
  pbrt::CacheWave bcw[kBranchSlots] = {};
  int ensure_branch_buffers(uint32_t slot, uint32_t queries);

  int device_arrays();
  int ensure_tiles(uint32_t tiles);
  int reset();
  pbrt::mlp::Bounds bounds() const;
  int gradient_device(const float* records, const float* targets, uint64_t n, cudaStream_t s);
  int adam_device(cudaStream_t s, const uint32_t* active = nullptr);
  int query_device(const float* records, uint64_t n, float* rgb, cudaStream_t s);
  void release();
};
