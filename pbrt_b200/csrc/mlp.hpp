// mlp.hpp — the learned radiance cache's network: host-visible constants and launchers.
//
// Network: 82 input features (12-band sin/cos encoding of the normalised position, 72
// values; the outgoing direction, normal, albedo, roughness, 10 values) padded to 96 ->
// 5 hidden layers of 64 ReLU units -> 3 linear outputs (RGB radiance), padded to 16 for the
// tensor cores. No biases. BF16 weights and activations, FP32 accumulation (tcgen05).
// Loss: relative L2, mean over samples and channels of (o - t)^2 / (o^2 + 0.01) with o
// treated as a constant in the denominator. Optimiser: Adam on FP32 master weights.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pbrt {
namespace mlp {

constexpr int kIn = 82, kInPad = 96, kHidden = 64, kLayers = 6, kOut = 3, kOutPad = 16;
constexpr int kTile = 128;       // samples per CTA tile (the MMA's M)
constexpr int kRecord = 16;      // floats per query record: p.xyz, rough, wo.xyz, 0, n.xyz, 0, albedo.xyz, 0
constexpr int kParams = 64 * 96 + 4 * 64 * 64 + 16 * 64;  // 23,552 (W6 padded to 16 rows)

__host__ __device__ constexpr int layer_k(int l) { return l == 0 ? kInPad : kHidden; }
__host__ __device__ constexpr int layer_n(int l) { return l == kLayers - 1 ? kOutPad : kHidden; }
__host__ __device__ constexpr int layer_off(int l) {
  return l == 0 ? 0 : (l == 1 ? 6144 : (l == 2 ? 10240 : (l == 3 ? 14336 : (l == 4 ? 18432 : 22528))));
}

struct Bounds {
  float lo[3], inv_extent[3];  // position normalisation to [0, 1]^3
};

struct Net {
  const uint16_t* wpk_fwd;  // BF16, per layer in the B-operand layout of the forward GEMM
  const uint16_t* wpk_bwd;  // BF16, per layer transposed, for the data-gradient GEMM
};

// out[3 * i + c] = network(record i), i < n.
cudaError_t launch_infer(const Net& net, const Bounds& b, const float* records, uint64_t n, float* out,
                         uint32_t* err, int sm_count, cudaStream_t s);
// The same for n = min(n_max, *n_dev), a count on the device (the grid is sized for n_max).
cudaError_t launch_infer_dev(const Net& net, const Bounds& b, const float* records, const uint32_t* n_dev,
                             uint64_t n_max, float* out, uint32_t* err, int sm_count, cudaStream_t s);
// Per-tile partial gradients (tiles = ceil(n / 128), each kParams floats) and loss sums.
cudaError_t launch_grad_tiles(const Net& net, const Bounds& b, const float* records, const float* targets, uint64_t n,
                              float grad_scale, float* partials, float* tile_loss, uint32_t* err, cudaStream_t s);
// grad[p] = sum over tiles of partials; loss[0] = sum of tile losses.
cudaError_t launch_reduce(const float* partials, const float* tile_loss, uint32_t tiles, float* grad, float* loss,
                          cudaStream_t s);
// One Adam step on the FP32 master weights, then the BF16 packs are rewritten; skipped
// entirely when `active` is given and *active == 0.
cudaError_t launch_adam(float* w, float* m, float* v, const float* grad, uint32_t step, float lr, float beta1,
                        float beta2, float eps, uint16_t* wpk_fwd, uint16_t* wpk_bwd, cudaStream_t s,
                        const uint32_t* active = nullptr);
cudaError_t launch_pack(const float* w, uint16_t* wpk_fwd, uint16_t* wpk_bwd, cudaStream_t s);

size_t infer_smem_bytes();
size_t train_smem_bytes();

}  // namespace mlp
}  // namespace pbrt
