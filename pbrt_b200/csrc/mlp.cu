// mlp.cu — forward (inference), per-tile backward, gradient reduction and Adam for the
// radiance cache's network; see mlp.hpp for the network and tcgen05.cuh for the layouts.
//
// One CTA of 128 threads owns a tile of 128 samples: thread r encodes sample r into row r of
// the BF16 input tile in shared memory; for every layer, thread 0 issues the tcgen05.mma
// chain (M = 128, N = 64 or 16, K = 96 or 64 in steps of 16) into a TMEM accumulator of 64
// FP32 columns and commits it to an mbarrier; every thread then reads its own accumulator
// row (TMEM lane = sample), applies ReLU and writes the BF16 activations back to shared
// memory as the next layer's A operand. The weights of all six layers (47 KB of BF16) stay
// resident in shared memory for the CTA's lifetime.
//
// Training: the same forward keeps every layer's activations; the loss gradient dO is
// written as a BF16 tile; for each layer both products run on the tensor cores, issued back
// to back and committed once: the data gradient dA = G·W (W transposed in its own pack) and
// the weight gradient dW = Gᵀ·A, which reduces over the tile's 128 samples by reading the
// resident G and A tiles as MN-major operands (M = 64; the output layer's 16-row dW is
// formed transposed, dWᵀ = Aᵀ·G). Per-tile partial gradients are reduced by a second kernel
// and Adam updates the FP32 master weights and rewrites both BF16 packs.
#include <cuda_bf16.h>

#include <atomic>
#include <cstdint>

#include "mlp.hpp"
#include "tcgen05.cuh"

namespace pbrt {
namespace mlp {

constexpr uint32_t kErrMma = 4u;  // a tensor-core completion wait ran out of its budget
constexpr uint32_t kWBytes = kParams * 2;           // 47,104
constexpr uint32_t kXBytes = kTile * kInPad * 2;    // 24,576
constexpr uint32_t kHBytes = kTile * kHidden * 2;   // 16,384
constexpr uint32_t kG16Bytes = kTile * kOutPad * 2;  // 4,096
constexpr uint32_t kTmemCols = 64;       // one 64-column accumulator
constexpr uint32_t kTrainTmemCols = 256;  // training: dA in columns 0-63, dW from column 64 (up to 96 wide)
constexpr uint32_t kWgradCol = 64;
static_assert(kXBytes >= kHBytes, "the inference kernel stores the hidden tile over the input tile");

__device__ __forceinline__ uint16_t to_bf16(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
__device__ __forceinline__ float from_bf16(uint16_t b) { return __uint_as_float(uint32_t(b) << 16); }
// Two values to BF16 (round to nearest even), `a` in the low half: one cvt.rn.bf16x2.f32,
// whose first source goes to the high half.
__device__ __forceinline__ uint32_t pack2(float a, float b) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
  return d;
}
// The same after a ReLU (.relu clamps negative results to 0): the hidden layers' epilogue.
__device__ __forceinline__ uint32_t pack2_relu(float a, float b) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
  return d;
}

// sin(pi x) and cos(pi x) in FP32, about 1.5 ulp: x reduced (k = rint(x / 2), r = x - 2k in
// [-1, 1]; q = rint(2r), t = r - q / 2 in [-1/4, 1/4]), the Taylor polynomials of sin(pi t)
// to t^9 and cos(pi t) to t^10 (truncation below 2e-9 there) in Horner form, each step one
// rounded multiply and one rounded add (no fused multiply-add, so a host computes the same
// bits), then the quadrant q. Coefficients: (-1)^k pi^(2k+1) / (2k+1)! and (-1)^k pi^(2k) /
// (2k)!, rounded to FP32.
__device__ __forceinline__ void sincospi_poly(float x, float& s, float& c) {
  const float k = rintf(__fmul_rn(x, 0.5f));
  const float r = __fsub_rn(x, __fmul_rn(k, 2.0f));
  const float q = rintf(__fmul_rn(r, 2.0f));
  const float t = __fsub_rn(r, __fmul_rn(q, 0.5f));
  const float t2 = __fmul_rn(t, t);
  float ps = 0x1.507834p-4f;
  ps = __fadd_rn(__fmul_rn(ps, t2), -0x1.32d2ccp-1f);
  ps = __fadd_rn(__fmul_rn(ps, t2), 0x1.466bc6p+1f);
  ps = __fadd_rn(__fmul_rn(ps, t2), -0x1.4abbcep+2f);
  ps = __fadd_rn(__fmul_rn(ps, t2), 0x1.921fb6p+1f);
  const float st = __fmul_rn(ps, t);
  float pc = -0x1.a6d1f2p-6f;
  pc = __fadd_rn(__fmul_rn(pc, t2), 0x1.e1f506p-3f);
  pc = __fadd_rn(__fmul_rn(pc, t2), -0x1.55d3c8p+0f);
  pc = __fadd_rn(__fmul_rn(pc, t2), 0x1.03c1f0p+2f);
  pc = __fadd_rn(__fmul_rn(pc, t2), -0x1.3bd3ccp+2f);
  const float ct = __fadd_rn(__fmul_rn(pc, t2), 1.0f);
  switch (int(q) & 3) {
    case 0: s = st; c = ct; break;
    case 1: s = ct; c = -st; break;
    case 2: s = -st; c = -ct; break;
    default: s = -ct; c = st; break;
  }
}

// The next octave of a band: sin 2a = 2 sin a cos a, cos 2a = (cos a - sin a)(cos a + sin a),
// each operation rounded (the error doubles per octave: 2e-4 at the twelfth band).
__device__ __forceinline__ void next_octave(float& s, float& c) {
  const float s2 = __fmul_rn(__fmul_rn(s, c), 2.0f);
  c = __fmul_rn(__fsub_rn(c, s), __fadd_rn(c, s));
  s = s2;
}

// Encodes one query record into 96 features (82 used, zero padded): sin / cos (pi 2^j x) of the
// normalised position, j < 12 (the first band by sincospi_poly, the others by next_octave),
// then wo, n, albedo, roughness.
__device__ void encode(const float* __restrict__ rec, const Bounds& b, float* f) {
  const float4 q0 = __ldg(reinterpret_cast<const float4*>(rec));
  const float4 q1 = __ldg(reinterpret_cast<const float4*>(rec) + 1);
  const float4 q2 = __ldg(reinterpret_cast<const float4*>(rec) + 2);
  const float4 q3 = __ldg(reinterpret_cast<const float4*>(rec) + 3);
  const float p[3] = {q0.x, q0.y, q0.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float s, c;
    sincospi_poly(__fmul_rn(__fsub_rn(p[a], b.lo[a]), b.inv_extent[a]), s, c);
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      f[a * 24 + 2 * j] = s;
      f[a * 24 + 2 * j + 1] = c;
      next_octave(s, c);
    }
  }
  f[72] = q1.x; f[73] = q1.y; f[74] = q1.z;
  f[75] = q2.x; f[76] = q2.y; f[77] = q2.z;
  f[78] = q3.x; f[79] = q3.y; f[80] = q3.z;
  f[81] = q0.w;
#pragma unroll
  for (int k = kIn; k < kInPad; ++k) f[k] = 0.f;
}

// Writes `n` (multiple of 8) values of row r into an R=128-row tile as BF16.
__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t r, const float* v, int n) {
  for (int c = 0; c < n; c += 8) {
    uint4 q;
    q.x = pack2(v[c], v[c + 1]);
    q.y = pack2(v[c + 2], v[c + 3]);
    q.z = pack2(v[c + 4], v[c + 5]);
    q.w = pack2(v[c + 6], v[c + 7]);
    *reinterpret_cast<uint4*>(tile + tc::tile_offset(r, uint32_t(c), kTile)) = q;
  }
}

__device__ __forceinline__ float tile_at(const uint8_t* tile, uint32_t r, uint32_t k, uint32_t rows) {
  return from_bf16(*reinterpret_cast<const uint16_t*>(tile + tc::tile_offset(r, k, rows)));
}

// D[128 x n] = A[128 x k] · B[n x k]^T, both K-major in the core-matrix layout; thread 0 only.
// Commits to mbar unless mbar is null.
__device__ __forceinline__ void issue_gemm(const uint8_t* a, const uint8_t* b, uint32_t n, uint32_t k, uint32_t tmem,
                                           uint64_t* mbar) {
  const uint32_t a_addr = tc::smem_u32(a), b_addr = tc::smem_u32(b);
  const uint32_t lbo_a = (kTile / 8) * 128, lbo_b = (n / 8) * 128;
  const uint32_t idesc = tc::idesc_bf16(kTile, n);
  for (uint32_t s = 0; s < k / 16; ++s)
    tc::mma_bf16(tmem, tc::make_desc(a_addr + s * 2 * lbo_a, lbo_a, 128), tc::make_desc(b_addr + s * 2 * lbo_b, lbo_b, 128),
                 idesc, s > 0 ? 1u : 0u);
  if (mbar) tc::mma_commit(mbar);  // null: a later issue commits both
}

// D[64 x n] = P^T · Q over the 128 samples of two resident 128-row tiles: the 64 columns of P
// become D's rows, the n columns of Q its columns, and the tiles' row (sample) index is the
// reduction. Both tiles are read MN-major (SBO = 16 core matrices down the tile = 2048 bytes
// between 8-column blocks, LBO = 128 bytes between 8-sample blocks); K steps of 16 samples
// advance 256 bytes. Thread 0 only; commits to mbar.
__device__ __forceinline__ void issue_gemm_tn(const uint8_t* p, const uint8_t* q, uint32_t n, uint32_t tmem,
                                              uint64_t* mbar) {
  const uint32_t p_addr = tc::smem_u32(p), q_addr = tc::smem_u32(q);
  constexpr uint32_t sbo = (kTile / 8) * 128, lbo = 128;
  const uint32_t idesc = tc::idesc_bf16_mn(64, n);
  for (uint32_t s = 0; s < kTile / 16; ++s)
    tc::mma_bf16(tmem, tc::make_desc(p_addr + s * 2 * lbo, lbo, sbo), tc::make_desc(q_addr + s * 2 * lbo, lbo, sbo),
                 idesc, s > 0 ? 1u : 0u);
  tc::mma_commit(mbar);
}

// All threads: waits for the committed GEMM; false (and the error bit) if it never completes.
__device__ __forceinline__ bool wait_gemm(uint64_t* mbar, uint32_t& phase, uint32_t* err) {
  bool ok = tc::mbar_wait(mbar, phase);
  ok = __syncthreads_and(ok);
  if (!ok && threadIdx.x == 0) atomicOr(err, kErrMma);
  phase ^= 1u;
  tc::fence_after_sync();
  return ok;
}

// This thread's 64 accumulator columns (its TMEM lane is its row).
__device__ __forceinline__ void read_acc64(uint32_t tmem, float* v) {
  const uint32_t lane = (threadIdx.x >> 5) * 32u;
#pragma unroll
  for (int c = 0; c < 64; c += 16) tc::tmem_ld16(tmem + (lane << 16) + uint32_t(c), v + c);
}

__device__ __forceinline__ void load_smem(uint8_t* dst, const uint16_t* src, uint32_t bytes) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (uint32_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = __ldg(s + i);
}

__device__ __forceinline__ void setup_tmem(uint64_t* mbar, uint32_t* tslot, uint32_t ncols = kTmemCols) {
  if (threadIdx.x == 0) tc::mbar_init(mbar, 1);
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tslot, ncols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

__device__ __forceinline__ void release_tmem(uint32_t tmem, uint64_t* mbar, uint32_t phase, bool ok,
                                             uint32_t ncols = kTmemCols) {
  if (!ok) tc::mbar_wait(mbar, phase, 1u << 20);  // one more bounded wait for a GEMM still in flight
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(tmem, ncols);
}

// Inference: one CTA per SM holds the weights once and runs kInferGroups independent tile
// groups of 128 threads (four warps), each with its own activation tile, mbarrier, named
// barrier and 64 TMEM columns, so six tiles' GEMM chains are in flight per SM: while one
// group waits on its GEMM the others encode, read TMEM or store activations. (Three CTAs of
// one tile each, every CTA with its own copy of the weights, was the shared-memory limit.)
constexpr int kInferGroups = 6;  // 7 (72 registers, spills) measured 4 % slower
constexpr int kInferThreads = kInferGroups * kTile;  // 768
constexpr uint32_t kInferTmemCols = 512;             // 6 x 64 columns, rounded up to a power of two
static_assert(kInferGroups * kTmemCols <= kInferTmemCols, "the groups' accumulators must fit the allocation");

// Named barrier g + 1 over the 128 threads of tile group g (barrier 0 is __syncthreads).
__device__ __forceinline__ void group_sync(uint32_t g) {
  asm volatile("bar.sync %0, %1;" ::"r"(g + 1u), "r"(uint32_t(kTile)) : "memory");
}
// The same barrier, returning whether `v` holds in every thread of the group.
__device__ __forceinline__ bool group_and(uint32_t g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(uint32_t(v)), "r"(g + 1u), "r"(uint32_t(kTile))
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(kInferThreads, 1) k_mlp_infer(Net net, Bounds b, const float* __restrict__ rec,
                                                                uint64_t n, const uint32_t* __restrict__ n_dev,
                                                                float* __restrict__ out, uint32_t* err) {
  if (n_dev) n = min(n, uint64_t(*n_dev));  // a count the previous kernel left on the device
  if (uint64_t(blockIdx.x) * kInferGroups * kTile >= n) return;  // before any barrier or TMEM allocation
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sW = smem;
  const uint32_t g = threadIdx.x / kTile, r = threadIdx.x % kTile;
  // The group's tile: the hidden activations overwrite the input features (a layer's GEMM has
  // finished reading its A operand before any thread stores the next layer's, and the next
  // tile's features are stored only after the last layer's GEMM has completed).
  uint8_t* sX = sW + kWBytes + g * kXBytes;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(sW + kWBytes + kInferGroups * kXBytes);
  uint64_t* mbar = mbars + g;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbars + kInferGroups);
  load_smem(sW, net.wpk_fwd, kWBytes);
  if (r == 0) tc::mbar_init(mbar, 1);
  if (threadIdx.x < 32) {
    tc::tmem_alloc(tslot, kInferTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot + g * kTmemCols;                // this group's 64 columns
  const uint32_t lane_base = ((threadIdx.x >> 5) & 3u) * 32u;  // this warp's TMEM lanes = rows
  uint32_t phase = 0;
  bool ok = true;
  const uint64_t tiles = (n + kTile - 1) / kTile;
  const uint64_t tile_step = uint64_t(gridDim.x) * kInferGroups;
  // A row's record, loaded one tile ahead: the next tile's loads are in flight while this
  // tile's features are encoded and its GEMM chain runs.
  auto load_record = [&](uint64_t t, float4& a, float4& b1, float4& c1, float4& d1) {
    const uint64_t rw = t * kTile + r;
    if (t < tiles && rw < n) {
      const float4* qr = reinterpret_cast<const float4*>(rec + rw * kRecord);
      a = __ldg(qr);
      b1 = __ldg(qr + 1);
      c1 = __ldg(qr + 2);
      d1 = __ldg(qr + 3);
    } else {
      a = b1 = c1 = d1 = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  float4 n0, n1, n2, n3;
  load_record(uint64_t(blockIdx.x) * kInferGroups + g, n0, n1, n2, n3);
  for (uint64_t tile = uint64_t(blockIdx.x) * kInferGroups + g; tile < tiles && ok; tile += tile_step) {
    const uint64_t row = tile * kTile + r;
    {
      // encode(): the features in 8-column chunks, 3 axes x 3 chunks of sin/cos bands, then the
      // 10 record values, without a 96-value array in registers
      const float4 q0 = n0, q1 = n1, q2 = n2, q3 = n3;
      load_record(tile + tile_step, n0, n1, n2, n3);
      const bool valid = row < n;
      const float p[3] = {q0.x, q0.y, q0.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float sn, cs;
        sincospi_poly(__fmul_rn(__fsub_rn(p[a], b.lo[a]), b.inv_extent[a]), sn, cs);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float v[8];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            v[2 * j] = valid ? sn : 0.f;
            v[2 * j + 1] = valid ? cs : 0.f;
            next_octave(sn, cs);
          }
          uint4 qq;
          qq.x = pack2(v[0], v[1]);
          qq.y = pack2(v[2], v[3]);
          qq.z = pack2(v[4], v[5]);
          qq.w = pack2(v[6], v[7]);
          *reinterpret_cast<uint4*>(sX + tc::tile_offset(r, uint32_t(a * 24 + c * 8), kTile)) = qq;
        }
      }
      uint4 qa, qb;
      const uint4 qz = make_uint4(0u, 0u, 0u, 0u);
      qa.x = pack2(q1.x, q1.y);
      qa.y = pack2(q1.z, q2.x);
      qa.z = pack2(q2.y, q2.z);
      qa.w = pack2(q3.x, q3.y);
      qb.x = pack2(q3.z, q0.w);
      qb.y = 0u;
      qb.z = 0u;
      qb.w = 0u;
      *reinterpret_cast<uint4*>(sX + tc::tile_offset(r, 72u, kTile)) = qa;
      *reinterpret_cast<uint4*>(sX + tc::tile_offset(r, 80u, kTile)) = qb;
      *reinterpret_cast<uint4*>(sX + tc::tile_offset(r, 88u, kTile)) = qz;
    }
    tc::fence_smem_to_async();
    group_sync(g);
    for (int l = 0; l < kLayers && ok; ++l) {
      if (r == 0) {
        tc::fence_after_sync();
        issue_gemm(sX, sW + 2 * layer_off(l), uint32_t(layer_n(l)), uint32_t(layer_k(l)), tmem, mbar);
      }
      ok = group_and(g, tc::mbar_wait(mbar, phase));
      if (!ok) {
        if (r == 0) atomicOr(err, kErrMma);
        break;
      }
      phase ^= 1u;
      tc::fence_after_sync();
      if (l < kLayers - 1) {
#pragma unroll
        for (int c = 0; c < 64; c += 16) {
          float v[16];
          tc::tmem_ld16(tmem + (lane_base << 16) + uint32_t(c), v);
          uint4 lo, hi;
          lo.x = pack2_relu(v[0], v[1]);
          lo.y = pack2_relu(v[2], v[3]);
          lo.z = pack2_relu(v[4], v[5]);
          lo.w = pack2_relu(v[6], v[7]);
          hi.x = pack2_relu(v[8], v[9]);
          hi.y = pack2_relu(v[10], v[11]);
          hi.z = pack2_relu(v[12], v[13]);
          hi.w = pack2_relu(v[14], v[15]);
          *reinterpret_cast<uint4*>(sX + tc::tile_offset(r, uint32_t(c), kTile)) = lo;
          *reinterpret_cast<uint4*>(sX + tc::tile_offset(r, uint32_t(c + 8), kTile)) = hi;
        }
        tc::fence_before_sync();
        tc::fence_smem_to_async();
        group_sync(g);
      } else {
        float v[16];
        tc::tmem_ld16(tmem + (lane_base << 16), v);
        if (row < n) {
          out[3 * row] = v[0];
          out[3 * row + 1] = v[1];
          out[3 * row + 2] = v[2];
        }
        tc::fence_before_sync();
        group_sync(g);
      }
    }
  }
  if (!ok) tc::mbar_wait(mbar, phase, 1u << 20);  // one more bounded wait for a GEMM still in flight
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) tc::tmem_dealloc(*tslot, kInferTmemCols);
}

__global__ void __launch_bounds__(kTile, 1) k_mlp_grad(Net net, Bounds b, const float* __restrict__ rec,
                                                        const float* __restrict__ tgt, uint64_t n, float grad_scale,
                                                        float* __restrict__ partials, float* __restrict__ tile_loss,
                                                        uint32_t* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sWf = smem;
  uint8_t* sWb = sWf + kWBytes;
  uint8_t* sX = sWb + kWBytes;
  uint8_t* sA = sX + kXBytes;          // activations A_1..A_5, kHBytes each
  uint8_t* sG = sA + 5 * kHBytes;      // layer gradient (64 wide)
  uint8_t* sG16 = sG + kHBytes;        // output gradient (16 wide)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sG16 + kG16Bytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  float* s_loss = reinterpret_cast<float*>(tslot + 1);
  load_smem(sWf, net.wpk_fwd, kWBytes);
  load_smem(sWb, net.wpk_bwd, kWBytes);
  if (threadIdx.x == 0) *s_loss = 0.f;
  setup_tmem(mbar, tslot, kTrainTmemCols);
  const uint32_t tmem = *tslot;
  uint32_t phase = 0;
  bool ok = true;
  const uint64_t tile = blockIdx.x;
  const uint32_t r = threadIdx.x;
  const uint64_t row = tile * kTile + r;
  auto act = [&](int l) -> uint8_t* { return l == 0 ? sX : sA + (l - 1) * kHBytes; };

  {
    float f[kInPad];
    if (row < n) {
      encode(rec + row * kRecord, b, f);
    } else {
#pragma unroll
      for (int k = 0; k < kInPad; ++k) f[k] = 0.f;
    }
    store_row(sX, r, f, kInPad);
    tc::fence_smem_to_async();
    __syncthreads();
  }
  // forward, keeping every activation
  float o[3] = {0.f, 0.f, 0.f};
  for (int l = 0; l < kLayers && ok; ++l) {
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      issue_gemm(act(l), sWf + 2 * layer_off(l), uint32_t(layer_n(l)), uint32_t(layer_k(l)), tmem, mbar);
    }
    ok = wait_gemm(mbar, phase, err);
    if (!ok) break;
    if (l < kLayers - 1) {
      float v[64];
      read_acc64(tmem, v);
#pragma unroll
      for (int c = 0; c < 64; ++c) v[c] = fmaxf(v[c], 0.f);
      store_row(act(l + 1), r, v, 64);
      tc::fence_before_sync();
      tc::fence_smem_to_async();
      __syncthreads();
    } else {
      float v[16];
      tc::tmem_ld16(tmem + (((threadIdx.x >> 5) * 32u) << 16), v);
      o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
      tc::fence_before_sync();
      __syncthreads();
    }
  }
  if (ok) {
    // relative L2 loss and its gradient (the denominator is held constant)
    float g[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) g[c] = 0.f;
    float loss = 0.f;
    if (row < n) {
      for (int c = 0; c < 3; ++c) {
        const float d = o[c] - __ldg(tgt + 3 * row + c);
        const float w = 1.0f / (o[c] * o[c] + 0.01f);
        loss += d * d * w;
        g[c] = 2.0f * d * w * grad_scale;
      }
    }
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(s_loss, loss);
    store_row(sG16, r, g, 16);
    tc::fence_smem_to_async();
    __syncthreads();
  }
  // backward
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t quarter = (warp * 32u) << 16;  // this warp's TMEM lanes
  for (int l = kLayers - 1; l >= 0 && ok; --l) {
    const int N = layer_n(l), K = layer_k(l);
    const uint8_t* G = (l == kLayers - 1) ? sG16 : sG;
    const uint8_t* A = act(l);
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      // dA_l = G_l · W_l, (128 x K) with K = 64, into columns 0-63
      if (l > 0) issue_gemm(G, sWb + 2 * layer_off(l), uint32_t(K), uint32_t(N), tmem, nullptr);
      // dW_l = G_lᵀ · A_l (64 x K), or for the 16-row output layer dW_lᵀ = A_lᵀ · G_l (64 x 16)
      if (l < kLayers - 1)
        issue_gemm_tn(G, A, uint32_t(K), tmem + kWgradCol, mbar);
      else
        issue_gemm_tn(A, G, uint32_t(N), tmem + kWgradCol, mbar);
    }
    ok = wait_gemm(mbar, phase, err);
    if (!ok) break;
    {
      // M = 64 accumulator: lanes 0-15 of warp q hold rows 16q .. 16q + 15
      const uint32_t row = warp * 16u + lane;
      float* dst = partials + tile * uint64_t(kParams) + layer_off(l);
      const int cols = l < kLayers - 1 ? K : N;
      for (int c = 0; c < cols; c += 16) {
        float v[16];
        tc::tmem_ld16(tmem + quarter + kWgradCol + uint32_t(c), v);
        if (lane < 16) {
          if (l < kLayers - 1) {  // row = output unit o, columns = inputs i
#pragma unroll
            for (int j = 0; j < 16; j += 4)
              *reinterpret_cast<float4*>(dst + row * uint32_t(K) + uint32_t(c + j)) =
                  make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
          } else {  // transposed: row = input i, columns = outputs o
#pragma unroll
            for (int j = 0; j < 16; ++j) dst[uint32_t(c + j) * uint32_t(K) + row] = v[j];
          }
        }
      }
    }
    if (l > 0) {
      float v[64];
      read_acc64(tmem, v);
#pragma unroll
      for (int c = 0; c < 64; ++c) v[c] = tile_at(A, r, uint32_t(c), kTile) > 0.f ? v[c] : 0.f;
      store_row(sG, r, v, 64);
      tc::fence_smem_to_async();
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_loss[tile] = *s_loss;
  release_tmem(tmem, mbar, phase, ok, kTrainTmemCols);
}

__global__ void k_reduce(const float* __restrict__ partials, const float* __restrict__ tile_loss, uint32_t tiles,
                         float* __restrict__ grad, float* __restrict__ loss) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < uint32_t(kParams)) {
    float s = 0.f;
    for (uint32_t t = 0; t < tiles; ++t) s += partials[uint64_t(t) * kParams + p];
    grad[p] = s;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float s = 0.f;
    for (uint32_t t = 0; t < tiles; ++t) s += tile_loss[t];
    *loss = s;
  }
}

__device__ __forceinline__ void pack_one(uint32_t p, float w, uint16_t* fwd, uint16_t* bwd) {
  int l = 0;
  while (l + 1 < kLayers && uint32_t(layer_off(l + 1)) <= p) ++l;
  const uint32_t local = p - uint32_t(layer_off(l));
  const uint32_t K = uint32_t(layer_k(l)), N = uint32_t(layer_n(l));
  const uint32_t o = local / K, i = local % K;
  const uint16_t bits = to_bf16(w);
  fwd[layer_off(l) + tc::tile_offset(o, i, N) / 2] = bits;
  bwd[layer_off(l) + tc::tile_offset(i, o, K) / 2] = bits;
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grad, float c1, float c2, float lr, float b1, float b2, float eps,
                       uint16_t* fwd, uint16_t* bwd, const uint32_t* __restrict__ active) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= uint32_t(kParams)) return;
  if (active && *active == 0) return;  // no training data this step
  // Rounded operations spelled out (no contraction) so the step is reproducible on the host.
  const float g = grad[p];
  const float mm = __fadd_rn(__fmul_rn(b1, m[p]), __fmul_rn(1.0f - b1, g));
  const float vv = __fadd_rn(__fmul_rn(b2, v[p]), __fmul_rn(__fmul_rn(1.0f - b2, g), g));
  m[p] = mm;
  v[p] = vv;
  const float step = __fdiv_rn(__fmul_rn(lr, __fdiv_rn(mm, c1)), __fadd_rn(__fsqrt_rn(__fdiv_rn(vv, c2)), eps));
  const float ww = __fsub_rn(w[p], step);
  w[p] = ww;
  pack_one(p, ww, fwd, bwd);
}

__global__ void k_pack(const float* __restrict__ w, uint16_t* fwd, uint16_t* bwd) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < uint32_t(kParams)) pack_one(p, w[p], fwd, bwd);
}

size_t infer_smem_bytes() { return kWBytes + kInferGroups * kXBytes + kInferGroups * 8 + 16; }
size_t train_smem_bytes() { return 2 * kWBytes + kXBytes + 5 * kHBytes + kHBytes + kG16Bytes + 64; }

cudaError_t launch_infer(const Net& net, const Bounds& b, const float* records, uint64_t n, float* out, uint32_t* err,
                         int sm_count, cudaStream_t s) {
  return launch_infer_dev(net, b, records, nullptr, n, out, err, sm_count, s);
}

// The dynamic shared-memory limit of a kernel is a per-device attribute: set it once on each
// device the kernel runs on (one bit per device; setting it twice is harmless).
static cudaError_t allow_smem(std::atomic<uint64_t>& done, const void* kernel, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev >= 0 && dev < 64 ? uint64_t(1) << dev : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

cudaError_t launch_infer_dev(const Net& net, const Bounds& b, const float* records, const uint32_t* n_dev,
                             uint64_t n, float* out, uint32_t* err, int sm_count, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  static std::atomic<uint64_t> configured{0};
  cudaError_t e = allow_smem(configured, reinterpret_cast<const void*>(k_mlp_infer), infer_smem_bytes());
  if (e != cudaSuccess) return e;
  const uint64_t ctas = (n + uint64_t(kInferGroups) * kTile - 1) / (uint64_t(kInferGroups) * kTile);
  const uint64_t cap = uint64_t(sm_count);  // one CTA (six tile groups) per SM
  k_mlp_infer<<<unsigned(ctas < cap ? ctas : cap), kInferThreads, infer_smem_bytes(), s>>>(net, b, records, n, n_dev,
                                                                                           out, err);
  return cudaGetLastError();
}

cudaError_t launch_grad_tiles(const Net& net, const Bounds& b, const float* records, const float* targets, uint64_t n,
                              float grad_scale, float* partials, float* tile_loss, uint32_t* err, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  static std::atomic<uint64_t> configured{0};
  cudaError_t e = allow_smem(configured, reinterpret_cast<const void*>(k_mlp_grad), train_smem_bytes());
  if (e != cudaSuccess) return e;
  const uint64_t tiles = (n + kTile - 1) / kTile;
  k_mlp_grad<<<unsigned(tiles), kTile, train_smem_bytes(), s>>>(net, b, records, targets, n, grad_scale, partials,
                                                                 tile_loss, err);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const float* partials, const float* tile_loss, uint32_t tiles, float* grad, float* loss,
                          cudaStream_t s) {
  k_reduce<<<(kParams + 255) / 256, 256, 0, s>>>(partials, tile_loss, tiles, grad, loss);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* w, float* m, float* v, const float* grad, uint32_t step, float lr, float beta1,
                        float beta2, float eps, uint16_t* wpk_fwd, uint16_t* wpk_bwd, cudaStream_t s,
                        const uint32_t* active) {
  const float c1 = 1.0f - powf(beta1, float(step)), c2 = 1.0f - powf(beta2, float(step));
  k_adam<<<(kParams + 255) / 256, 256, 0, s>>>(w, m, v, grad, c1, c2, lr, beta1, beta2, eps, wpk_fwd, wpk_bwd,
                                               active);
  return cudaGetLastError();
}

cudaError_t launch_pack(const float* w, uint16_t* wpk_fwd, uint16_t* wpk_bwd, cudaStream_t s) {
  k_pack<<<(kParams + 255) / 256, 256, 0, s>>>(w, wpk_fwd, wpk_bwd);
  return cudaGetLastError();
}

}  // namespace mlp
}  // namespace pbrt
