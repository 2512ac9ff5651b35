// kernels_trace.cu — batched ray-cast kernels (nearest hit / any hit) over one mesh.
//
// Ray planes are read and results written with streaming cache hints (each byte is touched
// once), so L1/L2 stay dedicated to the tree and triangles, which every ray revisits.
//
// The nearest-hit pass on a batch runs in two stages:
//   1. k_cull_root streams every ray once (four rays per thread, 16-byte loads), tests the
//      root box, writes a miss for every ray, and appends the rays that enter the root to a
//      queue with one atomicAdd per block, each with a 32-byte copy of the ray beside its
//      index (when a record buffer is given), so that stage 2 reads its rays coalesced
//      instead of gathering eight planes per ray;
//   2. k_mesh_closest_persistent: persistent warps over the queue, idle lanes refilled with
//      ballot/popc and one atomicAdd per warp once 8 are idle; each iteration is one
//      warp-voted step: a burst of up to 8 interior nodes for the lanes on interior nodes
//      or, once 8 lanes stand on a leaf (or no lane has interior work), a leaf step for those.
//      k_mesh_closest_ww is the classic while-while schedule it replaced (interior nodes
//      until every lane stands on a leaf, then all leaves), kept for measurements. Each lane
//      still visits its nodes in the reference's order, so ids and t stay bit-exact either way.
// k_mesh_closest (one thread per ray) is the instrumented form that counts the work.
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "kernels.hpp"
#include "tcgen05.cuh"
#include "trace_mesh.cuh"

namespace pbrt {

template <bool kCount>
__global__ void __launch_bounds__(128) k_mesh_closest(MeshView m, const float* __restrict__ rays, uint64_t stride,
                                                      uint64_t n, uint32_t* __restrict__ prim, float* __restrict__ tout,
                                                      uint32_t* __restrict__ obj, unsigned long long* __restrict__ counters,
                                                      uint32_t* __restrict__ err) {
  const uint64_t step = uint64_t(gridDim.x) * blockDim.x;
  unsigned long long acc[3] = {0, 0, 0};
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += step) {
    const F3 o = mk3(__ldcs(rays + i), __ldcs(rays + stride + i), __ldcs(rays + 2 * stride + i));
    const F3 d = mk3(__ldcs(rays + 3 * stride + i), __ldcs(rays + 4 * stride + i), __ldcs(rays + 5 * stride + i));
    const float near = __ldcs(rays + 6 * stride + i), far = __ldcs(rays + 7 * stride + i);
    const PRay r = prepare_ray(o, d);
    TraceCounters c{0, 0, 0};
    float t;
    const uint32_t id = mesh_closest<kCount>(m, r, near, far, &t, &c, err);
    __stcs(prim + i, id);
    __stcs(tout + i, id == 0xFFFFFFFFu ? __int_as_float(0x7f800000) : t);
    if (obj) __stcs(obj + i, id == 0xFFFFFFFFu ? 0xFFFFFFFFu : 0u);
    if (kCount) {
      acc[0] += c.nodes_visited;
      acc[1] += c.box_tests;
      acc[2] += c.triangle_tests;
    }
  }
  if (kCount) {
    // Every lane reaches this point, so a full-warp reduction is safe.
    for (int k = 0; k < 3; ++k) {
      unsigned long long v = acc[k];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if ((threadIdx.x & 31) == 0 && v) atomicAdd(&counters[k], v);
    }
  }
}

__global__ void __launch_bounds__(128) k_mesh_any(MeshView m, const float* __restrict__ rays, uint64_t stride, uint64_t n,
                                                  uint8_t* __restrict__ occ, uint32_t* __restrict__ err) {
  const uint64_t step = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += step) {
    const F3 o = mk3(__ldcs(rays + i), __ldcs(rays + stride + i), __ldcs(rays + 2 * stride + i));
    const F3 d = mk3(__ldcs(rays + 3 * stride + i), __ldcs(rays + 4 * stride + i), __ldcs(rays + 5 * stride + i));
    const float near = __ldcs(rays + 6 * stride + i), far = __ldcs(rays + 7 * stride + i);
    const PRay r = prepare_ray(o, d);
    occ[i] = mesh_any(m, r, near, far, err) ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------------------
// Stage 1: root-box cull and compaction.
// ---------------------------------------------------------------------------------------
constexpr int kCullThreads = 256;
constexpr int kCullRays = 4;  // rays per thread and iteration

// kVec: every plane and every output pointer is 16-byte aligned and the plane stride is a
// multiple of 4, so a thread's four rays are one float4 per plane.
// kDense: no miss answers; instead each block iteration (one 1,024-ray chunk) writes the
// chunk's survivor bitmask (32 words, bit i = ray chunk * 1024 + i entered the root) and the
// queue position of its first survivor; the queue itself is not needed (the traversal writes
// results by queue position and k_dense_finalize maps them back to rays).
static_assert(kDenseChunk == uint64_t(kCullThreads) * kCullRays, "a dense chunk is one cull block iteration");
// Registers: the plain form is left unbounded (54; an explicit minimum of one block per SM
// lets ptxas take 77); the dense form is bounded to 4 blocks per SM (64 instead of 78).
template <bool kVec, bool kDense>
__global__ void __launch_bounds__(kCullThreads, kDense ? 4 : 0) k_cull_root(MeshView m, const float* __restrict__ rays, uint64_t stride,
                                                            uint64_t n, uint32_t* __restrict__ prim,
                                                            float* __restrict__ tout, uint32_t* __restrict__ obj,
                                                            uint32_t* __restrict__ queue,
                                                            unsigned long long* __restrict__ queue_count,
                                                            float4* __restrict__ rec, uint32_t* __restrict__ mask,
                                                            uint32_t* __restrict__ bases) {
  __shared__ uint32_t warp_off[2][kCullThreads / 32];
  __shared__ unsigned long long blk_base[2];
  const float4 rlo = __ldg(&m.nodes[0]);
  const float4 rhi = __ldg(&m.nodes[1]);
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint64_t per_iter = uint64_t(gridDim.x) * blockDim.x * kCullRays;  // blockDim.x <= kCullThreads
  const uint64_t iters = (n + per_iter - 1) / per_iter;  // uniform across the grid: __syncthreads is safe
  for (uint64_t it = 0; it < iters; ++it) {
    const uint64_t i0 = it * per_iter + (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) * kCullRays;
    float v[8][kCullRays];
    const bool full = i0 + kCullRays <= n;
    if (kVec && full) {
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const float4 q = __ldcs(reinterpret_cast<const float4*>(rays + p * stride + i0));
        v[p][0] = q.x; v[p][1] = q.y; v[p][2] = q.z; v[p][3] = q.w;
      }
    } else {
#pragma unroll
      for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int j = 0; j < kCullRays; ++j) v[p][j] = (i0 + j < n) ? __ldcs(rays + p * stride + i0 + j) : 0.f;
    }
    unsigned enter = 0;
#pragma unroll
    for (int j = 0; j < kCullRays; ++j) {
      if (i0 + j < n) {
        float entry;
        const PRay r = prepare_ray(mk3(v[0][j], v[1][j], v[2][j]), mk3(v[3][j], v[4][j], v[5][j]));
        // entered, and not dropped at its first pop for entry >= min_t = FLT_MAX (bvh.rs:462-472)
        if (box_hit(r, rlo, rhi, v[6][j], v[7][j], entry) && entry < FLT_MAX) enter |= 1u << j;
      }
    }
    const uint64_t chunk = it * gridDim.x + blockIdx.x;
    if (kDense) {  // the 4-bit survivor nibbles of 8 lanes form one mask word
      uint32_t word = uint32_t(enter) << ((lane & 7u) * 4u);
      word |= __shfl_xor_sync(0xffffffffu, word, 1);
      word |= __shfl_xor_sync(0xffffffffu, word, 2);
      word |= __shfl_xor_sync(0xffffffffu, word, 4);
      if ((lane & 7u) == 0 && chunk * kDenseChunk < n) mask[chunk * 32 + warp * 4 + (lane >> 3)] = word;
    } else if (kVec && full) {  // every ray gets the miss answer now; stage 2 overwrites the rays it traverses
      __stcs(reinterpret_cast<uint4*>(prim + i0), make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu));
      const float inf = __int_as_float(0x7f800000);
      __stcs(reinterpret_cast<float4*>(tout + i0), make_float4(inf, inf, inf, inf));
      if (obj)
        __stcs(reinterpret_cast<uint4*>(obj + i0), make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu));
    } else if (!kDense) {
      for (int j = 0; j < kCullRays; ++j)
        if (i0 + j < n) {
          __stcs(prim + i0 + j, 0xFFFFFFFFu);
          __stcs(tout + i0 + j, __int_as_float(0x7f800000));
          if (obj) __stcs(obj + i0 + j, 0xFFFFFFFFu);
        }
    }
    // Block-wide exclusive scan of the survivor counts: one atomicAdd per block.
    const uint32_t c = __popc(enter);
    uint32_t incl = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= unsigned(off)) incl += y;
    }
    const int buf = int(it & 1);
    if (lane == 31) warp_off[buf][warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int w = 0; w < int(blockDim.x / 32); ++w) {
        const uint32_t t = warp_off[buf][w];
        warp_off[buf][w] = run;
        run += t;
      }
      blk_base[buf] = run ? atomicAdd(queue_count, (unsigned long long)run) : 0ull;
      if (kDense && chunk * kDenseChunk < n) bases[chunk] = uint32_t(blk_base[buf]);
    }
    __syncthreads();
    uint64_t pos = blk_base[buf] + warp_off[buf][warp] + (incl - c);
#pragma unroll
    for (int j = 0; j < kCullRays; ++j)
      if (enter & (1u << j)) {
        if (rec) {  // read back soon by stage 2: default caching, the planes stream past
          rec[2 * pos] = make_float4(v[0][j], v[1][j], v[2][j], v[6][j]);
          rec[2 * pos + 1] = make_float4(v[3][j], v[4][j], v[5][j], v[7][j]);
        }
        if (!kDense) queue[pos] = uint32_t(i0 + j);
        ++pos;
      }
  }
}

// The cull with its rays staged through shared memory by bulk asynchronous copies (the plain
// cp.async.bulk, no tensor map, no multicast), double-buffered: while a block tests, scans and
// compacts one 512-ray chunk, the next chunk's eight plane segments (2 KB each) are already on
// their way. The answers are k_cull_root's (same tests, same compaction, same records).
// Requires kVec's alignment (planes and outputs 16-byte aligned, stride a multiple of 4). The
// last, partial chunk is read directly. A copy wait that runs out of its budget sets kErrCopy.
constexpr int kBulkThreads = 128;
constexpr uint32_t kBulkChunk = kBulkThreads * kCullRays;  // rays per chunk
constexpr uint32_t kBulkPlaneBytes = kBulkChunk * 4;         // one plane's segment

__global__ void __launch_bounds__(kBulkThreads) k_cull_root_bulk(MeshView m, const float* __restrict__ rays,
                                                                 uint64_t stride, uint64_t n,
                                                                 uint32_t* __restrict__ prim, float* __restrict__ tout,
                                                                 uint32_t* __restrict__ obj, uint32_t* __restrict__ queue,
                                                                 unsigned long long* __restrict__ queue_count,
                                                                 float4* __restrict__ rec, uint32_t* __restrict__ err) {
  __shared__ __align__(128) float sbuf[2][8][kBulkChunk];  // 32 KB
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t warp_off[2][kBulkThreads / 32];
  __shared__ unsigned long long blk_base[2];
  const float4 rlo = __ldg(&m.nodes[0]);
  const float4 rhi = __ldg(&m.nodes[1]);
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint64_t full_chunks = n / kBulkChunk;  // chunks read by bulk copies
  const uint64_t chunks = (n + kBulkChunk - 1) / kBulkChunk;
  const uint64_t iters = (chunks + gridDim.x - 1) / gridDim.x;  // uniform across the grid
  // thread 0 starts chunk c's copies into buffer b (c < full_chunks)
  auto issue = [&](uint64_t c, int b) {
    tc::fence_smem_to_async();  // the buffer's previous contents were read by ordinary loads
    tc::mbar_arrive_expect_tx(&mbar[b], 8u * kBulkPlaneBytes);
#pragma unroll
    for (int p = 0; p < 8; ++p) tc::bulk_g2s(&sbuf[b][p][0], rays + p * stride + c * kBulkChunk, kBulkPlaneBytes, &mbar[b]);
  };
  if (threadIdx.x == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    if (uint64_t(blockIdx.x) < full_chunks) issue(blockIdx.x, 0);
  }
  __syncthreads();
  bool copies_ok = true;  // false after a wait ran out: this thread reads directly from then on
  for (uint64_t it = 0; it < iters; ++it) {
    const uint64_t c = uint64_t(blockIdx.x) + it * gridDim.x;
    const int b = int(it & 1);
    // The next chunk's copies go out now; its buffer was last read in the previous
    // iteration, before that iteration's barriers.
    if (threadIdx.x == 0 && c + gridDim.x < full_chunks) issue(c + gridDim.x, b ^ 1);
    const uint64_t i0 = c * kBulkChunk + uint64_t(threadIdx.x) * kCullRays;
    float v[8][kCullRays];
    // buffer b's (it >> 1)-th use: full chunks come first, so every earlier use was a copy
    if (c < full_chunks && copies_ok && !tc::mbar_wait(&mbar[b], uint32_t((it >> 1) & 1u))) {
      atomicOr(err, kErrCopy);
      copies_ok = false;
    }
    if (c < full_chunks && copies_ok) {
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const float4 q = *reinterpret_cast<const float4*>(&sbuf[b][p][threadIdx.x * kCullRays]);
        v[p][0] = q.x; v[p][1] = q.y; v[p][2] = q.z; v[p][3] = q.w;
      }
    } else {
#pragma unroll
      for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int j = 0; j < kCullRays; ++j) v[p][j] = (i0 + j < n) ? __ldcs(rays + p * stride + i0 + j) : 0.f;
    }
    unsigned enter = 0;
#pragma unroll
    for (int j = 0; j < kCullRays; ++j) {
      if (i0 + j < n) {
        float entry;
        const PRay r = prepare_ray(mk3(v[0][j], v[1][j], v[2][j]), mk3(v[3][j], v[4][j], v[5][j]));
        // entered, and not dropped at its first pop for entry >= min_t = FLT_MAX (bvh.rs:462-472)
        if (box_hit(r, rlo, rhi, v[6][j], v[7][j], entry) && entry < FLT_MAX) enter |= 1u << j;
      }
    }
    if (i0 + kCullRays <= n) {  // every ray gets the miss answer now; stage 2 overwrites the hits
      __stcs(reinterpret_cast<uint4*>(prim + i0), make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu));
      const float inf = __int_as_float(0x7f800000);
      __stcs(reinterpret_cast<float4*>(tout + i0), make_float4(inf, inf, inf, inf));
      if (obj)
        __stcs(reinterpret_cast<uint4*>(obj + i0), make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu));
    } else {
      for (int j = 0; j < kCullRays; ++j)
        if (i0 + j < n) {
          __stcs(prim + i0 + j, 0xFFFFFFFFu);
          __stcs(tout + i0 + j, __int_as_float(0x7f800000));
          if (obj) __stcs(obj + i0 + j, 0xFFFFFFFFu);
        }
    }
    // Block-wide exclusive scan of the survivor counts: one atomicAdd per block.
    const uint32_t cnt = __popc(enter);
    uint32_t incl = cnt;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= unsigned(off)) incl += y;
    }
    if (lane == 31) warp_off[b][warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int w = 0; w < kBulkThreads / 32; ++w) {
        const uint32_t t = warp_off[b][w];
        warp_off[b][w] = run;
        run += t;
      }
      blk_base[b] = run ? atomicAdd(queue_count, (unsigned long long)run) : 0ull;
    }
    __syncthreads();
    uint64_t pos = blk_base[b] + warp_off[b][warp] + (incl - cnt);
#pragma unroll
    for (int j = 0; j < kCullRays; ++j)
      if (enter & (1u << j)) {
        if (rec) {  // read back soon by stage 2: default caching
          rec[2 * pos] = make_float4(v[0][j], v[1][j], v[2][j], v[6][j]);
          rec[2 * pos + 1] = make_float4(v[3][j], v[4][j], v[5][j], v[7][j]);
        }
        queue[pos] = uint32_t(i0 + j);
        ++pos;
      }
  }
}

// ---------------------------------------------------------------------------------------
// Stage 2: persistent traversal of the survivors.
// ---------------------------------------------------------------------------------------
struct TraversalStack {
  uint32_t lf[kTraceStack];
  uint32_t cnt[kTraceStack];
  float e[kTraceStack];
};

// Next node to visit after a leaf or a node with no child worth visiting: pops, dropping
// entries whose entry distance is >= min_t (bvh.rs:470-472). False when the stack is empty.
PBRT_DEV bool pop_next(TraversalStack& s, int& sp, float min_t, uint32_t& lf, uint32_t& count) {
  while (sp > 0) {
    --sp;
    if (s.e[sp] < min_t) {
      lf = s.lf[sp];
      count = s.cnt[sp];
      return true;
    }
  }
  return false;
}

// Resident 128-thread blocks per SM the traversal kernels are compiled for (the register cap
// follows: 10 -> 48 registers a thread).
#ifndef PBRT_TRAVERSAL_MIN_BLOCKS
#define PBRT_TRAVERSAL_MIN_BLOCKS 10
#endif

// The while-while schedule: refill the idle lanes, walk interior nodes until every lane
// stands on a leaf (or its ray is finished), then test the leaves of all lanes in one pass.
// Compiled for PBRT_TRAVERSAL_MIN_BLOCKS resident blocks per SM: for this schedule 12 blocks
// (40 registers) measured 1.01 ms against 1.10 ms at the compiler's 72 registers for the
// 16M-ray step.
template <bool kRec>
__global__ void __launch_bounds__(128, PBRT_TRAVERSAL_MIN_BLOCKS) k_mesh_closest_ww(MeshView m, const float* __restrict__ rays,
                                                                 uint64_t stride, const uint32_t* __restrict__ queue,
                                                                 const unsigned long long* __restrict__ queue_count,
                                                                 uint32_t* __restrict__ prim,
                                                                 float* __restrict__ tout, uint32_t* __restrict__ obj,
                                                                 unsigned long long* __restrict__ next_ray,
                                                                 uint32_t* __restrict__ err,
                                                                 const float4* __restrict__ rec) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  const uint64_t n = *queue_count;
  bool active = false;
  uint32_t idx = 0;
  PRay r;
  float near = 0.f, far = 0.f, min_t = FLT_MAX;
  uint32_t best = 0xFFFFFFFFu, lf = 0, count = 0, budget = 0;
  int sp = 0;
  TraversalStack stk;
  const uint32_t root_lf = __float_as_uint(__ldg(&m.nodes[0]).w);
  const uint32_t root_cnt = __float_as_uint(__ldg(&m.nodes[1]).w);

  for (;;) {
    // Refill the lanes whose ray is finished: one atomicAdd per warp.
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    bool exhausted = false;
    if (idle) {
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if (int(lane) == leader) base = atomicAdd(next_ray, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, leader);
      exhausted = base + __popc(idle) >= n;
      if (!active) {
        const uint64_t k = base + __popc(idle & lt_mask);
        if (k < n) {
          idx = __ldg(queue + k);
          F3 o, d;
          if (kRec) {  // the copy stage 1 wrote: consecutive lanes read consecutive records
            const float4 a = __ldcs(rec + 2 * k), b = __ldcs(rec + 2 * k + 1);
            o = mk3(a.x, a.y, a.z);
            d = mk3(b.x, b.y, b.z);
            near = a.w;
            far = b.w;
          } else {
            o = mk3(__ldg(rays + idx), __ldg(rays + stride + idx), __ldg(rays + 2 * stride + idx));
            d = mk3(__ldg(rays + 3 * stride + idx), __ldg(rays + 4 * stride + idx), __ldg(rays + 5 * stride + idx));
            near = __ldg(rays + 6 * stride + idx);
            far = __ldg(rays + 7 * stride + idx);
          }
          r = prepare_ray(o, d);
          min_t = FLT_MAX;
          best = 0xFFFFFFFFu;
          lf = root_lf;  // the root entered the ray's interval in stage 1 (bvh.rs:458-461)
          count = root_cnt;
          sp = 0;
          budget = m.node_count;
          active = true;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, active) == 0) {
      if (exhausted) break;
      continue;
    }
    if (active) {
      bool done = false;
      // Interior walk until this lane stands on a leaf (or its ray is finished).
      while (count == 0) {
        if (budget-- == 0) {
          atomicOr(err, kErrBudget);
          done = true;
          break;
        }
        float4 l0, l1, r0, r1;
        load_node(&m.nodes[2 * lf], l0, l1);
        load_node(&m.nodes[2 * lf + 2], r0, r1);
        float dl, dr;
        const bool hl = box_hit(r, l0, l1, near, far, dl);
        const bool hr = box_hit(r, r0, r1, near, far, dr);
        const bool swap = hl && hr && dr < dl;  // right first only when strictly nearer
        const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
        const float dn = swap ? dr : dl, df = swap ? dl : dr;
        const bool take_f = hf && df < min_t;
        const bool take_n = hn && dn < min_t;
        if (take_n) {
          if (take_f) {
            if (sp >= kTraceStack) {
              atomicOr(err, kErrStack);
              done = true;
              break;
            }
            stk.lf[sp] = __float_as_uint(swap ? l0.w : r0.w);
            stk.cnt[sp] = __float_as_uint(swap ? l1.w : r1.w);
            stk.e[sp] = df;
            ++sp;
          }
          lf = __float_as_uint(swap ? r0.w : l0.w);
          count = __float_as_uint(swap ? r1.w : l1.w);
        } else if (take_f) {
          lf = __float_as_uint(swap ? l0.w : r0.w);
          count = __float_as_uint(swap ? l1.w : r1.w);
        } else if (!pop_next(stk, sp, min_t, lf, count)) {
          done = true;
          break;
        }
      }
      // Leaf: every lane that reached one tests its triangles in the same pass.
      if (!done) {
        if (budget-- == 0) {
          atomicOr(err, kErrBudget);
          done = true;
        } else {
          for (uint32_t k = lf; k < lf + count; ++k) {
            const float4 A = __ldg(&m.tri_a[k]);
            const float4 B = __ldg(&m.tri_b[k]);
            const float2 C = __ldg(&m.tri_c[k]);
            float t;
            if (tri_hit(r, A, B, C.x, t) && t < min_t && t >= near && t <= far) {
              min_t = t;
              best = __float_as_uint(C.y);
            }
          }
          if (!pop_next(stk, sp, min_t, lf, count)) done = true;
        }
      }
      if (done) {
        if (best != 0xFFFFFFFFu) {  // stage 1 already wrote the miss answer
          __stcs(prim + idx, best);
          __stcs(tout + idx, min_t);
          if (obj) __stcs(obj + idx, 0u);
        }
        active = false;
      }
    }
  }
}

// One warp-voted step per iteration: either a node step for the lanes standing on an
// interior node (up to `burst` nodes each, fewer when a lane reaches a leaf) or a leaf step
// for the lanes standing on a leaf, never both. A leaf step is taken once at least `leaf_min`
// lanes stand on a leaf (or no lane has interior work left); until then the lanes on a leaf
// wait and the others keep descending. Idle lanes are refilled from the queue once at least
// `refill_min` of them are idle (or all are). Waiting for every lane to reach a leaf before
// any leaf is tested (the classic while-while loop) left 3/4 of the lanes idle on this
// workload; this schedule keeps most lanes on interior nodes, where the work is, and the
// bursts spread the vote's cost over several nodes (single-node steps lost to while-while).
// Each lane still visits its nodes in the reference's order, so ids and t are unchanged.
//
// 10 resident blocks of 128 threads per SM (at most 48 registers a thread, 4 bytes spilled):
// 0.882-0.887 ms per 16M-ray step against 0.888-0.894 at 9 blocks (56 registers), 0.897-0.900
// at 8 (64, no spill), 0.928-0.932 at 12 (40, 64 bytes spilled) and 1.146-1.152 at 13-16
// (32, 176 bytes spilled): the stack spills cost more than the extra warps hide.
// kDense (with records): a lane's result goes to its queue slot in `res` (every survivor, hit
// or miss) instead of to its ray's place in prim / tout; the queue's ray indices are not read.
template <bool kRec, bool kDense>
__global__ void __launch_bounds__(128, PBRT_TRAVERSAL_MIN_BLOCKS) k_mesh_closest_persistent(
    MeshView m, const float* __restrict__ rays, uint64_t stride, const uint32_t* __restrict__ queue,
    const unsigned long long* __restrict__ queue_count, uint32_t* __restrict__ prim, float* __restrict__ tout,
    uint32_t* __restrict__ obj, unsigned long long* __restrict__ next_ray, uint32_t* __restrict__ err,
    const float4* __restrict__ rec, int leaf_min, int refill_min, int burst, uint2* __restrict__ res) {
  static_assert(kRec || !kDense, "dense results need the ray records");
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  const uint64_t n = *queue_count;
  bool active = false, exhausted = false;  // exhausted is warp-uniform
  uint32_t idx = 0;
  PRay r;
  float near = 0.f, far = 0.f, min_t = FLT_MAX;
  uint32_t best = 0xFFFFFFFFu, lf = 0, count = 0, budget = 0;
  int sp = 0;
  TraversalStack stk;
  const uint32_t root_lf = __float_as_uint(__ldg(&m.nodes[0]).w);
  const uint32_t root_cnt = __float_as_uint(__ldg(&m.nodes[1]).w);

  for (;;) {
    // Refill the idle lanes: one atomicAdd per warp.
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if (int(lane) == leader) base = atomicAdd(next_ray, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, leader);
      exhausted = base + __popc(idle) >= n;
      if (!active) {
        const uint64_t k = base + __popc(idle & lt_mask);
        if (k < n) {
          idx = kDense ? uint32_t(k) : __ldg(queue + k);  // dense: the queue slot (results go there)
          F3 o, d;
          if (kRec) {  // the copy stage 1 wrote: consecutive lanes read consecutive records
            const float4 a = __ldcs(rec + 2 * k), b = __ldcs(rec + 2 * k + 1);
            o = mk3(a.x, a.y, a.z);
            d = mk3(b.x, b.y, b.z);
            near = a.w;
            far = b.w;
          } else {
            o = mk3(__ldg(rays + idx), __ldg(rays + stride + idx), __ldg(rays + 2 * stride + idx));
            d = mk3(__ldg(rays + 3 * stride + idx), __ldg(rays + 4 * stride + idx), __ldg(rays + 5 * stride + idx));
            near = __ldg(rays + 6 * stride + idx);
            far = __ldg(rays + 7 * stride + idx);
          }
          r = prepare_ray(o, d);
          min_t = FLT_MAX;
          best = 0xFFFFFFFFu;
          lf = root_lf;  // the root entered the ray's interval in stage 1 (bvh.rs:458-461)
          count = root_cnt;
          sp = 0;
          budget = m.node_count;
          active = true;
        }
      }
    }
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (act == 0) {
      if (exhausted) break;
      continue;  // all idle and the queue not yet drained: the next iteration refills
    }
    const unsigned on_leaf = __ballot_sync(0xffffffffu, active && count > 0);
    // (leaf_min and burst carry the schedule of the drained queue in their second byte)
    const int lmin = exhausted ? (leaf_min >> 8) : (leaf_min & 255);
    const bool leaf_step = __popc(on_leaf) >= lmin || on_leaf == act;
    bool done = false;
    if (active && (count > 0) == leaf_step) {
      if (budget-- == 0) {
        atomicOr(err, kErrBudget);
        done = true;
      } else if (leaf_step) {
        for (uint32_t k = lf; k < lf + count; ++k) {
          const float4 A = __ldg(&m.tri_a[k]);
          const float4 B = __ldg(&m.tri_b[k]);
          const float2 C = __ldg(&m.tri_c[k]);
          float t;
          if (tri_hit(r, A, B, C.x, t) && t < min_t && t >= near && t <= far) {
            min_t = t;
            best = __float_as_uint(C.y);
          }
        }
        if (!pop_next(stk, sp, min_t, lf, count)) done = true;
      } else {
        // up to `burst` interior nodes before the next vote (fewer when a leaf is reached)
        const int nb = exhausted ? (burst >> 8) : (burst & 255);
        for (int b = 0; b < nb && !done && count == 0; ++b) {
          if (b > 0 && budget-- == 0) {
            atomicOr(err, kErrBudget);
            done = true;
            break;
          }
          float4 l0, l1, r0, r1;
          load_node(&m.nodes[2 * lf], l0, l1);
          load_node(&m.nodes[2 * lf + 2], r0, r1);
          float dl, dr;
          const bool hl = box_hit(r, l0, l1, near, far, dl);
          const bool hr = box_hit(r, r0, r1, near, far, dr);
          const bool swap = hl && hr && dr < dl;  // right first only when strictly nearer
          const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
          const float dn = swap ? dr : dl, df = swap ? dl : dr;
          const bool take_f = hf && df < min_t;
          const bool take_n = hn && dn < min_t;
          if (take_n) {
            if (take_f) {
              if (sp >= kTraceStack) {
                atomicOr(err, kErrStack);
                done = true;
                break;
              }
              stk.lf[sp] = __float_as_uint(swap ? l0.w : r0.w);
              stk.cnt[sp] = __float_as_uint(swap ? l1.w : r1.w);
              stk.e[sp] = df;
              ++sp;
            }
            lf = __float_as_uint(swap ? r0.w : l0.w);
            count = __float_as_uint(swap ? r1.w : l1.w);
          } else if (take_f) {
            lf = __float_as_uint(swap ? l0.w : r0.w);
            count = __float_as_uint(swap ? l1.w : r1.w);
          } else if (!pop_next(stk, sp, min_t, lf, count)) {
            done = true;
          }
        }
      }
    }
    if (done) {
      if (kDense) {
        res[idx] = make_uint2(best, best != 0xFFFFFFFFu ? __float_as_uint(min_t) : 0x7f800000u);
      } else if (best != 0xFFFFFFFFu) {  // stage 1 already wrote the miss answer
        __stcs(prim + idx, best);
        __stcs(tout + idx, min_t);
        if (obj) __stcs(obj + idx, 0u);
      }
      active = false;
    }
  }
}

// The persistent traversal's schedule: the voted kernel with a leaf step once `leaf_min`
// lanes of a warp stand on a leaf, a refill once `refill_min` lanes are idle and up to
// `burst` interior nodes per node step (default 8, 8, 8: 0.913 ms per 16,777,216-ray step
// against 1.021 ms for the while-while kernel and 1.052 ms for single-node steps), or the
// while-while kernel (voted = false). Once the queue is drained no refill can come, and a
// lane waiting on a leaf only lengthens the tail: there a leaf step is taken as soon as one
// lane stands on a leaf (tail_leaf_min 1: 1.7 % faster than keeping 8).
// PBRT_TRACE_SCHEDULE="ww" or "leaf_min,refill_min[,burst[,tail_leaf_min[,tail_burst]]]"
// (each in 1..32; without tail values the bulk's apply) overrides it for measurements;
// results do not depend on it. `dense` (PBRT_TRACE_DENSE=1, when the caller gives its scratch): the
// voted kernel's results go out through the dense pass instead of the cull's miss answers
// plus scattered hit stores. On the 16,777,216-ray step it cuts DRAM traffic from 997 MB to
// 851 MB but takes 0.923-0.926 ms against 0.916-0.920 ms: the cull saves 18 us by writing
// no answers, the ray-order pass costs 37 us, and the hit stores it replaces were hidden
// under the issue-bound traversal.
struct TraversalSchedule {
  bool voted = true, dense = false;
  int leaf_min = 8, refill_min = 8, burst = 8;
  int tail_leaf_min = 1, tail_burst = 8;  // once the queue is drained (no refill can come)
  int leaf_arg() const { return leaf_min | (tail_leaf_min << 8); }
  int burst_arg() const { return burst | (tail_burst << 8); }
};

static TraversalSchedule traversal_schedule() {
  static const TraversalSchedule v = [] {
    TraversalSchedule d;
    if (const char* e = std::getenv("PBRT_TRACE_SCHEDULE")) {
      int a = 0, b = 0, c = 1, ta = 0, tc = 0;
      const int got = std::sscanf(e, "%d,%d,%d,%d,%d", &a, &b, &c, &ta, &tc);
      if (std::strcmp(e, "ww") == 0) {
        d.voted = false;
      } else if (got >= 2 && a >= 1 && a <= 32 && b >= 1 && b <= 32 && c >= 1 && c <= 32) {
        d.leaf_min = a;
        d.refill_min = b;
        d.burst = got >= 3 ? c : 1;
        d.tail_leaf_min = got >= 4 && ta >= 1 && ta <= 32 ? ta : d.leaf_min;
        d.tail_burst = got >= 5 && tc >= 1 && tc <= 32 ? tc : d.burst;
      }
    }
    if (const char* e = std::getenv("PBRT_TRACE_DENSE")) d.dense = std::strcmp(e, "1") == 0;
    return d;
  }();
  return v;
}

// Stage 3 of the dense form: every ray's answer in ray order. One block per 1,024-ray chunk:
// the chunk's 32 mask words and their exclusive prefix popcounts in shared memory; thread t
// owns rays 4t .. 4t + 3 of the chunk, finds its survivors' ranks and reads their results
// from consecutive queue slots, and writes 4 ids and 4 distances as one 16-byte store each.
template <bool kVec>
__global__ void __launch_bounds__(kCullThreads) k_dense_finalize(const uint2* __restrict__ res,
                                                                 const uint32_t* __restrict__ mask,
                                                                 const uint32_t* __restrict__ bases, uint64_t n,
                                                                 uint32_t* __restrict__ prim, float* __restrict__ tout,
                                                                 uint32_t* __restrict__ obj) {
  __shared__ uint32_t msk[32], pre[32];
  const uint64_t chunks = (n + kDenseChunk - 1) / kDenseChunk;
  const uint32_t t = threadIdx.x, lane = t & 31u;
  for (uint64_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    if (t < 32) {
      const uint32_t w = __ldg(mask + ch * 32 + t);
      const uint32_t c = __popc(w);
      uint32_t incl = c;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= unsigned(off)) incl += y;
      }
      msk[t] = w;
      pre[t] = incl - c;
    }
    __syncthreads();
    const uint32_t w = t >> 3, sh = (t & 7u) * 4u;
    const uint32_t word = msk[w], bits = (word >> sh) & 0xFu;
    uint64_t rank = uint64_t(__ldg(bases + ch)) + pre[w] + __popc(word & ((1u << sh) - 1u));
    const uint64_t i0 = ch * kDenseChunk + 4u * t;
    uint32_t p[4];
    float tt[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      p[j] = 0xFFFFFFFFu;
      tt[j] = __int_as_float(0x7f800000);
      if (bits & (1u << j)) {
        const uint2 r = __ldg(res + rank);
        ++rank;
        p[j] = r.x;
        tt[j] = __uint_as_float(r.y);
      }
    }
    if (kVec && i0 + 4 <= n) {
      __stcs(reinterpret_cast<uint4*>(prim + i0), make_uint4(p[0], p[1], p[2], p[3]));
      __stcs(reinterpret_cast<float4*>(tout + i0), make_float4(tt[0], tt[1], tt[2], tt[3]));
      if (obj)
        __stcs(reinterpret_cast<uint4*>(obj + i0),
               make_uint4(p[0] != 0xFFFFFFFFu ? 0u : 0xFFFFFFFFu, p[1] != 0xFFFFFFFFu ? 0u : 0xFFFFFFFFu,
                          p[2] != 0xFFFFFFFFu ? 0u : 0xFFFFFFFFu, p[3] != 0xFFFFFFFFu ? 0u : 0xFFFFFFFFu));
    } else {
      for (int j = 0; j < 4; ++j)
        if (i0 + j < n) {
          __stcs(prim + i0 + j, p[j]);
          __stcs(tout + i0 + j, tt[j]);
          if (obj) __stcs(obj + i0 + j, p[j] != 0xFFFFFFFFu ? 0u : 0xFFFFFFFFu);
        }
    }
    __syncthreads();  // msk and pre are reused by the next chunk
  }
}

static unsigned grid_for(uint64_t n, int threads, int sm_count) {
  const uint64_t want = (n + threads - 1) / threads;
  const uint64_t cap = uint64_t(sm_count) * 64;  // grid-stride beyond this
  return unsigned(want < cap ? (want ? want : 1) : cap);
}

cudaError_t launch_mesh_closest(const MeshView& m, const float* rays, uint64_t stride, uint64_t n, uint32_t* prim,
                                float* t, uint32_t* obj, unsigned long long* counters, uint32_t* err, int sm_count,
                                cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned g = grid_for(n, 128, sm_count);
  if (counters)
    k_mesh_closest<true><<<g, 128, 0, s>>>(m, rays, stride, n, prim, t, obj, counters, err);
  else
    k_mesh_closest<false><<<g, 128, 0, s>>>(m, rays, stride, n, prim, t, obj, nullptr, err);
  return cudaGetLastError();
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Resident 128-thread blocks per SM of the persistent traversal (the same on every B200);
// computed once, thread-safely, by the first launch.
template <bool kRec>
static int persistent_blocks_per_sm() {
  static const int v = [] {
    int b = 0;
    const cudaError_t e =
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_mesh_closest_persistent<kRec, false>, 128, 0);
    return e == cudaSuccess && b > 0 ? b : 8;
  }();
  return v;
}

cudaError_t launch_mesh_closest_persistent(const MeshView& m, const float* rays, uint64_t stride, uint64_t n,
                                           uint32_t* prim, float* t, uint32_t* obj, uint32_t* queue,
                                           unsigned long long* counters, uint32_t* err, int sm_count, cudaStream_t s,
                                           float4* rec, const DenseScratch* dense) {
  if (n == 0) return cudaSuccess;
  const int blocks_per_sm = persistent_blocks_per_sm<true>();
  cudaError_t e = cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  const bool vec = stride % 4 == 0 && aligned16(rays) && aligned16(prim) && aligned16(t) && (!obj || aligned16(obj));
  const uint64_t per_block = uint64_t(kCullThreads) * kCullRays;
  const uint64_t cull_need = (n + per_block - 1) / per_block, cull_cap = uint64_t(sm_count) * 8;
  const unsigned cg = unsigned(cull_need < cull_cap ? cull_need : cull_cap);
  const uint64_t full = uint64_t(sm_count) * blocks_per_sm;
  const uint64_t need = (n + 127) / 128;
  const unsigned g = unsigned(need < full ? need : full);
  const TraversalSchedule ts = traversal_schedule();
  if (ts.voted && ts.dense && rec && vec && dense && dense->res && dense->mask && dense->bases) {
    // dense results: cull (bitmask, chunk bases, records), traversal (results by queue slot),
    // then every ray's answer in ray order
    k_cull_root<true, true><<<cg, kCullThreads, 0, s>>>(m, rays, stride, n, prim, t, obj, queue, counters, rec,
                                                         dense->mask, dense->bases);
    k_mesh_closest_persistent<true, true><<<g, 128, 0, s>>>(m, rays, stride, queue, counters, prim, t, obj,
                                                            counters + 1, err, rec, ts.leaf_arg(), ts.refill_min,
                                                            ts.burst_arg(), dense->res);
    k_dense_finalize<true><<<cg, kCullThreads, 0, s>>>(dense->res, dense->mask, dense->bases, n, prim, t, obj);
    return cudaGetLastError();
  }
  // The cull staged through shared memory by bulk copies (k_cull_root_bulk) whenever the
  // planes are aligned: 0.8 % faster per 16M-ray step than direct loads (three alternating
  // pairs). PBRT_CULL_BULK=0 selects the direct-load cull for measurements.
  static const bool cull_bulk = [] {
    const char* e = std::getenv("PBRT_CULL_BULK");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  if (vec && cull_bulk) {
    static const int bulk_per_sm = [] {
      int b = 0;
      const cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cull_root_bulk, kBulkThreads, 0);
      return oe == cudaSuccess && b > 0 ? b : 4;
    }();
    const uint64_t bneed = (n + kBulkChunk - 1) / kBulkChunk, bcap = uint64_t(sm_count) * bulk_per_sm;
    k_cull_root_bulk<<<unsigned(bneed < bcap ? bneed : bcap), kBulkThreads, 0, s>>>(m, rays, stride, n, prim, t, obj,
                                                                                   queue, counters, rec, err);
  }
  // The cull in 128-thread blocks, twice as many as 256-thread ones: more independent
  // load / scan / atomicAdd chains per SM (0.5 % faster per 16M-ray step, three alternating
  // pairs). PBRT_CULL_THREADS=256 selects the larger blocks for measurements.
  static const unsigned cull_threads = [] {
    const char* e = std::getenv("PBRT_CULL_THREADS");
    return e && std::strcmp(e, "256") == 0 ? unsigned(kCullThreads) : 128u;
  }();
  const uint64_t cpb = uint64_t(cull_threads) * kCullRays;
  const uint64_t cneed = (n + cpb - 1) / cpb, ccap = uint64_t(sm_count) * 8 * (kCullThreads / cull_threads);
  const unsigned cgt = unsigned(cneed < ccap ? cneed : ccap);
  if (vec && !cull_bulk)
    k_cull_root<true, false><<<cgt, cull_threads, 0, s>>>(m, rays, stride, n, prim, t, obj, queue, counters, rec,
                                                           nullptr, nullptr);
  else if (!vec)
    k_cull_root<false, false><<<cgt, cull_threads, 0, s>>>(m, rays, stride, n, prim, t, obj, queue, counters, rec,
                                                            nullptr, nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (!ts.voted) {
    if (rec)
      k_mesh_closest_ww<true><<<g, 128, 0, s>>>(m, rays, stride, queue, counters, prim, t, obj, counters + 1, err, rec);
    else
      k_mesh_closest_ww<false><<<g, 128, 0, s>>>(m, rays, stride, queue, counters, prim, t, obj, counters + 1, err,
                                                 nullptr);
  } else if (rec) {
    k_mesh_closest_persistent<true, false><<<g, 128, 0, s>>>(m, rays, stride, queue, counters, prim, t, obj,
                                                             counters + 1, err, rec, ts.leaf_arg(), ts.refill_min,
                                                             ts.burst_arg(), nullptr);
  } else {
    k_mesh_closest_persistent<false, false><<<g, 128, 0, s>>>(m, rays, stride, queue, counters, prim, t, obj,
                                                              counters + 1, err, nullptr, ts.leaf_arg(), ts.refill_min,
                                                              ts.burst_arg(), nullptr);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of the two-stage nearest-hit pass.
//
// Its scratch (the two 64-bit counters, the device error word and the survivor queue) is
// this file-scope array instead of memory the context allocates: 256 header bytes plus
// kNoAllocMaxRays queue entries, i.e. 4 MiB + 256 B that every GPU which loads the library
// holds until the process exits. Header layout in 32-bit words: [0..1] queue length,
// [2..3] fetch position, [4] error word; the queue starts at word 64.
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) uint32_t g_noalloc_scratch[64 + kNoAllocMaxRays];

// Device address of g_noalloc_scratch on the current device (host code cannot use the
// symbol itself as a device address). The context looks it up when it is created, with its
// device current, and keeps it: a context made after a device reset gets the new address.
cudaError_t noalloc_scratch_lookup(uint32_t** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<uint32_t*>(p);
  return cudaSuccess;
}

cudaError_t launch_mesh_closest_noalloc(const MeshView& m, const float* rays, uint64_t n, uint32_t* prim, float* t,
                                        uint32_t* scratch, int sm_count, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (n > kNoAllocMaxRays || !scratch) return cudaErrorInvalidValue;
  // The array keeps the previous call's contents: the counters and the error word must
  // start at zero; the queue is written before it is read.
  cudaError_t e = cudaMemsetAsync(scratch, 0, 64 * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(scratch);
  uint32_t* err = scratch + 4;
  uint32_t* queue = scratch + 64;
  const int blocks_per_sm = persistent_blocks_per_sm<false>();
  const bool vec = n % 4 == 0 && aligned16(rays) && aligned16(prim) && aligned16(t);
  const uint64_t per_block = uint64_t(kCullThreads) * kCullRays;
  const uint64_t cull_need = (n + per_block - 1) / per_block, cull_cap = uint64_t(sm_count) * 8;
  const unsigned cg = unsigned(cull_need < cull_cap ? cull_need : cull_cap);
  if (vec)
    k_cull_root<true, false><<<cg, kCullThreads, 0, s>>>(m, rays, n, n, prim, t, nullptr, queue, counters, nullptr,
                                                          nullptr, nullptr);
  else
    k_cull_root<false, false><<<cg, kCullThreads, 0, s>>>(m, rays, n, n, prim, t, nullptr, queue, counters, nullptr,
                                                           nullptr, nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const uint64_t full = uint64_t(sm_count) * blocks_per_sm;
  const uint64_t need = (n + 127) / 128;
  const unsigned g = unsigned(need < full ? need : full);
  const TraversalSchedule ts = traversal_schedule();
  if (!ts.voted)
    k_mesh_closest_ww<false><<<g, 128, 0, s>>>(m, rays, n, queue, counters, prim, t, nullptr, counters + 1, err,
                                               nullptr);
  else
    k_mesh_closest_persistent<false, false><<<g, 128, 0, s>>>(m, rays, n, queue, counters, prim, t, nullptr,
                                                              counters + 1, err, nullptr, ts.leaf_arg(), ts.refill_min,
                                                              ts.burst_arg(), nullptr);
  return cudaGetLastError();
}

cudaError_t launch_mesh_any(const MeshView& m, const float* rays, uint64_t stride, uint64_t n, uint8_t* occ,
                            uint32_t* err, int sm_count, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mesh_any<<<grid_for(n, 128, sm_count), 128, 0, s>>>(m, rays, stride, n, occ, err);
  return cudaGetLastError();
}

}  // namespace pbrt
