// bvh_build_gpu.cu — a triangle mesh's BVH built on the GPU: node for node, and triangle for
// triangle in every leaf, the tree mesh_bvh.cpp builds on the host (and so the reference's
// binned-SAH tree, src/shapes/triangle_mesh/bvh.rs:221-309, 609-735).
//
// What has to be identical, and how it is kept so:
//   - the centroid extents, bins, SAH costs and split decisions: min / max / counts are
//     order-independent, and the cost arithmetic is the host's, operation for operation
//     (FP32, round-to-nearest intrinsics, no FMA);
//   - the order of the triangles inside every node: the host partitions with one forward
//     pass that swaps each left triangle to the front (bvh.rs:260-267). Its result is
//     computed here in parallel: a left triangle with ordinal q (q lefts before it) lands at
//     q; a right triangle at i >= nl (nl lefts in all) stays; a right triangle at p < nl moves
//     along p -> pos(p) -> pos(pos(p)) ... (pos(q) = where the left of ordinal q stands) to
//     the first position >= nl — resolved by pointer jumping;
//   - the node numbering: the host numbers nodes depth first (children pushed as a pair when
//     their parent splits, left subtree first); here nodes are made in any order and
//     renumbered from their subtree sizes;
//   - stored zero bounds are +0 in both builders (the sign of a zero bound depends on visiting
//     order and no slab test can observe it).
// Large nodes (more than kSmall triangles) are split level by level by many blocks at once;
// a subtree of at most kSmall triangles is built by one thread with the host's algorithm.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>

#include "bvh_build_gpu.hpp"

namespace pbrt {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kSmall = 96;      // subtrees of at most this many triangles: one thread each
constexpr uint32_t kChunk = 2048;    // elements per block in the level kernels
constexpr int kLevelThreads = 256;
constexpr int kMaxBins = 64;
constexpr uint32_t kMaxSubtreeStack = 128;
enum : uint32_t { kBuildErrInput = 1u, kBuildErrStack = 2u };

struct __align__(16) TriRec {
  float4 c;   // centroid xyz, w = bits of the original triangle index
  float4 lo;  // triangle box
  float4 hi;
};

struct PoolNode {  // a node in making, in any order; renumbered at the end
  float lo[3], hi[3];
  uint32_t first, count, depth, child;  // child: the left child's pool index (right = +1), or kNone
};

struct LevelNode {  // a large node split by the level kernels
  uint32_t pool, first, count, depth;
  uint32_t ext[6];  // orderable centroid min xyz, max xyz
  float cmin[3], width[3];
  uint32_t use;     // bit a: axis a has distinct centroids
  uint32_t split, axis, boundary, nl;
  uint32_t child;
  uint32_t cbox[2][6];  // orderable child boxes (lo xyz, hi xyz)
};

struct Chunk {
  uint32_t node, start, len;  // start relative to the node's first triangle
};

struct SmallJob {
  uint32_t pool, first, count, depth, buf;
};

struct LevelResult {  // what the host needs back from a level: the split and the children
  uint32_t split, nl, child, pad;
};

// ---- FP32 helpers (the host builder's expressions) ----------------------------------------
__device__ __forceinline__ float mn(float x, float y) { return y < x ? y : x; }
__device__ __forceinline__ float mx(float x, float y) { return x < y ? y : x; }
__device__ __forceinline__ float canon(float x) { return x == 0.0f ? 0.0f : x; }
// a monotone map of floats to unsigned integers, for atomic min / max
__device__ __forceinline__ uint32_t f2o(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}
__device__ __forceinline__ float half_area(const float* lo, const float* hi) {
  if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) return 0.0f;
  const float dx = __fsub_rn(hi[0], lo[0]), dy = __fsub_rn(hi[1], lo[1]), dz = __fsub_rn(hi[2], lo[2]);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}
// bin_index (bvh.rs:173-176) as the host restates it
__device__ __forceinline__ int bin_of(float pos, float cmin, float width, int bins) {
  const float q = __fdiv_rn(__fsub_rn(pos, cmin), width);
  if (!(q >= 0.0f)) return 0;
  if (q >= float(bins - 1)) return bins - 1;
  return int(q);
}
__device__ __forceinline__ float comp(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// ---- block reductions ---------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}
__device__ __forceinline__ uint32_t warp_max(uint32_t v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}
// Reduces k values per thread (min for the first half, max for the second) across the block
// and applies one atomic per value into dst.
template <int K>
__device__ void block_minmax_atomic(uint32_t (&v)[K], uint32_t* dst) {
  __shared__ uint32_t red[K][kLevelThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k < K; ++k) {
    const uint32_t r = k < K / 2 ? warp_min(v[k]) : warp_max(v[k]);
    if (lane == 0) red[k][w] = r;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    const int k = threadIdx.x;
    uint32_t r = red[k][0];
    for (int j = 1; j < kLevelThreads / 32; ++j) r = k < K / 2 ? min(r, red[k][j]) : max(r, red[k][j]);
    if (k < K / 2) atomicMin(dst + k, r);
    else atomicMax(dst + k, r);
  }
  __syncthreads();
}

// ---- preparation ----------------------------------------------------------------------------
// tri_centroid and aabound_from_triangle (bvh.rs:564-584) per triangle; bad input sets err
__global__ void k_tri_prep(const float* __restrict__ v, uint32_t nv, const uint32_t* __restrict__ idx, uint32_t n,
                           TriRec* __restrict__ out, uint32_t* err) {
  const float third = __fdiv_rn(1.0f, 3.0f);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t i0 = idx[3 * size_t(i)], i1 = idx[3 * size_t(i) + 1], i2 = idx[3 * size_t(i) + 2];
    if (i0 >= nv || i1 >= nv || i2 >= nv) {
      atomicOr(err, kBuildErrInput);
      out[i] = TriRec{};
      continue;
    }
    float p[3][3];
    for (int a = 0; a < 3; ++a) {
      p[0][a] = v[3 * size_t(i0) + a];
      p[1][a] = v[3 * size_t(i1) + a];
      p[2][a] = v[3 * size_t(i2) + a];
    }
    float c[3], lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = mn(mn(p[0][a], p[1][a]), p[2][a]);
      hi[a] = mx(mx(p[0][a], p[1][a]), p[2][a]);
      c[a] = __fmul_rn(__fadd_rn(__fadd_rn(p[0][a], p[1][a]), p[2][a]), third);
    }
    out[i] = TriRec{make_float4(c[0], c[1], c[2], __uint_as_float(i)), make_float4(lo[0], lo[1], lo[2], 0.f),
                    make_float4(hi[0], hi[1], hi[2], 0.f)};
  }
}

// vertex bounds (TriangleMesh::get_bounding_box) and finiteness of every coordinate
__global__ void k_vertex_bounds(const float* __restrict__ v, uint32_t nv, uint32_t* box, uint32_t* err) {
  uint32_t r[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
    for (int a = 0; a < 3; ++a) {
      const float x = v[3 * size_t(i) + a];
      if (!isfinite(x)) atomicOr(err, kBuildErrInput);
      const uint32_t o = f2o(canon(x));
      r[a] = min(r[a], o);
      r[3 + a] = max(r[3 + a], o);
    }
  block_minmax_atomic<6>(r, box);
}

// the root's box: bounds over every triangle (bvh.rs:232-238)
__global__ void k_root_box(const TriRec* __restrict__ t, uint32_t n, uint32_t* box) {
  uint32_t r[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const TriRec x = t[i];
    r[0] = min(r[0], f2o(canon(x.lo.x))); r[1] = min(r[1], f2o(canon(x.lo.y))); r[2] = min(r[2], f2o(canon(x.lo.z)));
    r[3] = max(r[3], f2o(canon(x.hi.x))); r[4] = max(r[4], f2o(canon(x.hi.y))); r[5] = max(r[5], f2o(canon(x.hi.z)));
  }
  block_minmax_atomic<6>(r, box);
}

__global__ void k_root_node(PoolNode* pool, const uint32_t* box, uint32_t n) {
  PoolNode& p = pool[0];
  for (int a = 0; a < 3; ++a) {
    p.lo[a] = canon(o2f(box[a]));
    p.hi[a] = canon(o2f(box[3 + a]));
  }
  p.first = 0;
  p.count = n;
  p.depth = 1;
  p.child = kNone;
}

// ---- the level kernels (large nodes) -------------------------------------------------------
__global__ void k_ext(const TriRec* __restrict__ t, LevelNode* nodes, const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  LevelNode& nd = nodes[ch.node];
  const uint32_t base = nd.first + ch.start;
  uint32_t r[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  for (uint32_t k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const float4 c = t[base + k].c;
    r[0] = min(r[0], f2o(c.x)); r[1] = min(r[1], f2o(c.y)); r[2] = min(r[2], f2o(c.z));
    r[3] = max(r[3], f2o(c.x)); r[4] = max(r[4], f2o(c.y)); r[5] = max(r[5], f2o(c.z));
  }
  block_minmax_atomic<6>(r, nd.ext);
}

// per node: the splittable axes and bin widths (find_best_split_plane's first lines), bins reset
__global__ void k_bin_prep(LevelNode* nodes, uint32_t nn, uint32_t* bins, int B) {
  const uint32_t j = blockIdx.x;
  if (j >= nn) return;
  LevelNode& nd = nodes[j];
  if (threadIdx.x == 0) {
    nd.use = 0;
    for (int a = 0; a < 3; ++a) {
      const float lo = o2f(nd.ext[a]), hi = o2f(nd.ext[3 + a]);
      nd.cmin[a] = lo;
      nd.width[a] = __fdiv_rn(__fsub_rn(hi, lo), float(B));
      if (!(lo == hi)) nd.use |= 1u << a;
    }
  }
  uint32_t* b = bins + size_t(j) * 3 * B * 7;
  for (int k = threadIdx.x; k < 3 * B; k += blockDim.x) {
    uint32_t* e = b + 7 * k;
    e[0] = e[1] = e[2] = f2o(FLT_MAX);
    e[3] = e[4] = e[5] = f2o(-FLT_MAX);
    e[6] = 0;
  }
}

// fill_bins (bvh.rs:694-711) for the three axes: box of the triangles whose centroid falls in
// each bin, and their count
__global__ void k_bins(const TriRec* __restrict__ t, const LevelNode* __restrict__ nodes,
                       const Chunk* __restrict__ chunks, uint32_t* bins, int B) {
  __shared__ uint32_t sb[3 * kMaxBins * 7];
  const Chunk ch = chunks[blockIdx.x];
  const LevelNode& nd = nodes[ch.node];
  for (int k = threadIdx.x; k < 3 * B; k += blockDim.x) {
    uint32_t* e = sb + 7 * k;
    e[0] = e[1] = e[2] = f2o(FLT_MAX);
    e[3] = e[4] = e[5] = f2o(-FLT_MAX);
    e[6] = 0;
  }
  __syncthreads();
  const uint32_t base = nd.first + ch.start;
  for (uint32_t k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const TriRec x = t[base + k];
    const uint32_t lo[3] = {f2o(x.lo.x), f2o(x.lo.y), f2o(x.lo.z)}, hi[3] = {f2o(x.hi.x), f2o(x.hi.y), f2o(x.hi.z)};
    for (int a = 0; a < 3; ++a) {
      if (!(nd.use & (1u << a))) continue;
      uint32_t* e = sb + 7 * (a * B + bin_of(comp(x.c, a), nd.cmin[a], nd.width[a], B));
      for (int q = 0; q < 3; ++q) {
        atomicMin(e + q, lo[q]);
        atomicMax(e + 3 + q, hi[q]);
      }
      atomicAdd(e + 6, 1u);
    }
  }
  __syncthreads();
  uint32_t* g = bins + size_t(ch.node) * 3 * B * 7;
  for (int k = threadIdx.x; k < 3 * B; k += blockDim.x) {
    const uint32_t* e = sb + 7 * k;
    if (e[6] == 0) continue;
    uint32_t* d = g + 7 * k;
    for (int q = 0; q < 3; ++q) {
      atomicMin(d + q, e[q]);
      atomicMax(d + 3 + q, e[3 + q]);
    }
    atomicAdd(d + 6, e[6]);
  }
}

// The split decision of one node from its bins, exactly as the host evaluates it: axes in
// order, boundaries in order, the first strictly cheapest candidate; `get(b, lo, hi)` gives
// bin b of the axis (its box) and returns its count.
struct Split {
  bool have;
  int axis, boundary;
  float cost;
};

template <class Get>
__device__ void eval_axis(int a, int B, Split& s, Get get) {
  const int S = B - 1;
  float la[kMaxBins];
  uint32_t lc[kMaxBins];
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  uint32_t sum = 0;
  for (int i = 0; i < S; ++i) {  // prefix unions: boundary i has bins 0..i on the left
    float blo[3], bhi[3];
    sum += get(i, blo, bhi);
    for (int q = 0; q < 3; ++q) {
      lo[q] = mn(lo[q], blo[q]);
      hi[q] = mx(hi[q], bhi[q]);
    }
    la[i] = half_area(lo, hi);
    lc[i] = sum;
  }
  float ra[kMaxBins];
  uint32_t rc[kMaxBins];
  for (int q = 0; q < 3; ++q) { lo[q] = FLT_MAX; hi[q] = -FLT_MAX; }
  sum = 0;
  for (int i = 0; i < S; ++i) {  // suffix unions from the far end: boundary m has bins m+1.. on the right
    const int m = S - 1 - i;
    float blo[3], bhi[3];
    sum += get(m + 1, blo, bhi);
    for (int q = 0; q < 3; ++q) {
      lo[q] = mn(lo[q], blo[q]);
      hi[q] = mx(hi[q], bhi[q]);
    }
    ra[m] = half_area(lo, hi);
    rc[m] = sum;
  }
  for (int b = 0; b < S; ++b) {
    if (lc[b] == 0 || rc[b] == 0) continue;
    const float cost = __fadd_rn(__fmul_rn(la[b], __uint2float_rn(lc[b])), __fmul_rn(ra[b], __uint2float_rn(rc[b])));
    if (!s.have || cost < s.cost) {
      s.have = true;
      s.axis = a;
      s.boundary = b;
      s.cost = cost;
    }
  }
}

__global__ void k_sah(LevelNode* nodes, uint32_t nn, const uint32_t* __restrict__ bins, int B, uint32_t max_leaf,
                      const PoolNode* __restrict__ pool) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nn) return;
  LevelNode& nd = nodes[j];
  nd.split = 0;
  nd.nl = 0;
  if (nd.count <= max_leaf) return;
  const PoolNode& p = pool[nd.pool];
  const float leaf_cost = __fmul_rn(half_area(p.lo, p.hi), __uint2float_rn(nd.count));
  const uint32_t* g = bins + size_t(j) * 3 * B * 7;
  Split s{false, 0, 0, 0.0f};
  for (int a = 0; a < 3; ++a) {
    if (!(nd.use & (1u << a))) continue;
    eval_axis(a, B, s, [&](int b, float* lo, float* hi) {
      const uint32_t* e = g + 7 * (a * B + b);
      for (int q = 0; q < 3; ++q) {
        lo[q] = o2f(e[q]);
        hi[q] = o2f(e[3 + q]);
      }
      return e[6];
    });
  }
  if (!s.have || !(s.cost < leaf_cost)) return;
  nd.split = 1;
  nd.axis = uint32_t(s.axis);
  nd.boundary = uint32_t(s.boundary);
}

// the partition's classification, a block-wide exclusive scan of the left flags per chunk
__global__ void k_classify(const TriRec* __restrict__ t, const LevelNode* __restrict__ nodes,
                           const Chunk* __restrict__ chunks, uint32_t* __restrict__ ord, uint32_t* chunk_tot, int B) {
  __shared__ uint32_t warp_tot[kLevelThreads / 32];
  __shared__ uint32_t carry;
  const Chunk ch = chunks[blockIdx.x];
  const LevelNode& nd = nodes[ch.node];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const uint32_t base = nd.first + ch.start;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t k0 = 0; k0 < ch.len; k0 += blockDim.x) {
    const uint32_t k = k0 + threadIdx.x;
    uint32_t f = 0;
    if (k < ch.len && nd.split)
      f = bin_of(comp(t[base + k].c, int(nd.axis)), nd.cmin[nd.axis], nd.width[nd.axis], B) <= int(nd.boundary);
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, f);
    const uint32_t in_warp = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[w] = __popc(bal);
    __syncthreads();
    uint32_t before = carry;
    for (int j = 0; j < w; ++j) before += warp_tot[j];
    if (k < ch.len) ord[base + k] = (before + in_warp) | (f ? 0x80000000u : 0u);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int j = 0; j < kLevelThreads / 32; ++j) carry += warp_tot[j];
    __syncthreads();
  }
  if (threadIdx.x == 0) chunk_tot[blockIdx.x] = carry;
}

// per node: the chunks' offsets in the lefts' order and nl; the children's places
__global__ void k_chunk_offsets(LevelNode* nodes, uint32_t nn, const uint32_t* __restrict__ cfirst,
                                uint32_t* chunk_tot, PoolNode* pool, uint32_t* pool_count, LevelResult* res) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nn) return;
  LevelNode& nd = nodes[j];
  res[j] = LevelResult{0, 0, kNone, 0};
  uint32_t run = 0;
  for (uint32_t c = cfirst[j]; c < cfirst[j + 1]; ++c) {
    const uint32_t v = chunk_tot[c];
    chunk_tot[c] = run;
    run += v;
  }
  nd.nl = run;
  for (int q = 0; q < 6; ++q) {
    nd.cbox[0][q] = nd.cbox[1][q] = q < 3 ? 0xFFFFFFFFu : 0u;
  }
  nd.child = kNone;
  if (!nd.split) return;
  if (run == 0 || run == nd.count) {  // unreachable: the bins counted both sides non-empty
    nd.split = 0;
    return;
  }
  const uint32_t c = atomicAdd(pool_count, 2u);
  nd.child = c;
  res[j] = LevelResult{1, run, c, 0};
  pool[nd.pool].child = c;
  pool[nd.pool].count = 0;
  PoolNode l{}, r{};
  l.first = nd.first;
  l.count = run;
  r.first = nd.first + run;
  r.count = nd.count - run;
  l.depth = r.depth = nd.depth + 1;
  l.child = r.child = kNone;
  pool[c] = l;
  pool[c + 1] = r;
}

// each left's ordinal in its node; pos[q] = where the left of ordinal q stands (relative)
__global__ void k_scatter(const LevelNode* __restrict__ nodes, const Chunk* __restrict__ chunks,
                          const uint32_t* __restrict__ chunk_off, uint32_t* ord, uint32_t* pos) {
  const Chunk ch = chunks[blockIdx.x];
  const LevelNode& nd = nodes[ch.node];
  if (!nd.split) return;
  const uint32_t base = nd.first + ch.start;
  for (uint32_t k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const uint32_t o = ord[base + k];
    const uint32_t q = chunk_off[blockIdx.x] + (o & 0x7FFFFFFFu);
    ord[base + k] = q | (o & 0x80000000u);
    if (o & 0x80000000u) pos[nd.first + q] = ch.start + k;
  }
}

// pointer jumping on pos[] over [0, nl): a misplaced right at p follows p -> pos(p) -> ... to
// the first position >= nl (its final place)
__global__ void k_jump(const LevelNode* __restrict__ nodes, const Chunk* __restrict__ chunks, uint32_t* pos,
                       uint32_t* changed) {
  const Chunk ch = chunks[blockIdx.x];
  const LevelNode& nd = nodes[ch.node];
  if (!nd.split) return;
  uint32_t any = 0;
  for (uint32_t k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const uint32_t q = ch.start + k;
    if (q >= nd.nl) break;
    const uint32_t j = pos[nd.first + q];
    if (j < nd.nl) {
      const uint32_t jj = pos[nd.first + j];
      if (jj != j) {
        pos[nd.first + q] = jj;
        any = 1;
      }
    }
  }
  if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(changed, 1u);
}

// the partition's result written to the next buffer; a node that does not split is final
__global__ void k_permute(const TriRec* __restrict__ cur, TriRec* __restrict__ nxt, TriRec* __restrict__ fin,
                          const LevelNode* __restrict__ nodes, const Chunk* __restrict__ chunks,
                          const uint32_t* __restrict__ ord, const uint32_t* __restrict__ pos) {
  const Chunk ch = chunks[blockIdx.x];
  const LevelNode& nd = nodes[ch.node];
  const uint32_t base = nd.first + ch.start;
  for (uint32_t k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const TriRec x = cur[base + k];
    if (!nd.split) {
      fin[base + k] = x;
      continue;
    }
    const uint32_t i = ch.start + k, o = ord[base + k];
    uint32_t dest;
    if (o & 0x80000000u) dest = o & 0x7FFFFFFFu;  // a left: its ordinal
    else if (i >= nd.nl) dest = i;                // a right already on the right
    else dest = pos[nd.first + i];                // a misplaced right: the end of its chain
    nxt[nd.first + dest] = x;
  }
}

// the children's boxes (bounds over their triangles, bvh.rs:232-238)
__global__ void k_child_box(const TriRec* __restrict__ nxt, LevelNode* nodes, const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  LevelNode& nd = nodes[ch.node];
  if (!nd.split) return;
  const uint32_t base = nd.first + ch.start;
  uint32_t r[2][6];
  for (int s = 0; s < 2; ++s)
    for (int q = 0; q < 6; ++q) r[s][q] = q < 3 ? 0xFFFFFFFFu : 0u;
  for (uint32_t k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const TriRec x = nxt[base + k];
    const int s = ch.start + k < nd.nl ? 0 : 1;
    r[s][0] = min(r[s][0], f2o(canon(x.lo.x))); r[s][1] = min(r[s][1], f2o(canon(x.lo.y)));
    r[s][2] = min(r[s][2], f2o(canon(x.lo.z)));
    r[s][3] = max(r[s][3], f2o(canon(x.hi.x))); r[s][4] = max(r[s][4], f2o(canon(x.hi.y)));
    r[s][5] = max(r[s][5], f2o(canon(x.hi.z)));
  }
  block_minmax_atomic<6>(r[0], nd.cbox[0]);
  block_minmax_atomic<6>(r[1], nd.cbox[1]);
}

__global__ void k_child_finalize(const LevelNode* __restrict__ nodes, uint32_t nn, PoolNode* pool) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nn) return;
  const LevelNode& nd = nodes[j];
  if (!nd.split) return;
  for (int s = 0; s < 2; ++s) {
    PoolNode& p = pool[nd.child + s];
    for (int a = 0; a < 3; ++a) {
      p.lo[a] = canon(o2f(nd.cbox[s][a]));
      p.hi[a] = canon(o2f(nd.cbox[s][3 + a]));
    }
  }
}

// ---- small subtrees: one thread runs the host's algorithm -----------------------------------
__device__ void range_box(const TriRec* t, uint32_t first, uint32_t count, float* lo, float* hi) {
  for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
  for (uint32_t k = first; k < first + count; ++k) {
    const TriRec x = t[k];
    lo[0] = mn(lo[0], x.lo.x); lo[1] = mn(lo[1], x.lo.y); lo[2] = mn(lo[2], x.lo.z);
    hi[0] = mx(hi[0], x.hi.x); hi[1] = mx(hi[1], x.hi.y); hi[2] = mx(hi[2], x.hi.z);
  }
  for (int a = 0; a < 3; ++a) { lo[a] = canon(lo[a]); hi[a] = canon(hi[a]); }
}

__global__ void __launch_bounds__(64) k_small(const SmallJob* __restrict__ jobs, uint32_t nj, const TriRec* b0,
                                              const TriRec* b1, TriRec* fin, PoolNode* pool, uint32_t* pool_count,
                                              int B, uint32_t max_leaf, uint32_t* err) {
  const uint32_t jid = blockIdx.x * blockDim.x + threadIdx.x;
  if (jid >= nj) return;
  const SmallJob jb = jobs[jid];
  const TriRec* src = jb.buf ? b1 : b0;
  for (uint32_t k = jb.first; k < jb.first + jb.count; ++k) fin[k] = src[k];
  uint32_t stack[kMaxSubtreeStack];
  int sp = 0;
  stack[sp++] = jb.pool;
  float blo[kMaxBins][3], bhi[kMaxBins][3];
  uint32_t bcnt[kMaxBins];
  while (sp > 0) {
    const uint32_t ni = stack[--sp];
    const uint32_t first = pool[ni].first, count = pool[ni].count;
    if (count <= max_leaf) continue;
    const float leaf_cost = __fmul_rn(half_area(pool[ni].lo, pool[ni].hi), __uint2float_rn(count));
    float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t k = first; k < first + count; ++k) {
      const float4 c = fin[k].c;
      cmin[0] = mn(cmin[0], c.x); cmin[1] = mn(cmin[1], c.y); cmin[2] = mn(cmin[2], c.z);
      cmax[0] = mx(cmax[0], c.x); cmax[1] = mx(cmax[1], c.y); cmax[2] = mx(cmax[2], c.z);
    }
    uint32_t use = 0;
    float width[3];
    for (int a = 0; a < 3; ++a) {
      if (!(cmin[a] == cmax[a])) use |= 1u << a;
      width[a] = __fdiv_rn(__fsub_rn(cmax[a], cmin[a]), float(B));
    }
    Split s{false, 0, 0, 0.0f};
    for (int a = 0; a < 3; ++a) {  // fill_bins per axis, then its candidates
      if (!(use & (1u << a))) continue;
      for (int b = 0; b < B; ++b) {
        for (int q = 0; q < 3; ++q) {
          blo[b][q] = FLT_MAX;
          bhi[b][q] = -FLT_MAX;
        }
        bcnt[b] = 0;
      }
      for (uint32_t k = first; k < first + count; ++k) {
        const TriRec x = fin[k];
        const int b = bin_of(comp(x.c, a), cmin[a], width[a], B);
        blo[b][0] = mn(blo[b][0], x.lo.x); blo[b][1] = mn(blo[b][1], x.lo.y); blo[b][2] = mn(blo[b][2], x.lo.z);
        bhi[b][0] = mx(bhi[b][0], x.hi.x); bhi[b][1] = mx(bhi[b][1], x.hi.y); bhi[b][2] = mx(bhi[b][2], x.hi.z);
        bcnt[b]++;
      }
      eval_axis(a, B, s, [&](int b, float* lo, float* hi) {
        for (int q = 0; q < 3; ++q) {
          lo[q] = blo[b][q];
          hi[q] = bhi[b][q];
        }
        return bcnt[b];
      });
    }
    if (!s.have || !(s.cost < leaf_cost)) continue;
    // forward-swap partition by bin index (bvh.rs:260-267)
    const float bm = cmin[s.axis], bw = width[s.axis];
    uint32_t left_end = first;
    for (uint32_t k = first; k < first + count; ++k) {
      if (bin_of(comp(fin[k].c, s.axis), bm, bw, B) <= s.boundary) {
        const TriRec tmp = fin[k];
        fin[k] = fin[left_end];
        fin[left_end] = tmp;
        left_end++;
      }
    }
    const uint32_t lcnt = left_end - first;
    if (lcnt == 0 || lcnt == count) continue;
    const uint32_t c = atomicAdd(pool_count, 2u);
    PoolNode l{}, r{};
    l.first = first;
    l.count = lcnt;
    r.first = left_end;
    r.count = count - lcnt;
    l.depth = r.depth = pool[ni].depth + 1;
    l.child = r.child = kNone;
    range_box(fin, l.first, l.count, l.lo, l.hi);
    range_box(fin, r.first, r.count, r.lo, r.hi);
    pool[c] = l;
    pool[c + 1] = r;
    pool[ni].child = c;
    pool[ni].count = 0;
    if (sp + 2 > int(kMaxSubtreeStack)) {
      atomicOr(err, kBuildErrStack);
      return;
    }
    stack[sp++] = c + 1;
    stack[sp++] = c;
  }
}

// ---- depth-first renumbering and the GPU layout -----------------------------------------------
// Nodes grouped by depth. Every node adds to one of a few dozen counters, so the lanes of a
// warp that share a depth (neighbouring nodes usually do) add once, together; the order
// within a depth does not matter to the sizes and numbers computed from it.
__global__ void k_depth_hist(const PoolNode* __restrict__ pool, uint32_t n, uint32_t* hist) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t dep = min(pool[i].depth, 255u);
    const unsigned peers = __match_any_sync(__activemask(), dep);
    if ((threadIdx.x & 31u) == unsigned(__ffs(peers) - 1)) atomicAdd(hist + dep, uint32_t(__popc(peers)));
  }
}
__global__ void k_depth_scatter(const PoolNode* __restrict__ pool, uint32_t n, uint32_t* cursor, uint32_t* by_depth) {
  const unsigned lane = threadIdx.x & 31u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t dep = min(pool[i].depth, 255u);
    const unsigned peers = __match_any_sync(__activemask(), dep);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(cursor + dep, uint32_t(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    by_depth[base + __popc(peers & ((1u << lane) - 1u))] = i;
  }
}
// subtree sizes, deepest level first
__global__ void k_sizes(const PoolNode* __restrict__ pool, const uint32_t* __restrict__ ids, uint32_t n,
                        uint32_t* size) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t i = ids[k];
  const uint32_t c = pool[i].child;
  size[i] = c == kNone ? 1u : 1u + size[c] + size[c + 1];
}
// depth-first indexes, root level first: a node's children take the next two free indexes,
// its left subtree's descendants follow, then the right's
__global__ void k_number(const PoolNode* __restrict__ pool, const uint32_t* __restrict__ ids, uint32_t n,
                         const uint32_t* __restrict__ size, uint32_t* ref, uint32_t* cbase) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t i = ids[k];
  const uint32_t c = pool[i].child;
  if (c == kNone) return;
  const uint32_t b = cbase[i];
  ref[c] = b;
  ref[c + 1] = b + 1;
  cbase[c] = b + 2;
  cbase[c + 1] = b + 2 + (size[c] - 1u);
}
__global__ void k_layout(const PoolNode* __restrict__ pool, uint32_t n, const uint32_t* __restrict__ ref,
                         GpuNode* out, uint32_t* stats) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const PoolNode& p = pool[i];
    const uint32_t r = ref[i];
    GpuNode g;
    for (int a = 0; a < 3; ++a) {
      g.bmin[a] = p.lo[a];
      g.bmax[a] = p.hi[a];
    }
    if (p.child == kNone) {
      g.left_first = p.first;
      g.count = p.count;
      atomicAdd(stats, 1u);
      atomicMax(stats + 1, p.count);
    } else {
      g.left_first = ref[p.child] + 1;
      g.count = 0;
    }
    atomicMax(stats + 2, p.depth);
    out[r == 0 ? 0 : r + 1] = g;
  }
}

// the triangles in leaf order, with their precomputed edges (mesh_bvh.hpp)
__global__ void k_tri_layout(const TriRec* __restrict__ fin, uint32_t n, const float* __restrict__ v,
                             const uint32_t* __restrict__ idx, float4* ta, float4* tb, float2* tc, uint32_t* order) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const uint32_t t = __float_as_uint(fin[k].c.w);
    const float* p0 = v + 3 * size_t(idx[3 * size_t(t)]);
    const float* p1 = v + 3 * size_t(idx[3 * size_t(t) + 1]);
    const float* p2 = v + 3 * size_t(idx[3 * size_t(t) + 2]);
    const float e1[3] = {__fsub_rn(p1[0], p0[0]), __fsub_rn(p1[1], p0[1]), __fsub_rn(p1[2], p0[2])};
    const float e2[3] = {__fsub_rn(p2[0], p0[0]), __fsub_rn(p2[1], p0[1]), __fsub_rn(p2[2], p0[2])};
    ta[k] = make_float4(p0[0], p0[1], p0[2], e1[0]);
    tb[k] = make_float4(e1[1], e1[2], e2[0], e2[1]);
    tc[k] = make_float2(e2[2], __uint_as_float(t));
    order[k] = t;
  }
}

// ---- host driver ------------------------------------------------------------------------------
struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return e;
  }
};

#define BUILD_TRY(x)                                                                  \
  do {                                                                                \
    const cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) {                                                          \
      *err = std::string("device BVH build: ") + cudaGetErrorString(e_) + " at " #x; \
      return false;                                                                   \
    }                                                                                 \
  } while (0)

unsigned grid_for(uint64_t n, int threads, int sm_count) {
  const uint64_t want = (n + threads - 1) / threads;
  const uint64_t cap = uint64_t(sm_count) * 16;
  return unsigned(std::max<uint64_t>(1, std::min(want, cap)));
}

}  // namespace

bool build_mesh_bvh_device(const float* d_v, uint32_t nv, const uint32_t* d_idx, uint32_t n,
                           const MeshBuildParams& p, cudaStream_t st, int sm_count, DeviceMeshBuild* out,
                           std::string* err) {
  *out = DeviceMeshBuild{};
  if (n == 0) { *err = "a TriangleMesh needs at least one triangle"; return false; }
  if (p.bins < 2 || p.bins > kMaxBins) { *err = "bvh_bins must be in [2, 64]"; return false; }
  const int B = p.bins;
  Scratch s;
  TriRec *b0, *b1, *fin;
  PoolNode* pool;
  uint32_t *ord, *pos, *flags;  // flags: [0] error, [1] pool count, [2] changed, [3..8] root box, [9..14] vertex box
  BUILD_TRY(s.alloc(&b0, n));
  BUILD_TRY(s.alloc(&b1, n));
  BUILD_TRY(s.alloc(&fin, n));
  BUILD_TRY(s.alloc(&pool, size_t(2) * n));
  BUILD_TRY(s.alloc(&ord, n));
  BUILD_TRY(s.alloc(&pos, n));
  BUILD_TRY(s.alloc(&flags, 16));
  uint32_t init[16] = {0, 1, 0, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0, 0, 0,
                       0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0, 0, 0, 0};
  BUILD_TRY(cudaMemcpyAsync(flags, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_tri_prep<<<grid_for(n, 256, sm_count), 256, 0, st>>>(d_v, nv, d_idx, n, b0, flags);
  k_vertex_bounds<<<grid_for(nv, kLevelThreads, sm_count), kLevelThreads, 0, st>>>(d_v, nv, flags + 9, flags);
  k_root_box<<<grid_for(n, kLevelThreads, sm_count), kLevelThreads, 0, st>>>(b0, n, flags + 3);
  k_root_node<<<1, 1, 0, st>>>(pool, flags + 3, n);
  BUILD_TRY(cudaGetLastError());
  uint32_t h[16];
  BUILD_TRY(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, st));
  BUILD_TRY(cudaStreamSynchronize(st));
  if (h[0] & kBuildErrInput) {
    *err = "a triangle vertex index out of range or a non-finite vertex coordinate";
    return false;
  }

  // large nodes, level by level
  std::vector<SmallJob> small;
  std::vector<LevelNode> level;
  if (n > kSmall && n > p.max_leaf) {
    LevelNode r{};
    r.pool = 0;
    r.first = 0;
    r.count = n;
    r.depth = 1;
    level.push_back(r);
  } else {
    small.push_back(SmallJob{0, 0, n, 1, 0});
  }
  LevelNode* d_nodes = nullptr;
  LevelResult* d_res = nullptr;
  Chunk* d_chunks = nullptr;
  uint32_t *d_cfirst = nullptr, *d_ctot = nullptr, *d_bins = nullptr;
  size_t cap_nodes = 0, cap_chunks = 0;
  int cur = 0;
  TriRec* bufs[2] = {b0, b1};
  while (!level.empty()) {
    const uint32_t nn = uint32_t(level.size());
    std::vector<Chunk> chunks;
    std::vector<uint32_t> cfirst;
    for (uint32_t j = 0; j < nn; ++j) {
      for (int q = 0; q < 6; ++q) level[j].ext[q] = q < 3 ? 0xFFFFFFFFu : 0u;
      cfirst.push_back(uint32_t(chunks.size()));
      for (uint32_t o = 0; o < level[j].count; o += kChunk) chunks.push_back(Chunk{j, o, std::min(kChunk, level[j].count - o)});
    }
    cfirst.push_back(uint32_t(chunks.size()));
    const uint32_t nc = uint32_t(chunks.size());
    if (nn > cap_nodes) {
      cap_nodes = std::max<size_t>(nn, 2 * cap_nodes);
      BUILD_TRY(s.alloc(&d_nodes, cap_nodes));
      BUILD_TRY(s.alloc(&d_res, cap_nodes));
      BUILD_TRY(s.alloc(&d_cfirst, cap_nodes + 1));
      BUILD_TRY(s.alloc(&d_bins, cap_nodes * 3 * B * 7));
    }
    if (nc > cap_chunks) {
      cap_chunks = std::max<size_t>(nc, 2 * cap_chunks);
      BUILD_TRY(s.alloc(&d_chunks, cap_chunks));
      BUILD_TRY(s.alloc(&d_ctot, cap_chunks));
    }
    BUILD_TRY(cudaMemcpyAsync(d_nodes, level.data(), nn * sizeof(LevelNode), cudaMemcpyHostToDevice, st));
    BUILD_TRY(cudaMemcpyAsync(d_chunks, chunks.data(), nc * sizeof(Chunk), cudaMemcpyHostToDevice, st));
    BUILD_TRY(cudaMemcpyAsync(d_cfirst, cfirst.data(), (nn + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    const TriRec* tc = bufs[cur];
    TriRec* tn = bufs[cur ^ 1];
    k_ext<<<nc, kLevelThreads, 0, st>>>(tc, d_nodes, d_chunks);
    k_bin_prep<<<nn, 128, 0, st>>>(d_nodes, nn, d_bins, B);
    k_bins<<<nc, kLevelThreads, 0, st>>>(tc, d_nodes, d_chunks, d_bins, B);
    k_sah<<<(nn + 63) / 64, 64, 0, st>>>(d_nodes, nn, d_bins, B, p.max_leaf, pool);
    k_classify<<<nc, kLevelThreads, 0, st>>>(tc, d_nodes, d_chunks, ord, d_ctot, B);
    k_chunk_offsets<<<(nn + 127) / 128, 128, 0, st>>>(d_nodes, nn, d_cfirst, d_ctot, pool, flags + 1, d_res);
    k_scatter<<<nc, kLevelThreads, 0, st>>>(d_nodes, d_chunks, d_ctot, ord, pos);
    BUILD_TRY(cudaGetLastError());
    for (int round = 0; round < 40; ++round) {
      BUILD_TRY(cudaMemsetAsync(flags + 2, 0, sizeof(uint32_t), st));
      k_jump<<<nc, kLevelThreads, 0, st>>>(d_nodes, d_chunks, pos, flags + 2);
      uint32_t changed = 0;
      BUILD_TRY(cudaMemcpyAsync(&changed, flags + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      BUILD_TRY(cudaStreamSynchronize(st));
      if (!changed) break;
      if (round == 39) { *err = "device BVH build: the partition did not converge"; return false; }
    }
    k_permute<<<nc, kLevelThreads, 0, st>>>(tc, tn, fin, d_nodes, d_chunks, ord, pos);
    k_child_box<<<nc, kLevelThreads, 0, st>>>(tn, d_nodes, d_chunks);
    k_child_finalize<<<(nn + 127) / 128, 128, 0, st>>>(d_nodes, nn, pool);
    BUILD_TRY(cudaGetLastError());
    std::vector<LevelResult> res(nn);
    BUILD_TRY(cudaMemcpyAsync(res.data(), d_res, nn * sizeof(LevelResult), cudaMemcpyDeviceToHost, st));
    BUILD_TRY(cudaStreamSynchronize(st));
    std::vector<LevelNode> next;
    for (uint32_t j = 0; j < nn; ++j) {
      const LevelNode& nd = level[j];
      const LevelResult& r = res[j];
      if (!r.split) continue;
      const uint32_t cnt[2] = {r.nl, nd.count - r.nl};
      const uint32_t fst[2] = {nd.first, nd.first + r.nl};
      for (int side = 0; side < 2; ++side) {
        if (cnt[side] > kSmall && cnt[side] > p.max_leaf) {
          LevelNode c{};
          c.pool = r.child + side;
          c.first = fst[side];
          c.count = cnt[side];
          c.depth = nd.depth + 1;
          next.push_back(c);
        } else {
          small.push_back(SmallJob{r.child + uint32_t(side), fst[side], cnt[side], nd.depth + 1, uint32_t(cur ^ 1)});
        }
      }
    }
    level.swap(next);
    cur ^= 1;
  }

  // small subtrees
  if (!small.empty()) {
    SmallJob* d_jobs;
    BUILD_TRY(s.alloc(&d_jobs, small.size()));
    BUILD_TRY(cudaMemcpyAsync(d_jobs, small.data(), small.size() * sizeof(SmallJob), cudaMemcpyHostToDevice, st));
    const uint32_t nj = uint32_t(small.size());
    k_small<<<(nj + 63) / 64, 64, 0, st>>>(d_jobs, nj, b0, b1, fin, pool, flags + 1, B, p.max_leaf, flags);
    BUILD_TRY(cudaGetLastError());
  }
  BUILD_TRY(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, st));
  BUILD_TRY(cudaStreamSynchronize(st));
  if (h[0] & kBuildErrStack) { *err = "device BVH build: a subtree is deeper than its stack"; return false; }
  const uint32_t nodes = h[1];

  // renumbering: nodes grouped by depth, subtree sizes bottom-up, indexes top-down
  uint32_t *hist, *by_depth, *size, *ref, *cbase, *stats;
  BUILD_TRY(s.alloc(&hist, 512));
  BUILD_TRY(s.alloc(&by_depth, nodes));
  BUILD_TRY(s.alloc(&size, nodes));
  BUILD_TRY(s.alloc(&ref, nodes));
  BUILD_TRY(s.alloc(&cbase, nodes));
  BUILD_TRY(s.alloc(&stats, 4));
  BUILD_TRY(cudaMemsetAsync(hist, 0, 512 * sizeof(uint32_t), st));
  k_depth_hist<<<grid_for(nodes, 256, sm_count), 256, 0, st>>>(pool, nodes, hist);
  uint32_t hh[256];
  BUILD_TRY(cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, st));
  BUILD_TRY(cudaStreamSynchronize(st));
  if (hh[255]) { *err = "device BVH build: the tree is deeper than 254 levels"; return false; }
  uint32_t off[257];
  off[0] = 0;
  uint32_t maxd = 0;
  for (int d = 0; d < 256; ++d) {
    off[d + 1] = off[d] + hh[d];
    if (hh[d]) maxd = uint32_t(d);
  }
  BUILD_TRY(cudaMemcpyAsync(hist + 256, off, 256 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  k_depth_scatter<<<grid_for(nodes, 256, sm_count), 256, 0, st>>>(pool, nodes, hist + 256, by_depth);
  for (uint32_t d = maxd; d >= 1; --d) {
    const uint32_t cnt = hh[d];
    if (cnt) k_sizes<<<(cnt + 255) / 256, 256, 0, st>>>(pool, by_depth + off[d], cnt, size);
  }
  const uint32_t zero = 0, one = 1;
  BUILD_TRY(cudaMemcpyAsync(ref, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  BUILD_TRY(cudaMemcpyAsync(cbase, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  for (uint32_t d = 1; d <= maxd; ++d) {
    const uint32_t cnt = hh[d];
    if (cnt) k_number<<<(cnt + 255) / 256, 256, 0, st>>>(pool, by_depth + off[d], cnt, size, ref, cbase);
  }
  BUILD_TRY(cudaGetLastError());

  // outputs
  DeviceMeshBuild o{};
  BUILD_TRY(cudaMalloc(&o.nodes, (size_t(nodes) + 1) * sizeof(GpuNode)));
  o.node_slots = uint64_t(nodes) + 1;
  auto fail_free = [&o]() {
    cudaFree(o.nodes);
    cudaFree(o.tri_a);
    cudaFree(o.tri_b);
    cudaFree(o.tri_c);
    cudaFree(o.tri_index);
  };
  cudaError_t e = cudaMalloc(&o.tri_a, size_t(n) * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&o.tri_b, size_t(n) * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&o.tri_c, size_t(n) * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&o.tri_index, size_t(n) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemsetAsync(o.nodes, 0, (size_t(nodes) + 1) * sizeof(GpuNode), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, 4 * sizeof(uint32_t), st);
  if (e == cudaSuccess) {
    k_layout<<<grid_for(nodes, 256, sm_count), 256, 0, st>>>(pool, nodes, ref, o.nodes, stats);
    k_tri_layout<<<grid_for(n, 256, sm_count), 256, 0, st>>>(fin, n, d_v, d_idx, o.tri_a, o.tri_b, o.tri_c,
                                                             o.tri_index);
    e = cudaGetLastError();
  }
  uint32_t hs[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    fail_free();
    *err = std::string("device BVH build: ") + cudaGetErrorString(e);
    return false;
  }
  o.stats.node_count = nodes;
  o.stats.leaf_count = hs[0];
  o.stats.max_leaf_tris = hs[1];
  o.stats.max_depth = hs[2];
  for (int a = 0; a < 3; ++a) {
    const uint32_t lo = h[9 + a], hi = h[12 + a];
    auto dec = [](uint32_t x) {
      const uint32_t u = (x & 0x80000000u) ? (x & 0x7FFFFFFFu) : ~x;
      float f;
      std::memcpy(&f, &u, sizeof(f));
      return f == 0.0f ? 0.0f : f;
    };
    o.bounds_min[a] = dec(lo);
    o.bounds_max[a] = dec(hi);
  }
  *out = o;
  return true;
}

void free_device_mesh_build(DeviceMeshBuild* b) {
  cudaFree(b->nodes);
  cudaFree(b->tri_a);
  cudaFree(b->tri_b);
  cudaFree(b->tri_c);
  cudaFree(b->tri_index);
  *b = DeviceMeshBuild{};
}

}  // namespace pbrt
