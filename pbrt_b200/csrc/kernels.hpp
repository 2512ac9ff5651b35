// kernels.hpp — host-side launchers of the device kernels (no device code here).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pbrt {

struct MeshView;

// Ray buffers: eight planes (ox oy oz dx dy dz tmin tmax) of `stride` floats each, of which
// the first `n` are used.
cudaError_t launch_mesh_closest(const MeshView& m, const float* rays, uint64_t stride, uint64_t n, uint32_t* prim,
                                float* t, uint32_t* obj, unsigned long long* counters, uint32_t* err, int sm_count,
                                cudaStream_t s);
// Two-stage nearest hit: a streaming root-box cull that answers misses and compacts the
// survivors' indices into `queue` (scratch, capacity >= n, n < 2^32), then the persistent
// dynamic-fetch traversal over the queue. `counters` is two 64-bit words of scratch (queue
// length, fetch position), zeroed on `s` by the launcher. `rec` (optional scratch, 2 x n
// float4): the survivors' rays copied beside their queue entries, read back coalesced.
// Dense results (optional scratch, with `rec`): the cull writes no miss answers but a survivor
// bitmask per ray (`mask`, n/32 words) and the queue position of each 1,024-ray chunk's first
// survivor (`bases`); the traversal writes each survivor's (id, t) to its queue slot (`res`,
// capacity n); a last pass writes every ray's answer in ray order, coalesced.
struct DenseScratch {
  uint2* res = nullptr;
  uint32_t* mask = nullptr;
  uint32_t* bases = nullptr;
};
constexpr uint64_t kDenseChunk = 1024;  // rays per bitmask chunk (one cull block iteration)
cudaError_t launch_mesh_closest_persistent(const MeshView& m, const float* rays, uint64_t stride, uint64_t n,
                                           uint32_t* prim, float* t, uint32_t* obj, uint32_t* queue,
                                           unsigned long long* counters, uint32_t* err, int sm_count, cudaStream_t s,
                                           float4* rec = nullptr, const DenseScratch* dense = nullptr);
// The two-stage pass over `n` rays in up to kPipeMaxParts parts, the cull of part j + 1
// running beside the traversal of part j: culls on `cull` (the first with a full grid, the
// rest with one block per SM), part j's traversal on trav[j % 2] after part j's cull, at
// `trav_blocks_per_sm` resident blocks per SM so that a cull block fits beside them. Part j
// uses queue / records from its first ray's index on, and counters 2j, 2j + 1 (zeroed on
// `s`). `s` forks into the three streams through `fork` and waits for the ones it used
// through `joined`; the plane stride must be a multiple of 4 and every pointer 16-byte aligned.
// Stream ordering alone orders the parts (no kernel waits on another).
constexpr int kPipeMaxParts = 16;
struct TracePipeline {
  cudaStream_t cull = nullptr;
  cudaStream_t trav[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr;
  cudaEvent_t culled[kPipeMaxParts] = {};
  cudaEvent_t joined[3] = {nullptr, nullptr, nullptr};  // the cull stream, trav[0], trav[1]
  unsigned long long* counters = nullptr;  // 2 * kPipeMaxParts words
};
cudaError_t launch_mesh_closest_pipelined(const MeshView& m, const float* rays, uint64_t stride, uint64_t n,
                                          uint32_t* prim, float* t, uint32_t* obj, uint32_t* queue, float4* rec,
                                          uint32_t* err, int sm_count, cudaStream_t s, const TracePipeline& p,
                                          int parts, int trav_blocks_per_sm);
// The part count and traversal blocks per SM of the pipelined pass on this build (1 part: the
// plain two-stage pass); PBRT_TRACE_PARTS="K[,B]" overrides them for measurements.
void trace_pipeline_shape(int* parts, int* trav_blocks_per_sm);
// Allocation-free form of launch_mesh_closest_persistent for device buffers (plane stride
// = n): its scratch is a file-scope __device__ array of kNoAllocMaxRays queue entries
// shared by every call on a device. `scratch` is that array's device address on the current
// device, from noalloc_scratch_lookup (word 4 is the error word). cudaErrorInvalidValue when
// n > kNoAllocMaxRays. Calls that overlap on the GPU race.
constexpr uint64_t kNoAllocMaxRays = uint64_t(1) << 20;
cudaError_t launch_mesh_closest_noalloc(const MeshView& m, const float* rays, uint64_t n, uint32_t* prim, float* t,
                                        uint32_t* scratch, int sm_count, cudaStream_t s);
// Device address of the allocation-free pass's scratch array on the current device. The
// lookup loads this file's module there (under lazy loading), which commits the array.
cudaError_t noalloc_scratch_lookup(uint32_t** scratch);
cudaError_t launch_mesh_any(const MeshView& m, const float* rays, uint64_t stride, uint64_t n, uint8_t* occ,
                            uint32_t* err, int sm_count, cudaStream_t s);

}  // namespace pbrt
