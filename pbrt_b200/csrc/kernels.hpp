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
