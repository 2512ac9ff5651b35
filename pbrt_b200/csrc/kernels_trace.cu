// kernels_trace.cu — batched ray-cast kernels (nearest hit / any hit) over one mesh.
//
// One thread per ray. Ray planes are read and results written with streaming cache
// hints (each byte is touched once), so L1/L2 stay dedicated to the tree and triangles,
// which every ray revisits.
#include <cfloat>
#include <cstdint>

#include "kernels.hpp"
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

cudaError_t launch_mesh_any(const MeshView& m, const float* rays, uint64_t stride, uint64_t n, uint8_t* occ,
                            uint32_t* err, int sm_count, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mesh_any<<<grid_for(n, 128, sm_count), 128, 0, s>>>(m, rays, stride, n, occ, err);
  return cudaGetLastError();
}

}  // namespace pbrt
