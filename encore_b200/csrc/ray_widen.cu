// Widening of the reference's ray payload to the traversal's ray layout.
//
// The reference traces a Ray of an origin and a direction (Ray.h:44-45) with
// no distance bounds: a hit only needs t > 0 (TrianglePrim.cpp:222-223).  The
// host-buffer call that takes rays in that form (enc_intersect_closest_od)
// moves 24 bytes per ray across PCIe instead of 32, and this kernel writes
// each chunk out in the traversal's 32-byte form (ox, oy, oz, 0, dx, dy, dz,
// +inf) in device memory before the chunk's trace.
//
// Algorithmic bytes: 24 read + 32 written per ray; a streaming, HBM-bound
// pass (about 30 MB for a 512K-ray chunk, a few microseconds).  Each thread
// takes one ray per grid step with three 8-byte loads (a 24-byte record is
// 8-byte aligned) and two 16-byte stores; a warp's three loads cover 768
// contiguous bytes, so every sector fetched is used.
#include <cuda_runtime.h>

#include <cmath>

#include "engine.h"

namespace enc {
namespace {

__global__ void __launch_bounds__(256) widen_rays_kernel(const float2* __restrict__ od, size_t n,
                                                         float4* __restrict__ rays) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float2 a = __ldcs(od + 3 * i);
    const float2 b = __ldcs(od + 3 * i + 1);
    const float2 c = __ldcs(od + 3 * i + 2);
    rays[2 * i] = make_float4(a.x, a.y, b.x, 0.f);
    rays[2 * i + 1] = make_float4(b.y, c.x, c.y, INFINITY);
  }
}

}  // namespace

int launch_widen_rays(const float* d_od, size_t n, float* d_rays, int device, void* stream) {
  if (n == 0) return 0;
  // one wave of 8 blocks per SM, grid-stride beyond it
  const size_t need = (n + 255) / 256;
  const size_t wave = (size_t)device_sm_count(device) * 8;
  const unsigned grid = (unsigned)(need < wave ? need : wave);
  widen_rays_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(d_od), n, reinterpret_cast<float4*>(d_rays));
  return (int)cudaGetLastError();
}

}  // namespace enc
