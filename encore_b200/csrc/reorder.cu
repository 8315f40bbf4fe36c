// Ray binning ahead of the closest-hit launch.
//
// An incoherent batch (primaries and diffuse bounces in random order) puts
// rays that share no nodes side by side in a warp.  Binning groups rays by a
// key of their origin cell and direction, so the rays a warp takes from the
// queue walk similar paths through the tree: fewer distinct nodes per warp
// step, more lanes active per instruction, more L1 hits.
//
// Three kernels, all streaming over the batch:
//   bin_keys     key per ray (origin cell x direction cell, interleaved bit by
//                bit into one integer) + a histogram of the keys (warp-
//                aggregated global atomics: lanes of a warp with the same key
//                add once);
//   bin_scan     exclusive prefix sum of the histogram (one block);
//   bin_scatter  each ray's slot in its bucket (warp-aggregated atomics on the
//                bucket offsets), order[slot] = ray index.
// The traversal then takes queue index q as ray order[q] and writes its hit
// at that ray's own index, so callers see no reordering.  The order inside a
// bucket depends on atomic timing; the hits do not (each ray's result is a
// function of the ray alone).
//
// Algorithmic bytes: 32 (ray read) + 4 (key write) in the first pass, 4 (key
// read) + 4 (order write) in the third; the histogram is 4 bytes per bucket.
#include <cuda_runtime.h>

#include <cmath>

#include "engine.h"

namespace enc {
namespace {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt_bin() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t quantise(float x, float lo, float scale, int bits) {
  if (bits <= 0) return 0u;
  const float mx = (float)((1u << bits) - 1u);
  float q = (x - lo) * scale;
  q = fminf(fmaxf(q, 0.0f), mx);  // fmaxf drops a NaN: it lands in cell 0
  return (uint32_t)q;
}

// The key of one ray.  Dimensions: origin (or the probe point o + len * d)
// x, y, z over the scene box, then the direction's octahedral coordinates
// u, v in [-1, 1] (the unit direction projected onto the octahedron
// |x| + |y| + |z| = 1, the lower half folded out).  Bits are interleaved from
// the most significant level down, so each prefix of the key is a coarser
// cell of the same five-dimensional grid.
__device__ __forceinline__ uint32_t ray_key(const float4 r0, const float4 r1, const BinSpec& k) {
  float ox = r0.x, oy = r0.y, oz = r0.z;
  const float dx = r1.x, dy = r1.y, dz = r1.z;
  if (k.probe_len > 0.0f) {
    ox = fmaf(k.probe_len, dx, ox);
    oy = fmaf(k.probe_len, dy, oy);
    oz = fmaf(k.probe_len, dz, oz);
  }
  const float ad = fabsf(dx) + fabsf(dy) + fabsf(dz);
  float u = 0.0f, v = 0.0f;
  if (ad > 0.0f) {
    u = dx / ad;
    v = dz / ad;
    if (dy < 0.0f) {
      const float fu = (1.0f - fabsf(v)) * (u < 0.0f ? -1.0f : 1.0f);
      const float fv = (1.0f - fabsf(u)) * (v < 0.0f ? -1.0f : 1.0f);
      u = fu;
      v = fv;
    }
  }
  uint32_t q[5];
  q[0] = quantise(ox, k.lo[0], k.scale[0], k.bits[0]);
  q[1] = quantise(oy, k.lo[1], k.scale[1], k.bits[1]);
  q[2] = quantise(oz, k.lo[2], k.scale[2], k.bits[2]);
  q[3] = quantise(u, -1.0f, 0.5f * (float)(1u << k.bits[3]), k.bits[3]);
  q[4] = quantise(v, -1.0f, 0.5f * (float)(1u << k.bits[4]), k.bits[4]);
  uint32_t key = 0;
#pragma unroll
  for (int level = kBinMaxDimBits - 1; level >= 0; --level) {
#pragma unroll
    for (int d = 0; d < 5; ++d) {
      if (level < k.bits[d]) key = (key << 1) | ((q[d] >> level) & 1u);
    }
  }
  return key;
}

__global__ void __launch_bounds__(256) bin_keys(const float4* __restrict__ rays, uint32_t n,
                                                BinSpec spec, uint32_t* __restrict__ keys,
                                                uint32_t* __restrict__ hist) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  // the loop runs warp-uniformly: base is the warp's first index
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
    const uint32_t i = base + lane;
    const bool ok = i < n;
    uint32_t key = 0xffffffffu;
    if (ok) {
      key = ray_key(__ldg(rays + 2 * (size_t)i), __ldg(rays + 2 * (size_t)i + 1), spec);
      keys[i] = key;
    }
    const unsigned act = __ballot_sync(kFullMask, ok);
    const unsigned peers = __match_any_sync(kFullMask, key) & act;
    if (ok && lane == (unsigned)(__ffs(peers) - 1)) atomicAdd(hist + key, (uint32_t)__popc(peers));
  }
}

// Exclusive prefix sum of hist[0..nb) in place, one block of 1024 threads:
// each thread sums a contiguous run, the block scans the run totals, and each
// thread writes its run's offsets.
__global__ void __launch_bounds__(1024) bin_scan(uint32_t* hist, uint32_t nb) {
  __shared__ uint32_t s_warp[32];
  const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
  const uint32_t b = threadIdx.x * per;
  const uint32_t e = min(b + per, nb);
  uint32_t sum = 0;
  for (uint32_t i = b; i < e; ++i) sum += hist[i];
  // block-wide exclusive scan of `sum`
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t incl = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(kFullMask, incl, d);
    if ((int)lane >= d) incl += t;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const unsigned nw = blockDim.x >> 5;
    uint32_t w = lane < nw ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(kFullMask, wi, d);
      if ((int)lane >= d) wi += t;
    }
    if (lane < nw) s_warp[lane] = wi - w;
  }
  __syncthreads();
  uint32_t run = s_warp[wid] + incl - sum;
  for (uint32_t i = b; i < e; ++i) {
    const uint32_t c = hist[i];
    hist[i] = run;
    run += c;
  }
}

__global__ void __launch_bounds__(256) bin_scatter(const uint32_t* __restrict__ keys, uint32_t n,
                                                   uint32_t* __restrict__ offs,
                                                   uint32_t* __restrict__ order) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = lanemask_lt_bin();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
    const uint32_t i = base + lane;
    const bool ok = i < n;
    const uint32_t key = ok ? __ldg(keys + i) : 0xffffffffu;
    const unsigned act = __ballot_sync(kFullMask, ok);
    const unsigned peers = __match_any_sync(kFullMask, key) & act;
    const unsigned leader = ok ? (unsigned)(__ffs(peers) - 1) : lane;
    uint32_t slot = 0;
    if (ok && lane == leader) slot = atomicAdd(offs + key, (uint32_t)__popc(peers));
    slot = __shfl_sync(kFullMask, slot, leader);
    if (ok) order[slot + __popc(peers & lt)] = i;
  }
}

}  // namespace

size_t bin_scratch_bytes(size_t nrays, int key_bits) {
  const size_t a = 256;
  auto up = [&](size_t x) { return (x + a - 1) / a * a; };
  return up(nrays * 4) + up(nrays * 4) + up(((size_t)1 << key_bits) * 4);
}

BinSpec make_bin_spec(const float lo[3], const float hi[3], int key_bits, int dir_bits,
                      float probe_frac) {
  BinSpec k{};
  for (int d = 0; d < 5; ++d) k.bits[d] = 0;
  if (key_bits < 1) key_bits = 1;
  if (key_bits > kBinMaxKeyBits) key_bits = kBinMaxKeyBits;
  if (dir_bits < 0) dir_bits = 0;
  if (dir_bits > key_bits) dir_bits = key_bits;
  float ext[3];
  double diag2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    ext[i] = hi[i] > lo[i] ? hi[i] - lo[i] : 0.0f;
    diag2 += (double)ext[i] * ext[i];
  }
  const float diag = (float)std::sqrt(diag2);
  k.probe_len = probe_frac > 0.0f ? probe_frac * diag : 0.0f;
  // the probe point can leave the scene box by probe_len on every side
  for (int i = 0; i < 3; ++i) {
    k.lo[i] = lo[i] - k.probe_len;
    ext[i] += 2.0f * k.probe_len;
  }
  // direction bits split between u and v, u first
  k.bits[3] = (dir_bits + 1) / 2;
  k.bits[4] = dir_bits / 2;
  // origin bits go one at a time to the axis whose cells are widest, so the
  // cells stay close to cubes (a flat scene spends few bits on its thin axis)
  int left = key_bits - dir_bits;
  float cell[3] = {ext[0], ext[1], ext[2]};
  while (left > 0) {
    int best = 0;
    for (int i = 1; i < 3; ++i)
      if (cell[i] > cell[best]) best = i;
    if (cell[best] <= 0.0f || k.bits[best] >= kBinMaxDimBits) break;
    ++k.bits[best];
    cell[best] *= 0.5f;
    --left;
  }
  for (int i = 0; i < 3; ++i)
    k.scale[i] = ext[i] > 0.0f ? (float)(1u << k.bits[i]) / ext[i] : 0.0f;
  for (int d = 3; d < 5; ++d)
    if (k.bits[d] > kBinMaxDimBits) k.bits[d] = kBinMaxDimBits;
  return k;
}

int launch_bin(const float* d_rays, size_t n, const BinSpec& spec, void* d_scratch,
               uint32_t** d_order, int device, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int total = 0;
  for (int d = 0; d < 5; ++d) total += spec.bits[d];
  if (total < 1) total = 1;
  const size_t a = 256;
  auto up = [&](size_t x) { return (x + a - 1) / a * a; };
  char* base = static_cast<char*>(d_scratch);
  uint32_t* keys = reinterpret_cast<uint32_t*>(base);
  uint32_t* order = reinterpret_cast<uint32_t*>(base + up(n * 4));
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + 2 * up(n * 4));
  const uint32_t nb = 1u << total;
  cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)nb * 4, s);
  if (e != cudaSuccess) return (int)e;
  const int sms = device_sm_count(device);
  const size_t warps = (n + 31) / 32;
  int grid = (int)std::min<size_t>((warps + 7) / 8, (size_t)sms * 8);
  if (grid < 1) grid = 1;
  bin_keys<<<grid, 256, 0, s>>>(reinterpret_cast<const float4*>(d_rays), (uint32_t)n, spec, keys,
                                hist);
  bin_scan<<<1, 1024, 0, s>>>(hist, nb);
  bin_scatter<<<grid, 256, 0, s>>>(keys, (uint32_t)n, hist, order);
  *d_order = order;
  return (int)cudaGetLastError();
}

}  // namespace enc
