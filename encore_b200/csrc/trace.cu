// Ray traversal kernels for sm_100a.
//
//  * wbvh_trace<W, CLAMP, ANY, COUNT>: persistent warps over the quantised
//    wide BVH.  Each warp takes rays from a global atomic queue in chunks and
//    hands them to idle lanes as lanes finish (no lane waits for the slowest
//    ray of a batch).  The traversal stack lives in shared memory, one column
//    per thread.  Hit children of a node are ordered by entry distance with a
//    sorting network; the nearest is visited next, the rest are pushed.
//  * kd_trace<CLAMP>: the reference's kd-tree walk (Kdtree.cpp:682-784), one
//    thread per ray, over the flattened kd layout.  Bit-exact parity mode.
//
// The triangle test follows TrianglePrim::intersect (TrianglePrim.cpp:204-248)
// operation for operation: every product and sum is a separately rounded FP32
// operation (__fmul_rn / __fadd_rn / __fsub_rn are never contracted into FMA),
// 1/det is an IEEE division, and with CLAMP the Cross() components with
// |c| < 0.001 are set to zero as Vector3::ClampfloatoZero does
// (Vector3.h:148-161, Vector3.cpp:126-140).
//
// Every loop is bounded: a ray that exceeds kMaxSteps work items, or would
// overflow its stack, is stopped, reported as a miss, and sets a bit in the
// accelerator's status word, which the host turns into ENC_ERR_WATCHDOG.
#include <cuda_runtime.h>

#include <cstdio>

#include "engine.h"

namespace enc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned kMaxSteps = 1u << 22;
constexpr uint32_t kStatusWatchdog = 1u;
constexpr uint32_t kStatusStack = 2u;
constexpr uint32_t kStatusBounds = 4u;

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// ClampfloatoZero: (-ENC_EPSILON < x && x < ENC_EPSILON) with the double
// constant 0.001; for a float x this is the same comparison against 0.001f.
__device__ __forceinline__ float clamp_eps(float x) {
  return (x > -0.001f && x < 0.001f) ? 0.0f : x;
}

// Dot(v1, v2) = v1[0]*v2[0] + v1[1]*v2[1] + v1[2]*v2[2], left to right.
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

// The reference predicate.  a/b/c: the three float4 of a DevTri.
template <bool CLAMP>
__device__ __forceinline__ bool tri_test(const float4 a, const float4 b, const float4 c, float ox,
                                         float oy, float oz, float dx, float dy, float dz,
                                         float tmin, float& t, float& alpha, float& beta) {
  const float e1x = a.w, e1y = b.x, e1z = b.y;
  const float e2x = b.z, e2y = b.w, e2z = c.x;
  // pvec = Cross(dir, edge2)
  float px = fs(fm(dy, e2z), fm(dz, e2y));
  float py = -fs(fm(dx, e2z), fm(dz, e2x));
  float pz = fs(fm(dx, e2y), fm(dy, e2x));
  if (CLAMP) {
    px = clamp_eps(px);
    py = clamp_eps(py);
    pz = clamp_eps(pz);
  }
  const float invdet = __fdiv_rn(1.0f, dot3(e1x, e1y, e1z, px, py, pz));
  // svec = Vector3(v0, origin) = origin - v0
  const float sx = fs(ox, a.x), sy = fs(oy, a.y), sz = fs(oz, a.z);
  // qvec = Cross(svec, edge1)
  float qx = fs(fm(sy, e1z), fm(sz, e1y));
  float qy = -fs(fm(sx, e1z), fm(sz, e1x));
  float qz = fs(fm(sx, e1y), fm(sy, e1x));
  if (CLAMP) {
    qx = clamp_eps(qx);
    qy = clamp_eps(qy);
    qz = clamp_eps(qz);
  }
  alpha = fm(dot3(sx, sy, sz, px, py, pz), invdet);
  beta = fm(dot3(dx, dy, dz, qx, qy, qz), invdet);
  t = fm(dot3(e2x, e2y, e2z, qx, qy, qz), invdet);
  return (alpha >= 0.0f) && (beta >= 0.0f) && (fa(alpha, beta) <= 1.0f) && (t > tmin);
}

struct TraceParams {
  const uint8_t* nodes;
  const float4* tris;  // 3 per triangle
  const float4* rays;  // 2 per ray
  void* out;           // enc_hit* (closest) or uint8_t* (any)
  uint32_t* visits;    // COUNT: 2 per ray
  unsigned* counter;
  uint32_t* status;
  unsigned nrays;
  unsigned nnodes;
  unsigned ntris;
  int stack_depth;
  int chunk;
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t byte_of(const uint4* w, int off) {
  const uint32_t* u = reinterpret_cast<const uint32_t*>(w);
  return (u[off >> 2] >> (8 * (off & 3))) & 0xffu;
}

template <int W>
struct NodeWords {
  static constexpr int N = WNodeLayout<W>::kBytes / 16;
  uint4 w[N];
};

// Item encoding on the stack: internal node index, or leaf with bit 31 set,
// triangle count in bits 28..30 and first triangle in bits 0..27.
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kNoItem = 0xffffffffu;

template <int W>
__device__ __forceinline__ void sort_net(float (&k)[W], uint32_t (&v)[W]);

#define ENC_CSWAP(i, j)                   \
  {                                       \
    if (k[j] < k[i]) {                    \
      float tk = k[i];                    \
      k[i] = k[j];                        \
      k[j] = tk;                          \
      uint32_t tv = v[i];                 \
      v[i] = v[j];                        \
      v[j] = tv;                          \
    }                                     \
  }

template <>
__device__ __forceinline__ void sort_net<2>(float (&k)[2], uint32_t (&v)[2]) {
  ENC_CSWAP(0, 1);
}
template <>
__device__ __forceinline__ void sort_net<4>(float (&k)[4], uint32_t (&v)[4]) {
  ENC_CSWAP(0, 1);
  ENC_CSWAP(2, 3);
  ENC_CSWAP(0, 2);
  ENC_CSWAP(1, 3);
  ENC_CSWAP(1, 2);
}
template <>
__device__ __forceinline__ void sort_net<8>(float (&k)[8], uint32_t (&v)[8]) {
  // Batcher odd-even merge sort, 19 comparators.
  ENC_CSWAP(0, 1); ENC_CSWAP(2, 3); ENC_CSWAP(4, 5); ENC_CSWAP(6, 7);
  ENC_CSWAP(0, 2); ENC_CSWAP(1, 3); ENC_CSWAP(4, 6); ENC_CSWAP(5, 7);
  ENC_CSWAP(1, 2); ENC_CSWAP(5, 6);
  ENC_CSWAP(0, 4); ENC_CSWAP(1, 5); ENC_CSWAP(2, 6); ENC_CSWAP(3, 7);
  ENC_CSWAP(2, 4); ENC_CSWAP(3, 5);
  ENC_CSWAP(1, 2); ENC_CSWAP(3, 4); ENC_CSWAP(5, 6);
}
#undef ENC_CSWAP

template <int W, bool CLAMP, bool ANY, bool COUNT>
__global__ void __launch_bounds__(128) wbvh_trace(TraceParams P) {
  using L = WNodeLayout<W>;
  extern __shared__ uint2 s_stack[];
  const int B = blockDim.x;
  uint2* stk = s_stack + threadIdx.x;  // entry i at stk[i * B]
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = lanemask_lt();

  // Warp-private ray pool [pool_next, pool_end), refilled in chunks.
  unsigned pool_next = 0, pool_end = 0;
  bool exhausted = false;

  int ray = -1;
  float ox = 0, oy = 0, oz = 0, dx = 0, dy = 0, dz = 0, ix = 0, iy = 0, iz = 0, tmin = 0, tmax = 0;
  float best_t = 0, bu = 0, bv = 0;
  int best_id = -1;
  int sp = 0;
  uint32_t item = kNoItem;
  unsigned steps = 0;
  uint32_t nvis = 0, ntest = 0;

  while (true) {
    // ---- refill idle lanes from the warp pool --------------------------
    unsigned need = __ballot_sync(kFull, ray < 0);
    while (need && !exhausted) {
      if (pool_next >= pool_end) {
        unsigned b = 0;
        if (lane == 0) b = atomicAdd(P.counter, (unsigned)P.chunk);
        b = __shfl_sync(kFull, b, 0);
        if (b >= P.nrays) {
          exhausted = true;
          break;
        }
        pool_next = b;
        pool_end = min(b + (unsigned)P.chunk, P.nrays);
      }
      const unsigned avail = pool_end - pool_next;
      const unsigned rank = __popc(need & lt);
      if (((need >> lane) & 1u) && rank < avail) {
        ray = (int)(pool_next + rank);
        const float4 r0 = __ldg(P.rays + 2 * (size_t)ray);
        const float4 r1 = __ldg(P.rays + 2 * (size_t)ray + 1);
        ox = r0.x; oy = r0.y; oz = r0.z; tmin = r0.w;
        dx = r1.x; dy = r1.y; dz = r1.z; tmax = r1.w;
        ix = 1.0f / dx; iy = 1.0f / dy; iz = 1.0f / dz;
        best_t = tmax; best_id = -1; bu = 0.f; bv = 0.f;
        sp = 0;
        item = 0;  // root
        steps = 0;
        nvis = 0; ntest = 0;
      }
      const unsigned took = min(avail, (unsigned)__popc(need));
      pool_next += took;
      need = __ballot_sync(kFull, ray < 0);
    }
    if (__all_sync(kFull, ray < 0)) break;

    if (ray >= 0) {
      bool done = false;
      bool hit_any = false;
      ++steps;
      if (steps > kMaxSteps) {
        atomicOr(P.status, kStatusWatchdog);
        best_id = -1;
        done = true;
      } else if (!(item & kLeafBit)) {
        // ---- internal node: test all children ---------------------------
        if (item >= P.nnodes) {
          atomicOr(P.status, kStatusBounds);
          best_id = -1;
          done = true;
        } else {
          if (COUNT) ++nvis;
          NodeWords<W> nw;
          const uint4* src = reinterpret_cast<const uint4*>(P.nodes + (size_t)item * L::kBytes);
#pragma unroll
          for (int i = 0; i < NodeWords<W>::N; ++i) nw.w[i] = __ldg(src + i);
          const float px = __uint_as_float(nw.w[0].x);
          const float py = __uint_as_float(nw.w[0].y);
          const float pz = __uint_as_float(nw.w[0].z);
          const uint32_t ew = nw.w[0].w;
          const float sx = __uint_as_float((ew & 0xffu) << 23);
          const float sy = __uint_as_float(((ew >> 8) & 0xffu) << 23);
          const float sz = __uint_as_float(((ew >> 16) & 0xffu) << 23);
          const uint32_t child_base = nw.w[1].x;
          const uint32_t tri_base = nw.w[1].y;
          const float bx = (px - ox) * ix, by = (py - oy) * iy, bz = (pz - oz) * iz;
          const float cx = sx * ix, cy = sy * iy, cz = sz * iz;
          float key[W];
          uint32_t val[W];
          int nh = 0;
#pragma unroll
          for (int c = 0; c < W; ++c) {
            const float qlx = (float)byte_of(nw.w, L::kQOff + 0 * W + c);
            const float qly = (float)byte_of(nw.w, L::kQOff + 1 * W + c);
            const float qlz = (float)byte_of(nw.w, L::kQOff + 2 * W + c);
            const float qhx = (float)byte_of(nw.w, L::kQOff + 3 * W + c);
            const float qhy = (float)byte_of(nw.w, L::kQOff + 4 * W + c);
            const float qhz = (float)byte_of(nw.w, L::kQOff + 5 * W + c);
            const float t0x = fmaf(qlx, cx, bx), t1x = fmaf(qhx, cx, bx);
            const float t0y = fmaf(qly, cy, by), t1y = fmaf(qhy, cy, by);
            const float t0z = fmaf(qlz, cz, bz), t1z = fmaf(qhz, cz, bz);
            const float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), tmin));
            const float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), best_t));
            const uint32_t meta = byte_of(nw.w, L::kMetaOff + c);
            const bool hit = meta != 0u && tn <= tf;
            uint32_t it;
            if (meta >= 32u)
              it = kLeafBit | ((meta >> 5) << 28) | (tri_base + (meta & 31u));
            else
              it = child_base + meta - 1u;
            key[c] = hit ? fminf(tn, 3.0e38f) : INFINITY;  // hits sort before empty slots
            val[c] = it;
            nh += hit ? 1 : 0;
          }
          if (nh > 0) {
            sort_net<W>(key, val);
            if (sp + nh - 1 > P.stack_depth) {
              atomicOr(P.status, kStatusStack);
              best_id = -1;
              done = true;
            } else {
              // push hits 1..nh-1 farthest first
#pragma unroll
              for (int c = W - 1; c >= 1; --c) {
                if (c < nh) {
                  stk[(sp + (nh - 1 - c)) * B] = make_uint2(val[c], __float_as_uint(key[c]));
                }
              }
              sp += nh - 1;
              item = val[0];
            }
          } else {
            item = kNoItem;
          }
        }
      } else {
        // ---- leaf: test its triangles ----------------------------------
        const uint32_t first = item & 0x0fffffffu;
        const uint32_t cnt = (item >> 28) & 7u;
        if (first + cnt > P.ntris) {
          atomicOr(P.status, kStatusBounds);
          best_id = -1;
          done = true;
        } else {
          for (uint32_t k = 0; k < cnt; ++k) {
            const float4* tp = P.tris + 3 * (size_t)(first + k);
            const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
            if (COUNT) ++ntest;
            float t, u, v;
            if (tri_test<CLAMP>(a, b, c, ox, oy, oz, dx, dy, dz, tmin, t, u, v)) {
              const int id = __float_as_int(c.y);
              if (ANY) {
                if (t < tmax) {
                  hit_any = true;
                  break;
                }
              } else if (t < best_t || (t == best_t && id < best_id)) {
                best_t = t;
                best_id = id;
                bu = u;
                bv = v;
              }
            }
          }
          item = kNoItem;
        }
        if (ANY && hit_any) done = true;
      }
      // ---- pop the next item whose entry distance can still matter ------
      if (!done && item == kNoItem) {
        while (sp > 0) {
          const uint2 e = stk[(sp - 1) * B];
          --sp;
          if (ANY || __uint_as_float(e.y) <= best_t) {
            item = e.x;
            break;
          }
        }
        if (item == kNoItem) done = true;
      }
      if (done) {
        if (ANY) {
          reinterpret_cast<uint8_t*>(P.out)[ray] = hit_any ? 1 : 0;
        } else {
          int4 h;
          h.x = best_id;
          h.y = best_id >= 0 ? __float_as_int(best_t) : 0;
          h.z = best_id >= 0 ? __float_as_int(bu) : 0;
          h.w = best_id >= 0 ? __float_as_int(bv) : 0;
          reinterpret_cast<int4*>(P.out)[ray] = h;
        }
        if (COUNT) {
          P.visits[2 * (size_t)ray] = nvis;
          P.visits[2 * (size_t)ray + 1] = ntest;
        }
        ray = -1;
        item = kNoItem;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// kd-tree walk in the reference's order (Kdtree.cpp:682-784).

struct KdParams {
  const KdNode* nodes;
  const uint32_t* items;
  const float4* tris;  // triangle-ID order
  const float4* rays;
  void* out;
  uint32_t* status;
  unsigned nrays, nnodes, nitems, ntris;
  float lo[3], hi[3];  // root box min corner and pos + size
};

constexpr int kKdStack = 64;

template <bool CLAMP, bool ANY>
__global__ void __launch_bounds__(128) kd_trace(KdParams P) {
  for (unsigned ray = blockIdx.x * blockDim.x + threadIdx.x; ray < P.nrays;
       ray += gridDim.x * blockDim.x) {
    const float4 r0 = __ldg(P.rays + 2 * (size_t)ray);
    const float4 r1 = __ldg(P.rays + 2 * (size_t)ray + 1);
    const float o[3] = {r0.x, r0.y, r0.z};
    const float d[3] = {r1.x, r1.y, r1.z};
    const float rtmin = r0.w, rtmax = r1.w;
    const float inv[3] = {__fdiv_rn(1.f, d[0]), __fdiv_rn(1.f, d[1]), __fdiv_rn(1.f, d[2])};
    float best_t = INFINITY, bu = 0.f, bv = 0.f;
    int best_id = -1;
    // m_Bounds.Intersect(r, tmin, tmax)  (AABB.cpp:117-143)
    float t0 = 0.f, t1 = INFINITY;
    bool in = true;
    for (int i = 0; i < 3 && in; ++i) {
      float tin = __fdiv_rn(fs(P.lo[i], o[i]), d[i]);
      float tout = __fdiv_rn(fs(P.hi[i], o[i]), d[i]);
      if (tin > tout) {
        float tt = tin;
        tin = tout;
        tout = tt;
      }
      t0 = tin > t0 ? tin : t0;
      t1 = tout < t1 ? tout : t1;
      if (t0 > t1) in = false;
    }
    if (in) {
      float tmin = t0, tmax = t1;
      uint32_t st_node[kKdStack];
      float st_min[kKdStack], st_max[kKdStack];
      int sp = 0;
      uint32_t node = 0;
      unsigned steps = 0;
      while (true) {
        if (++steps > kMaxSteps) {
          atomicOr(P.status, kStatusWatchdog);
          best_id = -1;
          break;
        }
        if (best_t < tmin) break;
        if (node >= P.nnodes) {
          atomicOr(P.status, kStatusBounds);
          best_id = -1;
          break;
        }
        const KdNode n = P.nodes[node];
        if ((n.word0 & 3u) != 3u) {
          const int axis = (int)(n.word0 & 3u);
          float split = __uint_as_float(n.word0);
          split = (split > -0.001f && split < 0.001f) ? 0.0f : split;
          const float tplane = fm(fs(split, o[axis]), inv[axis]);
          const bool below = o[axis] <= split;
          const uint32_t first = below ? n.word1 : n.word1 + 1;
          const uint32_t second = below ? n.word1 + 1 : n.word1;
          if (tplane == 0.0f) {
            node = inv[axis] > 0.0f ? second : first;
          } else if (tplane >= tmax || tplane < 0.0f) {
            node = first;
          } else if (tplane <= tmin) {
            node = second;
          } else {
            if (sp >= kKdStack) {
              atomicOr(P.status, kStatusStack);
              best_id = -1;
              break;
            }
            st_node[sp] = second;
            st_min[sp] = tplane;
            st_max[sp] = tmax;
            ++sp;
            node = first;
            tmax = tplane;
          }
        } else {
          const uint32_t cnt = n.word0 >> 2;
          const uint32_t beg = n.word1;
          if ((size_t)beg + cnt > P.nitems) {
            atomicOr(P.status, kStatusBounds);
            best_id = -1;
            break;
          }
          for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t id = __ldg(P.items + beg + k);
            if (id >= P.ntris) {
              atomicOr(P.status, kStatusBounds);
              continue;
            }
            const float4* tp = P.tris + 3 * (size_t)id;
            float t, u, v;
            if (tri_test<CLAMP>(__ldg(tp), __ldg(tp + 1), __ldg(tp + 2), o[0], o[1], o[2], d[0],
                                d[1], d[2], rtmin, t, u, v) &&
                t < best_t) {
              best_t = t;
              best_id = (int)id;
              bu = u;
              bv = v;
            }
          }
          if (sp > 0) {
            --sp;
            node = st_node[sp];
            tmin = st_min[sp];
            tmax = st_max[sp];
          } else {
            break;
          }
        }
      }
    }
    // IsInShadow form: closest hit && t < distance; closest: hits at or
    // beyond the ray's tmax are reported as misses.
    const bool hit = best_id >= 0 && best_t < rtmax;
    if (ANY) {
      reinterpret_cast<uint8_t*>(P.out)[ray] = hit ? 1 : 0;
    } else {
      int4 h;
      h.x = hit ? best_id : -1;
      h.y = hit ? __float_as_int(best_t) : 0;
      h.z = hit ? __float_as_int(bu) : 0;
      h.w = hit ? __float_as_int(bv) : 0;
      reinterpret_cast<int4*>(P.out)[ray] = h;
    }
  }
}

template <int W, bool CLAMP, bool ANY, bool COUNT>
int launch_w(const DevAccel& a, const float* rays, size_t n, void* out, uint32_t* visits,
             const Launch& L, cudaStream_t s) {
  TraceParams p;
  p.nodes = static_cast<const uint8_t*>(a.d_nodes);
  p.tris = reinterpret_cast<const float4*>(a.d_tris);
  p.rays = reinterpret_cast<const float4*>(rays);
  p.out = out;
  p.visits = visits;
  p.counter = a.d_counter;
  p.status = a.d_status;
  p.nrays = (unsigned)n;
  p.nnodes = a.nnodes;
  p.ntris = a.ntris;
  p.stack_depth = L.stack;
  p.chunk = L.chunk;
  size_t smem = (size_t)L.stack * L.block * sizeof(uint2);
  auto k = wbvh_trace<W, CLAMP, ANY, COUNT>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  cudaError_t e = cudaMemsetAsync(a.d_counter, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return (int)e;
  int grid = device_sm_count(a.device) * L.blocks_per_sm;
  k<<<grid, L.block, smem, s>>>(p);
  return (int)cudaGetLastError();
}

template <bool ANY, bool COUNT>
int dispatch_w(const DevAccel& a, const float* rays, size_t n, void* out, uint32_t* visits,
               const Launch& L, cudaStream_t s) {
  const bool clamp = a.predicate == ENC_PRED_REFERENCE;
  switch (a.width) {
    case 2:
      return clamp ? launch_w<2, true, ANY, COUNT>(a, rays, n, out, visits, L, s)
                   : launch_w<2, false, ANY, COUNT>(a, rays, n, out, visits, L, s);
    case 4:
      return clamp ? launch_w<4, true, ANY, COUNT>(a, rays, n, out, visits, L, s)
                   : launch_w<4, false, ANY, COUNT>(a, rays, n, out, visits, L, s);
    default:
      return clamp ? launch_w<8, true, ANY, COUNT>(a, rays, n, out, visits, L, s)
                   : launch_w<8, false, ANY, COUNT>(a, rays, n, out, visits, L, s);
  }
}

template <bool ANY>
int launch_kd(const DevAccel& a, const float* rays, size_t n, void* out, cudaStream_t s) {
  KdParams p;
  p.nodes = a.d_kd;
  p.items = a.d_kd_items;
  p.tris = reinterpret_cast<const float4*>(a.d_tris);
  p.rays = reinterpret_cast<const float4*>(rays);
  p.out = out;
  p.status = a.d_status;
  p.nrays = (unsigned)n;
  p.nnodes = a.nnodes;
  p.nitems = a.kd_nitems;
  p.ntris = a.ntris;
  for (int i = 0; i < 3; ++i) {
    p.lo[i] = a.kd_root_lo[i];
    p.hi[i] = a.kd_root_hi[i];
  }
  int grid = device_sm_count(a.device) * 8;
  unsigned need = (unsigned)((n + 127) / 128);
  if ((unsigned)grid > need) grid = (int)need;
  if (grid < 1) grid = 1;
  if (a.predicate == ENC_PRED_REFERENCE)
    kd_trace<true, ANY><<<grid, 128, 0, s>>>(p);
  else
    kd_trace<false, ANY><<<grid, 128, 0, s>>>(p);
  return (int)cudaGetLastError();
}

}  // namespace

int device_sm_count(int device) {
  static int cache[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (cache[device] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0)
      v = 148;
    cache[device] = v;
  }
  return cache[device];
}

int launch_closest(const DevAccel& a, const float* d_rays, size_t n, enc_hit* d_hits,
                   const Launch& L, void* stream, uint32_t* d_visits) {
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (a.kind == ENC_ACCEL_KDTREE) return launch_kd<false>(a, d_rays, n, d_hits, s);
  if (d_visits) return dispatch_w<false, true>(a, d_rays, n, d_hits, d_visits, L, s);
  return dispatch_w<false, false>(a, d_rays, n, d_hits, nullptr, L, s);
}

int launch_any(const DevAccel& a, const float* d_rays, size_t n, uint8_t* d_occ, const Launch& L,
               void* stream) {
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (a.kind == ENC_ACCEL_KDTREE) return launch_kd<true>(a, d_rays, n, d_occ, s);
  return dispatch_w<true, false>(a, d_rays, n, d_occ, nullptr, L, s);
}

}  // namespace enc
