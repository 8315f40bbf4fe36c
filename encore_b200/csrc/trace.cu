// Ray traversal kernels for sm_100a.
//
//  * wbvh_trace<W, CLAMP, ANY, COUNT, MULTI, LANE>: persistent warps over the
//    quantised wide BVH.  Each warp takes rays from a global atomic queue in
//    chunks and hands them to idle lanes as lanes finish (no lane waits for
//    the slowest ray of a batch).  The traversal stack lives in shared
//    memory, one column per thread.  A visited node continues with its first
//    hit internal child; the others stay on the stack as one group entry.
//    The triangles of its hit leaves are tested in the same step: for closest
//    hit by the whole warp together (all lanes' triangles, one per lane per
//    round), for any hit and with LANE by each lane in turn.  Width 8 orders
//    children by octant (the builder places each child in the slot of its
//    octant, so slot k ^ octm for k = 0..7 is roughly front to back for a ray
//    with direction sign bits octm); widths 2 and 4 sort hit children by
//    entry distance.  MULTI launches trace many scenes' batches at once.
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

// Resident 128-thread blocks per SM that each kernel's register budget is
// fitted to (also the default grid: SMs x this).  The closest-hit kernel
// tests triangles cooperatively across the warp (below).  At 9 blocks it fits
// 56 registers without spilling and ran 1.7 % faster than at 8 (64
// registers) on the 2M-triangle heightfield workload; at 10 blocks (48
// registers) it spills 42 bytes and lost 8 %.  The multi-scene form keeps 8
// blocks: at 9 it spills 78 bytes.  The any-hit kernel keeps the per-lane
// loop (its rays rarely reach a triangle before the first hit) at 9 blocks
// (no spill; 3.9 % faster than 10 with a 28-byte spill).  The per-lane
// closest-hit form, which the host-buffer pipeline runs beside its copies,
// keeps 10 (at 9 the pipeline measured about 1 % slower).
constexpr int kBlocksClosest = 9;
constexpr int kBlocksMulti = 8;
constexpr int kBlocksAny = 9;
constexpr int kBlocksLane = 10;

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

// A float's bits made monotone as an unsigned integer (negative values
// below positive ones, order kept within each sign), and back.
__device__ __forceinline__ uint32_t order_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float from_order_key(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct TraceParams {
  const uint8_t* nodes;
  const float4* tris;  // 3 per triangle
  const float4* rays;  // 2 per ray
  const uint32_t* order;  // null, or: queue index q traces ray order[q] (binned batches)
  void* out;           // enc_hit* (closest) or uint8_t* (any)
  uint32_t* visits;    // COUNT: 2 per ray
  unsigned* counter;
  uint32_t* status;
  unsigned nrays;
  unsigned nnodes;
  unsigned ntris;
  int stack_depth;
  int chunk;
  // multi-scene launches (MULTI = true): per-batch scene and buffers
  const SceneDesc* scenes;
  const BatchDesc* batches;
  const uint32_t* starts;  // nbatches + 1 chunk-aligned queue offsets
  unsigned nbatches;
  uint32_t* batch_status;  // MULTI: one status word per batch, or null (all in *status)
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

// An 8-bit quantised coordinate as a float: the byte placed under the
// exponent of 2^23 gives 2^23 + q exactly; subtracting 2^23 is exact.
__device__ __forceinline__ float u8f(uint32_t q) {
  return __uint_as_float(0x4B000000u | q) - 8388608.0f;
}

template <int W>
struct NodeWords {
  static constexpr int N = WNodeLayout<W>::kBytes / 16;
  uint4 w[N];
};

constexpr uint32_t kNoItem = 0xffffffffu;

// Packed FP32 pairs (sm_100 `add/sub/mul/fma.rn.f32x2`): two floats per
// instruction, each half rounded exactly as the scalar operation, so results
// are bit-identical to the scalar form.  The width-8 slab test computes its
// 48 plane distances as 24 pairs (measured +2 % closest hit and +5 % any hit
// on the 2M-triangle heightfield, identical hits); kPairs = false keeps the
// scalar form.
#ifndef ENC_F32X2
#define ENC_F32X2 1
#endif
#ifndef ENC_GROUP_BOUND
#define ENC_GROUP_BOUND 0
#endif
// Width 8, closest hit: the stack group's lower bound (the smallest entry
// distance among the node's hit internal children) includes the child the
// walk continues into, and the hit found under that child is rarely nearer
// than its entry, so a popped group was culled by it 0.0002 times per ray on
// the 2M-triangle heightfield batch.  Without it such a group's node is
// visited and every child fails the box test against the same closest hit
// (so the hits are identical) and the per-child bound work is saved.
constexpr bool kGroupBound = ENC_GROUP_BOUND != 0;
constexpr bool kPairs = ENC_F32X2 != 0;

__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}


// L2 eviction priorities: rays are read once and hits written once, so they
// go in as evict_first, and the nodes, read by every ray, as evict_last; the
// streaming data then displaces less of the node and triangle working set
// (about the L2's size on the 2M-triangle heightfield).  +0.36 % for the
// cooperative closest-hit kernel, identical hits.
__device__ __forceinline__ uint64_t l2_policy_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float4 ldg_hint(const float4* a, uint64_t pol) {
  float4 v;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint4 ldg_hint_u(const uint4* a, uint64_t pol) {
  uint4 v;
  asm("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void stg_hint(int4* a, int4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.s32 [%0], {%1,%2,%3,%4}, %5;" ::"l"(a), "r"(v.x),
               "r"(v.y), "r"(v.z), "r"(v.w), "l"(pol)
               : "memory");
}

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
#undef ENC_CSWAP

template <int W, bool CLAMP, bool ANY, bool COUNT, bool MULTI = false, bool LANE = false,
          bool ORD = false>
__global__ void __launch_bounds__(128, ANY    ? kBlocksAny
                                      : LANE ? kBlocksLane
                                             : (MULTI ? kBlocksMulti : kBlocksClosest))
    wbvh_trace(TraceParams P) {
  using L = WNodeLayout<W>;
  // Stack of node groups: one entry per visited node that still has hit
  // internal children, so the depth never exceeds the tree depth.
  //   W == 8: x = child_base, y = remaining hit children as bits k in
  //           octant order (slot = k ^ octm) | internal-slot mask << 8;
  //           lb = smallest entry distance among the group's hit children.
  //   W < 8:  x = child_base, y = ranks of the remaining children sorted by
  //           entry distance (3 bits each, nearest first) | count << 24;
  //           lb = entry distance of the nearest remaining child.
  // lb is a lower bound for every child still in the group, so a group
  // whose lb exceeds the closest hit so far is dropped whole.
  //   Width-8 entries carry lb in the top 16 bits of y (the float's high
  //   half: rounded toward zero, so never above lb for lb >= 0; a negative
  //   lb is stored as -inf), which keeps an entry at 8 bytes of shared
  //   memory and leaves more of the SM's L1 to node and triangle loads.
  constexpr bool kCompact = W == 8;
  extern __shared__ uint2 s_stack[];
  // Closest hit tests the triangles of the lanes' hit leaves as one warp
  // (see below); any hit, and closest hit with LANE, keep one loop per lane.
  constexpr bool kCoop = !ANY && !LANE;
  // the per-lane form keeps the group bound (without it ptxas spills more)
  constexpr bool kBound = kGroupBound || LANE;
  // L2 priorities in the single-scene cooperative closest-hit form only: in
  // any hit they measured 1 % slower, and in the per-lane form, which the
  // host-buffer pipeline runs, the evict_first hits left L2 before their copy
  // out (2 %); the multi-scene form, whose hits the server copies out after
  // each launch, keeps plain loads and stores too
  constexpr bool kL2Hints = kCoop && !MULTI;
  __shared__ uint32_t s_coop_tri[kCoop ? 128 : 1];
  __shared__ uint32_t s_coop_own[kCoop ? 128 : 1];
  __shared__ unsigned long long s_coop_key[kCoop ? 128 : 1];
  __shared__ float2 s_coop_uv[kCoop ? 128 : 1];
  __shared__ int s_coop_cnt[kCoop ? 4 : 1];  // per warp: items listed this round
  // Each lane's ray, its reciprocal direction and sign bits, stored when the
  // lane takes the ray: the rounds' workers read their owners' rays here, and
  // with kRayShared the lane itself rereads them at every node instead of
  // holding eleven registers across the traversal loop.
  constexpr bool kRayShared = kCoop;
  __shared__ float4 s_ray[kCoop ? 384 : 1];
  const int B = blockDim.x;
  uint2* stk = s_stack + threadIdx.x;  // entry i at stk[i * B]
  float* slb = reinterpret_cast<float*>(s_stack + (size_t)P.stack_depth * B) + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = lanemask_lt();

  // Warp-private ray pool [pool_next, pool_end), refilled in chunks.
  unsigned pool_next = 0, pool_end = 0;
  bool exhausted = false;
  // Binned batches: lane j holds order[pool_base + j] of the current chunk,
  // loaded once when the chunk is taken (one coalesced load per chunk instead
  // of a dependent load per refill); chunks above 32 rays read the rest
  // directly.
  // binned batches (closest hit only): a separate instantiation, so the plain
  // launch carries none of the order handling
  constexpr bool kOrdered = ORD && !MULTI && !ANY;
  unsigned pool_base = 0, ord_reg = 0;

  int ray = -1;
  float ox = 0, oy = 0, oz = 0, dx = 0, dy = 0, dz = 0, ix = 0, iy = 0, iz = 0, tmin = 0, tmax = 0;
  float best_t = 0, bu = 0, bv = 0;
  int best_id = -1;
  int sp = 0;
  uint32_t node = kNoItem;
  uint32_t octm = 0;  // direction sign bits: bit a set = negative along axis a
  unsigned steps = 0;
  uint32_t nvis = 0, ntest = 0;
  // The scene a lane's ray belongs to (MULTI: per batch, else the launch's).
  const uint8_t* l_nodes = P.nodes;
  const float4* l_tris = P.tris;
  unsigned l_nnodes = P.nnodes, l_ntris = P.ntris;
  void* l_out = P.out;
  unsigned l_idx = 0;          // index of the ray in its output array
  unsigned pool_batch = 0;     // MULTI: batch of the current pool
  uint32_t* l_status = P.status;  // the status word of the lane's ray (MULTI: its batch's)

  while (true) {
    // ---- refill idle lanes from the warp pool --------------------------
    unsigned need = __ballot_sync(kFull, ray < 0);
    while (need && !exhausted) {
      if (pool_next >= pool_end) {
        unsigned b = 0;
        if (lane == 0) {
          b = atomicAdd(P.counter, (unsigned)P.chunk);
          // Rays are read once, so every refill would wait on DRAM: bring the
          // chunk one full grid of claims ahead into L2 now (one bulk
          // prefetch; the warp that claims it later finds it in L2).  With the
          // round's atomic listing below: +1.7 % on the 2M-triangle
          // heightfield batch (the listing alone measured -1.2 %).
          if (!MULTI && !kOrdered) {
            const unsigned ahead = gridDim.x * (blockDim.x >> 5) * (unsigned)P.chunk;
            const unsigned pb = b + ahead;
            if (pb > b && pb < P.nrays) {
              const unsigned cnt = min((unsigned)P.chunk, P.nrays - pb);
              asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(P.rays + 2 * (size_t)pb),
                           "r"(cnt * 32u)
                           : "memory");
            }
          }
        }
        b = __shfl_sync(kFull, b, 0);
        if (b >= P.nrays) {
          exhausted = true;
          break;
        }
        pool_next = b;
        pool_base = b;
        if (kOrdered && P.order != nullptr && b + lane < P.nrays) ord_reg = __ldg(P.order + b + lane);
        if constexpr (MULTI) {
          // batch = last start <= b (starts are chunk-aligned, so the whole
          // chunk lies in it); its real rays end before the padding
          unsigned lo = 0, hi = P.nbatches;
          while (hi - lo > 1) {
            const unsigned mid = (lo + hi) >> 1;
            if (__ldg(P.starts + mid) <= b) lo = mid;
            else hi = mid;
          }
          pool_batch = lo;
          pool_end = min(b + (unsigned)P.chunk, __ldg(P.starts + lo) + P.batches[lo].nrays);
        } else {
          pool_end = min(b + (unsigned)P.chunk, P.nrays);
        }
      }
      const unsigned avail = pool_end > pool_next ? pool_end - pool_next : 0u;
      const unsigned rank = __popc(need & lt);
      const unsigned qoff = pool_next - pool_base + rank;  // offset of this lane's ray in the chunk
      const unsigned via = kOrdered ? __shfl_sync(kFull, ord_reg, qoff & 31u) : 0u;
      bool bad_order = false;
      if (((need >> lane) & 1u) && rank < avail) {
        ray = (int)(pool_next + rank);
        if (kOrdered && P.order != nullptr) {
          const unsigned oi = qoff < 32u ? via : __ldg(P.order + pool_next + rank);
          // an order entry outside the batch is skipped and reported
          bad_order = oi >= P.nrays;
          ray = bad_order ? -1 : (int)oi;
        }
      }
      if (bad_order) atomicOr(l_status, kStatusBounds);
      if (ray >= 0 && ((need >> lane) & 1u) && rank < avail) {
        const float4* rp;
        if constexpr (MULTI) {
          const BatchDesc& bd = P.batches[pool_batch];
          const SceneDesc& sd = P.scenes[bd.scene];
          l_idx = (unsigned)ray - bd.start;
          l_out = bd.out;
          l_nodes = sd.nodes;
          l_tris = reinterpret_cast<const float4*>(sd.tris);
          l_nnodes = sd.nnodes;
          l_ntris = sd.ntris;
          if (P.batch_status) l_status = P.batch_status + pool_batch;
          rp = reinterpret_cast<const float4*>(bd.rays) + 2 * (size_t)l_idx;
        } else {
          l_idx = (unsigned)ray;
          rp = P.rays + 2 * (size_t)ray;
        }
        const float4 r0 = kL2Hints ? ldg_hint(rp, l2_policy_first()) : __ldg(rp);
        const float4 r1 = kL2Hints ? ldg_hint(rp + 1, l2_policy_first()) : __ldg(rp + 1);
        ox = r0.x; oy = r0.y; oz = r0.z; tmin = r0.w;
        dx = r1.x; dy = r1.y; dz = r1.z; tmax = r1.w;

        // Box tests use a reciprocal with |d| floored at 1e-20 so that a zero
        // direction component (the reference's Normalize clamps small ones to
        // exactly 0) gives finite slab distances instead of 0 * inf = NaN,
        // which would leave that axis unconstrained.  The triangle predicate
        // keeps the exact direction.
        // The hardware reciprocal (rcp.approx, within 1 ulp) is enough here:
        // an error of an ulp scales one axis's slab distances by 1 +- 2^-23,
        // far inside the 1e-5 padding that keeps every accepted hit point off
        // its box's faces, and it saves an IEEE division per axis each time a
        // lane takes a new ray (measured +2.4 % closest, +3 % any hit).
        auto rcp = [](float x) {
          float r;
          asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
          return r;
        };
        ix = rcp(fabsf(dx) > 1e-20f ? dx : copysignf(1e-20f, dx));
        iy = rcp(fabsf(dy) > 1e-20f ? dy : copysignf(1e-20f, dy));
        iz = rcp(fabsf(dz) > 1e-20f ? dz : copysignf(1e-20f, dz));
        octm = (dx < 0.f ? 1u : 0u) | (dy < 0.f ? 2u : 0u) | (dz < 0.f ? 4u : 0u);
        if (kCoop) {
          s_ray[3 * threadIdx.x] = r0;
          s_ray[3 * threadIdx.x + 1] = r1;
          s_ray[3 * threadIdx.x + 2] = make_float4(ix, iy, iz, __uint_as_float(octm));
        }
        best_t = tmax; best_id = -1; bu = 0.f; bv = 0.f;
        sp = 0;
        node = 0;  // root
        steps = 0;
        nvis = 0; ntest = 0;
      }
      const unsigned took = min(avail, (unsigned)__popc(need));
      pool_next += took;
      need = __ballot_sync(kFull, ray < 0);
    }
    if (__all_sync(kFull, ray < 0)) break;

    bool done = false;
    bool hit_any = false;
    uint32_t tmask = 0, tbase = 0;  // triangles of the node's hit leaves
    if (ray >= 0) {
      if (++steps > kMaxSteps) {
        atomicOr(l_status, kStatusWatchdog);
        best_id = -1;
        done = true;
      } else if (node >= l_nnodes) {
        atomicOr(l_status, kStatusBounds);
        best_id = -1;
        done = true;
      } else {
        // ---- visit one node: its hit leaves now, its hit internal children
        //      in front-to-back order (one continues, the rest become one
        //      group on the stack) ------------------------------------------
        if (COUNT) ++nvis;
        NodeWords<W> nw;
        const uint4* src = reinterpret_cast<const uint4*>(l_nodes + (size_t)node * L::kBytes);
#pragma unroll
        for (int i = 0; i < NodeWords<W>::N; ++i)
          nw.w[i] = kL2Hints ? ldg_hint_u(src + i, l2_policy_last()) : __ldg(src + i);
        const float px = __uint_as_float(nw.w[0].x);
        const float py = __uint_as_float(nw.w[0].y);
        const float pz = __uint_as_float(nw.w[0].z);
        const uint32_t ew = nw.w[0].w;
        const float sx = __uint_as_float((ew & 0xffu) << 23);
        const float sy = __uint_as_float(((ew >> 8) & 0xffu) << 23);
        const float sz = __uint_as_float(((ew >> 16) & 0xffu) << 23);
        const uint32_t child_base = nw.w[1].x;
        const uint32_t tri_base = nw.w[1].y;
        float vox = ox, voy = oy, voz = oz, vtmin = tmin, vix = ix, viy = iy, viz = iz;
        uint32_t voct = octm;
        if constexpr (kRayShared) {
          const float4 sa = s_ray[3 * threadIdx.x], sc = s_ray[3 * threadIdx.x + 2];
          vox = sa.x; voy = sa.y; voz = sa.z; vtmin = sa.w;
          vix = sc.x; viy = sc.y; viz = sc.z;
          voct = __float_as_uint(sc.w);
        }
        const float bx = (px - vox) * vix, by = (py - voy) * viy, bz = (pz - voz) * viz;
        const float cx = sx * vix, cy = sy * viy, cz = sz * viz;
        // Near and far planes per axis by the ray's direction sign: the
        // near plane of a child box is its lo corner for a positive
        // direction and its hi corner for a negative one.
        const bool nxs = (voct & 1u) != 0, nys = (voct & 2u) != 0, nzs = (voct & 4u) != 0;
        float key[W];
        uint32_t rnk[W];
        uint32_t trimask = 0;
        uint32_t hitk = 0;      // W == 8: hit internal children, bit k = slot k ^ voct
        float lbmin = INFINITY;  // W == 8: smallest entry distance of those
        int nh = 0;
        // Width 8: the six plane arrays are whole words (qlo x at words 8-9,
        // y 10-11, z 12-13, qhi x 14-15, y 16-17, z 18-19), so near/far are
        // chosen once per word and each byte becomes 2^23 + q with one PRMT.
        uint32_t wn[6], wf[6];
        if constexpr (W == 8) {
          const uint32_t* u = reinterpret_cast<const uint32_t*>(nw.w);
          const bool neg[3] = {nxs, nys, nzs};
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const uint32_t lo = u[8 + 2 * a + h], hi = u[14 + 2 * a + h];
              wn[2 * a + h] = neg[a] ? hi : lo;
              wf[2 * a + h] = neg[a] ? lo : hi;
            }
        }
        if constexpr (W == 8) {
          // Slab test of the eight children into a hit-slot mask; the header's
          // internal-slot mask splits it into internal and leaf hits.  Empty
          // slots hold an inverted box (lo 255, hi 0), whose near plane lies
          // beyond its far plane for either direction sign, so they never hit
          // (and a leaf entry with meta 0 would contribute no triangles).
          const uint32_t imask = ew >> 24;
          uint32_t hm = 0;
          // pairs: x and y share one pair for the near planes and one for the
          // far planes; z pairs its near and far plane
          const unsigned long long m23 = pack2(-8388608.0f, -8388608.0f);
          // (bx, by) and (cx, cy) as pairs: the node origin, the ray origin and
          // the reciprocal direction already sit in adjacent halves of their
          // 16-byte loads
          const unsigned long long vixy = pack2(vix, viy);
          const unsigned long long bxy = mul2(sub2(pack2(px, py), pack2(vox, voy)), vixy);
          const unsigned long long cxy = mul2(pack2(sx, sy), vixy);
          const unsigned long long czz = pack2(cz, cz), bzz = pack2(bz, bz);
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const uint32_t sel = 0x7650u | (uint32_t)(c & 3);
            const int h = c >> 2;
            float tnx, tfx, tny, tfy, tnz, tfz;
            if constexpr (kPairs) {
              // 2^23 + q, minus 2^23, times the scaled reciprocal plus the
              // origin offset, two planes at a time
              auto q2 = [&](uint32_t a, uint32_t b) {
                return add2(pack2(__uint_as_float(__byte_perm(a, 0x4B000000u, sel)),
                                  __uint_as_float(__byte_perm(b, 0x4B000000u, sel))),
                            m23);
              };
              unpack2(fma2(q2(wn[0 + h], wn[2 + h]), cxy, bxy), tnx, tny);
              unpack2(fma2(q2(wf[0 + h], wf[2 + h]), cxy, bxy), tfx, tfy);
              unpack2(fma2(q2(wn[4 + h], wf[4 + h]), czz, bzz), tnz, tfz);
            } else {
              tnx = fmaf(__uint_as_float(__byte_perm(wn[0 + h], 0x4B000000u, sel)) - 8388608.0f, cx, bx);
              tfx = fmaf(__uint_as_float(__byte_perm(wf[0 + h], 0x4B000000u, sel)) - 8388608.0f, cx, bx);
              tny = fmaf(__uint_as_float(__byte_perm(wn[2 + h], 0x4B000000u, sel)) - 8388608.0f, cy, by);
              tfy = fmaf(__uint_as_float(__byte_perm(wf[2 + h], 0x4B000000u, sel)) - 8388608.0f, cy, by);
              tnz = fmaf(__uint_as_float(__byte_perm(wn[4 + h], 0x4B000000u, sel)) - 8388608.0f, cz, bz);
              tfz = fmaf(__uint_as_float(__byte_perm(wf[4 + h], 0x4B000000u, sel)) - 8388608.0f, cz, bz);
            }
            // sm_100's three-input max/min (NaN operands ignored, as fmaxf /
            // fminf do): +0.45 % over the two-input tree
            float tn, tf;
            {
              float m;
              asm("max.f32 %0, %1, %2, %3;" : "=f"(m) : "f"(tnx), "f"(tny), "f"(tnz));
              tn = fmaxf(m, vtmin);
              asm("min.f32 %0, %1, %2, %3;" : "=f"(m) : "f"(tfx), "f"(tfy), "f"(tfz));
              tf = fminf(m, best_t);
            }
            if (tn <= tf) {
              hm |= 1u << c;
              // (any hit never culls by distance, so it keeps no bound)
              if (!ANY && kBound && ((imask >> c) & 1u)) lbmin = fminf(lbmin, tn);
            }
          }
          // triangles of the hit leaves (meta = count << 5 | offset)
          // (the meta bytes are words 6 and 7 of the node, bytes 24-31; they
          // are picked by select and shift, not by indexing the node array
          // with the runtime slot c, which would move it to local memory)
          uint32_t lh = hm & ~imask;
          const uint32_t mlo = nw.w[1].z, mhi = nw.w[1].w;
          while (lh) {
            const uint32_t c = __ffs(lh) - 1;
            lh &= lh - 1;
            const uint32_t meta = (((c & 4u) ? mhi : mlo) >> ((c & 3u) * 8u)) & 0xffu;
            trimask |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
          }
          // hit internal children in octant order: bit k = slot k ^ voct
          uint32_t x = hm & imask;
          if (voct & 1u) x = ((x & 0x55u) << 1) | ((x >> 1) & 0x55u);
          if (voct & 2u) x = ((x & 0x33u) << 2) | ((x >> 2) & 0x33u);
          if (voct & 4u) x = ((x & 0x0fu) << 4) | ((x >> 4) & 0x0fu);
          hitk = x;
        } else {
#pragma unroll
          for (int c = 0; c < W; ++c) {
            const uint32_t qlx = byte_of(nw.w, L::kQOff + 0 * W + c);
            const uint32_t qly = byte_of(nw.w, L::kQOff + 1 * W + c);
            const uint32_t qlz = byte_of(nw.w, L::kQOff + 2 * W + c);
            const uint32_t qhx = byte_of(nw.w, L::kQOff + 3 * W + c);
            const uint32_t qhy = byte_of(nw.w, L::kQOff + 4 * W + c);
            const uint32_t qhz = byte_of(nw.w, L::kQOff + 5 * W + c);
            const float tnx = fmaf(u8f(nxs ? qhx : qlx), cx, bx);
            const float tfx = fmaf(u8f(nxs ? qlx : qhx), cx, bx);
            const float tny = fmaf(u8f(nys ? qhy : qly), cy, by);
            const float tfy = fmaf(u8f(nys ? qly : qhy), cy, by);
            const float tnz = fmaf(u8f(nzs ? qhz : qlz), cz, bz);
            const float tfz = fmaf(u8f(nzs ? qlz : qhz), cz, bz);
            const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, vtmin));
            const float tf = fminf(fminf(tfx, tfy), fminf(tfz, best_t));
            const uint32_t meta = byte_of(nw.w, L::kMetaOff + c);
            const bool hit = meta != 0u && tn <= tf;
            const bool leaf = meta >= 32u;
            if (hit && leaf) trimask |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
            const bool ih = hit && !leaf;
            key[c] = ih ? fminf(tn, 3.0e38f) : INFINITY;  // hits sort before the rest
            rnk[c] = meta - 1u;
            nh += ih ? 1 : 0;
          }
        }
        // ---- next node, and the group of the other hit children ----------
        if constexpr (W == 8) {
          if (hitk) {
            const uint32_t imask = ew >> 24;
            const uint32_t k = __ffs(hitk) - 1;
            const uint32_t slot = k ^ voct;
            node = child_base + __popc(imask & ((1u << slot) - 1u));
            const uint32_t rest = hitk & (hitk - 1u);
            if (rest) {
              if (sp >= P.stack_depth) {
                atomicOr(l_status, kStatusStack);
                best_id = -1;
                done = true;
              } else {
                if constexpr (kCompact) {
                  const uint32_t lb16 =
                      (ANY || !kBound) ? 0u
                                            : (lbmin >= 0.0f ? (__float_as_uint(lbmin) >> 16) : 0xff80u);
                  stk[sp * B] = make_uint2(child_base, rest | (imask << 8) | (lb16 << 16));
                } else {
                  stk[sp * B] = make_uint2(child_base, rest | (imask << 8));
                  slb[sp * B] = lbmin;
                }
                ++sp;
              }
            }
          } else {
            node = kNoItem;
          }
        } else {
          if (nh > 0) {
            sort_net<W>(key, rnk);
            node = child_base + rnk[0];
            if (nh > 1) {
              if (sp >= P.stack_depth) {
                atomicOr(l_status, kStatusStack);
                best_id = -1;
                done = true;
              } else {
                uint32_t packed = 0;
#pragma unroll
                for (int c = W - 1; c >= 1; --c)
                  if (c < nh) packed = (packed << 3) | (rnk[c] & 7u);
                stk[sp * B] = make_uint2(child_base, packed | ((uint32_t)(nh - 1) << 24));
                slb[sp * B] = key[1];
                ++sp;
              }
            }
          } else {
            node = kNoItem;
          }
        }
        // ---- triangles of the hit leaves ---------------------------------
        tmask = trimask;
        tbase = tri_base;
        if (kCoop) trimask = 0;  // tested below by the whole warp
        while (!kCoop && trimask) {
          const uint32_t k = __ffs(trimask) - 1;
          trimask &= trimask - 1;
          const uint32_t ti = tri_base + k;
          if (ti >= l_ntris) {
            atomicOr(l_status, kStatusBounds);
            continue;
          }
          const float4* tp = l_tris + 3 * (size_t)ti;
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
        if (ANY && hit_any) done = true;
      }
    }
    if constexpr (kCoop) {
    // ---- the warp tests all lanes' pending triangles together -------------
    // Each round lists up to 32 (lane, triangle) items in shared memory; lane
    // w tests item w with the owner lane's ray, and the owner's closest hit
    // is the minimum of (t, ID) over its accepted candidates, taken with a
    // 64-bit shared atomicMin on an order-preserving key (t's bits made
    // monotone, then the ID) -- the same choice as the per-lane loop's
    // "t < best_t, or equal t and a lower ID", whatever the order.
    {
      unsigned pend = __ballot_sync(kFull, tmask != 0);
      const unsigned wib = threadIdx.x >> 5;
      uint32_t* it_tri = s_coop_tri + wib * 32;
      uint32_t* it_own = s_coop_own + wib * 32;
      unsigned long long* key = s_coop_key + wib * 32;
      float2* uv = s_coop_uv + wib * 32;
      while (pend) {
        const int ni = __popc(tmask);
        // each lane with items claims its slots with one shared atomic (the
        // list order does not matter: the closest hit is a minimum)
        if (lane == 0) s_coop_cnt[wib] = 0;
        __syncwarp();
        const int excl = ni ? atomicAdd(&s_coop_cnt[wib], ni) : 0;
        __syncwarp();
        const int total = s_coop_cnt[wib];
        int j = 0;
        while (tmask && excl + j < 32) {
          const uint32_t k = __ffs(tmask) - 1;
          tmask &= tmask - 1;
          it_tri[excl + j] = tbase + k;
          it_own[excl + j] = lane;
          ++j;
        }
        if (COUNT) ntest += j;
        const unsigned long long mykey =
            ((unsigned long long)order_key(best_t) << 32) | (uint32_t)best_id;
        key[lane] = mykey;
        __syncwarp();
        const int nitems = total < 32 ? total : 32;
        const int own = (int)lane < nitems ? (int)it_own[lane] : (int)lane;
        // the owner's ray, kept in shared memory since its refill (two
        // 16-byte loads instead of seven shuffles; measured +1 %)
        const float4 wr0 = s_ray[3 * (wib * 32 + own)], wr1 = s_ray[3 * (wib * 32 + own) + 1];
        const float wox = wr0.x, woy = wr0.y, woz = wr0.z, wtmin = wr0.w;
        const float wdx = wr1.x, wdy = wr1.y, wdz = wr1.z;
        const float wlim = __shfl_sync(kFull, ANY ? tmax : best_t, own);
        const int wbid = __shfl_sync(kFull, best_id, own);
        const float4* wtris = l_tris;
        unsigned wntris = l_ntris;
        uint32_t* wstatus = P.status;
        if constexpr (MULTI) {
          const unsigned long long tp = __shfl_sync(kFull, (unsigned long long)l_tris, own);
          wtris = reinterpret_cast<const float4*>(tp);
          wntris = __shfl_sync(kFull, l_ntris, own);
          wstatus = reinterpret_cast<uint32_t*>(
              __shfl_sync(kFull, (unsigned long long)l_status, own));
        }
        bool cand = false;
        unsigned long long ckey = 0;
        float cu = 0.f, cv = 0.f;
        if ((int)lane < nitems) {
          const uint32_t ti = it_tri[lane];
          if (ti >= wntris) {
            atomicOr(wstatus, kStatusBounds);
          } else {
            const float4* tp = wtris + 3 * (size_t)ti;
            const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, u, v;
            if (tri_test<CLAMP>(a, b, c, wox, woy, woz, wdx, wdy, wdz, wtmin, t, u, v)) {
              const int id = __float_as_int(c.y);
              if (ANY) {
                if (t < wlim) key[own] = 0ull;  // any hit: the owner is done
              } else if (t < wlim || (t == wlim && id < wbid)) {
                cand = true;
                ckey = ((unsigned long long)order_key(t) << 32) | (uint32_t)id;
                cu = u;
                cv = v;
                atomicMin(&key[own], ckey);
              }
            }
          }
        }
        __syncwarp();
        if (cand && key[own] == ckey) uv[own] = make_float2(cu, cv);
        __syncwarp();
        const unsigned long long nk = key[lane];
        if (ANY) {
          if (nk == 0ull && ray >= 0) {
            hit_any = true;
            done = true;
            tmask = 0;
          }
        } else if (nk != mykey) {
          best_t = from_order_key((uint32_t)(nk >> 32));
          best_id = (int)(uint32_t)nk;
        }
        __syncwarp();
        pend = __ballot_sync(kFull, tmask != 0);
      }
    }
    }
    if (ray >= 0) {
      // ---- pop the next group child that can still matter ----------------
      if (!done && node == kNoItem) {
        while (sp > 0) {
          uint2 e;
          if constexpr (kCompact) {
            e = stk[(sp - 1) * B];
            if (!ANY && kBound && __uint_as_float(e.y & 0xffff0000u) > best_t) {
              --sp;
              continue;
            }
          } else {
            if (!ANY && slb[(sp - 1) * B] > best_t) {
              --sp;
              continue;
            }
            e = stk[(sp - 1) * B];
          }
          if constexpr (W == 8) {
            const uint32_t hk = e.y & 0xffu;
            const uint32_t k = __ffs(hk) - 1;
            const uint32_t slot =
                k ^ (kRayShared ? __float_as_uint(s_ray[3 * threadIdx.x + 2].w) : octm);
            const uint32_t imask = (e.y >> 8) & 0xffu;
            node = e.x + __popc(imask & ((1u << slot) - 1u));
            const uint32_t rest = hk & (hk - 1u);
            if (rest == 0) {
              --sp;
            } else {
              e.y = (e.y & 0xffff0000u) | rest | (imask << 8);
              stk[(sp - 1) * B] = e;
            }
          } else {
            const uint32_t cnt = e.y >> 24;
            node = e.x + (e.y & 7u);
            if (cnt <= 1) {
              --sp;
            } else {
              e.y = (((e.y & 0xffffffu) >> 3)) | ((cnt - 1) << 24);
              stk[(sp - 1) * B] = e;
            }
          }
          break;
        }
        if (node == kNoItem) done = true;
      }
      if (done) {
        if (ANY) {
          reinterpret_cast<uint8_t*>(l_out)[l_idx] = hit_any ? 1 : 0;
        } else {
          int4 h;
          h.x = best_id;
          h.y = best_id >= 0 ? __float_as_int(best_t) : 0;
          float hu = bu, hv = bv;
          if constexpr (kCoop) {
            // the round that found the hit left its barycentrics in shared memory
            const float2 w = s_coop_uv[threadIdx.x];
            hu = w.x;
            hv = w.y;
          }
          h.z = best_id >= 0 ? __float_as_int(hu) : 0;
          h.w = best_id >= 0 ? __float_as_int(hv) : 0;
          if (kL2Hints)
            stg_hint(reinterpret_cast<int4*>(l_out) + l_idx, h, l2_policy_first());
          else
            reinterpret_cast<int4*>(l_out)[l_idx] = h;
        }
        if (COUNT) {
          P.visits[2 * (size_t)ray] = nvis;
          P.visits[2 * (size_t)ray + 1] = ntest;
        }
        ray = -1;
        node = kNoItem;
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
  const uint32_t* order;  // null, or: the i-th ray walked is ray order[i] (binned batches)
  void* out;
  uint32_t* status;
  unsigned nrays, nnodes, nitems, ntris;
  float lo[3], hi[3];  // root box min corner and pos + size
};

// Deferred far children of the walk: at most one per level, so a tree of
// depth <= 32 (the reference's depth limit 11 + 1.3 ln N stays below 32 up
// to about 10M triangles) needs 32 entries; deeper trees get 64.  The
// stack lives in local memory: the smaller one halves its traffic.
// Resident blocks per SM for the kd walk: one thread walks one ray, so its
// latency is hidden only by other warps.  At 10 blocks (48 registers, a
// 16-byte spill) it ran 6.8 % faster than at 8 (53 registers); 12 and 16
// spill 80 and 216 bytes and lose.
constexpr int kKdBlocks = 10;

template <bool CLAMP, bool ANY, int kKdStack>
__global__ void __launch_bounds__(128, kKdBlocks) kd_trace(KdParams P) {
  for (unsigned qi = blockIdx.x * blockDim.x + threadIdx.x; qi < P.nrays;
       qi += gridDim.x * blockDim.x) {
    const unsigned ray = P.order ? __ldg(P.order + qi) : qi;
    if (ray >= P.nrays) {  // an order entry outside the batch: skipped and reported
      atomicOr(P.status, kStatusBounds);
      continue;
    }
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
          // the axis's origin and reciprocal by select, not by indexing the
          // arrays with the runtime axis (which would put them in local memory)
          const float oa = axis == 0 ? o[0] : (axis == 1 ? o[1] : o[2]);
          const float ia = axis == 0 ? inv[0] : (axis == 1 ? inv[1] : inv[2]);
          const float tplane = fm(fs(split, oa), ia);
          const bool below = oa <= split;
          const uint32_t first = below ? n.word1 : n.word1 + 1;
          const uint32_t second = below ? n.word1 + 1 : n.word1;
          if (tplane == 0.0f) {
            node = ia > 0.0f ? second : first;
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

// Shared memory per stack entry: width 8 packs lb into the 8-byte entry;
// widths 2 and 4 keep it in a separate float array.
constexpr size_t stack_entry_bytes(int W) {
  return W == 8 ? sizeof(uint2) : sizeof(uint2) + sizeof(float);
}

template <int W, bool CLAMP, bool ANY, bool COUNT>
int launch_w(const DevAccel& a, const float* rays, size_t n, void* out, uint32_t* visits,
             const Launch& L, cudaStream_t s, const uint32_t* order) {
  TraceParams p{};
  p.nodes = static_cast<const uint8_t*>(a.d_nodes);
  p.tris = reinterpret_cast<const float4*>(a.d_tris);
  p.rays = reinterpret_cast<const float4*>(rays);
  p.order = order;
  p.out = out;
  p.visits = visits;
  const uint32_t slot =
      __atomic_fetch_add(const_cast<uint32_t*>(&a.counter_seq), 1u, __ATOMIC_RELAXED) % kQueueSlots;
  p.counter = a.d_counter + slot;
  p.status = a.d_status;
  p.nrays = (unsigned)n;
  p.nnodes = a.nnodes;
  p.ntris = a.ntris;
  // Each visited node leaves at most one group entry, so tree_depth - 1
  // entries always suffice; 0 selects that bound.
  p.stack_depth = L.stack > 0 ? L.stack : (a.tree_depth > 8 ? a.tree_depth : 8);
  p.chunk = L.chunk;
  size_t smem = (size_t)p.stack_depth * L.block * stack_entry_bytes(W);
  const bool lane = !ANY && L.per_lane;
  // Binned (ordered) launches use their own instantiation (closest hit
  // only); without the order handling the plain cooperative kernel ran 1.6 %
  // faster.  The per-lane form, which the host-buffer pipeline runs beside
  // its copies, keeps it whatever the order: leaner, it ran faster but slowed
  // the concurrent copies more (the whole call 4 % slower).
  const bool ord = !ANY && order != nullptr;
  auto k = lane ? wbvh_trace<W, CLAMP, ANY, COUNT, false, true, true>
                : (ord ? wbvh_trace<W, CLAMP, ANY, COUNT, false, false, true>
                       : wbvh_trace<W, CLAMP, ANY, COUNT>);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  cudaError_t e = cudaMemsetAsync(p.counter, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return (int)e;
  int grid = device_sm_count(a.device) *
             (L.blocks_per_sm > 0 ? L.blocks_per_sm
                                  : (ANY ? kBlocksAny : (lane ? kBlocksLane : kBlocksClosest)));
  k<<<grid, L.block, smem, s>>>(p);
  return (int)cudaGetLastError();
}

template <bool ANY, bool COUNT>
int dispatch_w(const DevAccel& a, const float* rays, size_t n, void* out, uint32_t* visits,
               const Launch& L, cudaStream_t s, const uint32_t* order = nullptr) {
  const bool clamp = a.predicate == ENC_PRED_REFERENCE;
  switch (a.width) {
    case 2:
      return clamp ? launch_w<2, true, ANY, COUNT>(a, rays, n, out, visits, L, s, order)
                   : launch_w<2, false, ANY, COUNT>(a, rays, n, out, visits, L, s, order);
    case 4:
      return clamp ? launch_w<4, true, ANY, COUNT>(a, rays, n, out, visits, L, s, order)
                   : launch_w<4, false, ANY, COUNT>(a, rays, n, out, visits, L, s, order);
    default:
      return clamp ? launch_w<8, true, ANY, COUNT>(a, rays, n, out, visits, L, s, order)
                   : launch_w<8, false, ANY, COUNT>(a, rays, n, out, visits, L, s, order);
  }
}

template <bool ANY>
int launch_kd(const DevAccel& a, const float* rays, size_t n, void* out, cudaStream_t s,
              const uint32_t* order = nullptr) {
  KdParams p;
  p.nodes = a.d_kd;
  p.items = a.d_kd_items;
  p.tris = reinterpret_cast<const float4*>(a.d_tris);
  p.rays = reinterpret_cast<const float4*>(rays);
  p.order = order;
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
  int grid = device_sm_count(a.device) * kKdBlocks;
  unsigned need = (unsigned)((n + 127) / 128);
  if ((unsigned)grid > need) grid = (int)need;
  if (grid < 1) grid = 1;
  const bool small = a.tree_depth > 0 && a.tree_depth <= 32;
  if (a.predicate == ENC_PRED_REFERENCE) {
    if (small) kd_trace<true, ANY, 32><<<grid, 128, 0, s>>>(p);
    else kd_trace<true, ANY, 64><<<grid, 128, 0, s>>>(p);
  } else {
    if (small) kd_trace<false, ANY, 32><<<grid, 128, 0, s>>>(p);
    else kd_trace<false, ANY, 64><<<grid, 128, 0, s>>>(p);
  }
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
                   const Launch& L, void* stream, uint32_t* d_visits, const uint32_t* d_order) {
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (a.kind == ENC_ACCEL_KDTREE) return launch_kd<false>(a, d_rays, n, d_hits, s, d_order);
  if (d_visits) return dispatch_w<false, true>(a, d_rays, n, d_hits, d_visits, L, s, d_order);
  return dispatch_w<false, false>(a, d_rays, n, d_hits, nullptr, L, s, d_order);
}

int launch_any(const DevAccel& a, const float* d_rays, size_t n, uint8_t* d_occ, const Launch& L,
               void* stream) {
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (a.kind == ENC_ACCEL_KDTREE) return launch_kd<true>(a, d_rays, n, d_occ, s);
  return dispatch_w<true, false>(a, d_rays, n, d_occ, nullptr, L, s);
}

namespace {

// Closest hit over the wide BVH with the queue head and status word supplied
// by the caller instead of taken from the accelerator.
template <int W, bool CLAMP>
int launch_w_external(const DevAccel& a, const float* rays, size_t n, enc_hit* hits,
                      const Launch& L, cudaStream_t s, uint32_t* counter, uint32_t* status) {
  TraceParams p{};
  p.nodes = static_cast<const uint8_t*>(a.d_nodes);
  p.tris = reinterpret_cast<const float4*>(a.d_tris);
  p.rays = reinterpret_cast<const float4*>(rays);
  p.out = hits;
  p.visits = nullptr;
  p.counter = counter;
  p.status = status;
  p.nrays = (unsigned)n;
  p.nnodes = a.nnodes;
  p.ntris = a.ntris;
  p.stack_depth = L.stack > 0 ? L.stack : (a.tree_depth > 8 ? a.tree_depth : 8);
  p.chunk = L.chunk;
  size_t smem = (size_t)p.stack_depth * L.block * stack_entry_bytes(W);
  auto k = wbvh_trace<W, CLAMP, false, false>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  int grid = device_sm_count(a.device) * (L.blocks_per_sm > 0 ? L.blocks_per_sm : kBlocksClosest);
  k<<<grid, L.block, smem, s>>>(p);
  return (int)cudaGetLastError();
}

}  // namespace

int warm_closest_kernel(const DevAccel& a, uint32_t* counter, uint32_t* status) {
  // An empty batch: every warp finds the queue exhausted at once.  The launch
  // loads the kernel's module and sizes the context's local memory for it.
  Launch L = resolve_launch(nullptr, a.kind, a.width);
  L.blocks_per_sm = 1;
  int e = 0;
  const bool clamp = a.predicate == ENC_PRED_REFERENCE;
  float* no_rays = nullptr;
  switch (a.width) {
    case 2:
      e = clamp ? launch_w_external<2, true>(a, no_rays, 0, nullptr, L, 0, counter, status)
                : launch_w_external<2, false>(a, no_rays, 0, nullptr, L, 0, counter, status);
      break;
    case 4:
      e = clamp ? launch_w_external<4, true>(a, no_rays, 0, nullptr, L, 0, counter, status)
                : launch_w_external<4, false>(a, no_rays, 0, nullptr, L, 0, counter, status);
      break;
    default:
      e = clamp ? launch_w_external<8, true>(a, no_rays, 0, nullptr, L, 0, counter, status)
                : launch_w_external<8, false>(a, no_rays, 0, nullptr, L, 0, counter, status);
  }
  if (e != 0) return e;
  return (int)cudaStreamSynchronize(0);
}

int launch_closest_external_scratch(const DevAccel& a, const float* d_rays, size_t n,
                                    enc_hit* d_hits, const Launch& L, void* stream,
                                    uint32_t* counter, uint32_t* status) {
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool clamp = a.predicate == ENC_PRED_REFERENCE;
  switch (a.width) {
    case 2:
      return clamp ? launch_w_external<2, true>(a, d_rays, n, d_hits, L, s, counter, status)
                   : launch_w_external<2, false>(a, d_rays, n, d_hits, L, s, counter, status);
    case 4:
      return clamp ? launch_w_external<4, true>(a, d_rays, n, d_hits, L, s, counter, status)
                   : launch_w_external<4, false>(a, d_rays, n, d_hits, L, s, counter, status);
    default:
      return clamp ? launch_w_external<8, true>(a, d_rays, n, d_hits, L, s, counter, status)
                   : launch_w_external<8, false>(a, d_rays, n, d_hits, L, s, counter, status);
  }
}

}  // namespace enc

namespace enc {
namespace {

template <int W, bool CLAMP, bool ANY>
int launch_multi_w(const MultiLaunch& m, const Launch& L, cudaStream_t s) {
  TraceParams p{};
  p.counter = m.d_counter;
  p.status = m.d_status;
  p.nrays = m.total;
  p.stack_depth = L.stack > 0 ? L.stack : (m.stack_depth > 8 ? m.stack_depth : 8);
  p.chunk = L.chunk;
  p.scenes = m.d_scenes;
  p.batches = m.d_batches;
  p.starts = m.d_starts;
  p.nbatches = m.nbatches;
  p.batch_status = m.d_batch_status;
  size_t smem = (size_t)p.stack_depth * L.block * stack_entry_bytes(W);
  auto k = wbvh_trace<W, CLAMP, ANY, false, true>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
  }
  cudaError_t e = cudaMemsetAsync(m.d_counter, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return (int)e;
  int grid = device_sm_count(m.device) *
             (L.blocks_per_sm > 0 ? L.blocks_per_sm : (ANY ? kBlocksAny : kBlocksMulti));
  k<<<grid, L.block, smem, s>>>(p);
  return (int)cudaGetLastError();
}

template <bool ANY>
int launch_multi(const MultiLaunch& m, const Launch& L, void* stream) {
  if (m.total == 0 || m.nbatches == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool clamp = m.predicate == ENC_PRED_REFERENCE;
  switch (m.width) {
    case 2:
      return clamp ? launch_multi_w<2, true, ANY>(m, L, s) : launch_multi_w<2, false, ANY>(m, L, s);
    case 4:
      return clamp ? launch_multi_w<4, true, ANY>(m, L, s) : launch_multi_w<4, false, ANY>(m, L, s);
    default:
      return clamp ? launch_multi_w<8, true, ANY>(m, L, s) : launch_multi_w<8, false, ANY>(m, L, s);
  }
}

}  // namespace

int launch_multi_closest(const MultiLaunch& m, const Launch& L, void* stream) {
  return launch_multi<false>(m, L, stream);
}

int launch_multi_any(const MultiLaunch& m, const Launch& L, void* stream) {
  return launch_multi<true>(m, L, stream);
}

}  // namespace enc
