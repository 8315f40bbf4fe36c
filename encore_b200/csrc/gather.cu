// Photon k-nearest gather and radiance estimate for sm_100a.
//
// One warp per query point.  The warp walks the 32-ary box tree over the
// photon kd leaves (photon.h) with a per-warp stack in shared memory: at an
// inner node each lane tests one child box against the search sphere and the
// children that can hold an accepted photon are pushed together (a leaf as
// its photon range); at a leaf each lane tests one photon, and two sibling
// leaves share one step when their photons fit in the warp (one coalesced
// 16-byte load per lane per array).  A box is pruned by its FP32 squared
// distance to the query, formed with the photon test's own operations on the
// box's clamped coordinates; rounding is monotone, so that distance never
// exceeds the squared distance of a photon inside the box and pruning drops
// nothing the photon test would accept.  The k best candidates are kept in a
// warp-distributed bounded max-heap: S = ceil(k/32) register slots per lane,
// slot i on lane i % 32; the maximum and its slot are found with two warp max
// reductions (redux.sync), and an accepted candidate replaces it.  The search
// radius is max_dist^2 until k photons are held and the heap maximum
// afterwards, as in PhotonMap::GetNearestNPhotons (PhotonMap.cpp:224-297), so
// the result is the exact k-nearest set.
//
// Acceptance is the reference's: FP32 dist^2 = (x*x + y*y) + z*z with separate
// roundings, dist^2 < r^2, and the stored surface normal equal to the query
// normal component by component unless ENC_GATHER_IGNORE_NORMAL
// (PhotonMap.cpp:239-244).  The estimate follows GetRadianceEstimate
// (PhotonMap.cpp:121-164): r = largest dist^2 found; weight 1 (global map) or
// (r - d)/d (caustic map); density 1 or k / (pi r^2) with pi = 3.14159f
// (Common.h:36); FP32 accumulation.
#include <cuda_runtime.h>

#include "../../include/encore_b200.h"
#include "photon.h"

namespace enc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 8;
// Each inner node pushes at most 32 children and the walk is depth first, so
// 32 entries per level suffice.
constexpr int kStack = 32 * kPhotonMaxLevels;
constexpr unsigned kMaxSteps = 1u << 24;
// Queries a warp takes from the queue at a time.
constexpr unsigned kQueryChunk = 4;

struct GatherParams {
  const float* box;
  const uint2* leaf;
  int nlevels;
  uint32_t lvl_count[kPhotonMaxLevels];
  uint32_t lvl_off[kPhotonMaxLevels];
  uint32_t lvl_pad[kPhotonMaxLevels];
  const float4* pos4;
  const float4* nrm4;
  const float4* pow4;
  const float* qpos;
  const float* qnrm;
  float* rgb;
  int32_t* idx;
  float* d2;
  int32_t* count;
  uint32_t* status;
  uint32_t* counter;  // this launch's query-queue head, zeroed before it
  uint32_t* visits;   // COUNT: 4 words per query (see gather_kernel)
  unsigned nq;
  int k;
  float r2max;
  int ignore_normal;
  int caustic;
};

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// Stack entries.  An inner-node entry is level << 28 | item (level 1..7);
// a leaf entry is kLeafEntry | first photon, with the leaf's photon count
// kept beside it, so a leaf step reads its photons without first loading
// its range.
constexpr uint32_t kLeafEntry = 0x80000000u;

// Position of the r-th set bit of m (r counted from 0, r < popc(m)), by
// halving: keep the low half while it holds more than r set bits.
__device__ __forceinline__ int nth_set_bit(unsigned m, int r) {
  int pos = 0;
#pragma unroll
  for (int b = 16; b >= 1; b >>= 1) {
    const int c = __popc(m & ((1u << b) - 1u));
    if (r >= c) {
      r -= c;
      m >>= b;
      pos += b;
    }
  }
  return pos;
}

// Max over the slots marked valid (slot index s*32 + lane < limit) and its
// slot index, the highest slot among equal maxima; -INF / -1 if none.  The
// held values are squared distances, non-negative floats whose bit patterns
// order as unsigned integers, so two warp max reductions (redux.sync) find
// the value and then its slot.
template <int S>
__device__ __forceinline__ void warp_max(const float (&dd)[S], int lane, int limit, float& v,
                                         int& loc) {
  uint32_t lv = 0;
  int ls = -1;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int slot = s * 32 + lane;
    const uint32_t u = __float_as_uint(dd[s]);
    if (slot < limit && (ls < 0 || u >= lv)) {
      lv = u;
      ls = slot;
    }
  }
  const uint32_t mv = __reduce_max_sync(kFull, ls >= 0 ? lv : 0u);
  const uint32_t l1 = __reduce_max_sync(kFull, (ls >= 0 && lv == mv) ? (uint32_t)(ls + 1) : 0u);
  loc = (int)l1 - 1;
  v = l1 == 0 ? -INFINITY : __uint_as_float(mv);
}

// COUNT: also records per query the work behind the roofline's bytes:
// visits[4q] child boxes tested (24 bytes each), [4q+1] photons tested (a
// 16-byte position each), [4q+2] normals read (16 bytes each), [4q+3]
// photons found (their 16-byte power is read by the estimate).
template <int S, bool NEAREST, bool COUNT = false>
__global__ void __launch_bounds__(256) gather_kernel(GatherParams P) {
  // stack entries, their squared distances, and a leaf entry's photon count
  __shared__ uint32_t s_item[kWarpsPerBlock][kStack];
  __shared__ float s_pd[kWarpsPerBlock][kStack];
  __shared__ uint8_t s_cnt[kWarpsPerBlock][kStack];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int k = P.k;
  // Each warp takes kQueryChunk queries at a time from the launch's queue
  // head, so every warp stays busy until the queue is empty (a fixed share
  // per warp left a fifth of the warp slots idle at the end).  The head
  // overshoots nq by at most kQueryChunk per warp: nq < 2^31 keeps it below
  // 2^32.
  unsigned q = 0, qend = 0;
  for (;;) {
    if (q == qend) {
      unsigned b = 0;
      if (lane == 0) b = atomicAdd(P.counter, kQueryChunk);
      b = __shfl_sync(kFull, b, 0);
      if (b >= P.nq) break;
      q = b;
      qend = min(b + kQueryChunk, P.nq);
    }
    const float qx = __ldg(P.qpos + 3 * (size_t)q), qy = __ldg(P.qpos + 3 * (size_t)q + 1),
                qz = __ldg(P.qpos + 3 * (size_t)q + 2);
    const float nx = __ldg(P.qnrm + 3 * (size_t)q), ny = __ldg(P.qnrm + 3 * (size_t)q + 1),
                nz = __ldg(P.qnrm + 3 * (size_t)q + 2);
    float dd[S];
    int ds[S];
    int dorig[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      dd[s] = INFINITY;
      ds[s] = 0;
      dorig[s] = -1;
    }
    int count = 0;
    float worst = INFINITY;
    int worst_loc = -1;
    float r2 = P.r2max;
    // the root: the top level's items are its children
    int sp = 0;
    if (k > 0) {
      if (lane == 0) {
        s_item[wib][0] = (uint32_t)P.nlevels << 28;
        s_pd[wib][0] = 0.f;
        s_cnt[wib][0] = 0;
      }
      sp = 1;
    }
    __syncwarp();
    unsigned steps = 0;
    uint32_t n_box = 0, n_pos = 0, n_nrm = 0;
    while (sp > 0) {
      if (++steps > kMaxSteps) {
        if (lane == 0) atomicOr(P.status, 1u);
        break;
      }
      --sp;
      const float pd = s_pd[wib][sp];
      const uint32_t e = s_item[wib][sp];
      const int c0 = s_cnt[wib][sp];
      if (!(pd < r2)) {  // nothing in it can be accepted any more
        __syncwarp();
        continue;
      }
      if (!(e & kLeafEntry)) {
        __syncwarp();
        // inner node: lane c tests child 32 * it + c of level lv - 1
        const int cl = (int)(e >> 28) - 1;
        const uint32_t child = 32u * (e & 0x0fffffffu) + (uint32_t)lane;
        bool pass = false;
        float cd = 0.f;
        if (child < P.lvl_count[cl]) {
          const float* b = P.box + P.lvl_off[cl];
          const uint32_t pad = P.lvl_pad[cl];
          const float lx = __ldg(b + child), ly = __ldg(b + pad + child),
                      lz = __ldg(b + 2 * pad + child);
          const float hx = __ldg(b + 3 * pad + child), hy = __ldg(b + 4 * pad + child),
                      hz = __ldg(b + 5 * pad + child);
          const float gx = fmaxf(fmaxf(fs(lx, qx), fs(qx, hx)), 0.f);
          const float gy = fmaxf(fmaxf(fs(ly, qy), fs(qy, hy)), 0.f);
          const float gz = fmaxf(fmaxf(fs(lz, qz), fs(qz, hz)), 0.f);
          cd = fa(fa(fm(gx, gx), fm(gy, gy)), fm(gz, gz));
          pass = cd < r2;
        }
        const unsigned m = __ballot_sync(kFull, pass);
        if (COUNT) n_box += __popc(__ballot_sync(kFull, child < P.lvl_count[cl]));
        const int n = __popc(m);
        if (sp + n > kStack) {
          if (lane == 0) atomicOr(P.status, 2u);
          break;
        }
        // Nearest child on top: the passing children are pushed farthest
        // first, so the walk visits them nearest first, the heap fills with
        // nearer photons and its maximum (the search radius once full)
        // shrinks sooner.  A child's place = the passing children farther
        // than it (equal distances: the higher lane counts as farther).
        int farther = 0;
        for (unsigned mm = m; mm; mm &= mm - 1u) {
          const int j = __ffs(mm) - 1;
          const float dj = __shfl_sync(kFull, cd, j);
          farther += (dj > cd || (dj == cd && j > (int)lane)) ? 1 : 0;
        }
        if (pass) {
          const int at = sp + farther;
          uint32_t item = ((uint32_t)cl << 28) | child;
          uint32_t cnt = 0;
          if (cl == 0) {  // a leaf: its photon range goes onto the stack
            const uint2 rng = __ldg(P.leaf + child);
            item = kLeafEntry | rng.x;
            cnt = rng.y - rng.x;
          }
          s_item[wib][at] = item;
          s_pd[wib][at] = cd;
          s_cnt[wib][at] = (uint8_t)cnt;
        }
        sp += n;
        __syncwarp();
        continue;
      }
      // leaf: lane j tests photon j of the leaf; when the entry below is a
      // leaf too and both fit in the warp, lanes c0.. test its photons
      uint32_t b1 = 0;
      int c1 = 0;
      if (sp > 0) {
        const uint32_t e1 = s_item[wib][sp - 1];
        const int n1 = s_cnt[wib][sp - 1];
        if ((e1 & kLeafEntry) && c0 + n1 <= 32 && s_pd[wib][sp - 1] < r2) {
          b1 = e1 & ~kLeafEntry;
          c1 = n1;
          --sp;
        }
      }
      __syncwarp();
      const unsigned pidx = lane < c0 ? (e & ~kLeafEntry) + (unsigned)lane
                                      : b1 + (unsigned)(lane - c0);
      bool acc = false;
      float d2 = 0.f;
      int orig = -1;
      if (COUNT) {
        n_pos += (uint32_t)(c0 + c1);
      }
      if (lane < c0 + c1) {
        const float4 p = __ldg(P.pos4 + pidx);
        const float x = fs(qx, p.x), y = fs(qy, p.y), z = fs(qz, p.z);
        d2 = fa(fa(fm(x, x), fm(y, y)), fm(z, z));
        orig = __float_as_int(p.w);
        acc = d2 < r2;
        if (acc && !P.ignore_normal) {
          const float4 pn = __ldg(P.nrm4 + pidx);
          acc = (pn.x == nx) && (pn.y == ny) && (pn.z == nz);
        }
      }
      if (COUNT && !P.ignore_normal)
        n_nrm += __popc(__ballot_sync(kFull, lane < c0 + c1 && d2 < r2));
      unsigned m = __ballot_sync(kFull, acc);
      if (m && count < k) {
        // fill free heap slots in one step: the accepted candidate of rank r
        // (r-th set bit of m) goes to slot count + r, which lives on lane
        // (count + r) % 32, register (count + r) / 32
        const int na = __popc(m);
        const int nfill = min(na, k - count);
        const int r = (lane - count) & 31;
        const bool take = r < nfill;
        const int src = nth_set_bit(m, take ? r : 0);
        const float cd = __shfl_sync(kFull, d2, src);
        const int co = __shfl_sync(kFull, orig, src);
        const int cs = __shfl_sync(kFull, (int)pidx, src);
        const int slot = count + r;
        if (take) {
#pragma unroll
          for (int s = 0; s < S; ++s)
            if (s == (slot >> 5)) {
              dd[s] = cd;
              ds[s] = cs;
              dorig[s] = co;
            }
        }
        // the first nfill set bits are done
        if (nfill == na) {
          m = 0;
        } else {
          for (int i = 0; i < nfill; ++i) m &= m - 1;
        }
        count += nfill;
        if (count == k) {
          warp_max<S>(dd, lane, k, worst, worst_loc);
          r2 = worst;
        }
      }
      // the heap is full (a fill step leaves candidates only then): each
      // closer candidate replaces the maximum
      while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        const float cd = __shfl_sync(kFull, d2, j);
        const int co = __shfl_sync(kFull, orig, j);
        const int cs = __shfl_sync(kFull, (int)pidx, j);
        if (cd < worst) {
#pragma unroll
          for (int s = 0; s < S; ++s)
            if (lane == (worst_loc & 31) && s == (worst_loc >> 5)) {
              dd[s] = cd;
              ds[s] = cs;
              dorig[s] = co;
            }
          warp_max<S>(dd, lane, k, worst, worst_loc);
          r2 = worst;
        }
      }
    }

    if (NEAREST) {
      // rank = number of held entries ordered before this one (dist^2, index)
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const int slot = s * 32 + lane;
        int rank = 0;
#pragma unroll
        for (int s2 = 0; s2 < S; ++s2)
          for (int l = 0; l < 32; ++l) {
            const float od = __shfl_sync(kFull, dd[s2], l);
            const int oo = __shfl_sync(kFull, dorig[s2], l);
            const int oslot = s2 * 32 + l;
            if (oslot < count && (od < dd[s] || (od == dd[s] && oo < dorig[s]))) ++rank;
          }
        if (slot < count) {
          P.idx[(size_t)q * k + rank] = dorig[s];
          P.d2[(size_t)q * k + rank] = dd[s];
        }
      }
      for (int p = count + lane; p < k; p += 32) {
        P.idx[(size_t)q * k + p] = -1;
        P.d2[(size_t)q * k + p] = 0.f;
      }
      if (lane == 0) P.count[q] = count;
    } else {
      float R = 0.f, G = 0.f, B = 0.f;
      if (count > 0) {
        float r;
        int loc;
        warp_max<S>(dd, lane, count, r, loc);
#pragma unroll
        for (int s = 0; s < S; ++s) {
          if (s * 32 + lane < count) {
            const float w = P.caustic ? __fdiv_rn(fs(r, dd[s]), dd[s]) : 1.0f;
            const float4 pw = __ldg(P.pow4 + ds[s]);
            R = fa(R, fm(pw.x, w));
            G = fa(G, fm(pw.y, w));
            B = fa(B, fm(pw.z, w));
          }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          R += __shfl_xor_sync(kFull, R, off);
          G += __shfl_xor_sync(kFull, G, off);
          B += __shfl_xor_sync(kFull, B, off);
        }
        if (P.caustic) {
          const float dens = __fdiv_rn((float)k, fm(fm(3.14159f, r), r));
          R = fm(R, dens);
          G = fm(G, dens);
          B = fm(B, dens);
        }
      }
      if (lane == 0) {
        P.rgb[3 * (size_t)q] = R;
        P.rgb[3 * (size_t)q + 1] = G;
        P.rgb[3 * (size_t)q + 2] = B;
      }
    }
    if (COUNT && lane == 0) {
      P.visits[4 * (size_t)q] = n_box;
      P.visits[4 * (size_t)q + 1] = n_pos;
      P.visits[4 * (size_t)q + 2] = n_nrm;
      P.visits[4 * (size_t)q + 3] = (uint32_t)count;
    }
    ++q;
  }
}

template <bool NEAREST, bool COUNT = false>
int launch_gather(const DevPhotonMap& m, const float* qpos, const float* qnrm, size_t nq, int k,
                  float max_dist, int flags, float* rgb, int32_t* idx, float* d2, int32_t* count,
                  cudaStream_t s, uint32_t* visits = nullptr) {
  if (nq == 0) return 0;
  GatherParams p;
  p.box = m.d_box;
  p.leaf = reinterpret_cast<const uint2*>(m.d_leaf);
  p.nlevels = m.nlevels;
  for (int l = 0; l < kPhotonMaxLevels; ++l) {
    p.lvl_count[l] = m.lvl_count[l];
    p.lvl_off[l] = m.lvl_off[l];
    p.lvl_pad[l] = m.lvl_pad[l];
  }
  p.pos4 = reinterpret_cast<const float4*>(m.d_pos4);
  p.nrm4 = reinterpret_cast<const float4*>(m.d_nrm4);
  p.pow4 = reinterpret_cast<const float4*>(m.d_pow4);
  p.qpos = qpos;
  p.qnrm = qnrm;
  p.rgb = rgb;
  p.idx = idx;
  p.d2 = d2;
  p.count = count;
  p.visits = visits;
  p.status = m.d_status;
  const uint32_t slot = __atomic_fetch_add(const_cast<uint32_t*>(&m.counter_seq), 1u,
                                           __ATOMIC_RELAXED) % kGatherSlots;
  p.counter = m.d_counter + slot;
  p.nq = (unsigned)nq;
  p.k = m.n == 0 ? 0 : k;
  p.r2max = max_dist * max_dist;  // maxDistance*maxDistance in FP32 (PhotonMap.cpp:89)
  p.ignore_normal = (flags & ENC_GATHER_IGNORE_NORMAL) ? 1 : 0;
  p.caustic = m.caustic;
  const int S = k <= 32 ? 1 : (k <= 64 ? 2 : (k <= 128 ? 4 : 8));
  void (*kern)(GatherParams) = S == 1   ? gather_kernel<1, NEAREST, COUNT>
                               : S == 2 ? gather_kernel<2, NEAREST, COUNT>
                               : S == 4 ? gather_kernel<4, NEAREST, COUNT>
                                        : gather_kernel<8, NEAREST, COUNT>;
  // One resident wave of persistent warps (the register count allows 5
  // blocks of 256 threads per SM): a larger grid would only queue blocks
  // that find the query queue empty.
  int sms = 148, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemsetAsync(p.counter, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return (int)e;
  if (per_sm < 1) per_sm = 1;
  const unsigned need = (unsigned)((nq + kWarpsPerBlock - 1) / kWarpsPerBlock);
  unsigned grid = (unsigned)sms * (unsigned)per_sm;
  if (grid > need) grid = need;
  kern<<<grid, 256, 0, s>>>(p);
  return (int)cudaGetLastError();
}

}  // namespace

int launch_radiance(const DevPhotonMap& m, const float* d_qpos, const float* d_qnrm, size_t nq,
                    int k, float max_dist, int flags, float* d_rgb, void* stream) {
  return launch_gather<false>(m, d_qpos, d_qnrm, nq, k, max_dist, flags, d_rgb, nullptr, nullptr,
                              nullptr, static_cast<cudaStream_t>(stream));
}

int launch_radiance_counted(const DevPhotonMap& m, const float* d_qpos, const float* d_qnrm,
                            size_t nq, int k, float max_dist, int flags, float* d_rgb,
                            uint32_t* d_visits, void* stream) {
  return launch_gather<false, true>(m, d_qpos, d_qnrm, nq, k, max_dist, flags, d_rgb, nullptr,
                                    nullptr, nullptr, static_cast<cudaStream_t>(stream), d_visits);
}

int launch_nearest(const DevPhotonMap& m, const float* d_qpos, const float* d_qnrm, size_t nq,
                   int k, float max_dist, int flags, int32_t* d_idx, float* d_d2,
                   int32_t* d_count, void* stream) {
  return launch_gather<true>(m, d_qpos, d_qnrm, nq, k, max_dist, flags, nullptr, d_idx, d_d2,
                             d_count, static_cast<cudaStream_t>(stream));
}

}  // namespace enc
