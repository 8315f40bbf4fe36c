// Internal declarations shared by the host builders, the CUDA kernels and the
// C ABI.  Device layouts are defined here once so the builder that writes a
// structure and the kernel that walks it agree by construction.
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/encore_b200.h"

namespace enc {

// ---------------------------------------------------------------------------
// Triangles on the device: 3 x float4 = 48 bytes, read with three 16-byte
// vector loads.  e1 = v1 - v0 and e2 = v2 - v0 are precomputed on the host in
// FP32, which yields the same floats the reference forms per test as
// Vector3(v0, v1) and Vector3(v0, v2) (TrianglePrim.cpp:210-211).
//   a = (v0.x, v0.y, v0.z, e1.x)
//   b = (e1.y, e1.z, e2.x, e2.y)
//   c = (e2.z, id as int bits, 0, 0)
struct alignas(16) DevTri {
  float a[4], b[4], c[4];
};
static_assert(sizeof(DevTri) == 48, "DevTri is three float4");

// ---------------------------------------------------------------------------
// Wide BVH node, width W in {2, 4, 8}.  Child boxes are stored as 8-bit
// offsets from the node origin p in units of 2^(e-127) per axis, rounded
// outward (lo floored, hi ceiled) so a decoded box always contains the
// child's true box.
//
// meta[c]: 0 = empty slot; 1..8 = internal child, node index child_base +
// (meta-1); >= 32 = leaf, triangle count meta>>5 (1..7) starting at
// tri_base + (meta & 31).
template <int W>
struct WNodeLayout {
  static constexpr int kRaw = 24 + 7 * W;
  static constexpr int kBytes = (kRaw + 15) / 16 * 16;  // 48, 64, 80
  static constexpr int kMetaOff = 24;
  static constexpr int kQOff = 24 + W;  // qlo x,y,z then qhi x,y,z; W bytes each
};

struct WNodeHeader {  // first 24 bytes of every wide node
  float p[3];
  uint8_t e[3];
  uint8_t imask;  // bit c set: slot c holds an internal child (its meta is 1 + rank)
  uint32_t child_base;
  uint32_t tri_base;
};
static_assert(sizeof(WNodeHeader) == 24, "wide node header is 24 bytes");

// ---------------------------------------------------------------------------
// kd-tree node, 8 bytes.  The reference stores flags/split/count in one union
// and the child index / primitive list pointer in another (Kdtree.h:25-58);
// its initNode writes the axis into the two low bits of the split float
// (Kdtree.h:47-52), so the split value its traversal reads differs from the
// build's split position in those bits.  This layout keeps exactly that word:
//   word0 low 2 bits == 3  -> leaf, count = word0 >> 2, word1 = first index
//                             into the leaf-index array
//   otherwise              -> internal, axis = word0 & 3, split = as_float(word0),
//                             children at word1 and word1 + 1
struct KdNode {
  uint32_t word0;
  uint32_t word1;
};

// ---------------------------------------------------------------------------
// Device-resident accelerator.
constexpr int kQueueSlots = 256;
struct DevAccel {
  int kind = 0;
  int width = 8;
  int predicate = 0;
  uint32_t ntris = 0;
  uint32_t nnodes = 0;
  int tree_depth = 0;  // WBVH levels; the traversal stack needs at most depth - 1 entries
  // WBVH
  void* d_nodes = nullptr;      // nnodes * WNodeLayout<W>::kBytes
  DevTri* d_tris = nullptr;     // WBVH: leaf order; kd: triangle-ID order
  uint32_t* d_tri_pos = nullptr;  // triangle ID -> index into d_tris (WBVH; kd: identity, null)
  // kd-tree
  KdNode* d_kd = nullptr;
  uint32_t* d_kd_items = nullptr;  // leaf triangle IDs
  uint32_t kd_nitems = 0;
  float kd_root_lo[3] = {0, 0, 0}, kd_root_hi[3] = {0, 0, 0};
  // status word written by kernels (watchdog / bounds)
  uint32_t* d_status = nullptr;
  // Work-queue heads: each launch takes the next of kQueueSlots words (and
  // zeroes it on its stream), so up to kQueueSlots launches on one
  // accelerator can be in flight on different streams.
  uint32_t* d_counter = nullptr;
  uint32_t counter_seq = 0;
  size_t node_bytes = 0, tri_bytes = 0, device_bytes = 0;
  int device = 0;
  double build_seconds = 0;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// ---------------------------------------------------------------------------
// Multi-scene launch tables (device memory).  One persistent launch traces
// the ray batches of many scenes: batch b owns queue indices
// [start[b], start[b] + nrays), and start[b] is a multiple of the launch's
// chunk, so a warp's chunk never spans two batches.
struct alignas(16) SceneDesc {
  const uint8_t* nodes;
  const void* tris;  // DevTri[], leaf order
  uint32_t nnodes;
  uint32_t ntris;
};
struct alignas(16) BatchDesc {
  const float* rays;  // 8 floats per ray
  void* out;          // enc_hit[] (closest) or uint8_t[] (any)
  uint32_t scene;
  uint32_t nrays;
  uint32_t start;     // first queue index of the batch
  uint32_t any;       // 0 = closest hit, 1 = any hit (kept for the table's use by callers)
};

struct MultiLaunch {
  const SceneDesc* d_scenes = nullptr;
  const BatchDesc* d_batches = nullptr;
  const uint32_t* d_starts = nullptr;  // nbatches + 1 chunk-aligned starts
  uint32_t nbatches = 0;
  uint32_t total = 0;  // queue indices including the alignment padding
  int width = 8;
  int predicate = 0;
  int device = 0;
  int stack_depth = 8;  // deepest scene's tree depth
  uint32_t* d_counter = nullptr;
  uint32_t* d_status = nullptr;
  // optional: one status word per batch (a ray's loop-bound stop is recorded
  // in its own batch's word instead of d_status)
  uint32_t* d_batch_status = nullptr;
};

// Host results of the builders (before upload).
struct WBVHHost {
  int width = 8;
  std::vector<uint8_t> nodes;  // nnodes * kBytes
  uint32_t nnodes = 0;
  std::vector<DevTri> tris;    // leaf order
  std::vector<uint32_t> tri_pos;  // triangle ID -> position in `tris`
  std::vector<uint32_t> tri_order;  // position in `tris` -> triangle ID
  float lo[3], hi[3];
  int depth = 0;               // levels of wide nodes (root = 1)
};

struct KdHost {
  std::vector<KdNode> nodes;
  std::vector<uint32_t> items;
  float root_lo[3], root_hi[3];  // reference root box (pos, pos + size)
  int max_depth = 0;
};

// Builders (host).  tri_verts: 9 floats per triangle.
void build_wbvh(const float* tri_verts, uint32_t ntris, int width, int max_leaf, WBVHHost* out);
void build_kd_reference(const float* tri_verts, uint32_t ntris, KdHost* out);
// Recomputes the boxes of a built wide BVH for moved triangles (same IDs,
// same tree shape) and rewrites its triangle records.
void refit_wbvh(WBVHHost* h, const float* tri_verts, uint32_t ntris);
void make_dev_tris(const float* tri_verts, uint32_t ntris, const uint32_t* order, DevTri* out);

// Launch parameters after defaults are applied.
struct Launch {
  int block = 128;
  int blocks_per_sm = 4;
  int chunk = 32;
  int stack = 32;
  // Closest hit with one triangle loop per lane instead of the warp-wide
  // triangle rounds: the host-buffer pipeline uses it (see host_form).
  bool per_lane = false;
};
Launch resolve_launch(const enc_launch_opts* o, int kind, int width);

// ---------------------------------------------------------------------------
// Ray binning (reorder.cu): a key per ray from its origin cell and direction
// cell, counting-sorted into a permutation the traversal reads its queue
// through.
constexpr int kBinMaxDimBits = 10;  // bits per key dimension
constexpr int kBinMaxKeyBits = 20;  // histogram of at most 2^20 buckets
struct BinSpec {
  float lo[3];     // low corner of the binned box
  float scale[3];  // cells per unit length on each axis
  float probe_len; // > 0: bin the point o + probe_len * d instead of o
  int bits[5];     // key bits: origin x, y, z, direction u, v
};
// Scratch layout: keys (n words), order (n words), histogram (2^key_bits
// words), each 256-byte aligned.
size_t bin_scratch_bytes(size_t nrays, int key_bits);
// key_bits total, dir_bits of them for the direction; the rest go to the
// origin axes, widest cells first.  probe_frac: probe distance as a fraction
// of the box diagonal (0 = the origin itself).
BinSpec make_bin_spec(const float lo[3], const float hi[3], int key_bits, int dir_bits,
                      float probe_frac);
// Enqueues the three binning kernels on `s`; *d_order points into d_scratch.
int launch_bin(const float* d_rays, size_t n, const BinSpec& spec, void* d_scratch,
               uint32_t** d_order, int device, void* stream);

// Writes n rays of 6 floats (origin, direction; 8-byte aligned) as n rays of
// the 8-float layout with tmin = 0 and tmax = +inf (ray_widen.cu).
// Asynchronous on `stream`.
int launch_widen_rays(const float* d_od, size_t n, float* d_rays, int device, void* stream);

// Kernel launchers (trace.cu).  All asynchronous on `stream`.  d_order (may
// be null): queue index q traces ray d_order[q].
int launch_closest(const DevAccel& a, const float* d_rays, size_t n, enc_hit* d_hits,
                   const Launch& L, void* stream, uint32_t* d_visits,
                   const uint32_t* d_order = nullptr);
int launch_any(const DevAccel& a, const float* d_rays, size_t n, uint8_t* d_occ,
               const Launch& L, void* stream);
// Wide-BVH closest hit whose queue head (*counter, zeroed by the caller on
// `stream`) and status word are caller-provided device words.
int launch_closest_external_scratch(const DevAccel& a, const float* d_rays, size_t n,
                                    enc_hit* d_hits, const Launch& L, void* stream,
                                    uint32_t* counter, uint32_t* status);
// Launches the closest-hit kernel of launch_closest_external_scratch for `a`
// once over an empty batch and waits (trace.cu): its module is loaded and the
// context's local memory sized for it, so a later launch allocates nothing.
// `a.device` must be current; counter and status are device words.
int warm_closest_kernel(const DevAccel& a, uint32_t* counter, uint32_t* status);
// Resolves the no-allocation entry point's fixed scratch on `a.device` and
// preloads its kernel (noalloc.cu); called by enc_accel_build, where
// allocating is allowed.  `a.device` must be current.
int noalloc_prepare(const DevAccel& a);
// Closest hit for every batch of a multi-scene table in one persistent launch.
int launch_multi_closest(const MultiLaunch& m, const Launch& L, void* stream);
// Any hit (uint8 occluded per ray) for every batch of the table.
int launch_multi_any(const MultiLaunch& m, const Launch& L, void* stream);
int device_sm_count(int device);

// Error reporting (capi.cpp).
void set_error(const std::string& msg);

// The device view of an accelerator handle, or nullptr (capi.cpp).
const DevAccel* accel_device_view(enc_accel a);

// Device scratch of the wavefront photon tracer, kept with the accelerator
// and grown on demand, so repeated calls allocate nothing.  `mu` serialises
// the tracer's calls on one accelerator.
struct WaveScratch {
  float* rays[2] = {nullptr, nullptr};
  uint32_t* path[2] = {nullptr, nullptr};
  float* srays[2] = {nullptr, nullptr};    // shadow-photon rays
  uint32_t* spath[2] = {nullptr, nullptr};
  void* hits = nullptr;
  uint32_t* counters = nullptr;  // device: photons offered per store, next wave's and
                                 // next shadow wave's rays, shadow rays dropped
  uint32_t* h_counts = nullptr;  // pinned host copy of the counters
  size_t cap = 0;                // photons the buffers hold
  std::mutex mu;
};
WaveScratch* accel_wave_scratch(enc_accel a);
void free_wave_scratch(WaveScratch* w);

}  // namespace enc
