// Photon map: device layout shared by the host builder (photon.cpp) and the
// gather kernel (gather.cu).
//
// The tree is a complete binary kd-tree over photon index ranges: every
// internal node splits its range at the median index on the axis of the
// range's largest extent (the reference balances at the median too,
// PhotonMap.cpp:176-221), and leaves hold at most 32 photons, one per lane of
// the warp that gathers a query.  Photons are stored in leaf order as SoA
// float4 arrays so a leaf is one coalesced 512-byte read per array.
#pragma once

#include <cstdint>
#include <vector>

namespace enc {

constexpr int kPhotonLeaf = 32;

struct PNode {
  float split;     // internal: split coordinate
  int32_t axis;    // internal: 0..2; leaf: -1
  uint32_t begin;  // photon range [begin, end)
  uint32_t end;
};

// The gather walks a 32-ary box tree over the kd leaves, so that one warp
// step tests 32 children (one per lane) instead of one binary split:
//   level 0 = the kd leaves in leaf order (photon ranges, at most 32 each);
//   level l = groups of 32 consecutive level-(l-1) items (a kd subtree five
//             levels deep), item j covering items 32j .. 32j+31 below;
//   the top level has at most 32 items and is the root's children.
// Each level stores its items' boxes (the photons' bounds) as six float
// arrays lo.x, lo.y, lo.z, hi.x, hi.y, hi.z of `pad` entries (count rounded
// up to 32, padding boxes inverted so nothing enters them).
constexpr int kPhotonMaxLevels = 8;

struct PhotonHost {
  std::vector<PNode> nodes;   // heap order: children of i at 2i+1, 2i+2
  std::vector<float> pos4;    // x, y, z, original index (int bits)
  std::vector<float> nrm4;    // nx, ny, nz, 0
  std::vector<float> pow4;    // r, g, b, 0
  int depth = 0;
  std::vector<uint32_t> leaf;  // (begin, end) per level-0 item
  std::vector<float> box;      // all levels' box arrays, level 0 first
  int nlevels = 0;
  uint32_t lvl_count[kPhotonMaxLevels] = {};
  uint32_t lvl_off[kPhotonMaxLevels] = {};  // float offset of the level in `box`
  uint32_t lvl_pad[kPhotonMaxLevels] = {};
};

void build_photon_tree(const float* pos, const float* nrm, const float* power, size_t n,
                       PhotonHost* out);

constexpr int kGatherSlots = 256;

struct DevPhotonMap {
  float* d_box = nullptr;      // PhotonHost::box
  uint32_t* d_leaf = nullptr;  // PhotonHost::leaf
  int nlevels = 0;
  uint32_t lvl_count[kPhotonMaxLevels] = {};
  uint32_t lvl_off[kPhotonMaxLevels] = {};
  uint32_t lvl_pad[kPhotonMaxLevels] = {};
  float* d_pos4 = nullptr;
  float* d_nrm4 = nullptr;
  float* d_pow4 = nullptr;
  uint32_t* d_status = nullptr;
  // Query-queue heads: each launch takes the next of kGatherSlots words and
  // zeroes it on its stream, so up to kGatherSlots launches in flight at once
  // never share one (the next launch after those reuses the first's head).
  uint32_t* d_counter = nullptr;
  uint32_t counter_seq = 0;
  uint32_t nnodes = 0;
  uint32_t n = 0;
  int depth = 0;
  int caustic = 0;
  int device = 0;
  size_t box_floats = 0;   // PhotonHost::box.size()
  size_t leaf_words = 0;   // PhotonHost::leaf.size()
};

// Launchers (gather.cu).  k <= 256.  Asynchronous on `stream`.
int launch_radiance(const DevPhotonMap& m, const float* d_qpos, const float* d_qnrm, size_t nq,
                    int k, float max_dist, int flags, float* d_rgb, void* stream);
// The radiance launch that also writes 4 counters per query (gather.cu:
// child boxes tested, photons tested, normals read, photons found).
int launch_radiance_counted(const DevPhotonMap& m, const float* d_qpos, const float* d_qnrm,
                            size_t nq, int k, float max_dist, int flags, float* d_rgb,
                            uint32_t* d_visits, void* stream);
int launch_nearest(const DevPhotonMap& m, const float* d_qpos, const float* d_qnrm, size_t nq,
                   int k, float max_dist, int flags, int32_t* d_idx, float* d_d2,
                   int32_t* d_count, void* stream);

}  // namespace enc
