// Host build of the photon kd-tree (layout in photon.h).
//
// Replaces PhotonMap::BalanceAndConstruct (PhotonMap.cpp:167-221).  The
// reference keeps one photon per node and picks the split axis from a running
// box that starts at +-1e10 (PhotonMap.cpp:27-28, 182-191); the result of a
// k-nearest query does not depend on the tree, so this build uses bucketed
// leaves of 32 photons and the range's largest extent, which is what a warp
// gather wants.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <stdexcept>

#include "photon.h"

namespace enc {
namespace {

struct TreeBuilder {
  const float* pos;
  std::vector<uint32_t>& idx;
  std::vector<PNode>& nodes;
  int depth;

  void build(uint32_t node, uint32_t b, uint32_t e, int d) {
    PNode& nd = nodes[node];
    nd.begin = b;
    nd.end = e;
    if (d == depth) {
      nd.axis = -1;
      nd.split = 0.f;
      return;
    }
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = b; i < e; ++i)
      for (int a = 0; a < 3; ++a) {
        float c = pos[3 * (size_t)idx[i] + a];
        mn[a] = std::min(mn[a], c);
        mx[a] = std::max(mx[a], c);
      }
    int axis = 0;
    if (mx[1] - mn[1] > mx[axis] - mn[axis]) axis = 1;
    if (mx[2] - mn[2] > mx[axis] - mn[axis]) axis = 2;
    uint32_t m = b + (e - b) / 2;
    if (e > b) {
      std::nth_element(idx.begin() + b, idx.begin() + m, idx.begin() + e,
                       [&](uint32_t p, uint32_t q) { return pos[3 * (size_t)p + axis] < pos[3 * (size_t)q + axis]; });
    }
    nd.axis = axis;
    nd.split = (m < e) ? pos[3 * (size_t)idx[m] + axis] : 0.f;
    if (d < 3 && e - b > (1u << 16)) {
      auto f = std::async(std::launch::async, [=] { build(2 * node + 1, b, m, d + 1); });
      build(2 * node + 2, m, e, d + 1);
      f.get();
    } else {
      build(2 * node + 1, b, m, d + 1);
      build(2 * node + 2, m, e, d + 1);
    }
  }
};

}  // namespace

void build_photon_tree(const float* pos, const float* nrm, const float* power, size_t n,
                       PhotonHost* out) {
  if (n > 0x7fffffffu) throw std::runtime_error("too many photons");
  int depth = 0;
  while (((n + ((size_t)1 << depth) - 1) >> depth) > (size_t)kPhotonLeaf) ++depth;
  out->depth = depth;
  std::vector<uint32_t> idx(n);
  for (size_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
  out->nodes.assign(((size_t)2 << depth) - 1, PNode{0.f, -1, 0, 0});
  TreeBuilder tb{pos, idx, out->nodes, depth};
  tb.build(0, 0, (uint32_t)n, 0);
  out->pos4.resize(4 * n);
  out->nrm4.resize(4 * n);
  out->pow4.resize(4 * n);
  for (size_t i = 0; i < n; ++i) {
    size_t s = idx[i];
    int32_t orig = (int32_t)s;
    for (int a = 0; a < 3; ++a) {
      out->pos4[4 * i + a] = pos[3 * s + a];
      out->nrm4[4 * i + a] = nrm[3 * s + a];
      out->pow4[4 * i + a] = power[3 * s + a];
    }
    std::memcpy(&out->pos4[4 * i + 3], &orig, 4);
    out->nrm4[4 * i + 3] = 0.f;
    out->pow4[4 * i + 3] = 0.f;
  }
  // 32-ary box levels over the kd leaves (the leaves are the heap's last
  // level, left to right = leaf order)
  const size_t nleaf = (size_t)1 << depth;
  const size_t first = nleaf - 1;
  out->leaf.resize(2 * nleaf);
  std::vector<float> lo(3 * nleaf), hi(3 * nleaf);
  for (size_t j = 0; j < nleaf; ++j) {
    const PNode& nd = out->nodes[first + j];
    out->leaf[2 * j] = nd.begin;
    out->leaf[2 * j + 1] = nd.end;
    for (int a = 0; a < 3; ++a) {
      lo[3 * j + a] = INFINITY;
      hi[3 * j + a] = -INFINITY;
    }
    for (uint32_t i = nd.begin; i < nd.end; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[3 * j + a] = std::min(lo[3 * j + a], out->pos4[4 * (size_t)i + a]);
        hi[3 * j + a] = std::max(hi[3 * j + a], out->pos4[4 * (size_t)i + a]);
      }
  }
  size_t count = nleaf;
  int lvl = 0;
  for (;;) {
    if (lvl >= kPhotonMaxLevels) throw std::runtime_error("photon box tree too deep");
    const size_t pad = (count + 31) / 32 * 32;
    out->lvl_count[lvl] = (uint32_t)count;
    out->lvl_pad[lvl] = (uint32_t)pad;
    out->lvl_off[lvl] = (uint32_t)out->box.size();
    const size_t o = out->box.size();
    out->box.resize(o + 6 * pad);
    for (size_t j = 0; j < pad; ++j)
      for (int a = 0; a < 3; ++a) {
        out->box[o + a * pad + j] = j < count ? lo[3 * j + a] : INFINITY;
        out->box[o + (3 + a) * pad + j] = j < count ? hi[3 * j + a] : -INFINITY;
      }
    ++lvl;
    if (count <= 32) break;
    const size_t up = (count + 31) / 32;
    std::vector<float> ulo(3 * up, INFINITY), uhi(3 * up, -INFINITY);
    for (size_t j = 0; j < count; ++j)
      for (int a = 0; a < 3; ++a) {
        ulo[3 * (j / 32) + a] = std::min(ulo[3 * (j / 32) + a], lo[3 * j + a]);
        uhi[3 * (j / 32) + a] = std::max(uhi[3 * (j / 32) + a], hi[3 * j + a]);
      }
    lo.swap(ulo);
    hi.swap(uhi);
    count = up;
  }
  // The gather's stack keeps a level below its leaf-entry bit (bit 31), so
  // at most 7; 2^31 photons in leaves of 16 or more make at most 6.
  if (lvl > 7) throw std::runtime_error("photon box tree too deep");
  out->nlevels = lvl;
  if (out->box.size() > 0xffffffffu) throw std::runtime_error("photon box tree too large");
}

}  // namespace enc
