// Host builder for the wide BVH (width 2, 4 or 8) with 8-bit quantised child
// boxes.
//
// 1. Binned SAH (16 bins per axis, centroid bounds) builds a binary BVH with
//    at most `max_leaf` triangles per leaf.  The reference's Bvh splits at the
//    spatial median with one triangle per leaf (BVH.cpp:246-251); SAH gives
//    far fewer node visits per ray and the closest hit does not depend on the
//    tree shape, only on the set of triangles the predicate accepts.
// 2. The binary tree is collapsed to width W by repeatedly opening the child
//    with the largest surface area.
// 3. Each wide node stores its box origin p and per-axis power-of-two scale;
//    child boxes are quantised to 8 bits with lo rounded down and hi rounded
//    up, so the decoded box always contains the child's box.  Triangle boxes
//    are padded by 1e-5 of the scene size before anything else, which keeps
//    traversal conservative against FP32 rounding in the slab test and in the
//    triangle predicate: a triangle the predicate accepts always lies in a box
//    the ray is found to enter.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <stdexcept>
#include <thread>

#include "engine.h"

namespace enc {
namespace {

struct Box {
  float lo[3], hi[3];
  void empty() {
    for (int a = 0; a < 3; ++a) {
      lo[a] = INFINITY;
      hi[a] = -INFINITY;
    }
  }
  void grow(const Box& b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  void grow(const float* p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  float area() const {
    float dx = std::max(0.f, hi[0] - lo[0]), dy = std::max(0.f, hi[1] - lo[1]),
          dz = std::max(0.f, hi[2] - lo[2]);
    return 2.f * (dx * dy + dy * dz + dz * dx);
  }
};

struct BNode {
  Box box;
  int32_t left;    // child pair at left, left + 1; -1 for a leaf
  uint32_t first;  // leaf: first index into prim order
  uint32_t count;  // leaf: number of triangles
};

constexpr int kBins = 16;
// Cost of one binary traversal step relative to one triangle test in the
// SAH.  (1.5, 2 and 3 were measured on the 2M-triangle heightfield: with
// leaves of up to 3 triangles the trees barely change; with up to 4 the
// extra triangle tests cost 14-24 % more time than the fewer node visits
// save.)
#ifndef ENC_SAH_TRAV_COST
#define ENC_SAH_TRAV_COST 1.0f
#endif
constexpr float kTravCost = ENC_SAH_TRAV_COST;
constexpr uint32_t kParallelCutoff = 1u << 16;

struct BinaryBuilder {
  const Box* pbox;
  const float* cent;  // 3 per prim
  uint32_t* idx;
  BNode* nodes;
  std::atomic<uint32_t> next{1};
  int max_leaf;

  uint32_t alloc_pair() { return next.fetch_add(2); }

  void make_leaf(uint32_t ni, uint32_t b, uint32_t e, const Box& box) {
    nodes[ni].box = box;
    nodes[ni].left = -1;
    nodes[ni].first = b;
    nodes[ni].count = e - b;
  }

  // Builds node ni over idx[b, e).  box = bounds of the prims in the range.
  void build(uint32_t ni, uint32_t b, uint32_t e, const Box& box, int depth) {
    uint32_t n = e - b;
    if (n <= 1 || depth > 60) {
      if (n > (uint32_t)max_leaf) {  // pathological depth: split by count
        split_median(ni, b, e, box, depth);
        return;
      }
      make_leaf(ni, b, e, box);
      return;
    }
    Box cb;
    cb.empty();
    for (uint32_t i = b; i < e; ++i) cb.grow(cent + 3 * (size_t)idx[i]);
    int best_axis = -1, best_split = -1;
    float best_cost = INFINITY;
    for (int a = 0; a < 3; ++a) {
      float ext = cb.hi[a] - cb.lo[a];
      if (!(ext > 0.f)) continue;
      float k = kBins * (1.f - 1e-6f) / ext;
      Box bb[kBins];
      uint32_t bc[kBins] = {0};
      for (int i = 0; i < kBins; ++i) bb[i].empty();
      for (uint32_t i = b; i < e; ++i) {
        uint32_t p = idx[i];
        int bi = (int)((cent[3 * (size_t)p + a] - cb.lo[a]) * k);
        bi = std::min(std::max(bi, 0), kBins - 1);
        bc[bi]++;
        bb[bi].grow(pbox[p]);
      }
      float ra[kBins];
      uint32_t rc[kBins];
      Box acc;
      acc.empty();
      uint32_t cnt = 0;
      for (int i = kBins - 1; i > 0; --i) {
        acc.grow(bb[i]);
        cnt += bc[i];
        ra[i] = acc.area();
        rc[i] = cnt;
      }
      acc.empty();
      cnt = 0;
      for (int i = 0; i < kBins - 1; ++i) {
        acc.grow(bb[i]);
        cnt += bc[i];
        if (cnt == 0 || rc[i + 1] == 0) continue;
        float cost = acc.area() * cnt + ra[i + 1] * rc[i + 1];
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_split = i;
        }
      }
    }
    float parea = box.area();
    float leaf_cost = (float)n;
    float split_cost = parea > 0.f ? kTravCost + best_cost / parea : INFINITY;
    if (n <= (uint32_t)max_leaf && leaf_cost <= split_cost) {
      make_leaf(ni, b, e, box);
      return;
    }
    if (best_axis < 0) {  // all centroids equal: split by count
      split_median(ni, b, e, box, depth);
      return;
    }
    float k = kBins * (1.f - 1e-6f) / (cb.hi[best_axis] - cb.lo[best_axis]);
    float lo = cb.lo[best_axis];
    uint32_t* mid = std::partition(idx + b, idx + e, [&](uint32_t p) {
      int bi = (int)((cent[3 * (size_t)p + best_axis] - lo) * k);
      bi = std::min(std::max(bi, 0), kBins - 1);
      return bi <= best_split;
    });
    uint32_t m = (uint32_t)(mid - idx);
    if (m == b || m == e) {
      split_median(ni, b, e, box, depth);
      return;
    }
    recurse(ni, b, m, e, depth);
  }

  void split_median(uint32_t ni, uint32_t b, uint32_t e, const Box& box, int depth) {
    (void)box;
    uint32_t m = b + (e - b) / 2;
    recurse(ni, b, m, e, depth);
  }

  void recurse(uint32_t ni, uint32_t b, uint32_t m, uint32_t e, int depth) {
    Box lb, rb;
    lb.empty();
    rb.empty();
    for (uint32_t i = b; i < m; ++i) lb.grow(pbox[idx[i]]);
    for (uint32_t i = m; i < e; ++i) rb.grow(pbox[idx[i]]);
    uint32_t c = alloc_pair();
    nodes[ni].left = (int32_t)c;
    nodes[ni].count = 0;
    nodes[ni].first = 0;
    if (e - b > kParallelCutoff) {
      auto fut = std::async(std::launch::async, [&, c, b, m, lb, depth] { build(c, b, m, lb, depth + 1); });
      build(c + 1, m, e, rb, depth + 1);
      fut.get();
    } else {
      build(c, b, m, lb, depth + 1);
      build(c + 1, m, e, rb, depth + 1);
    }
    Box u = lb;
    u.grow(rb);
    nodes[ni].box = u;
  }
};

// Writes the node origin, scale exponents and the 8-bit child planes of a
// wide node: the grid has its origin at the node's lo corner and steps of
// 2^e with the node extent in at most 255 of them, 2^e no finer than the
// float spacing at the node (so tiny nodes far from the origin still
// quantise); each child's lo is rounded down and hi up, so the decoded box
// contains the child box.  Empty slots get an inverted box (lo 255, hi 0)
// that no ray enters.  (A grid one step wider on each side, which lets the
// kernel drop one add per plane, was measured: the looser boxes cost 7 % more
// node visits and more time than the add saves.)
template <int W>
void quantize_node(const Box& nb, const Box* slot_box, const bool* slot_used, WNodeHeader* h,
                   uint8_t* raw) {
  using L = WNodeLayout<W>;
  double scale[3];
  for (int a = 0; a < 3; ++a) {
    const double ext = (double)nb.hi[a] - (double)nb.lo[a];
    const float mag = std::max(std::fabs(nb.lo[a]), std::fabs(nb.hi[a]));
    const double spacing = (double)std::nextafter(mag, INFINITY) - (double)mag;
    int e = -126;
    while (std::ldexp(255.0, e) < ext || std::ldexp(1.0, e) < spacing) ++e;
    if (e > 127) throw std::runtime_error("scene extent too large to quantise");
    h->e[a] = (uint8_t)(e + 127);
    scale[a] = std::ldexp(1.0, e);
    h->p[a] = nb.lo[a];
  }
  uint8_t* q = raw + L::kQOff;
  for (int i = 0; i < W; ++i) {
    for (int a = 0; a < 3; ++a) {
      if (!slot_used[i]) {
        q[a * W + i] = 255;
        q[(3 + a) * W + i] = 0;
        continue;
      }
      const double lo = std::floor(((double)slot_box[i].lo[a] - (double)h->p[a]) / scale[a]);
      const double hi = std::ceil(((double)slot_box[i].hi[a] - (double)h->p[a]) / scale[a]);
      if (lo < 0.0 || hi > 255.0) throw std::runtime_error("child box outside its quantisation grid");
      q[a * W + i] = (uint8_t)lo;
      q[(3 + a) * W + i] = (uint8_t)hi;
    }
  }
}

template <int W>
void collapse(const std::vector<BNode>& bn, const std::vector<uint32_t>& order,
              const float* tri_verts, WBVHHost* out) {
  using L = WNodeLayout<W>;
  std::vector<uint32_t> queue;  // binary node per wide node, BFS order
  std::vector<uint16_t> level;  // depth of each wide node (root = 1)
  queue.push_back(0);
  level.push_back(1);
  int max_level = 1;
  std::vector<uint8_t>& nodes = out->nodes;
  std::vector<uint32_t> tri_order;
  tri_order.reserve(order.size());
  nodes.clear();
  for (size_t qi = 0; qi < queue.size(); ++qi) {
    uint32_t b = queue[qi];
    // Children of this wide node.
    uint32_t kids[W];
    int nk = 0;
    if (bn[b].left < 0) {
      kids[nk++] = b;  // root is a leaf
    } else {
      kids[nk++] = (uint32_t)bn[b].left;
      kids[nk++] = (uint32_t)bn[b].left + 1;
      while (nk < W) {
        int best = -1;
        float ba = -1.f;
        for (int i = 0; i < nk; ++i)
          if (bn[kids[i]].left >= 0 && bn[kids[i]].box.area() > ba) {
            ba = bn[kids[i]].box.area();
            best = i;
          }
        if (best < 0) break;
        uint32_t o = kids[best];
        kids[best] = (uint32_t)bn[o].left;
        kids[nk++] = (uint32_t)bn[o].left + 1;
      }
    }
    // Node box = union of children.
    Box nb;
    nb.empty();
    for (int i = 0; i < nk; ++i) nb.grow(bn[kids[i]].box);
    std::vector<uint8_t> raw(L::kBytes, 0);
    WNodeHeader h;
    std::memset(&h, 0, sizeof(h));
    h.child_base = (uint32_t)(queue.size());
    h.tri_base = (uint32_t)tri_order.size();
    // Slot order.  Width 8: slot s holds the child lying most in octant s
    // (bit a of s set = positive side of axis a) relative to the node centre,
    // assigned greedily by largest dot(child centre - node centre, octant
    // direction).  A ray whose direction is negative on the axes in mask m
    // then meets the children roughly front to back in slot order k ^ m,
    // k = 0..7, with no per-node sort.  Widths 2 and 4 keep build order.
    int slot_child[W];
    for (int s = 0; s < W; ++s) slot_child[s] = -1;
    if (W == 8) {
      float ctr[3];
      for (int a = 0; a < 3; ++a) ctr[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
      float score[8][8];
      for (int i = 0; i < nk; ++i) {
        const Box& cb = bn[kids[i]].box;
        float d[3];
        for (int a = 0; a < 3; ++a) d[a] = 0.5f * (cb.lo[a] + cb.hi[a]) - ctr[a];
        for (int s = 0; s < 8; ++s)
          score[i][s] = ((s & 1) ? d[0] : -d[0]) + ((s & 2) ? d[1] : -d[1]) + ((s & 4) ? d[2] : -d[2]);
      }
      bool used_child[8] = {false}, used_slot[8] = {false};
      for (int it = 0; it < nk; ++it) {
        int bi = -1, bs = -1;
        float bv = -INFINITY;
        for (int i = 0; i < nk; ++i)
          if (!used_child[i])
            for (int s = 0; s < 8; ++s)
              if (!used_slot[s] && (bi < 0 || score[i][s] > bv)) {
                bv = score[i][s];
                bi = i;
                bs = s;
              }
        used_child[bi] = true;
        used_slot[bs] = true;
        slot_child[bs] = bi;
      }
    } else {
      for (int i = 0; i < nk; ++i) slot_child[i] = i;
    }
    int n_internal = 0;
    uint8_t* meta = raw.data() + L::kMetaOff;
    Box slot_box[W];
    bool slot_used[W];
    for (int i = 0; i < W; ++i) {
      slot_used[i] = slot_child[i] >= 0;
      if (!slot_used[i]) continue;
      const BNode& c = bn[kids[slot_child[i]]];
      slot_box[i] = c.box;
      if (c.left >= 0) {
        meta[i] = (uint8_t)(1 + n_internal);
        h.imask |= (uint8_t)(1u << i);
        ++n_internal;
        queue.push_back(kids[slot_child[i]]);
        level.push_back((uint16_t)(level[qi] + 1));
        max_level = std::max(max_level, (int)level[qi] + 1);
      } else {
        uint32_t off = (uint32_t)tri_order.size() - h.tri_base;
        if (c.count < 1 || c.count > 7 || off + c.count > 32)
          throw std::runtime_error("leaf packing overflow");
        meta[i] = (uint8_t)((c.count << 5) | off);
        for (uint32_t k = 0; k < c.count; ++k) tri_order.push_back(order[c.first + k]);
      }
    }
    quantize_node<W>(nb, slot_box, slot_used, &h, raw.data());
    std::memcpy(raw.data(), &h, sizeof(h));
    nodes.insert(nodes.end(), raw.begin(), raw.end());
  }
  out->nnodes = (uint32_t)queue.size();
  out->depth = max_level;
  out->tri_order = tri_order;
  out->tri_pos.assign(tri_order.size(), 0);
  for (size_t i = 0; i < tri_order.size(); ++i) out->tri_pos[tri_order[i]] = (uint32_t)i;
  out->tris.resize(tri_order.size());
  make_dev_tris(tri_verts, (uint32_t)tri_order.size(), tri_order.data(), out->tris.data());
}

}  // namespace

void make_dev_tris(const float* v, uint32_t n, const uint32_t* order, DevTri* out) {
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t id = order ? order[i] : i;
    const float* t = v + 9 * (size_t)id;
    DevTri& d = out[i];
    float e1[3] = {t[3] - t[0], t[4] - t[1], t[5] - t[2]};
    float e2[3] = {t[6] - t[0], t[7] - t[1], t[8] - t[2]};
    d.a[0] = t[0];
    d.a[1] = t[1];
    d.a[2] = t[2];
    d.a[3] = e1[0];
    d.b[0] = e1[1];
    d.b[1] = e1[2];
    d.b[2] = e2[0];
    d.b[3] = e2[1];
    d.c[0] = e2[2];
    int32_t iid = (int32_t)id;
    std::memcpy(&d.c[1], &iid, 4);
    d.c[2] = 0.f;
    d.c[3] = 0.f;
  }
}

namespace {

// Triangle boxes padded by 1e-5 of the larger of the scene extent and the
// largest coordinate, the scene bounds, and (if asked) the unpadded box
// centres the SAH bins on.
std::vector<Box> padded_boxes(const float* v, uint32_t n, float lo[3], float hi[3],
                              std::vector<float>* cent = nullptr) {
  std::vector<Box> pbox(n);
  Box scene;
  scene.empty();
  float maxabs = 0.f;
  for (uint32_t i = 0; i < n; ++i) {
    const float* t = v + 9 * (size_t)i;
    Box b;
    b.empty();
    b.grow(t);
    b.grow(t + 3);
    b.grow(t + 6);
    pbox[i] = b;
    scene.grow(b);
    for (int k = 0; k < 9; ++k) maxabs = std::max(maxabs, std::fabs(t[k]));
  }
  const float ext = std::max(std::max(scene.hi[0] - scene.lo[0], scene.hi[1] - scene.lo[1]),
                             scene.hi[2] - scene.lo[2]);
  float pad = 1e-5f * std::max(ext, maxabs);
  if (!(pad > 0.f)) pad = 1e-30f;
  if (cent) cent->resize(3 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      if (cent) (*cent)[3 * (size_t)i + a] = 0.5f * (pbox[i].lo[a] + pbox[i].hi[a]);
      pbox[i].lo[a] -= pad;
      pbox[i].hi[a] += pad;
    }
  for (int a = 0; a < 3; ++a) {
    lo[a] = scene.lo[a];
    hi[a] = scene.hi[a];
  }
  return pbox;
}

// Bottom-up refit: the nodes are in breadth-first order, so every child has
// a larger index than its parent and one reverse pass sees children first.
template <int W>
void refit_w(WBVHHost* H, const float* v, uint32_t ntris) {
  using L = WNodeLayout<W>;
  std::vector<Box> pbox = padded_boxes(v, ntris, H->lo, H->hi);
  std::vector<Box> nbox(H->nnodes);
  for (int64_t i = (int64_t)H->nnodes - 1; i >= 0; --i) {
    uint8_t* raw = H->nodes.data() + (size_t)i * L::kBytes;
    WNodeHeader h;
    std::memcpy(&h, raw, sizeof(h));
    const uint8_t* meta = raw + L::kMetaOff;
    Box slot_box[W];
    bool used[W];
    Box nb;
    nb.empty();
    for (int c = 0; c < W; ++c) {
      const uint32_t m = meta[c];
      used[c] = m != 0;
      if (!used[c]) continue;
      if (m < 32) {
        const uint32_t child = h.child_base + (m - 1);
        if (child >= H->nnodes) throw std::runtime_error("refit: corrupt node table");
        slot_box[c] = nbox[child];
      } else {
        slot_box[c].empty();
        for (uint32_t k = 0; k < (m >> 5); ++k) {
          const uint32_t slot = h.tri_base + (m & 31u) + k;
          if (slot >= H->tri_order.size()) throw std::runtime_error("refit: corrupt node table");
          slot_box[c].grow(pbox[H->tri_order[slot]]);
        }
      }
      nb.grow(slot_box[c]);
    }
    nbox[(size_t)i] = nb;
    quantize_node<W>(nb, slot_box, used, &h, raw);
    std::memcpy(raw, &h, sizeof(h));
  }
  H->tris.resize(H->tri_order.size());
  make_dev_tris(v, (uint32_t)H->tri_order.size(), H->tri_order.data(), H->tris.data());
}

}  // namespace

void refit_wbvh(WBVHHost* h, const float* tri_verts, uint32_t ntris) {
  if (ntris != h->tri_order.size()) throw std::runtime_error("refit needs the same triangle count");
  if (h->width == 2) refit_w<2>(h, tri_verts, ntris);
  else if (h->width == 4) refit_w<4>(h, tri_verts, ntris);
  else refit_w<8>(h, tri_verts, ntris);
}

void build_wbvh(const float* tri_verts, uint32_t ntris, int width, int max_leaf, WBVHHost* out) {
  if (ntris == 0) throw std::runtime_error("empty scene");
  if (max_leaf < 1 || max_leaf > 4) throw std::runtime_error("max_leaf_tris must be 1..4");
  std::vector<float> cent;
  std::vector<Box> pbox = padded_boxes(tri_verts, ntris, out->lo, out->hi, &cent);
  std::vector<uint32_t> idx(ntris);
  for (uint32_t i = 0; i < ntris; ++i) idx[i] = i;
  std::vector<BNode> bn(2 * (size_t)ntris);
  BinaryBuilder bb;
  bb.pbox = pbox.data();
  bb.cent = cent.data();
  bb.idx = idx.data();
  bb.nodes = bn.data();
  bb.max_leaf = max_leaf;
  Box root;
  root.empty();
  for (uint32_t i = 0; i < ntris; ++i) root.grow(pbox[i]);
  bb.build(0, 0, ntris, root, 0);
  bn.resize(bb.next.load());
  out->width = width;
  if (width == 2) collapse<2>(bn, idx, tri_verts, out);
  else if (width == 4) collapse<4>(bn, idx, tri_verts, out);
  else if (width == 8) collapse<8>(bn, idx, tri_verts, out);
  else throw std::runtime_error("width must be 2, 4 or 8");
}

}  // namespace enc
