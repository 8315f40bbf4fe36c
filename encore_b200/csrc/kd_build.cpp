// Host builder of the kd-tree layout, following the reference's Kdtree build
// rules so that the device walk visits the same cells in the same order and
// tests the same triangles in the same order as Kdtree::intersect:
//
//  * root box = model bounds padded by 0.001 per axis, kept as the reference
//    keeps every AABB: min corner + size, max recomputed as pos + size in FP32
//    (Kdtree.cpp:116-117, AABB.h:34-40);
//  * max depth 11 + (unsigned)(1.3 ln N) and leaf capacity 2 (N <= 5000) or 10
//    (Kdtree.cpp:123-131, Kdtree.cpp:17);
//  * leaf when size <= capacity, depth >= max depth, or the list size changed
//    by at most 3 for three consecutive levels (Kdtree.cpp:314-324);
//  * split axis depth % 3 at the node box's midpoint (Kdtree.cpp:514-517);
//  * a triangle goes to each child whose voxel its box overlaps with the strict
//    test of AABB::Intersect(AABB) (AABB.cpp:9-18), and to both when it
//    overlaps neither (Kdtree.cpp:561-650); list order is preserved, so a
//    leaf's triangles are in ascending ID order as in the reference;
//  * the node word keeps the split float with its two low bits replaced by the
//    axis, which is the value the reference's traversal reads (Kdtree.h:47-53).
//
// The implementation is an explicit-stack recursion over index vectors; the
// reference's shared leftBOX/rightBOX buffers (Kdtree.cpp:164-176) only change
// where the lists live, not their contents.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <utility>

#include "engine.h"

namespace enc {
namespace {

// The reference's AABB: min corner and size (AABB.h:65-66).
struct RBox {
  float pos[3], size[3];
};

inline RBox from_corners(const float* mn, const float* mx) {
  RBox b;
  for (int a = 0; a < 3; ++a) {
    b.pos[a] = mn[a];
    b.size[a] = mx[a] - mn[a];
  }
  return b;
}

// AABB::Intersect(AABB b2) called on `self` (AABB.cpp:9-18).
inline bool overlaps(const RBox& self, const RBox& b2) {
  for (int a = 0; a < 3; ++a) {
    float v1 = b2.pos[a];
    float v2 = b2.pos[a] + b2.size[a];
    float v3 = self.pos[a];
    float v4 = self.pos[a] + self.size[a];
    if (!((v4 > v1) && (v3 < v2))) return false;
  }
  return true;
}

// TrianglePrim::getAABB (TrianglePrim.cpp:184-202) with the dmin/dmax macros
// of TrianglePrim.h:29-30.
inline RBox tri_box(const float* t) {
  float mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    float x0 = t[a], x1 = t[3 + a], x2 = t[6 + a];
    float m01 = (x0 > x1) ? x1 : x0;
    mn[a] = (m01 > x2) ? x2 : m01;
    float M01 = (x0 > x1) ? x0 : x1;
    mx[a] = (M01 > x2) ? M01 : x2;
  }
  return from_corners(mn, mx);
}

struct Task {
  uint32_t node;
  RBox box;
  std::vector<uint32_t> list;
  uint32_t depth, pre_size;
  bool dsize;
  int tries;
};

}  // namespace

void build_kd_reference(const float* v, uint32_t ntris, KdHost* out) {
  if (ntris == 0) throw std::runtime_error("empty scene");
  // Model bounds (the vertex bounds), then the 0.001 pad.
  float mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = v[a];
    mx[a] = v[a];
  }
  for (size_t i = 0; i < 3 * (size_t)ntris; ++i)
    for (int a = 0; a < 3; ++a) {
      float c = v[3 * i + a];
      if (c < mn[a]) mn[a] = c;
      if (c > mx[a]) mx[a] = c;
    }
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = mn[a] - 0.001f;
    hi[a] = mx[a] + 0.001f;
  }
  RBox root = from_corners(lo, hi);
  for (int a = 0; a < 3; ++a) {
    out->root_lo[a] = root.pos[a];
    out->root_hi[a] = root.pos[a] + root.size[a];
  }
  const uint32_t max_items = ntris <= 5000 ? 2u : 10u;
  const uint32_t max_depth = 11u + (uint32_t)(1.3 * (double)std::log((float)ntris));
  out->max_depth = (int)max_depth;

  std::vector<RBox> tbox(ntris);
  for (uint32_t i = 0; i < ntris; ++i) tbox[i] = tri_box(v + 9 * (size_t)i);

  out->nodes.assign(1, KdNode{0, 0});
  out->items.clear();
  std::vector<Task> stack;
  Task t0;
  t0.node = 0;
  t0.box = root;
  t0.list.resize(ntris);
  for (uint32_t i = 0; i < ntris; ++i) t0.list[i] = i;
  t0.depth = 0;
  t0.pre_size = 0;
  t0.dsize = false;
  t0.tries = 0;
  stack.push_back(std::move(t0));
  while (!stack.empty()) {
    Task t = std::move(stack.back());
    stack.pop_back();
    uint32_t size = (uint32_t)t.list.size();
    bool dsize = t.dsize;
    int tries = t.tries;
    if ((int)std::abs((int)(t.pre_size - size)) <= 3) {
      dsize = true;
      tries++;
    } else {
      dsize = false;
      tries = 0;
    }
    if (size <= max_items || t.depth >= max_depth || (dsize && tries == 3)) {
      KdNode& n = out->nodes[t.node];
      n.word0 = (size << 2) | 3u;
      n.word1 = (uint32_t)out->items.size();
      out->items.insert(out->items.end(), t.list.begin(), t.list.end());
      continue;
    }
    int axis = (int)(t.depth % 3);
    float minp[3], maxp[3];
    for (int a = 0; a < 3; ++a) {
      minp[a] = t.box.pos[a];
      maxp[a] = minp[a] + t.box.size[a];
    }
    float splitpos = (minp[axis] + maxp[axis]) / 2;
    float rminp[3], lmaxp[3], bmax[3];
    for (int a = 0; a < 3; ++a) {
      rminp[a] = t.box.pos[a];
      lmaxp[a] = t.box.pos[a] + t.box.size[a];
      bmax[a] = t.box.pos[a] + t.box.size[a];
    }
    rminp[axis] = splitpos;
    lmaxp[axis] = splitpos;
    RBox lvox = from_corners(t.box.pos, lmaxp);
    RBox rvox = from_corners(rminp, bmax);
    Task L, R;
    L.list.reserve(size);
    R.list.reserve(size);
    for (uint32_t p : t.list) {
      bool l = overlaps(lvox, tbox[p]);
      bool r = overlaps(rvox, tbox[p]);
      if (l || !r) L.list.push_back(p);
      if (r || !l) R.list.push_back(p);
    }
    uint32_t child = (uint32_t)out->nodes.size();
    out->nodes.push_back(KdNode{0, 0});
    out->nodes.push_back(KdNode{0, 0});
    uint32_t bits;
    std::memcpy(&bits, &splitpos, 4);
    KdNode& n = out->nodes[t.node];
    n.word0 = (bits & ~3u) | (uint32_t)axis;
    n.word1 = child;
    L.node = child;
    L.box = lvox;
    L.depth = t.depth + 1;
    L.pre_size = size;
    L.dsize = dsize;
    L.tries = tries;
    R.node = child + 1;
    R.box = rvox;
    R.depth = t.depth + 1;
    R.pre_size = size;
    R.dsize = dsize;
    R.tries = tries;
    stack.push_back(std::move(R));
    stack.push_back(std::move(L));
  }
}

}  // namespace enc
