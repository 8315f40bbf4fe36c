// Test-infrastructure program: runs the drop-in adapters
// (encore_b200/adapters/GpuAccel.h, GpuPhotonMap.h) beside the reference's
// own Kdtree and PhotonMap, inside one binary built from the reference's
// unmodified sources (oracle/Makefile, target `adapter`), and compares them
// call by call through the reference's interfaces:
//
//   AccelerationStructure::build / intersect / update (Kdtree.cpp:84-200,
//   682-784; Kdtree.h:138) against GpuAccel in kd mode (every HitInfo field
//   identical) and in wide-BVH mode (same primitive, or a tie at the same t);
//   PhotonMap::GetNearestNPhotons / GetRadianceEstimate (PhotonMap.cpp:76-164)
//   against GpuPhotonMap (same photon sets, radiance within 1e-4 relative).
//
// Compiled as C++98, like the reference, which also shows the adapters are.
// Needs a CUDA device.  Prints one line of `key value` pairs; exit status 0
// when every comparison passes.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <list>
#include <set>
#include <vector>

#include "IModel.h"
#include "Kdtree.h"
#include "PhotonMap.h"
#include "Photon.h"
#include "Triangle.h"
#include "TrianglePrim.h"
#include "Vertex.h"
#include "../../encore_b200/adapters/GpuAccel.h"
#include "../../encore_b200/adapters/GpuPhotonMap.h"

extern bool IGNORE_NORMAL;

namespace {

unsigned long long g_state = 0x9E3779B97F4A7C15ull;
float urand() {  // xorshift64*, uniform in [0, 1)
  g_state ^= g_state >> 12;
  g_state ^= g_state << 25;
  g_state ^= g_state >> 27;
  return (float)((g_state * 2685821657736338717ull) >> 40) / 16777216.0f;
}

// A model over a vertex array it owns: triangle i uses vertices 3i..3i+2.
class SoupModel : public IModel {
 public:
  SoupModel(const std::vector<float>& v) : m_n((int)(v.size() / 9)) {
    m_verts.reserve(3 * m_n);
    for (int i = 0; i < 3 * m_n; ++i)
      m_verts.push_back(Vertex(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.f, 0.f, 1.f));
    m_tris.reserve(m_n);
    for (int i = 0; i < m_n; ++i)
      m_tris.push_back(Triangle(m_verts[3 * i], m_verts[3 * i + 1], m_verts[3 * i + 2]));
    m_prims.reserve(m_n);
    for (int i = 0; i < m_n; ++i) m_prims.push_back(TrianglePrim(m_tris[i]));
    for (int i = 0; i < m_n; ++i) m_PrimitiveList.push_back(&m_prims[i]);
    bounds();
  }
  ~SoupModel() { m_PrimitiveList.clear(); }
  // Moves every vertex (the scene animates): same primitives, new positions.
  void move(float dx, float dy, float wave) {
    for (size_t i = 0; i < m_verts.size(); ++i) {
      Point3 c = m_verts[i].getCoordinates();
      c.X() += dx;
      c.Y() += dy + wave * std::sin(c.X() * 0.006f);
      m_verts[i].setCoordinates(c);
    }
    bounds();
  }
  const IPrimitive* prim(int i) const { return &m_prims[i]; }

 private:
  void bounds() {
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (size_t i = 0; i < m_verts.size(); ++i) {
      const Point3& c = m_verts[i].getCoordinates();
      for (int a = 0; a < 3; ++a) {
        if (c[a] < lo[a]) lo[a] = c[a];
        if (c[a] > hi[a]) hi[a] = c[a];
      }
    }
    m_minPoint = Point3(lo[0], lo[1], lo[2]);
    m_maxPoint = Point3(hi[0], hi[1], hi[2]);
  }
  int m_n;
  std::vector<Vertex> m_verts;
  std::vector<Triangle> m_tris;
  std::vector<TrianglePrim> m_prims;
};

struct Tally {
  long rays, hits, same, ties, other, batch_diff;
  Tally() : rays(0), hits(0), same(0), ties(0), other(0), batch_diff(0) {}
};

bool same_point(const Point3& a, const Point3& b) {
  return a.X() == b.X() && a.Y() == b.Y() && a.Z() == b.Z();
}
bool same_vec(const Vector3& a, const Vector3& b) {
  return a.X() == b.X() && a.Y() == b.Y() && a.Z() == b.Z();
}

// Compares gpu.intersect with ref.intersect ray by ray, and the batched call
// with the per-ray one.
Tally compare(AccelerationStructure& ref, GpuAccel& gpu, const std::vector<float>& rays) {
  Tally t;
  const size_t n = rays.size() / 6;
  std::vector<float> r8(8 * n);
  for (size_t i = 0; i < n; ++i) {
    const float* r = &rays[6 * i];
    Ray a(Point3(r[0], r[1], r[2]), Vector3(r[3], r[4], r[5]));
    Ray b(Point3(r[0], r[1], r[2]), Vector3(r[3], r[4], r[5]));
    HitInfo ha, hb;
    const bool oka = ref.intersect(a, &ha);
    const bool okb = gpu.intersect(b, &hb);
    GpuAccel::pack(b, &r8[8 * i]);
    ++t.rays;
    if (oka) ++t.hits;
    const bool same = oka == okb &&
                      (!oka || (ha.hitObject == hb.hitObject && (float)ha.hitTime == (float)hb.hitTime &&
                                same_point(ha.hitPoint, hb.hitPoint) &&
                                same_vec(ha.hitNormal, hb.hitNormal) && ha.isEntering == hb.isEntering));
    if (same)
      ++t.same;
    else if (oka && okb && (float)ha.hitTime == (float)hb.hitTime)
      ++t.ties;  // another triangle at the same FP32 t (a shared edge)
    else
      ++t.other;
  }
  std::vector<enc_hit> hits(n);
  if (gpu.intersectBatch(&r8[0], n, &hits[0]) != ENC_OK) {
    t.batch_diff = (long)n;
    return t;
  }
  for (size_t i = 0; i < n; ++i) {
    const float* r = &rays[6 * i];
    Ray b(Point3(r[0], r[1], r[2]), Vector3(r[3], r[4], r[5]));
    HitInfo hb;
    const bool okb = gpu.intersect(b, &hb);
    const IPrimitive* pb = okb ? hb.hitObject : NULL;
    if (gpu.primitive(hits[i].tri) != pb) ++t.batch_diff;
  }
  // the batched call on the Ray payload itself (origin, direction) gives the
  // 8-float batch's hits, field for field
  std::vector<enc_hit> hits6(n);
  if (gpu.intersectBatchOD(&rays[0], n, &hits6[0]) != ENC_OK) {
    t.batch_diff += (long)n;
    return t;
  }
  for (size_t i = 0; i < n; ++i)
    if (std::memcmp(&hits6[i], &hits[i], sizeof(enc_hit)) != 0) ++t.batch_diff;
  return t;
}

std::vector<float> scene(int n, float scale) {
  std::vector<float> v;
  for (int i = 0; i < n; ++i) {
    float c[3] = {urand(), urand(), urand()};
    const float len = 0.005f + 0.045f * urand();
    for (int k = 0; k < 3; ++k) {
      float d[3] = {urand() - 0.5f, urand() - 0.5f, urand() - 0.5f};
      const float m = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + 1e-6f;
      for (int a = 0; a < 3; ++a) v.push_back((c[a] + len * d[a] / m) * scale);
    }
  }
  return v;
}

std::vector<float> rays_into(int n, float scale) {
  std::vector<float> r;
  for (int i = 0; i < n; ++i) {
    float o[3] = {urand() * scale, urand() * scale, -1.5f * scale};
    float t[3] = {(0.2f + 0.6f * urand()) * scale, (0.2f + 0.6f * urand()) * scale, 0.5f * scale};
    if (i % 2) {  // half start inside the cube, any direction
      o[0] = urand() * scale, o[1] = urand() * scale, o[2] = urand() * scale;
      t[0] = o[0] + urand() - 0.5f, t[1] = o[1] + urand() - 0.5f, t[2] = o[2] + urand() - 0.5f;
    }
    float d[3] = {t[0] - o[0], t[1] - o[1], t[2] - o[2]};
    const float m = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int a = 0; a < 3; ++a) r.push_back(o[a]);
    for (int a = 0; a < 3; ++a) r.push_back(d[a] / m);
  }
  return r;
}

}  // namespace

int main() {
  int ndev = 0;
  if (enc_device_count(&ndev) != ENC_OK || ndev < 1) {
    std::printf("error no_cuda_device\n");
    return 2;
  }
  bool ok = true;
  const float scale = 1000.f;
  std::vector<float> v = scene(20000, scale);
  std::vector<float> rays = rays_into(20000, scale);
  SoupModel model(v);
  std::list<IModel*> models;
  models.push_back(&model);

  Kdtree* kd = new Kdtree();  // never deleted: ~Kdtree walks unwritten node slots
  kd->build(models);
  GpuAccel gkd(ENC_ACCEL_KDTREE), gbvh(ENC_ACCEL_WBVH);
  gkd.build(models);
  gbvh.build(models);
  if (gkd.status() != ENC_OK || gbvh.status() != ENC_OK) {
    std::printf("error build %s\n", enc_last_error());
    return 1;
  }
  Tally a = compare(*kd, gkd, rays);
  Tally b = compare(*kd, gbvh, rays);
  std::printf("kd rays %ld hits %ld same %ld ties %ld other %ld batch_diff %ld\n", a.rays, a.hits,
              a.same, a.ties, a.other, a.batch_diff);
  std::printf("wbvh rays %ld hits %ld same %ld ties %ld other %ld batch_diff %ld\n", b.rays,
              b.hits, b.same, b.ties, b.other, b.batch_diff);
  ok &= a.same == a.rays && a.batch_diff == 0 && a.hits > a.rays / 4;
  ok &= b.other == 0 && b.ties <= b.rays / 1000 && b.batch_diff == 0;

  // update(): the scene moves; Kdtree::update rebuilds, GpuAccel refits.
  model.move(3.f, -2.f, 4.f);
  kd = new Kdtree();  // what Kdtree::update does (Kdtree.h:138), on a fresh object
  kd->build(models);
  gbvh.update(models);
  gkd.update(models);
  Tally c = compare(*kd, gkd, rays);
  Tally d = compare(*kd, gbvh, rays);
  std::printf("moved_kd same %ld of %ld other %ld; moved_wbvh same %ld ties %ld other %ld\n", c.same,
              c.rays, c.other, d.same, d.ties, d.other);
  ok &= c.same == c.rays && d.other == 0 && d.ties <= d.rays / 1000;

  // Photon maps: photons on three planes with three normals, so the
  // reference's exact normal-equality test (PhotonMap.cpp:244) matters.
  const int np = 30000, nq = 2000;
  PhotonMap ref_map(np);
  GpuPhotonMap gpu_map(np);
  const float normals[3][3] = {{0, 1, 0}, {1, 0, 0}, {0, 0, 1}};
  for (int i = 0; i < np; ++i) {
    const int k = i % 3;
    Point3 p(urand(), urand(), urand());
    p[k == 0 ? 1 : (k == 1 ? 0 : 2)] = 0.5f;  // on the plane of its normal
    Photon ph(p, encore::Color(urand(), urand(), urand()), Vector3((float)i, 0.f, 0.f));
    ph.SurfNormal(Vector3(normals[k][0], normals[k][1], normals[k][2]));
    ref_map.AddPhoton(ph);
    gpu_map.AddPhoton(ph);
  }
  ref_map.BalanceAndConstruct();
  gpu_map.BalanceAndConstruct();
  double worst = 0.0;
  long set_diff = 0, heap_bad = 0;
  for (int pass = 0; pass < 2; ++pass) {
    IGNORE_NORMAL = pass == 1;
    gpu_map.SetIgnoreNormal(pass == 1);
    for (int i = 0; i < nq; ++i) {
      const int k = i % 3;
      Point3 q(urand(), urand(), urand());
      q[k == 0 ? 1 : (k == 1 ? 0 : 2)] = 0.5f;
      Vector3 qn(normals[k][0], normals[k][1], normals[k][2]);
      encore::Color cr = ref_map.GetRadianceEstimate(50, 0.1f, q, qn);
      encore::Color cg = gpu_map.GetRadianceEstimate(50, 0.1f, q, qn);
      const float rr[3] = {cr.R(), cr.G(), cr.B()}, gg[3] = {cg.R(), cg.G(), cg.B()};
      for (int c3 = 0; c3 < 3; ++c3) {
        const double den = std::fabs((double)rr[c3]) > 1e-30 ? std::fabs((double)rr[c3]) : 1.0;
        const double e = std::fabs((double)rr[c3] - (double)gg[c3]) / den;
        if (e > worst) worst = e;
      }
      std::vector<PhotonDistPair> nr = ref_map.GetNearestNPhotons(50, 0.1f, q, qn);
      std::vector<PhotonDistPair> ng = gpu_map.GetNearestNPhotons(50, 0.1f, q, qn);
      std::set<int> sr, sg;
      for (size_t j = 0; j < nr.size(); ++j) sr.insert((int)nr[j].m_pPhoton->Direction().X());
      for (size_t j = 0; j < ng.size(); ++j) sg.insert((int)ng[j].m_pPhoton->Direction().X());
      if (sr != sg) ++set_diff;
      for (size_t j = 1; j < ng.size(); ++j)  // max-heap: no child above its parent
        if (ng[(j - 1) / 2] < ng[j]) {
          ++heap_bad;
          break;
        }
    }
  }
  IGNORE_NORMAL = false;
  std::printf("photons queries %d set_diff %ld heap_bad %ld radiance_max_rel_err %.3g\n", 2 * nq,
              set_diff, heap_bad, worst);
  ok &= set_diff == 0 && heap_bad == 0 && worst <= 1e-4;

  // EmitPhotons on the device into two GpuPhotonMaps (PhotonMapperCPU's
  // direct and indirect maps): the indirect map is filled by the emission
  // loop, the direct map holds first hits and shadow photons, and both agree
  // with the C ABI's own split call on the same options.
  enc_photon_opts po;
  po.light_center[0] = 0.5f * scale;
  po.light_center[1] = 2.0f * scale;
  po.light_center[2] = 0.5f * scale;
  po.light_size = 0.1f * scale;
  po.nphotons = 20000;
  po.max_bounces = 3;
  po.albedo = 0.7f;
  po.seed = 5;
  po.emit_offset = 0.01f * scale;
  po.bounce_offset = 0.001f * scale;
  GpuPhotonMap direct(200000), indirect(2000);
  uint32_t emitted = 0;
  const enc_status es = GpuEmitPhotons(gbvh.handle(), po, 5.0f, true, direct, indirect, &emitted);
  std::vector<float> bd(9 * 200000 + 9), bi(9 * 2000 + 9);
  enc_photon_store sd = {&bd[0], &bd[0] + 3 * 200000, &bd[0] + 6 * 200000, NULL, 200000};
  enc_photon_store si = {&bi[0], &bi[0] + 3 * 2000, &bi[0] + 6 * 2000, NULL, 2000};
  uint32_t stored[2] = {0, 0}, emitted2 = 0;
  const enc_status es2 = enc_photons_trace_maps(gbvh.handle(), &po, 5.0f, 1, &sd, &si, stored,
                                                &emitted2, NULL);
  std::printf("emit status %d direct %d indirect %d emitted %u abi %u %u %u\n", (int)es,
              direct.GetCountStored(), indirect.GetCountStored(), emitted, stored[0], stored[1],
              emitted2);
  ok &= es == ENC_OK && es2 == ENC_OK && indirect.Full() && emitted >= po.nphotons &&
        emitted % po.nphotons == 0 &&
        emitted == emitted2 && (uint32_t)direct.GetCountStored() == stored[0] &&
        (uint32_t)indirect.GetCountStored() == stored[1] && stored[0] > 0;
  std::printf("result %s\n", ok ? "pass" : "fail");
  return ok ? 0 : 1;
}
