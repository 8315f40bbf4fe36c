// Test-infrastructure harness around the reference's own CPU query path.
//
// This file is compiled together with the reference's unmodified .cpp files
// (list in oracle/Makefile) into oracle/_ref/libencore_ref.so.  It only adapts
// plain arrays to the reference's object model and back; every hit, tree and
// photon search below is computed by the reference code itself:
//
//   Kdtree::build / Kdtree::intersect   ENCORE/src/accelerators/Kdtree.cpp:84-200, 682-784
//   Bvh::build / Bvh::intersect         ENCORE/src/accelerators/BVH.cpp:123-187, 778-884
//   BasicAS::intersect                  ENCORE/src/accelerators/BasicAS.cpp:167-194
//   TrianglePrim::intersect             ENCORE/src/scene/TrianglePrim.cpp:204-248
//   PhotonMap::BalanceAndConstruct      ENCORE/src/renderers/PhotonMap.cpp:167-221
//   PhotonMap::GetNearestNPhotons       ENCORE/src/renderers/PhotonMap.cpp:76-94, 224-297
//   PhotonMap::GetRadianceEstimate      ENCORE/src/renderers/PhotonMap.cpp:121-164
//   PhotonMapperCPU::IsInShadow         ENCORE/src/renderers/PhotonMapperCPU.cpp:1192-1207
//   Camera::Camera / CalcCamVectors     ENCORE/src/scene/Camera.cpp:12-18, 85-93, 157-166
//   TrianglePrim::intersect's hit point and normal  TrianglePrim.cpp:236-239
//
// It is the checker used by tests and the timed CPU arm of bench.py; nothing
// in the engine links it.
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>
#include <list>
#include <thread>
#include <algorithm>

#include "Vertex.h"
#include "Triangle.h"
#include "TrianglePrim.h"
#include "IModel.h"
#include "Kdtree.h"
#include "BVH.h"
#include "BasicAS.h"
#include "PhotonMap.h"
#include "Photon.h"
#include "Color.h"
#include "Model.h"
#include "Material.h"
#include "Camera.h"
#include "Common.h"
#include "Ray.h"

extern bool IGNORE_NORMAL;  // ENCORE/src/renderers/PhotonMap.cpp:23

namespace {

// An IModel whose vertices and triangles come from a flat float array
// (9 floats per triangle).  Primitive-list order = triangle index, which is
// how the reference identifies a hit triangle (Model.cpp:255-264).  The model
// bounds are set to the true vertex bounds: the accelerators read them through
// IModel::MinPoint/MaxPoint (IModel.h:34-35) and a zero box would cull every ray.
class ArrayModel : public IModel {
 public:
  ArrayModel(const float* v, int ntris) {
    verts_.reserve((size_t)ntris * 3);
    for (int i = 0; i < 3 * ntris; ++i)
      verts_.push_back(Vertex(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.f, 0.f, 1.f));
    tris_.reserve(ntris);
    for (int i = 0; i < ntris; ++i)
      tris_.push_back(Triangle(verts_[3 * i], verts_[3 * i + 1], verts_[3 * i + 2]));
    prims_.reserve(ntris);
    for (int i = 0; i < ntris; ++i) prims_.push_back(TrianglePrim(tris_[i]));
    for (int i = 0; i < ntris; ++i) m_PrimitiveList.push_back(&prims_[i]);
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int i = 0; i < 3 * ntris; ++i)
      for (int a = 0; a < 3; ++a) {
        float c = v[3 * i + a];
        if (i == 0 || c < lo[a]) lo[a] = c;
        if (i == 0 || c > hi[a]) hi[a] = c;
      }
    m_minPoint = Point3(lo[0], lo[1], lo[2]);
    m_maxPoint = Point3(hi[0], hi[1], hi[2]);
  }
  ~ArrayModel() { m_PrimitiveList.clear(); }
  int index_of(const IPrimitive* p) const {
    if (!p) return -1;
    return (int)((const TrianglePrim*)p - &prims_[0]);
  }
  const float* tri_coords(int i, int k) const {
    return coords_.empty() ? 0 : &coords_[(size_t)9 * i + 3 * k];
  }
  std::vector<float> coords_;

 private:
  std::vector<Vertex> verts_;
  std::vector<Triangle> tris_;
  std::vector<TrianglePrim> prims_;
};

struct Scene {
  ArrayModel* model;
  std::list<IModel*> models;
  AccelerationStructure* accel;
  int kind;
};

// Barycentrics of the winning triangle.  HitInfo carries neither alpha nor
// beta (HitInfo.h:14-28), so they are recomputed here with the operations and
// order of TrianglePrim::intersect (TrianglePrim.cpp:210-220) using the
// reference's own Vector3/Cross/Dot.
void barycentrics(const float* c, const float* o, const float* d, float* alpha, float* beta) {
  Point3 v0(c[0], c[1], c[2]), v1(c[3], c[4], c[5]), v2(c[6], c[7], c[8]);
  Vector3 dir(d[0], d[1], d[2]);
  Point3 org(o[0], o[1], o[2]);
  const Vector3 edge1(v0, v1);
  const Vector3 edge2(v0, v2);
  Vector3 pvec = Cross(dir, edge2);
  float invdet = 1.0f / Dot(edge1, pvec);
  Vector3 svec(v0, org);
  Vector3 qvec = Cross(svec, edge1);
  *alpha = Dot(svec, pvec) * invdet;
  *beta = Dot(dir, qvec) * invdet;
}

template <class F>
void parallel_for(long n, int nthreads, F f) {
  if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
  if (nthreads < 1) nthreads = 1;
  if (n < 1024 || nthreads == 1) {
    f(0L, n);
    return;
  }
  std::vector<std::thread> th;
  long chunk = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    long b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.push_back(std::thread(f, b, e));
  }
  for (size_t i = 0; i < th.size(); ++i) th[i].join();
}

double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

}  // namespace

extern "C" {

// kind: 0 = Kdtree, 1 = Bvh, 2 = BasicAS (brute force).  Returns NULL on a
// bad kind or empty scene.  *build_seconds receives the build wall time.
void* encref_scene_create(const float* tri_verts, int ntris, int kind, double* build_seconds) {
  if (ntris <= 0 || kind < 0 || kind > 2) return 0;
  Scene* s = new Scene();
  s->model = new ArrayModel(tri_verts, ntris);
  s->model->coords_.assign(tri_verts, tri_verts + (size_t)9 * ntris);
  s->models.push_back(s->model);
  s->kind = kind;
  if (kind == 0) s->accel = new Kdtree();
  else if (kind == 1) s->accel = new Bvh();
  else s->accel = new BasicAS();
  double t0 = now_s();
  s->accel->build(s->models);
  if (build_seconds) *build_seconds = now_s() - t0;
  return s;
}

void encref_scene_destroy(void* h) {
  Scene* s = (Scene*)h;
  if (!s) return;
  // Kdtree::~Kdtree -> deleteTree walks all m_MaxNode node slots and
  // delete[]s the primitive list of every slot that looks like a leaf
  // (Kdtree.cpp:62-66), but only m_NodeUsed slots were ever written
  // (Kdtree.cpp:157, 532); the rest hold heap garbage and the walk crashes.
  // The harness therefore leaks a Kdtree (and the model it points into).
  if (s->kind == 0) return;
  delete s->accel;
  delete s->model;
  delete s;
}

// Closest hit for n rays given as 6 floats each (origin, direction).
// Writes the hit triangle index (-1 = miss), t (as the float the predicate
// produced), and the barycentrics alpha/beta of the hit triangle.
void encref_closest(void* h, const float* rays, long n, int* tri_id, float* t, float* alpha,
                    float* beta, int nthreads) {
  Scene* s = (Scene*)h;
  parallel_for(n, nthreads, [&](long b, long e) {
    for (long i = b; i < e; ++i) {
      const float* r = rays + 6 * i;
      Ray ray(Point3(r[0], r[1], r[2]), Vector3(r[3], r[4], r[5]));
      HitInfo hit;
      bool ok = s->accel->intersect(ray, &hit);
      int id = ok ? s->model->index_of(hit.hitObject) : -1;
      tri_id[i] = id;
      t[i] = ok ? (float)hit.hitTime : 0.f;
      float a = 0.f, bb = 0.f;
      if (ok && id >= 0) barycentrics(s->model->tri_coords(id, 0), r, r + 3, &a, &bb);
      if (alpha) alpha[i] = a;
      if (beta) beta[i] = bb;
    }
  });
}

// Shadow query as PhotonMapperCPU::IsInShadow forms it: a full closest-hit
// intersect followed by hitTime < distance.  Rays are 7 floats each
// (origin, direction, distance); the caller has already applied the
// origin offset along the direction.
void encref_occluded(void* h, const float* rays, long n, unsigned char* occluded, int nthreads) {
  Scene* s = (Scene*)h;
  parallel_for(n, nthreads, [&](long b, long e) {
    for (long i = b; i < e; ++i) {
      const float* r = rays + 7 * i;
      Ray ray(Point3(r[0], r[1], r[2]), Vector3(r[3], r[4], r[5]));
      HitInfo hit;
      bool ok = s->accel->intersect(ray, &hit) && hit.hitTime < r[6];
      occluded[i] = ok ? 1 : 0;
    }
  });
}

// Photon map from plain arrays.  The photon's original index is kept in its
// incoming-direction x component, a field no search or estimate reads
// (PhotonMap.cpp:121-164 reads Direction() into an unused local only).
void* encref_pmap_create(const float* pos, const float* nrm, const float* power, long n,
                         int caustic, double* build_seconds) {
  PhotonMap* m = new PhotonMap((size_t)n);
  for (long i = 0; i < n; ++i) {
    Photon p(Point3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
             encore::Color(power[3 * i], power[3 * i + 1], power[3 * i + 2]),
             Vector3((float)i, 0.f, 0.f));
    p.SurfNormal(Vector3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]));
    m->AddPhoton(p);
  }
  m->SetCausticsMap(caustic != 0);
  double t0 = now_s();
  m->BalanceAndConstruct();
  if (build_seconds) *build_seconds = now_s() - t0;
  return m;
}

void encref_pmap_destroy(void* h) { delete (PhotonMap*)h; }

void encref_set_ignore_normal(int v) { IGNORE_NORMAL = (v != 0); }

// Radiance estimate per query point (position + surface normal).
void encref_pmap_radiance(void* h, const float* qpos, const float* qnrm, long nq, int k,
                          float max_dist, float* rgb, int nthreads) {
  PhotonMap* m = (PhotonMap*)h;
  parallel_for(nq, nthreads, [&](long b, long e) {
    for (long i = b; i < e; ++i) {
      encore::Color c = m->GetRadianceEstimate(
          k, max_dist, Point3(qpos[3 * i], qpos[3 * i + 1], qpos[3 * i + 2]),
          Vector3(qnrm[3 * i], qnrm[3 * i + 1], qnrm[3 * i + 2]));
      rgb[3 * i] = c.R();
      rgb[3 * i + 1] = c.G();
      rgb[3 * i + 2] = c.B();
    }
  });
}

// The k-nearest set per query: original photon indices and squared
// distances, in the heap order GetNearestNPhotons returns, padded with -1.
void encref_pmap_nearest(void* h, const float* qpos, const float* qnrm, long nq, int k,
                         float max_dist, int* idx, float* d2, int* count, int nthreads) {
  PhotonMap* m = (PhotonMap*)h;
  parallel_for(nq, nthreads, [&](long b, long e) {
    for (long i = b; i < e; ++i) {
      std::vector<PhotonDistPair> v = m->GetNearestNPhotons(
          k, max_dist, Point3(qpos[3 * i], qpos[3 * i + 1], qpos[3 * i + 2]),
          Vector3(qnrm[3 * i], qnrm[3 * i + 1], qnrm[3 * i + 2]));
      int c = (int)v.size();
      count[i] = c;
      for (int j = 0; j < k; ++j) {
        idx[(size_t)i * k + j] = j < c ? (int)v[j].m_pPhoton->Direction().X() : -1;
        d2[(size_t)i * k + j] = j < c ? v[j].m_Distance : 0.f;
      }
    }
  });
}

int encref_hardware_threads(void) { return (int)std::thread::hardware_concurrency(); }

// Model::Model(filename, center, size, angle, axis, material) -> Model::load
// (Model.cpp:34-107): the reference's loader and centring transform.  Writes
// up to `cap` triangles (9 floats each, primitive-list order, read back
// through TrianglePrim::getNewTesselation) and returns the primitive count.
long encref_model_load(const char* path, const float* center, float size, float angle,
                       const float* axis, float* out, long cap) {
  Model m(std::string(path), Point3(center[0], center[1], center[2]), size, angle,
          Vector3(axis[0], axis[1], axis[2]), Material());
  std::list<IPrimitive*>& pl = m.getPrimitiveList();
  long i = 0;
  for (std::list<IPrimitive*>::iterator p = pl.begin(); p != pl.end(); ++p, ++i) {
    if (i >= cap) continue;
    std::list<Triangle*>* ts = (*p)->getNewTesselation();
    Triangle* t = ts->front();
    const Vertex* v[3] = {t->getVertex0(), t->getVertex1(), t->getVertex2()};
    for (int k = 0; k < 3; ++k) {
      const Point3& c = v[k]->getCoordinates();
      out[9 * i + 3 * k + 0] = c.X();
      out[9 * i + 3 * k + 1] = c.Y();
      out[9 * i + 3 * k + 2] = c.Z();
    }
    for (std::list<Triangle*>::iterator q = ts->begin(); q != ts->end(); ++q) delete *q;
    delete ts;
  }
  return (long)pl.size();
}


// Eye rays of RayTracer::CalcEyeRaySamples (RayTracer.cpp:489-525) for one
// unjittered sample per pixel (m_BlockSize = 1, so x = col + 0.5), row-major
// from the bottom row.  The camera basis is the reference's own Camera (the
// three-argument constructor, which keeps `up`; Camera::set ignores its `up`
// argument, Camera.cpp:44) with SetViewVolume's view angle, aspect and near
// plane, and all vector arithmetic is the reference's Vector3.  The loop body
// is the expression of RayTracer.cpp:495-516 written out here, because
// RayTracer.cpp itself needs the renderer's GL classes.  out: 8 floats per ray
// (eye, 0, direction, +inf).
void encref_camera_rays(const float* eye, const float* look, const float* up, float fov_deg,
                        float aspect, float near_plane, int width, int height, float* out) {
  Camera cam(Point3(eye[0], eye[1], eye[2]), Point3(look[0], look[1], look[2]),
             Vector3(up[0], up[1], up[2]));
  cam.SetViewVolume(fov_deg, aspect, near_plane, 1000.0f);
  const int block = 1;
  float H = cam.GetNearClipPlane() * tan(cam.GetViewAngle() * (PI / 360.0));
  float W = H * cam.GetAspect();
  for (int row = 0; row < height; ++row) {
    for (int col = 0; col < width; ++col) {
      float x = col + (block / 2.0f);
      float y = row + (block / 2.0f);
      float Uc = -W + (W * (2 * x) / (float)width);
      float Vr = -H + (H * (2 * y) / (float)height);
      float N = cam.GetNearClipPlane();
      Vector3 n = cam.N() * -N;
      Vector3 u = cam.U() * Uc;
      Vector3 v = cam.V() * Vr;
      Vector3 direction = n + u + v;
      direction.Normalize();
      Point3 e = cam.GetEye();
      float* o = out + 8 * ((size_t)row * width + col);
      o[0] = e.X();
      o[1] = e.Y();
      o[2] = e.Z();
      o[3] = 0.0f;
      o[4] = direction.X();
      o[5] = direction.Y();
      o[6] = direction.Z();
      o[7] = INFINITY;
    }
  }
}

// The hit point and normal TrianglePrim::intersect stores for ray i against
// triangle ids[i] (TrianglePrim.cpp:236-239), computed by the reference's
// own intersect on that one triangle; NaN where ids[i] < 0 or the reference
// reports no hit.  rays: 8 floats each (origin, tmin, direction, tmax).
void encref_hit_surface(const float* tri_verts, const float* rays, const int* ids, long n,
                        float* pos, float* nrm) {
  const float qnan = NAN;
  for (long i = 0; i < n; ++i) {
    float* p = pos + 3 * i;
    float* q = nrm + 3 * i;
    p[0] = p[1] = p[2] = q[0] = q[1] = q[2] = qnan;
    if (ids[i] < 0) continue;
    const float* c = tri_verts + 9 * (size_t)ids[i];
    Vertex v0(c[0], c[1], c[2], 0.f, 0.f, 1.f), v1(c[3], c[4], c[5], 0.f, 0.f, 1.f),
        v2(c[6], c[7], c[8], 0.f, 0.f, 1.f);
    TrianglePrim prim(v0, v1, v2);
    const float* r = rays + 8 * i;
    Ray ray(Point3(r[0], r[1], r[2]), Vector3(r[4], r[5], r[6]));
    HitInfo hit;
    if (!prim.intersect(ray, &hit)) continue;
    p[0] = hit.hitPoint.X();
    p[1] = hit.hitPoint.Y();
    p[2] = hit.hitPoint.Z();
    q[0] = hit.hitNormal.X();
    q[1] = hit.hitNormal.Y();
    q[2] = hit.hitNormal.Z();
  }
}

}  // extern "C"
