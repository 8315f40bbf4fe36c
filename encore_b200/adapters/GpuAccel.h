// GpuAccel: an ENCORE AccelerationStructure backed by the encore_b200 engine.
//
// A drop-in for the accelerators behind ENCORE's AccelerationStructure
// interface (ENCORE/src/accelerators/AccelerationStructure.h:33-67).  It is
// compiled inside ENCORE's source tree (it includes ENCORE's headers; C++98
// like them) and links libencore_b200.so through include/encore_b200.h.
//
//   build(models)   flattens the models' primitive lists in order, so the
//                   engine's triangle IDs are primitive-list positions (the
//                   ID the reference recovers from HitInfo::hitObject,
//                   Model.cpp:255-264), then enc_accel_build.
//   intersect(r, h) the reference's per-ray call as a batch of one; the
//                   winning primitive fills HitInfo itself (hit point,
//                   normal, isEntering as TrianglePrim::intersect forms them,
//                   TrianglePrim.cpp:224-243), with the engine's t.
//   update(models)  enc_accel_refit with the moved vertices.
//   intersectBatch / occludedBatch: the batched calls a renderer uses for a
//                   bucket of eye rays (RayTracer::Refine, RayTracer.cpp:226-274)
//                   or shadow rays (PhotonMapperCPU::IsInShadow,
//                   PhotonMapperCPU.cpp:1192-1207).
//
// Primitives that are not triangles are traced as the triangles of their
// IPrimitive::getNewTesselation() (a RectangleLight is its two triangles);
// a hit on one reports the primitive.
#ifndef ENCORE_B200_GPU_ACCEL_H
#define ENCORE_B200_GPU_ACCEL_H

#include <limits>
#include <list>
#include <vector>

#include "AccelerationStructure.h"
#include "HitInfo.h"
#include "IModel.h"
#include "Ray.h"
#include "Triangle.h"
#include "encore_b200.h"

class GpuAccel : public AccelerationStructure {
 public:
  // kind: ENC_ACCEL_WBVH (fast) or ENC_ACCEL_KDTREE (the reference kd-tree's
  // exact answers, clamp artefacts included).
  explicit GpuAccel(int kind = ENC_ACCEL_WBVH, int device = 0)
      : m_accel(NULL), m_kind(kind), m_device(device), m_status(ENC_OK) {}
  virtual ~GpuAccel() {
    if (m_accel) enc_accel_destroy(m_accel);
  }

  virtual void usage(void) {}
  virtual void configure(Options*) {}
  virtual void keyboard(unsigned char) {}
#ifdef WIN32
  virtual void buildGPU(std::list<IModel*>&, std::list<Triangle*>&, GPUAccelerationStructureData&) {}
  virtual void setGPUParameters(CShader&, GPUAccelerationStructureData&) {}
#endif

  virtual void build(std::list<IModel*>& models) {
    std::vector<float> v;
    flatten(models, &v, true);
    if (m_accel) {
      enc_accel_destroy(m_accel);
      m_accel = NULL;
    }
    enc_scene scene = NULL;
    m_status = enc_scene_create(v.empty() ? NULL : &v[0], (uint32_t)(v.size() / 9), &scene);
    if (m_status != ENC_OK) return;
    enc_build_opts o;
    o.kind = m_kind;
    o.width = 8;
    o.max_leaf_tris = 3;
    o.predicate = ENC_PRED_REFERENCE;
    m_status = enc_accel_build(scene, &o, m_device, &m_accel);
    enc_scene_destroy(scene);
  }

  virtual void update(std::list<IModel*>& models) {
    std::vector<float> v;
    flatten(models, &v, false);
    if (!m_accel || v.size() / 9 != m_prim_of_tri.size()) {
      build(models);  // a different primitive set: rebuild
      return;
    }
    m_status = enc_accel_refit(m_accel, &v[0], (uint32_t)(v.size() / 9));
  }

  virtual bool intersect(Ray& r, HitInfo* info) {
    float ray[8];
    pack(r, ray);
    enc_hit h;
    m_status = m_accel ? enc_intersect_closest(m_accel, ray, 1, &h, NULL, NULL) : ENC_ERR_INVALID_ARG;
    if (m_status != ENC_OK || h.tri < 0) return false;
    fill(r, h, info);
    return true;
  }

  // n rays of 8 floats (ox oy oz tmin dx dy dz tmax) -> n hits (tri = -1: miss;
  // tri is an engine triangle ID, primitive(tri) gives the IPrimitive*).
  enc_status intersectBatch(const float* rays8, size_t n, enc_hit* hits) {
    return enc_intersect_closest(m_accel, rays8, n, hits, NULL, NULL);
  }
  // n rays of 6 floats (ox oy oz dx dy dz: a Ray's origin and direction, no
  // distance bounds) -> n hits; 24 bytes per ray cross PCIe instead of 32.
  enc_status intersectBatchOD(const float* rays6, size_t n, enc_hit* hits) {
    return enc_intersect_closest_od(m_accel, rays6, n, hits, NULL, NULL);
  }
  enc_status occludedBatch(const float* rays8, size_t n, uint8_t* occluded) {
    return enc_intersect_any(m_accel, rays8, n, occluded, NULL, NULL);
  }

  IPrimitive* primitive(int32_t tri) const {
    return tri >= 0 && (size_t)tri < m_prim_of_tri.size() ? m_prims[m_prim_of_tri[tri]] : NULL;
  }
  enc_status status() const { return m_status; }
  enc_accel handle() const { return m_accel; }

  // A reference Ray as the engine's record: t in (0, inf).
  static void pack(Ray& r, float out[8]) {
    out[0] = r.Origin().X();
    out[1] = r.Origin().Y();
    out[2] = r.Origin().Z();
    out[3] = 0.f;
    out[4] = r.Direction().X();
    out[5] = r.Direction().Y();
    out[6] = r.Direction().Z();
    out[7] = std::numeric_limits<float>::infinity();
  }

  // HitInfo for an engine hit: the primitive's own intersect forms the hit
  // point, normal and isEntering (TrianglePrim::intersect); t is the engine's,
  // which for a triangle is the same float.
  void fill(Ray& r, const enc_hit& h, HitInfo* info) const {
    IPrimitive* p = primitive(h.tri);
    HitInfo tmp;
    if (p && p->intersect(r, &tmp)) {
      *info = tmp;
    } else {  // a tessellated non-triangle primitive the analytic test misses
      info->hitPoint = Point3(r.Origin().X() + h.t * r.Direction().X(),
                              r.Origin().Y() + h.t * r.Direction().Y(),
                              r.Origin().Z() + h.t * r.Direction().Z());
      info->bHasInfo = true;
    }
    info->hitTime = h.t;
    info->hitObject = p;
  }

 private:
  void flatten(std::list<IModel*>& models, std::vector<float>* v, bool record) {
    if (record) {
      m_prims.clear();
      m_prim_of_tri.clear();
    }
    for (std::list<IModel*>::iterator m = models.begin(); m != models.end(); ++m) {
      std::list<IPrimitive*>& pl = (*m)->getPrimitiveList();
      for (std::list<IPrimitive*>::iterator p = pl.begin(); p != pl.end(); ++p) {
        std::list<Triangle*>* ts = (*p)->getNewTesselation();
        for (std::list<Triangle*>::iterator t = ts->begin(); t != ts->end(); ++t) {
          const Vertex* vs[3] = {(*t)->getVertex0(), (*t)->getVertex1(), (*t)->getVertex2()};
          for (int k = 0; k < 3; ++k) {
            v->push_back(vs[k]->getCoordinates().X());
            v->push_back(vs[k]->getCoordinates().Y());
            v->push_back(vs[k]->getCoordinates().Z());
          }
          if (record) m_prim_of_tri.push_back((int32_t)m_prims.size());
          delete *t;
        }
        delete ts;
        if (record) m_prims.push_back(*p);
      }
    }
  }

  enc_accel m_accel;
  int m_kind, m_device;
  enc_status m_status;
  std::vector<IPrimitive*> m_prims;      // primitive-list order
  std::vector<int32_t> m_prim_of_tri;    // engine triangle ID -> primitive index
};

#endif  // ENCORE_B200_GPU_ACCEL_H
