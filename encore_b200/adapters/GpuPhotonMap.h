// GpuPhotonMap: ENCORE's PhotonMap interface backed by the encore_b200 engine.
//
// The public methods of PhotonMap (ENCORE/src/renderers/PhotonMap.h:28-105)
// with the same names and meaning; PhotonMapperCPU's three maps
// (PhotonMapperCPU.cpp:516-528) can each be one.  Compiled inside ENCORE's
// source tree (C++98, ENCORE's headers), linked against libencore_b200.so.
//
//   AddPhoton               stores a copy, up to the maximum (PhotonMap.cpp:46-53)
//   BalanceAndConstruct     builds the device photon tree (enc_photonmap_create)
//   GetNearestNPhotons      the k nearest accepted photons as PhotonDistPair
//                           pointers into this map's copies, heapified with
//                           PhotonDistPair's operator< as the reference
//                           returns them (front = farthest, PhotonMap.cpp:90)
//   GetRadianceEstimate     enc_photonmap_radiance for one point
//   GetRadianceEstimates    the batched form for a bucket of gather points
//
// The normal test follows the flag given to SetIgnoreNormal (the reference
// reads its global IGNORE_NORMAL, PhotonMap.cpp:23, 244).
#ifndef ENCORE_B200_GPU_PHOTON_MAP_H
#define ENCORE_B200_GPU_PHOTON_MAP_H

#include <algorithm>
#include <vector>

#include "Color.h"
#include "Photon.h"
#include "encore_b200.h"

class GpuPhotonMap {
 public:
  explicit GpuPhotonMap(size_t maxPhotonCount, int device = 0)
      : m_CausticsMap(false), m_max(maxPhotonCount), m_device(device), m_map(NULL),
        m_balanced(false), m_ignore_normal(false), m_status(ENC_OK) {}
  virtual ~GpuPhotonMap() {
    if (m_map) enc_photonmap_destroy(m_map);
  }

  void AddPhoton(Photon& p) {
    if (m_photons.size() >= m_max) return;
    m_photons.push_back(p);
    m_balanced = false;
  }

  void BalanceAndConstruct() {
    if (m_balanced) return;
    if (m_map) {
      enc_photonmap_destroy(m_map);
      m_map = NULL;
    }
    m_balanced = true;
    if (m_photons.empty()) return;
    const size_t n = m_photons.size();
    std::vector<float> pos(3 * n), nrm(3 * n), pw(3 * n);
    for (size_t i = 0; i < n; ++i) {
      const Photon& p = m_photons[i];
      pos[3 * i] = p.Position().X();
      pos[3 * i + 1] = p.Position().Y();
      pos[3 * i + 2] = p.Position().Z();
      nrm[3 * i] = p.SurfNormal().X();
      nrm[3 * i + 1] = p.SurfNormal().Y();
      nrm[3 * i + 2] = p.SurfNormal().Z();
      pw[3 * i] = p.Power().R();
      pw[3 * i + 1] = p.Power().G();
      pw[3 * i + 2] = p.Power().B();
    }
    m_status = enc_photonmap_create(&pos[0], &nrm[0], &pw[0], n, m_CausticsMap ? 1 : 0, m_device,
                                    &m_map);
  }

  std::vector<PhotonDistPair> GetNearestNPhotons(const int N, const float maxDistance,
                                                 Point3 location, Vector3 normal) {
    std::vector<PhotonDistPair> out;
    if (N <= 0 || !ready()) return out;
    float q[3] = {location.X(), location.Y(), location.Z()};
    float qn[3] = {normal.X(), normal.Y(), normal.Z()};
    std::vector<int32_t> idx(N);
    std::vector<float> d2(N);
    int32_t count = 0;
    m_status = enc_photonmap_nearest(m_map, q, qn, 1, N, maxDistance, flags(), &idx[0], &d2[0],
                                     &count, NULL);
    if (m_status != ENC_OK) return out;
    for (int32_t j = 0; j < count; ++j) out.push_back(PhotonDistPair(&m_photons[idx[j]], d2[j]));
    std::make_heap(out.begin(), out.end());
    return out;
  }

  encore::Color GetRadianceEstimate(const int N, const float maxDistance, Point3 location,
                                    Vector3 normal) {
    float q[3] = {location.X(), location.Y(), location.Z()};
    float qn[3] = {normal.X(), normal.Y(), normal.Z()};
    float rgb[3] = {0.f, 0.f, 0.f};
    GetRadianceEstimates(N, maxDistance, q, qn, 1, rgb);
    return encore::Color(rgb[0], rgb[1], rgb[2]);
  }

  // nq points (3 floats each for position and normal) -> 3 floats each.
  enc_status GetRadianceEstimates(int N, float maxDistance, const float* q, const float* qn,
                                  size_t nq, float* rgb) {
    if (!ready()) {
      std::fill(rgb, rgb + 3 * nq, 0.f);
      return m_status;
    }
    m_status = enc_photonmap_radiance(m_map, q, qn, nq, N, maxDistance, flags(), rgb, NULL);
    return m_status;
  }

  void ScalePhotons(const float scaleFactor) {  // PhotonMap.cpp:97-104
    for (size_t i = 0; i < m_photons.size(); ++i) {
      encore::Color c = m_photons[i].Power();
      c.R() *= scaleFactor;
      c.G() *= scaleFactor;
      c.B() *= scaleFactor;
      m_photons[i].Power(c);
    }
    m_balanced = false;
  }

  bool Full() { return m_photons.size() == m_max; }
  int GetCountStored() { return (int)m_photons.size(); }
  size_t GetMaxPhotons() { return m_max; }
  void SetCausticsMap(bool isCausticsMap) {
    m_CausticsMap = isCausticsMap;
    m_balanced = false;
  }
  void SetIgnoreNormal(bool ignore) { m_ignore_normal = ignore; }
  enc_status status() const { return m_status; }

  bool m_CausticsMap;

 private:
  bool ready() {
    BalanceAndConstruct();
    return m_map != NULL && m_status == ENC_OK;
  }
  int32_t flags() const { return m_ignore_normal ? ENC_GATHER_IGNORE_NORMAL : 0; }

  std::vector<Photon> m_photons;
  size_t m_max;
  int m_device;
  enc_photonmap m_map;
  bool m_balanced, m_ignore_normal;
  enc_status m_status;
};

// PhotonMapperCPU::EmitPhotons (PhotonMapperCPU.cpp:503-586) on the device
// for a scene of diffuse surfaces: photons from the square light in `opts`
// traced by enc_photons_trace_maps, and stored where ReflectPhotonDiffusely
// and EmitShadowPhoton store them (PhotonMapperCPU.cpp:701-745, 776-798):
// first hits and shadow photons (shadowOffset > 0; the reference's offset
// is 2 at unit scale) into `direct`, later bounces into `indirect`.  With
// fillIndirect, batches of opts.nphotons are emitted until `indirect` is
// full, as EmitPhotons loops.  Each map takes at most its free capacity; the
// photons' power is 1 / photons emitted (the reference then rescales with
// ScalePhotons); their direction is the light's -y.  *emitted (may be NULL)
// receives the paths emitted.
inline enc_status GpuEmitPhotons(enc_accel accel, const enc_photon_opts& opts,
                                 float shadowOffset, bool fillIndirect, GpuPhotonMap& direct,
                                 GpuPhotonMap& indirect, uint32_t* emitted) {
  GpuPhotonMap* maps[2] = {&direct, &indirect};
  std::vector<float> buf[2];
  std::vector<uint32_t> tag[2];
  enc_photon_store st[2];
  for (int m = 0; m < 2; ++m) {
    const size_t cap = maps[m]->GetMaxPhotons() - (size_t)maps[m]->GetCountStored();
    buf[m].resize(9 * cap + 1);
    tag[m].resize(cap + 1);
    st[m].d_pos = &buf[m][0];
    st[m].d_nrm = &buf[m][0] + 3 * cap;
    st[m].d_pow = &buf[m][0] + 6 * cap;
    st[m].d_tag = &tag[m][0];
    st[m].capacity = (uint32_t)cap;
  }
  uint32_t stored[2] = {0, 0};
  const enc_status s = enc_photons_trace_maps(accel, &opts, shadowOffset, fillIndirect ? 1 : 0,
                                              &st[0], &st[1], stored, emitted, NULL);
  if (s != ENC_OK) return s;
  for (int m = 0; m < 2; ++m) {
    for (uint32_t i = 0; i < stored[m]; ++i) {
      const float* p = st[m].d_pos + 3 * i;
      const float* n = st[m].d_nrm + 3 * i;
      const float* w = st[m].d_pow + 3 * i;
      Photon ph(Point3(p[0], p[1], p[2]), encore::Color(w[0], w[1], w[2]), Vector3(0.f, -1.f, 0.f));
      ph.SurfNormal(Vector3(n[0], n[1], n[2]));
      ph.SetShadowPhoton((tag[m][i] & 8u) != 0);
      maps[m]->AddPhoton(ph);
    }
  }
  return ENC_OK;
}

#endif  // ENCORE_B200_GPU_PHOTON_MAP_H
