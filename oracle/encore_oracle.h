/*
 * Test oracle: a CPU restatement, in plain C, of the reference's ray-query
 * path.  It is the checker for the engine's CUDA kernels and is used only by
 * tests/, __graft_entry__.smoke() and the CPU arm of bench.py.  The engine
 * never links or calls it.
 *
 * Parity pins: tests/test_oracle_pins.py checks every function here against
 * the reference itself (oracle/_ref/libencore_ref.so, compiled from the
 * reference's own sources) and against the committed golden vectors in
 * tests/golden/, which that library produced.
 *
 * Rays are 8 floats (ox, oy, oz, tmin, dx, dy, dz, tmax); a hit needs
 * tmin < t < tmax (the reference's rays: tmin = 0, tmax = +inf).
 * Hits are 4 words (int32 id, float t, float alpha, float beta), id -1 = miss.
 */
#ifndef ENCORE_ORACLE_H
#define ENCORE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct eo_hit {
  int32_t id;
  float t, alpha, beta;
} eo_hit;

/* TrianglePrim::intersect (TrianglePrim.cpp:204-248), FP32, clamp = apply
 * ClampfloatoZero to the Cross() results (Vector3.h:148-161). */
int eo_tri_test(const float* tri9, const float* ray8, int clamp, float* t, float* alpha,
                float* beta);
/* eo_tri_test for ray i against triangle ids[i] (ids[i] < 0: not tested). */
void eo_tri_test_batch(const float* tris, const float* rays, const int* ids, long n, int clamp,
                       uint8_t* acc, float* t, float* alpha, float* beta);

/* Brute-force closest hit over all triangles in ID order, strict-less
 * replacement (BasicAS::intersect, BasicAS.cpp:167-194). */
void eo_closest_brute(const float* tris, int ntris, const float* rays, long n, int clamp,
                      eo_hit* out, int nthreads);
/* Any hit with tmin < t < tmax (PhotonMapperCPU::IsInShadow's boolean). */
void eo_occluded_brute(const float* tris, int ntris, const float* rays, long n, int clamp,
                       uint8_t* out, int nthreads);
/* Geometric truth: Moller-Trumbore in FP64, no clamp; t, alpha, beta rounded
 * to float on output. */
void eo_closest_f64(const float* tris, int ntris, const float* rays, long n, eo_hit* out,
                    int nthreads);

/* Geometric test of ray i against triangle ids[i] (FP64, no clamp): hit[i] = 1
 * iff tmin < t < tmax; t[i] = FP64 distance.  Used to classify mismatches. */
void eo_pairs_f64(const float* tris, const float* rays, const int32_t* ids, long n, uint8_t* hit,
                  double* t);

/* The reference kd-tree (Kdtree.cpp:84-200, 299-680) and its walk
 * (Kdtree.cpp:682-784). */
void* eo_kd_build(const float* tris, int ntris, int* max_depth, long* nnodes, long* nitems);
void eo_kd_closest(void* kd, const float* rays, long n, int clamp, eo_hit* out, int nthreads);
void eo_kd_free(void* kd);
/* The same walk, reporting per ray whether it tested triangle ids[i] at all
 * (ids[i] < 0: never).  Used to explain a closer hit the walk passed over. */
void eo_kd_tested(void* kd, const float* rays, const int32_t* ids, long n, int clamp,
                  uint8_t* tested, int nthreads);
/* Inspection of the walk: the leaves whose cells contain a point (both sides
 * of a split within eps), whether a leaf lists a triangle, and the leaves one
 * ray's walk visits with their [tmin, tmax]. */
int eo_kd_leaves_at(void* kd, const float* p, float eps, int32_t* leaves, int max);
int eo_kd_leaf_has(void* kd, int32_t leaf, int32_t id);
int eo_kd_walk(void* kd, const float* ray8, int clamp, int32_t* leaves, float* tmins,
               float* tmaxs, int max);

/* Photon gather: the k nearest accepted photons within max_dist
 * (PhotonMap::GetNearestNPhotons, PhotonMap.cpp:76-94, 224-297: accept
 * iff FP32 dist^2 < max_dist^2 and the stored normal equals the query
 * normal unless ignore_normal) and the radiance estimate
 * (GetRadianceEstimate, PhotonMap.cpp:121-164) accumulated in FP64.
 * idx/d2 (k per query, ascending d2, -1 padded) and count may be NULL. */
void* eo_pmap_build(const float* pos, const float* nrm, const float* power, long n);
void eo_pmap_gather(void* pm, const float* qpos, const float* qnrm, long nq, int k,
                    float max_dist, int ignore_normal, int caustic, double* rgb, int32_t* idx,
                    float* d2, int32_t* count, int nthreads);
void eo_pmap_free(void* pm);

/* Photon tracing as the engine traces photons (enc_photons_trace_device /
 * _maps_device; PhotonMapperCPU.cpp:503-798 with the engine's seeded random
 * numbers), path by path, with the brute-force closest hit (clamp selects
 * the reference predicate).  split: bounce 0 -> s0 (direct), later -> s1
 * (indirect); else all -> s0.  shadow_offset > 0: shadow photons into s0.
 * fill: batches of opts->nphotons until s1 is full (at most 64).  Photons
 * past a store's capacity are dropped in path order.  Powers: 1/emitted, the
 * shadow photons' negative.  Returns 1 if a shadow ray left 32 surfaces. */
typedef struct eo_photon_opts {
  float light_center[3];
  float light_size;
  uint32_t nphotons;
  uint32_t max_bounces;
  float albedo;
  uint32_t seed;
  float emit_offset;
  float bounce_offset;
} eo_photon_opts;
typedef struct eo_photon_out {
  float* pos;
  float* nrm;
  float* pow;
  uint32_t* tag; /* may be NULL */
  uint32_t capacity;
} eo_photon_out;
int eo_photon_trace(const float* tris, int ntris, const eo_photon_opts* o, int clamp, int split,
                    float shadow_offset, int fill, eo_photon_out* s0, eo_photon_out* s1,
                    uint32_t* stored, uint32_t* emitted, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
