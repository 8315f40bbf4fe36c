/*
 * Test oracle: CPU restatement of the reference's ray-query path in plain C.
 * Test infrastructure only (see encore_oracle.h); compiled by oracle/Makefile
 * with -ffp-contract=off and no fast-math, so every FP32 expression below is
 * evaluated with the same roundings as the reference's g++ -O2 x86-64 build
 * (SSE scalar float, no FMA contraction).
 */
#define _GNU_SOURCE
#include "encore_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* threading                                                                 */

typedef void (*range_fn)(void* ctx, long b, long e);
typedef struct {
  range_fn fn;
  void* ctx;
  long b, e;
} range_job;

static void* range_thread(void* p) {
  range_job* j = (range_job*)p;
  j->fn(j->ctx, j->b, j->e);
  return NULL;
}

static void parallel_range(long n, int nthreads, range_fn fn, void* ctx) {
  if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (n < 256 || nthreads == 1) {
    fn(ctx, 0, n);
    return;
  }
  pthread_t th[256];
  range_job jobs[256];
  long chunk = (n + nthreads - 1) / nthreads;
  int started = 0;
  for (int t = 0; t < nthreads; ++t) {
    long b = t * chunk, e = b + chunk < n ? b + chunk : n;
    if (b >= e) break;
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
    jobs[t].b = b;
    jobs[t].e = e;
    if (pthread_create(&th[t], NULL, range_thread, &jobs[t]) != 0) {
      fn(ctx, b, e);
      jobs[t].fn = NULL;
    }
    started = t + 1;
  }
  for (int t = 0; t < started; ++t)
    if (jobs[t].fn) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------ */
/* a1: the triangle predicate                                                */

/* Vector3::ClampfloatoZero (Vector3.cpp:126-140): ENC_EPSILON is the double
 * 0.001 (Vector3.h:18-20), compared after promoting the float. */
static float clamp_eps(float x) { return (-0.001 < x && x < 0.001) ? 0.0f : x; }

/* Cross (Vector3.h:148-162). */
static void cross_ref(const float* a, const float* b, int clamp, float* out) {
  float x = a[1] * b[2] - a[2] * b[1];
  float y = -1 * (a[0] * b[2] - a[2] * b[0]);
  float z = a[0] * b[1] - a[1] * b[0];
  if (clamp) {
    x = clamp_eps(x);
    y = clamp_eps(y);
    z = clamp_eps(z);
  }
  out[0] = x;
  out[1] = y;
  out[2] = z;
}

/* Dot (Vector3.h:137-144). */
static float dot_ref(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* TrianglePrim::intersect (TrianglePrim.cpp:204-224). */
int eo_tri_test(const float* tri, const float* r, int clamp, float* t, float* alpha, float* beta) {
  const float v0[3] = {tri[0], tri[1], tri[2]};
  const float edge1[3] = {tri[3] - tri[0], tri[4] - tri[1], tri[5] - tri[2]};
  const float edge2[3] = {tri[6] - tri[0], tri[7] - tri[1], tri[8] - tri[2]};
  const float dir[3] = {r[4], r[5], r[6]};
  float pvec[3], qvec[3];
  cross_ref(dir, edge2, clamp, pvec);
  float invdet = 1.0f / dot_ref(edge1, pvec);
  const float svec[3] = {r[0] - v0[0], r[1] - v0[1], r[2] - v0[2]};
  cross_ref(svec, edge1, clamp, qvec);
  float a = dot_ref(svec, pvec) * invdet;
  float b = dot_ref(dir, qvec) * invdet;
  float time = dot_ref(edge2, qvec) * invdet;
  *t = time;
  *alpha = a;
  *beta = b;
  return (a >= 0.0) && (b >= 0.0) && (a + b <= 1) && (time > r[3]);
}

/* eo_tri_test for ray i against triangle ids[i] (ids[i] < 0: not tested). */
void eo_tri_test_batch(const float* tris, const float* rays, const int* ids, long n, int clamp,
                       uint8_t* acc, float* t, float* alpha, float* beta) {
  for (long i = 0; i < n; ++i) {
    acc[i] = 0;
    t[i] = alpha[i] = beta[i] = 0.f;
    if (ids[i] < 0) continue;
    acc[i] = (uint8_t)eo_tri_test(tris + 9 * (size_t)ids[i], rays + 8 * (size_t)i, clamp, t + i,
                                  alpha + i, beta + i);
  }
}

/* ------------------------------------------------------------------------ */
/* brute force                                                               */

typedef struct {
  const float* tris;
  int ntris;
  const float* rays;
  int clamp;
  eo_hit* out;
  uint8_t* occ;
} brute_ctx;

static void closest_brute_range(void* p, long b, long e) {
  brute_ctx* c = (brute_ctx*)p;
  for (long i = b; i < e; ++i) {
    const float* r = c->rays + 8 * i;
    eo_hit h = {-1, 0.f, 0.f, 0.f};
    float best = r[7];
    for (int k = 0; k < c->ntris; ++k) {
      float t, a, bb;
      if (eo_tri_test(c->tris + 9 * (size_t)k, r, c->clamp, &t, &a, &bb) && t < best) {
        best = t;
        h.id = k;
        h.t = t;
        h.alpha = a;
        h.beta = bb;
      }
    }
    c->out[i] = h;
  }
}

void eo_closest_brute(const float* tris, int ntris, const float* rays, long n, int clamp,
                      eo_hit* out, int nthreads) {
  brute_ctx c = {tris, ntris, rays, clamp, out, NULL};
  parallel_range(n, nthreads, closest_brute_range, &c);
}

static void occluded_brute_range(void* p, long b, long e) {
  brute_ctx* c = (brute_ctx*)p;
  for (long i = b; i < e; ++i) {
    const float* r = c->rays + 8 * i;
    uint8_t o = 0;
    for (int k = 0; k < c->ntris && !o; ++k) {
      float t, a, bb;
      if (eo_tri_test(c->tris + 9 * (size_t)k, r, c->clamp, &t, &a, &bb) && t < r[7]) o = 1;
    }
    c->occ[i] = o;
  }
}

void eo_occluded_brute(const float* tris, int ntris, const float* rays, long n, int clamp,
                       uint8_t* out, int nthreads) {
  brute_ctx c = {tris, ntris, rays, clamp, NULL, out};
  parallel_range(n, nthreads, occluded_brute_range, &c);
}

static void closest_f64_range(void* p, long b, long e) {
  brute_ctx* c = (brute_ctx*)p;
  for (long i = b; i < e; ++i) {
    const float* r = c->rays + 8 * i;
    const double o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
    double best = r[7];
    eo_hit h = {-1, 0.f, 0.f, 0.f};
    for (int k = 0; k < c->ntris; ++k) {
      const float* t = c->tris + 9 * (size_t)k;
      double e1[3], e2[3], s[3], p[3], q[3];
      for (int a = 0; a < 3; ++a) {
        e1[a] = (double)t[3 + a] - t[a];
        e2[a] = (double)t[6 + a] - t[a];
        s[a] = o[a] - t[a];
      }
      p[0] = d[1] * e2[2] - d[2] * e2[1];
      p[1] = d[2] * e2[0] - d[0] * e2[2];
      p[2] = d[0] * e2[1] - d[1] * e2[0];
      double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
      if (det == 0.0) continue;
      double inv = 1.0 / det;
      double u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
      if (u < 0.0 || u > 1.0) continue;
      q[0] = s[1] * e1[2] - s[2] * e1[1];
      q[1] = s[2] * e1[0] - s[0] * e1[2];
      q[2] = s[0] * e1[1] - s[1] * e1[0];
      double v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
      if (v < 0.0 || u + v > 1.0) continue;
      double tt = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
      if (tt > r[3] && tt < best) {
        best = tt;
        h.id = k;
        h.t = (float)tt;
        h.alpha = (float)u;
        h.beta = (float)v;
      }
    }
    c->out[i] = h;
  }
}

void eo_closest_f64(const float* tris, int ntris, const float* rays, long n, eo_hit* out,
                    int nthreads) {
  brute_ctx c = {tris, ntris, rays, 0, out, NULL};
  parallel_range(n, nthreads, closest_f64_range, &c);
}

static int tri_f64(const float* t, const float* r, double* tout) {
  const double o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
  double e1[3], e2[3], s[3], p[3], q[3];
  for (int a = 0; a < 3; ++a) {
    e1[a] = (double)t[3 + a] - t[a];
    e2[a] = (double)t[6 + a] - t[a];
    s[a] = o[a] - t[a];
  }
  p[0] = d[1] * e2[2] - d[2] * e2[1];
  p[1] = d[2] * e2[0] - d[0] * e2[2];
  p[2] = d[0] * e2[1] - d[1] * e2[0];
  double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
  if (det == 0.0) return 0;
  double inv = 1.0 / det;
  double u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
  q[0] = s[1] * e1[2] - s[2] * e1[1];
  q[1] = s[2] * e1[0] - s[0] * e1[2];
  q[2] = s[0] * e1[1] - s[1] * e1[0];
  double v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
  double tt = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
  *tout = tt;
  return u >= 0.0 && v >= 0.0 && u + v <= 1.0 && tt > r[3] && tt < r[7];
}

void eo_pairs_f64(const float* tris, const float* rays, const int32_t* ids, long n, uint8_t* hit,
                  double* t) {
  for (long i = 0; i < n; ++i) {
    t[i] = 0.0;
    hit[i] = ids[i] >= 0 ? (uint8_t)tri_f64(tris + 9 * (size_t)ids[i], rays + 8 * i, &t[i]) : 0;
  }
}

/* ------------------------------------------------------------------------ */
/* a5 / a6: the reference kd-tree                                            */

typedef struct {
  float pos[3], size[3]; /* AABB: min corner + size (AABB.h:65-66) */
} rbox;

typedef struct {
  uint32_t w0, w1;
} kdnode;

typedef struct {
  const float* tris;
  int ntris;
  rbox* tb;
  kdnode* nodes;
  long nn, ncap;
  uint32_t* items;
  long ni, icap;
  uint32_t max_items, max_depth;
  float root_lo[3], root_hi[3];
} kdtree;

static rbox box_corners(const float* mn, const float* mx) {
  rbox b;
  for (int a = 0; a < 3; ++a) {
    b.pos[a] = mn[a];
    b.size[a] = mx[a] - mn[a];
  }
  return b;
}

/* AABB::Intersect(AABB) (AABB.cpp:9-18). */
static int box_overlap(const rbox* self, const rbox* b2) {
  for (int a = 0; a < 3; ++a) {
    float v1 = b2->pos[a], v2 = b2->pos[a] + b2->size[a];
    float v3 = self->pos[a], v4 = self->pos[a] + self->size[a];
    if (!((v4 > v1) && (v3 < v2))) return 0;
  }
  return 1;
}

#define DMIN(a, b) (((a) > (b) ? (b) : (a))) /* TrianglePrim.h:29 */
#define DMAX(a, b) (((a) > (b) ? (a) : (b))) /* TrianglePrim.h:30 */

/* TrianglePrim::getAABB (TrianglePrim.cpp:184-202). */
static rbox tri_aabb(const float* t) {
  float mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = DMIN(DMIN(t[a], t[3 + a]), t[6 + a]);
    mx[a] = DMAX(DMAX(t[a], t[3 + a]), t[6 + a]);
  }
  return box_corners(mn, mx);
}

static long kd_alloc_pair(kdtree* kd) {
  if (kd->nn + 2 > kd->ncap) {
    kd->ncap = kd->ncap * 2 + 16;
    kd->nodes = (kdnode*)realloc(kd->nodes, kd->ncap * sizeof(kdnode));
  }
  long c = kd->nn;
  kd->nn += 2;
  return c;
}

/* Kdtree::construct (Kdtree.cpp:299-680), non-SAH branch. */
static void kd_construct(kdtree* kd, long fn, rbox box, uint32_t* list, uint32_t size,
                         uint32_t depth, uint32_t pre_size, int dsize, int tries) {
  if ((int)abs((int)(pre_size - size)) <= 3) {
    dsize = 1;
    tries++;
  } else {
    dsize = 0;
    tries = 0;
  }
  if (size <= kd->max_items || depth >= kd->max_depth || (dsize && tries == 3)) {
    if (kd->ni + size > kd->icap) {
      kd->icap = (kd->ni + size) * 2 + 16;
      kd->items = (uint32_t*)realloc(kd->items, kd->icap * sizeof(uint32_t));
    }
    memcpy(kd->items + kd->ni, list, size * sizeof(uint32_t));
    kd->nodes[fn].w0 = (size << 2) | 3u;
    kd->nodes[fn].w1 = (uint32_t)kd->ni;
    kd->ni += size;
    return;
  }
  int axis = (int)(depth % 3);
  float minp[3], maxp[3], rminp[3], lmaxp[3], bmax[3];
  for (int a = 0; a < 3; ++a) {
    minp[a] = box.pos[a];
    maxp[a] = minp[a] + box.size[a];
  }
  float splitpos = (minp[axis] + maxp[axis]) / 2;
  for (int a = 0; a < 3; ++a) {
    rminp[a] = box.pos[a];
    lmaxp[a] = box.pos[a] + box.size[a];
    bmax[a] = box.pos[a] + box.size[a];
  }
  rminp[axis] = splitpos;
  lmaxp[axis] = splitpos;
  rbox lvox = box_corners(box.pos, lmaxp);
  rbox rvox = box_corners(rminp, bmax);
  uint32_t* left = (uint32_t*)malloc((size ? size : 1) * sizeof(uint32_t));
  uint32_t* right = (uint32_t*)malloc((size ? size : 1) * sizeof(uint32_t));
  uint32_t a_n = 0, b_n = 0;
  for (uint32_t i = 0; i < size; ++i) {
    const rbox* tb = &kd->tb[list[i]];
    int hit = 0;
    if (box_overlap(&lvox, tb)) {
      left[a_n++] = list[i];
      hit = 1;
    }
    if (box_overlap(&rvox, tb)) {
      right[b_n++] = list[i];
      hit = 1;
    }
    if (!hit) {
      left[a_n++] = list[i];
      right[b_n++] = list[i];
    }
  }
  long child = kd_alloc_pair(kd);
  uint32_t bits;
  memcpy(&bits, &splitpos, 4);
  kd->nodes[fn].w0 = (bits & ~3u) | (uint32_t)axis; /* Kdtree.h:47-52 */
  kd->nodes[fn].w1 = (uint32_t)child;
  kd_construct(kd, child, lvox, left, a_n, depth + 1, size, dsize, tries);
  free(left);
  kd_construct(kd, child + 1, rvox, right, b_n, depth + 1, size, dsize, tries);
  free(right);
}

/* Kdtree::build (Kdtree.cpp:84-200) with the model bounds = vertex bounds. */
void* eo_kd_build(const float* tris, int ntris, int* max_depth, long* nnodes, long* nitems) {
  if (ntris <= 0) return NULL;
  kdtree* kd = (kdtree*)calloc(1, sizeof(kdtree));
  kd->tris = tris;
  kd->ntris = ntris;
  float mn[3], mx[3];
  for (int a = 0; a < 3; ++a) mn[a] = mx[a] = tris[a];
  for (long i = 0; i < 3L * ntris; ++i)
    for (int a = 0; a < 3; ++a) {
      float c = tris[3 * i + a];
      if (c < mn[a]) mn[a] = c;
      if (c > mx[a]) mx[a] = c;
    }
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = mn[a] - 0.001f;
    hi[a] = mx[a] + 0.001f;
  }
  rbox root = box_corners(lo, hi);
  for (int a = 0; a < 3; ++a) {
    kd->root_lo[a] = root.pos[a];
    kd->root_hi[a] = root.pos[a] + root.size[a];
  }
  kd->max_items = ntris <= 5000 ? 2u : 10u;
  kd->max_depth = 11u + (uint32_t)(1.3 * (double)logf((float)ntris));
  kd->tb = (rbox*)malloc((size_t)ntris * sizeof(rbox));
  for (int i = 0; i < ntris; ++i) kd->tb[i] = tri_aabb(tris + 9 * (size_t)i);
  kd->ncap = 1024;
  kd->nodes = (kdnode*)malloc(kd->ncap * sizeof(kdnode));
  kd->nn = 1;
  uint32_t* all = (uint32_t*)malloc((size_t)ntris * sizeof(uint32_t));
  for (int i = 0; i < ntris; ++i) all[i] = (uint32_t)i;
  kd_construct(kd, 0, root, all, (uint32_t)ntris, 0, 0, 0, 0);
  free(all);
  if (max_depth) *max_depth = (int)kd->max_depth;
  if (nnodes) *nnodes = kd->nn;
  if (nitems) *nitems = kd->ni;
  return kd;
}

void eo_kd_free(void* p) {
  kdtree* kd = (kdtree*)p;
  if (!kd) return;
  free(kd->tb);
  free(kd->nodes);
  free(kd->items);
  free(kd);
}

typedef struct {
  kdtree* kd;
  const float* rays;
  int clamp;
  eo_hit* out;
  const int32_t* probe; /* optional: per ray, a triangle ID to watch for */
  uint8_t* tested;      /* with probe: 1 if the walk tested that triangle */
} kd_ctx;

/* Kdtree::intersect (Kdtree.cpp:682-784). */
static void kd_closest_range(void* p, long b, long e) {
  kd_ctx* c = (kd_ctx*)p;
  const kdtree* kd = c->kd;
  enum { STACK = 128 };
  uint32_t sn[STACK];
  float smin[STACK], smax[STACK];
  for (long i = b; i < e; ++i) {
    const float* r = c->rays + 8 * i;
    const float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
    const float inv[3] = {1.f / d[0], 1.f / d[1], 1.f / d[2]};
    float best = INFINITY, ba = 0.f, bb = 0.f;
    int best_id = -1;
    const int32_t watch = c->probe ? c->probe[i] : -1;
    if (c->tested) c->tested[i] = 0;
    /* AABB::Intersect(Ray&, float&, float&) (AABB.cpp:117-143) */
    float t0 = 0, t1 = INFINITY;
    int in = 1;
    for (int a = 0; a < 3 && in; ++a) {
      float tin = (kd->root_lo[a] - o[a]) / d[a];
      float tout = (kd->root_hi[a] - o[a]) / d[a];
      if (tin > tout) {
        float tt = tin;
        tin = tout;
        tout = tt;
      }
      t0 = tin > t0 ? tin : t0;
      t1 = tout < t1 ? tout : t1;
      if (t0 > t1) in = 0;
    }
    if (in) {
      float tmin = t0, tmax = t1;
      int sp = 0;
      uint32_t node = 0;
      for (;;) {
        if (best < tmin) break;
        kdnode nd = kd->nodes[node];
        if ((nd.w0 & 3u) != 3u) {
          int axis = (int)(nd.w0 & 3u);
          float split;
          memcpy(&split, &nd.w0, 4);
          split = (split > -0.001 && split < 0.001) ? 0 : split; /* EPSILON, Common.h:31 */
          float tplane = (split - o[axis]) * inv[axis];
          int below = o[axis] <= split;
          uint32_t first = below ? nd.w1 : nd.w1 + 1;
          uint32_t second = below ? nd.w1 + 1 : nd.w1;
          if (tplane == 0) {
            node = inv[axis] > 0 ? second : first;
          } else if (tplane >= tmax || tplane < 0) {
            node = first;
          } else if (tplane <= tmin) {
            node = second;
          } else {
            if (sp < STACK) {
              sn[sp] = second;
              smin[sp] = tplane;
              smax[sp] = tmax;
              ++sp;
            }
            node = first;
            tmax = tplane;
          }
        } else {
          uint32_t cnt = nd.w0 >> 2;
          for (uint32_t k = 0; k < cnt; ++k) {
            uint32_t id = kd->items[nd.w1 + k];
            if (watch >= 0 && (int32_t)id == watch) c->tested[i] = 1;
            float t, a, bt;
            if (eo_tri_test(kd->tris + 9 * (size_t)id, r, c->clamp, &t, &a, &bt) && t < best) {
              best = t;
              best_id = (int)id;
              ba = a;
              bb = bt;
            }
          }
          if (sp > 0) {
            --sp;
            node = sn[sp];
            tmin = smin[sp];
            tmax = smax[sp];
          } else {
            break;
          }
        }
      }
    }
    eo_hit h = {-1, 0.f, 0.f, 0.f};
    if (best_id >= 0 && best < r[7]) {
      h.id = best_id;
      h.t = best;
      h.alpha = ba;
      h.beta = bb;
    }
    c->out[i] = h;
  }
}

void eo_kd_closest(void* kd, const float* rays, long n, int clamp, eo_hit* out, int nthreads) {
  kd_ctx c = {(kdtree*)kd, rays, clamp, out, NULL, NULL};
  parallel_range(n, nthreads, kd_closest_range, &c);
}

void eo_kd_tested(void* kd, const float* rays, const int32_t* ids, long n, int clamp,
                  uint8_t* tested, int nthreads) {
  eo_hit* out = (eo_hit*)malloc((size_t)(n > 0 ? n : 1) * sizeof(eo_hit));
  kd_ctx c = {(kdtree*)kd, rays, clamp, out, ids, tested};
  parallel_range(n, nthreads, kd_closest_range, &c);
  free(out);
}

/* ------------------------------------------------------------------------ */
/* a8-a10: photon gather                                                     */

typedef struct {
  long n;
  float* pos;  /* 3n, implicit-tree order */
  float* nrm;  /* 3n */
  float* pow;  /* 3n */
  int32_t* orig;
  uint8_t* axis;
} pmap;

static float* g_sort_key; /* for the quickselect below (single-threaded build) */

static void swap_idx(long* a, long i, long j) {
  long t = a[i];
  a[i] = a[j];
  a[j] = t;
}

/* nth_element on idx[lo..hi] by coordinate g_sort_key[3*idx+axis]. */
static void select_nth(long* idx, long lo, long hi, long nth, int axis) {
  while (hi > lo) {
    float pv = g_sort_key[3 * idx[(lo + hi) / 2] + axis];
    long i = lo, j = hi;
    while (i <= j) {
      while (g_sort_key[3 * idx[i] + axis] < pv) ++i;
      while (g_sort_key[3 * idx[j] + axis] > pv) --j;
      if (i <= j) {
        swap_idx(idx, i, j);
        ++i;
        --j;
      }
    }
    if (nth <= j) hi = j;
    else if (nth >= i) lo = i;
    else return;
  }
}

/* Implicit median-balanced tree as PhotonMap::BalanceAndConstruct lays it
 * out (node = (lo + hi) / 2 of its range, PhotonMap.cpp:176-221); the split
 * axis here is the range's largest extent. */
static void pm_balance(long* idx, uint8_t* axis_of, long lo, long hi) {
  if (hi - lo < 0) return;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long i = lo; i <= hi; ++i)
    for (int a = 0; a < 3; ++a) {
      float c = g_sort_key[3 * idx[i] + a];
      if (c < mn[a]) mn[a] = c;
      if (c > mx[a]) mx[a] = c;
    }
  int axis = 0;
  if (mx[1] - mn[1] > mx[axis] - mn[axis]) axis = 1;
  if (mx[2] - mn[2] > mx[axis] - mn[axis]) axis = 2;
  long m = (lo + hi) / 2;
  select_nth(idx, lo, hi, m, axis);
  axis_of[m] = (uint8_t)axis;
  pm_balance(idx, axis_of, lo, m - 1);
  pm_balance(idx, axis_of, m + 1, hi);
}

void* eo_pmap_build(const float* pos, const float* nrm, const float* power, long n) {
  pmap* pm = (pmap*)calloc(1, sizeof(pmap));
  pm->n = n;
  long* idx = (long*)malloc((n ? n : 1) * sizeof(long));
  for (long i = 0; i < n; ++i) idx[i] = i;
  pm->axis = (uint8_t*)calloc(n ? n : 1, 1);
  g_sort_key = (float*)pos;
  pm_balance(idx, pm->axis, 0, n - 1);
  pm->pos = (float*)malloc((n ? n : 1) * 3 * sizeof(float));
  pm->nrm = (float*)malloc((n ? n : 1) * 3 * sizeof(float));
  pm->pow = (float*)malloc((n ? n : 1) * 3 * sizeof(float));
  pm->orig = (int32_t*)malloc((n ? n : 1) * sizeof(int32_t));
  for (long i = 0; i < n; ++i) {
    memcpy(pm->pos + 3 * i, pos + 3 * idx[i], 12);
    memcpy(pm->nrm + 3 * i, nrm + 3 * idx[i], 12);
    memcpy(pm->pow + 3 * i, power + 3 * idx[i], 12);
    pm->orig[i] = (int32_t)idx[i];
  }
  free(idx);
  return pm;
}

void eo_pmap_free(void* p) {
  pmap* pm = (pmap*)p;
  if (!pm) return;
  free(pm->pos);
  free(pm->nrm);
  free(pm->pow);
  free(pm->orig);
  free(pm->axis);
  free(pm);
}

typedef struct {
  float* d2;
  long* node;
  int size, k;
} kheap;

static void heap_sift_down(kheap* h, int i) {
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < h->size && h->d2[l] > h->d2[m]) m = l;
    if (r < h->size && h->d2[r] > h->d2[m]) m = r;
    if (m == i) return;
    float td = h->d2[i];
    h->d2[i] = h->d2[m];
    h->d2[m] = td;
    long tn = h->node[i];
    h->node[i] = h->node[m];
    h->node[m] = tn;
    i = m;
  }
}

static void heap_push(kheap* h, float d2, long node) {
  int i = h->size++;
  h->d2[i] = d2;
  h->node[i] = node;
  while (i > 0) {
    int p = (i - 1) / 2;
    if (h->d2[p] >= h->d2[i]) break;
    float td = h->d2[i];
    h->d2[i] = h->d2[p];
    h->d2[p] = td;
    long tn = h->node[i];
    h->node[i] = h->node[p];
    h->node[p] = tn;
    i = p;
  }
}

/* PhotonMap::GetNearestNPhotons recursion (PhotonMap.cpp:224-297): the
 * search radius is the heap maximum once k photons are held. */
static void pm_search(const pmap* pm, const float* q, const float* qn, int ignore_normal,
                      float maxd2, kheap* h, long lo, long hi) {
  if (hi - lo < 0) return;
  long m = (lo + hi) / 2;
  const float* p = pm->pos + 3 * m;
  float x = q[0] - p[0], y = q[1] - p[1], z = q[2] - p[2];
  float d2 = (x * x) + (y * y) + (z * z);
  float r2 = h->size < h->k ? maxd2 : h->d2[0];
  const float* pn = pm->nrm + 3 * m;
  int nrm_ok = ignore_normal || (pn[0] == qn[0] && pn[1] == qn[1] && pn[2] == qn[2]);
  if (d2 < r2 && nrm_ok) {
    if (h->size < h->k) {
      heap_push(h, d2, m);
    } else {
      h->d2[0] = d2;
      h->node[0] = m;
      heap_sift_down(h, 0);
    }
  }
  int axis = pm->axis[m];
  float dp = q[axis] - p[axis];
  r2 = h->size < h->k ? maxd2 : h->d2[0];
  if (dp * dp > r2) {
    if (dp > 0) pm_search(pm, q, qn, ignore_normal, maxd2, h, m + 1, hi);
    else pm_search(pm, q, qn, ignore_normal, maxd2, h, lo, m - 1);
  } else {
    pm_search(pm, q, qn, ignore_normal, maxd2, h, lo, m - 1);
    r2 = h->size < h->k ? maxd2 : h->d2[0];
    pm_search(pm, q, qn, ignore_normal, maxd2, h, m + 1, hi);
  }
}

typedef struct {
  const pmap* pm;
  const float *qpos, *qnrm;
  int k;
  float max_dist;
  int ignore_normal, caustic;
  double* rgb;
  int32_t* idx;
  float* d2;
  int32_t* count;
} gather_ctx;

static void gather_range(void* p, long b, long e) {
  gather_ctx* c = (gather_ctx*)p;
  kheap h;
  h.k = c->k;
  h.d2 = (float*)malloc((c->k + 1) * sizeof(float));
  h.node = (long*)malloc((c->k + 1) * sizeof(long));
  const float maxd2 = c->max_dist * c->max_dist;
  for (long i = b; i < e; ++i) {
    h.size = 0;
    if (c->pm->n > 0 && c->k > 0)
      pm_search(c->pm, c->qpos + 3 * i, c->qnrm + 3 * i, c->ignore_normal, maxd2, &h, 0,
                c->pm->n - 1);
    /* sort ascending (insertion sort on a copy of the heap) */
    int n = h.size;
    for (int a = 1; a < n; ++a) {
      float kd = h.d2[a];
      long kn = h.node[a];
      int j = a - 1;
      while (j >= 0 && (h.d2[j] > kd || (h.d2[j] == kd && c->pm->orig[h.node[j]] > c->pm->orig[kn]))) {
        h.d2[j + 1] = h.d2[j];
        h.node[j + 1] = h.node[j];
        --j;
      }
      h.d2[j + 1] = kd;
      h.node[j + 1] = kn;
    }
    if (c->count) c->count[i] = n;
    if (c->idx)
      for (int j = 0; j < c->k; ++j) {
        c->idx[i * c->k + j] = j < n ? c->pm->orig[h.node[j]] : -1;
        c->d2[i * c->k + j] = j < n ? h.d2[j] : 0.f;
      }
    /* GetRadianceEstimate (PhotonMap.cpp:121-164) in FP64 */
    double R = 0, G = 0, B = 0;
    if (n > 0) {
      double r = h.d2[n - 1];
      for (int j = 0; j < n; ++j) {
        const float* pw = c->pm->pow + 3 * h.node[j];
        double radius = h.d2[j];
        double w = c->caustic ? (r - radius) / radius : 1.0;
        R += pw[0] * w;
        G += pw[1] * w;
        B += pw[2] * w;
      }
      double dens = c->caustic ? c->k / ((double)3.14159f * r * r) : 1.0;
      R *= dens;
      G *= dens;
      B *= dens;
    }
    if (c->rgb) {
      c->rgb[3 * i] = R;
      c->rgb[3 * i + 1] = G;
      c->rgb[3 * i + 2] = B;
    }
  }
  free(h.d2);
  free(h.node);
}

void eo_pmap_gather(void* pm, const float* qpos, const float* qnrm, long nq, int k,
                    float max_dist, int ignore_normal, int caustic, double* rgb, int32_t* idx,
                    float* d2, int32_t* count, int nthreads) {
  gather_ctx c = {(const pmap*)pm, qpos, qnrm, k, max_dist, ignore_normal, caustic,
                  rgb, idx, d2, count};
  parallel_range(nq, nthreads, gather_range, &c);
}

/* ------------------------------------------------------------------------ */
/* f1: photon tracing (the device tracer's algorithm, restated)              */
/*                                                                           */
/* The engine traces photons as PhotonMapperCPU::EmitPhotons / TracePhoton / */
/* ReflectPhotonDiffusely / EmitShadowPhoton do (PhotonMapperCPU.cpp:503-798) */
/* with its own seeded counter-based random numbers (the reference's rand()  */
/* is not reproducible, H12).  This is that algorithm written out path by    */
/* path in plain C, with the oracle's brute-force closest hit: given the    */
/* same closest hits it produces the same photons bit for bit.               */

static uint32_t ph_hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

static float ph_rnd(uint32_t seed, uint32_t path, uint32_t draw) {
  const uint32_t h = ph_hash32(seed ^ ph_hash32(path * 0x9E3779B9u ^ ph_hash32(draw + 0x632BE5ABu)));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

/* Vector3::Normalize (Vector3.cpp:105-124): divide by sqrt((x*x + y*y) + z*z),
 * then ClampfloatoZero each component. */
static void ph_normalize(float* v) {
  const float m = sqrtf((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
  for (int i = 0; i < 3; ++i) v[i] = clamp_eps(v[i] / m);
}

/* The cut cosine lobe about n: cos^2(theta) uniform on [lo, 1) from a point
 * on the unit disk drawn by rejection (16 tries, draws draw0 + 2j, + 1),
 * scaled by sqrt(1 - lo); frame t = normalize(a' x n), b = n x t. */
static void ph_lobe(const float* n_in, float lo, uint32_t seed, uint32_t path, uint32_t draw0,
                    float* d) {
  float n[3] = {n_in[0], n_in[1], n_in[2]};
  ph_normalize(n);
  const float R = sqrtf(1.0f - lo);
  float x = 0.f, y = 0.f, r2 = 0.f;
  for (int j = 0; j < 16; ++j) {
    const float a = 2.0f * ph_rnd(seed, path, draw0 + 2 * j) - 1.0f;
    const float b = 2.0f * ph_rnd(seed, path, draw0 + 2 * j + 1) - 1.0f;
    if (a * a + b * b <= 1.0f) {
      x = a * R;
      y = b * R;
      r2 = x * x + y * y;
      break;
    }
  }
  const float z = sqrtf(1.0f - r2);
  float t[3];
  if (fabsf(n[0]) > 0.9f) {
    t[0] = n[2];
    t[1] = 0.0f;
    t[2] = -n[0];
  } else {
    t[0] = 0.0f;
    t[1] = -n[2];
    t[2] = n[1];
  }
  const float tl = sqrtf((t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]);
  for (int i = 0; i < 3; ++i) t[i] = t[i] / tl;
  const float b[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2],
                      n[0] * t[1] - n[1] * t[0]};
  for (int i = 0; i < 3; ++i) d[i] = (x * t[i] + y * b[i]) + z * n[i];
  ph_normalize(d);
}

typedef struct {
  const float* tris;
  int ntris;
  int clamp;
} ph_scene;

/* Closest hit: the lowest t, then the lowest ID (BasicAS order). */
static int ph_closest(const ph_scene* S, const float* r, float* a, float* b) {
  int id = -1;
  float best = r[7];
  for (int k = 0; k < S->ntris; ++k) {
    float t, aa, bb;
    if (eo_tri_test(S->tris + 9 * (size_t)k, r, S->clamp, &t, &aa, &bb) && t < best) {
      best = t;
      id = k;
      *a = aa;
      *b = bb;
    }
  }
  return id;
}

/* TrianglePrim::intersect's hit point and stored normal. */
static void ph_surface(const float* tri, float a, float b, float* p, float* n) {
  const float e1[3] = {tri[3] - tri[0], tri[4] - tri[1], tri[5] - tri[2]};
  const float e2[3] = {tri[6] - tri[0], tri[7] - tri[1], tri[8] - tri[2]};
  for (int i = 0; i < 3; ++i) p[i] = (tri[i] + e1[i] * a) + e2[i] * b;
  cross_ref(e1, e2, 1, n);
  ph_normalize(n);
}

typedef struct {
  float pos[3], nrm[3], power;
  uint32_t tag;
  int store;
} ph_photon;

typedef struct {
  ph_scene S;
  eo_photon_opts o;
  uint32_t path0;
  int split;
  float shadow_offset;
  int max_per_path;
  ph_photon* out; /* max_per_path per path */
  int* count;     /* per path */
  long shadow_dropped;
} ph_ctx;

static void ph_ray(float* r, const float* o, const float* d) {
  r[0] = o[0];
  r[1] = o[1];
  r[2] = o[2];
  r[3] = 0.0f;
  r[4] = d[0];
  r[5] = d[1];
  r[6] = d[2];
  r[7] = INFINITY;
}

static void ph_trace_range(void* p, long b, long e) {
  ph_ctx* c = (ph_ctx*)p;
  const eo_photon_opts* o = &c->o;
  const uint32_t seed = o->seed ? o->seed : 1u;
  for (long i = b; i < e; ++i) {
    const uint32_t id = c->path0 + (uint32_t)i;
    ph_photon* out = c->out + (size_t)i * c->max_per_path;
    int k = 0;
    /* RectangleLight::EmitPhoton + TracePhoton's first ray */
    const float lp[3] = {o->light_center[0] + (ph_rnd(seed, id, 0) - 0.5f) * o->light_size,
                         o->light_center[1],
                         o->light_center[2] + (ph_rnd(seed, id, 1) - 0.5f) * o->light_size};
    const float down[3] = {0.f, -1.f, 0.f};
    float d[3];
    ph_lobe(down, 0.01f, seed, id, 2, d);
    float org[3] = {lp[0] + d[0] * o->emit_offset, lp[1] + d[1] * o->emit_offset,
                    lp[2] + d[2] * o->emit_offset};
    float r[8];
    ph_ray(r, org, d);
    for (uint32_t wave = 0; wave <= o->max_bounces; ++wave) {
      float a, bb;
      const int hid = ph_closest(&c->S, r, &a, &bb);
      if (hid < 0) break;
      const float* tri = c->S.tris + 9 * (size_t)hid;
      float hp[3], hn[3];
      ph_surface(tri, a, bb, hp, hn);
      ph_photon* ph = &out[k++];
      memcpy(ph->pos, hp, sizeof hp);
      memcpy(ph->nrm, hn, sizeof hn);
      ph->power = 1.0f;
      ph->tag = (id << 4) | (wave < 7 ? wave : 7u);
      ph->store = (c->split && wave > 0) ? 1 : 0;
      if (wave == 0 && c->shadow_offset > 0.0f) {
        /* EmitShadowPhoton: from hitPoint + dir * shadow_offset on */
        const float* sd = r + 4;
        float so[3] = {hp[0] + sd[0] * c->shadow_offset, hp[1] + sd[1] * c->shadow_offset,
                       hp[2] + sd[2] * c->shadow_offset};
        float sr[8];
        ph_ray(sr, so, sd);
        for (int step = 0; step < 32; ++step) {
          float sa, sb;
          const int sid = ph_closest(&c->S, sr, &sa, &sb);
          if (sid < 0) break;
          float sp[3], sn[3];
          ph_surface(c->S.tris + 9 * (size_t)sid, sa, sb, sp, sn);
          const float dn = (sd[0] * sn[0] + sd[1] * sn[1]) + sd[2] * sn[2];
          if (dn < 0.0f) {
            ph_photon* q = &out[k++];
            memcpy(q->pos, sp, sizeof sp);
            memcpy(q->nrm, sn, sizeof sn);
            q->power = -1.0f;
            q->tag = (id << 4) | 8u;
            q->store = 0;
            break;
          }
          if (step == 31) {
            __atomic_fetch_add(&c->shadow_dropped, 1, __ATOMIC_RELAXED);
            break;
          }
          so[0] = sp[0] + sd[0] * o->emit_offset;
          so[1] = sp[1] + sd[1] * o->emit_offset;
          so[2] = sp[2] + sd[2] * o->emit_offset;
          ph_ray(sr, so, sd);
        }
      }
      if (wave >= o->max_bounces) break;
      if (!(ph_rnd(seed, id, 64u + 64u * wave) < o->albedo)) break;
      float nd[3];
      ph_lobe(hn, 0.001f, seed, id, 65u + 64u * wave, nd);
      if (!(nd[0] == nd[0]) || !(nd[1] == nd[1]) || !(nd[2] == nd[2])) break;
      const float no[3] = {hp[0] + nd[0] * o->bounce_offset, hp[1] + nd[1] * o->bounce_offset,
                           hp[2] + nd[2] * o->bounce_offset};
      ph_ray(r, no, nd);
    }
    c->count[i] = k;
  }
}

int eo_photon_trace(const float* tris, int ntris, const eo_photon_opts* o, int clamp, int split,
                    float shadow_offset, int fill, eo_photon_out* s0, eo_photon_out* s1,
                    uint32_t* stored, uint32_t* emitted, int nthreads) {
  ph_ctx c;
  memset(&c, 0, sizeof c);
  c.S.tris = tris;
  c.S.ntris = ntris;
  c.S.clamp = clamp;
  c.o = *o;
  c.split = split;
  c.shadow_offset = shadow_offset;
  c.max_per_path = (int)o->max_bounces + 2;
  const long n = o->nphotons;
  uint64_t offered[2] = {0, 0};
  stored[0] = stored[1] = 0;
  uint32_t batches = 0;
  uint64_t total = 0;
  if (n == 0) {
    if (emitted) *emitted = 0;
    return 0;
  }
  c.out = (ph_photon*)malloc((size_t)n * c.max_per_path * sizeof(ph_photon));
  c.count = (int*)malloc((size_t)n * sizeof(int));
  eo_photon_out* st[2] = {s0, s1};
  for (;;) {
    c.path0 = (uint32_t)total;
    parallel_range(n, nthreads, ph_trace_range, &c);
    for (long i = 0; i < n; ++i) {
      for (int k = 0; k < c.count[i]; ++k) {
        const ph_photon* ph = &c.out[(size_t)i * c.max_per_path + k];
        const int m = ph->store;
        const uint64_t slot = offered[m]++;
        if (!st[m] || slot >= st[m]->capacity) continue;
        memcpy(st[m]->pos + 3 * slot, ph->pos, 3 * sizeof(float));
        memcpy(st[m]->nrm + 3 * slot, ph->nrm, 3 * sizeof(float));
        for (int q = 0; q < 3; ++q) st[m]->pow[3 * slot + q] = ph->power;
        if (st[m]->tag) st[m]->tag[slot] = ph->tag;
      }
    }
    total += (uint64_t)n;
    ++batches;
    if (!fill || !s1 || offered[1] >= s1->capacity || batches >= 64) break;
  }
  const float scale = (float)(1.0 / (double)total);
  for (int m = 0; m < 2; ++m) {
    if (!st[m]) continue;
    stored[m] = (uint32_t)(offered[m] < st[m]->capacity ? offered[m] : st[m]->capacity);
    for (uint64_t j = 0; j < 3ull * stored[m]; ++j) st[m]->pow[j] = st[m]->pow[j] * scale;
  }
  if (emitted) *emitted = (uint32_t)total;
  free(c.out);
  free(c.count);
  return c.shadow_dropped ? 1 : 0;
}

/* ------------------------------------------------------------------------ */
/* kd walk inspection (explains rays the reference walk passes over)         */

/* The leaves whose cells contain point p: descend by the node's split
 * (read as Kdtree::intersect reads it, snapped to 0 within 0.001), both
 * children where |p - split| <= eps.  Returns the number written (<= max). */
int eo_kd_leaves_at(void* p_kd, const float* p, float eps, int32_t* leaves, int max) {
  const kdtree* kd = (const kdtree*)p_kd;
  uint32_t stack[256];
  int sp = 0, n = 0;
  stack[sp++] = 0;
  while (sp > 0 && n < max) {
    const uint32_t node = stack[--sp];
    const kdnode nd = kd->nodes[node];
    if ((nd.w0 & 3u) == 3u) {
      leaves[n++] = (int32_t)node;
      continue;
    }
    const int axis = (int)(nd.w0 & 3u);
    float split;
    memcpy(&split, &nd.w0, 4);
    split = (split > -0.001 && split < 0.001) ? 0 : split;
    const float d = p[axis] - split;
    if (d <= eps && sp < 255) stack[sp++] = nd.w1;
    if (d >= -eps && sp < 255) stack[sp++] = nd.w1 + 1;
  }
  return n;
}

/* 1 if triangle id is in leaf `leaf`'s item list. */
int eo_kd_leaf_has(void* p_kd, int32_t leaf, int32_t id) {
  const kdtree* kd = (const kdtree*)p_kd;
  const kdnode nd = kd->nodes[leaf];
  if ((nd.w0 & 3u) != 3u) return 0;
  const uint32_t cnt = nd.w0 >> 2;
  for (uint32_t k = 0; k < cnt; ++k)
    if ((int32_t)kd->items[nd.w1 + k] == id) return 1;
  return 0;
}

/* The reference walk of one ray (kd_closest_range's steps): the leaves it
 * visits in order with their [tmin, tmax]; returns the count (<= max). */
int eo_kd_walk(void* p_kd, const float* r, int clamp, int32_t* leaves, float* tmins,
               float* tmaxs, int max) {
  const kdtree* kd = (const kdtree*)p_kd;
  const float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
  const float inv[3] = {1.f / d[0], 1.f / d[1], 1.f / d[2]};
  float best = INFINITY;
  float t0 = 0, t1 = INFINITY;
  for (int a = 0; a < 3; ++a) {
    float tin = (kd->root_lo[a] - o[a]) / d[a];
    float tout = (kd->root_hi[a] - o[a]) / d[a];
    if (tin > tout) {
      float tt = tin;
      tin = tout;
      tout = tt;
    }
    t0 = tin > t0 ? tin : t0;
    t1 = tout < t1 ? tout : t1;
    if (t0 > t1) return 0;
  }
  float tmin = t0, tmax = t1;
  uint32_t sn[128];
  float smin[128], smax[128];
  int sp = 0, n = 0;
  uint32_t node = 0;
  for (;;) {
    if (best < tmin) break;
    kdnode nd = kd->nodes[node];
    if ((nd.w0 & 3u) != 3u) {
      int axis = (int)(nd.w0 & 3u);
      float split;
      memcpy(&split, &nd.w0, 4);
      split = (split > -0.001 && split < 0.001) ? 0 : split;
      float tplane = (split - o[axis]) * inv[axis];
      int below = o[axis] <= split;
      uint32_t first = below ? nd.w1 : nd.w1 + 1;
      uint32_t second = below ? nd.w1 + 1 : nd.w1;
      if (tplane == 0) {
        node = inv[axis] > 0 ? second : first;
      } else if (tplane >= tmax || tplane < 0) {
        node = first;
      } else if (tplane <= tmin) {
        node = second;
      } else {
        if (sp < 128) {
          sn[sp] = second;
          smin[sp] = tplane;
          smax[sp] = tmax;
          ++sp;
        }
        node = first;
        tmax = tplane;
      }
    } else {
      if (n < max) {
        leaves[n] = (int32_t)node;
        tmins[n] = tmin;
        tmaxs[n] = tmax;
        ++n;
      }
      uint32_t cnt = nd.w0 >> 2;
      for (uint32_t k = 0; k < cnt; ++k) {
        uint32_t id = kd->items[nd.w1 + k];
        float t, a, bt;
        if (eo_tri_test(kd->tris + 9 * (size_t)id, r, clamp, &t, &a, &bt) && t < best) best = t;
      }
      if (sp > 0) {
        --sp;
        node = sn[sp];
        tmin = smin[sp];
        tmax = smax[sp];
      } else {
        break;
      }
    }
  }
  return n;
}
