// Ray and photon generation on the device, wavefront style: the callers'
// per-ray loops of the reference become kernels that write ray batches for
// the traversal kernels, and read their hits back.
//
//  * eye rays        RayTracer::CalcEyeRaySamples (RayTracer.cpp:489-525) with
//                    the basis of Camera::CalcCamVectors (Camera.cpp:157-166)
//  * hit surface     hit point and stored normal of TrianglePrim::intersect
//                    (TrianglePrim.cpp:236-239)
//  * diffuse rays    cosine-weighted secondaries from hits
//  * photon tracing  PhotonMapperCPU::EmitPhotons / TracePhoton /
//                    ReflectPhotonDiffusely (PhotonMapperCPU.cpp:503-745) with
//                    RectangleLight::EmitPhoton (RectangleLight.cpp:172-185)
//                    and the cosine lobes of randDirectionN/SuperN
//                    (Common.cpp:95-182): waves of emission or bounce rays are
//                    traced by the closest-hit kernel, then one kernel stores
//                    a photon at every hit and spawns the survivors of the
//                    Russian roulette into the next wave.
//
// Random numbers come from a counter-based hash of (seed, path, draw), so a
// photon path or a secondary ray is the same whatever the launch shape.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "engine.h"

namespace enc {
namespace {

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float clamp_eps(float x) { return (x > -0.001f && x < 0.001f) ? 0.0f : x; }

// Normalize() (Vector3.cpp:105-124): x / sqrt((x*x + y*y) + z*z), clamped.
__device__ __forceinline__ float3 normalize_ref(float3 v) {
  const float m = __fsqrt_rn(fa(fa(fm(v.x, v.x), fm(v.y, v.y)), fm(v.z, v.z)));
  return make_float3(clamp_eps(__fdiv_rn(v.x, m)), clamp_eps(__fdiv_rn(v.y, m)),
                     clamp_eps(__fdiv_rn(v.z, m)));
}

// Cross() with ClampfloatoZero (Vector3.h:148-161).
__device__ __forceinline__ float3 cross_ref(float3 a, float3 b) {
  return make_float3(clamp_eps(fs(fm(a.y, b.z), fm(a.z, b.y))),
                     clamp_eps(-fs(fm(a.x, b.z), fm(a.z, b.x))),
                     clamp_eps(fs(fm(a.x, b.y), fm(a.y, b.x))));
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Uniform [0, 1) from (seed, path, draw).
__device__ __forceinline__ float rnd(uint32_t seed, uint32_t path, uint32_t draw) {
  const uint32_t h = hash32(seed ^ hash32(path * 0x9E3779B9u ^ hash32(draw + 0x632BE5ABu)));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// Cosine lobe about n with the grazing tip cut as randDirectionN/SuperN cut
// it (Common.cpp:96, 146): cos^2(theta) uniform on [lo, 1), azimuth uniform.
// Drawn without trigonometry so that a plain C restatement reproduces it bit
// for bit (every step is a correctly rounded FP32 operation): a point (a, b)
// uniform on the unit disk by rejection from the square (at most kLobeTries
// tries, draws `draw0 + 2j` and `draw0 + 2j + 1`), scaled by R = sqrt(1 - lo),
// is the projection of a cosine-distributed direction: r^2 = R^2 (a^2 + b^2)
// is uniform on [0, 1 - lo], so cos^2(theta) = 1 - r^2 is uniform on [lo, 1).
// The frame is t = normalize(a' x n), b = n x t with a' = +y when |n.x| > 0.9,
// else +x; the result is normalised with the reference's Normalize, as
// randDirectionN/SuperN end with dir.Normalize().  n: the reference
// normalises it first (n.Normalize()); a zero or NaN normal gives NaN.
constexpr int kLobeTries = 16;
__device__ __forceinline__ float3 lobe_dir(float3 n, float lo, uint32_t seed, uint32_t path,
                                           uint32_t draw0) {
  n = normalize_ref(n);
  const float R = __fsqrt_rn(fs(1.0f, lo));
  float x = 0.f, y = 0.f, r2 = 0.f;
  for (int j = 0; j < kLobeTries; ++j) {
    const float a = fs(fm(2.0f, rnd(seed, path, draw0 + 2 * j)), 1.0f);
    const float b = fs(fm(2.0f, rnd(seed, path, draw0 + 2 * j + 1)), 1.0f);
    if (fa(fm(a, a), fm(b, b)) <= 1.0f) {
      x = fm(a, R);
      y = fm(b, R);
      r2 = fa(fm(x, x), fm(y, y));
      break;
    }
  }
  const float z = __fsqrt_rn(fs(1.0f, r2));
  const bool ax = fabsf(n.x) > 0.9f;
  // t = a' x n for a' = (0, 1, 0) or (1, 0, 0)
  float3 t = ax ? make_float3(n.z, 0.0f, -n.x) : make_float3(0.0f, -n.z, n.y);
  const float tl = __fsqrt_rn(fa(fa(fm(t.x, t.x), fm(t.y, t.y)), fm(t.z, t.z)));
  t = make_float3(__fdiv_rn(t.x, tl), __fdiv_rn(t.y, tl), __fdiv_rn(t.z, tl));
  const float3 b = make_float3(fs(fm(n.y, t.z), fm(n.z, t.y)), fs(fm(n.z, t.x), fm(n.x, t.z)),
                               fs(fm(n.x, t.y), fm(n.y, t.x)));
  const float3 d = make_float3(fa(fa(fm(x, t.x), fm(y, b.x)), fm(z, n.x)),
                               fa(fa(fm(x, t.y), fm(y, b.y)), fm(z, n.y)),
                               fa(fa(fm(x, t.z), fm(y, b.z)), fm(z, n.z)));
  return normalize_ref(d);
}

struct TriView {
  const float4* tris;
  const uint32_t* pos;  // id -> slot, or null for ID order
  uint32_t ntris;
};

// Hit point v0 + (v1 - v0) * alpha + (v2 - v0) * beta and the stored normal
// Normalize(Cross(edge1, edge2)) of TrianglePrim::intersect.
__device__ __forceinline__ bool hit_surface(const TriView& tv, const int4 h, float3& p, float3& n,
                                            float3& e1, float3& e2) {
  if (h.x < 0 || (uint32_t)h.x >= tv.ntris) return false;
  const uint32_t slot = tv.pos ? __ldg(tv.pos + h.x) : (uint32_t)h.x;
  if (slot >= tv.ntris) return false;
  const float4 a = __ldg(tv.tris + 3 * (size_t)slot), b = __ldg(tv.tris + 3 * (size_t)slot + 1),
               c = __ldg(tv.tris + 3 * (size_t)slot + 2);
  const float u = __int_as_float(h.z), v = __int_as_float(h.w);
  e1 = make_float3(a.w, b.x, b.y);
  e2 = make_float3(b.z, b.w, c.x);
  p = make_float3(fa(fa(a.x, fm(e1.x, u)), fm(e2.x, v)), fa(fa(a.y, fm(e1.y, u)), fm(e2.y, v)),
                  fa(fa(a.z, fm(e1.z, u)), fm(e2.z, v)));
  n = normalize_ref(cross_ref(e1, e2));
  return true;
}

// Unit geometric normal (not clamped) on the side the ray came from.
__device__ __forceinline__ float3 facing_normal(float3 e1, float3 e2, float3 d) {
  float3 g = make_float3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
  float l = rsqrtf(fmaxf(g.x * g.x + g.y * g.y + g.z * g.z, 1e-37f));
  if (g.x * d.x + g.y * d.y + g.z * d.z > 0.f) l = -l;
  return make_float3(g.x * l, g.y * l, g.z * l);
}

__device__ __forceinline__ void put_ray(float* out, size_t i, float3 o, float tmin, float3 d, float tmax) {
  float4* r = reinterpret_cast<float4*>(out) + 2 * i;
  r[0] = make_float4(o.x, o.y, o.z, tmin);
  r[1] = make_float4(d.x, d.y, d.z, tmax);
}

struct CamParams {
  float3 eye, u, v, dn;
  float W, H;
  uint32_t width, height, seed;
};

// Uc = -W + (W * (2 x)) / width and Vr = -H + (H * (2 y)) / height
// (RayTracer.cpp:505-506); direction = Normalize((-N near + U Uc) + V Vr).
__global__ void camera_kernel(CamParams c, float* out) {
  const size_t n = (size_t)c.width * c.height;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t row = (uint32_t)(i / c.width), col = (uint32_t)(i % c.width);
    float x, y;
    if (c.seed == 0) {
      x = fa((float)col, 0.5f);
      y = fa((float)row, 0.5f);
    } else {
      x = fa((float)col, rnd(c.seed, (uint32_t)i, 0));
      y = fa((float)row, rnd(c.seed, (uint32_t)i, 1));
    }
    const float uc = fa(-c.W, __fdiv_rn(fm(c.W, fm(2.0f, x)), (float)c.width));
    const float vr = fa(-c.H, __fdiv_rn(fm(c.H, fm(2.0f, y)), (float)c.height));
    const float3 d = make_float3(fa(fa(c.dn.x, fm(c.u.x, uc)), fm(c.v.x, vr)),
                                 fa(fa(c.dn.y, fm(c.u.y, uc)), fm(c.v.y, vr)),
                                 fa(fa(c.dn.z, fm(c.u.z, uc)), fm(c.v.z, vr)));
    put_ray(out, i, c.eye, 0.f, normalize_ref(d), INFINITY);
  }
}

__global__ void surface_kernel(TriView tv, const int4* hits, size_t n, float* pos, float* nrm) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float3 p, nn, e1, e2;
    if (!hit_surface(tv, hits[i], p, nn, e1, e2)) {
      p = nn = make_float3(NAN, NAN, NAN);
    }
    pos[3 * i] = p.x;
    pos[3 * i + 1] = p.y;
    pos[3 * i + 2] = p.z;
    nrm[3 * i] = nn.x;
    nrm[3 * i + 1] = nn.y;
    nrm[3 * i + 2] = nn.z;
  }
}

__global__ void diffuse_kernel(TriView tv, const float4* rays, const int4* hits, size_t n,
                               uint32_t per_hit, uint32_t seed, float offset, float* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float3 p, nn, e1, e2;
    const bool hit = hit_surface(tv, hits[i], p, nn, e1, e2);
    const float4 r1 = rays[2 * i + 1];
    const float3 f = hit ? facing_normal(e1, e2, make_float3(r1.x, r1.y, r1.z)) : make_float3(0, 0, 1);
    for (uint32_t k = 0; k < per_hit; ++k) {
      const size_t o = i * per_hit + k;
      if (!hit) {
        put_ray(out, o, make_float3(0, 0, 0), 0.f, make_float3(0, 0, 1), 0.f);  // empty ray
        continue;
      }
      // randDirectionSuperN's lobe: cos^2(theta) uniform on [0.001, 1)
      // (Common.cpp:146, 149)
      const float3 d = lobe_dir(f, 0.001f, seed, (uint32_t)o, 0);
      put_ray(out, o, make_float3(p.x + offset * f.x, p.y + offset * f.y, p.z + offset * f.z), 0.f,
              d, INFINITY);
    }
  }
}

// Photon tracing.  Random draws of path `id` (counter-based, so a path is the
// same whatever the launch shape or batch): 0, 1 the point on the light;
// 2.. its emission lobe; at bounce w, 64 + 64 w the Russian roulette and
// 65 + 64 w.. the bounce lobe.
constexpr uint32_t kDrawEmitLobe = 2;
__device__ __forceinline__ uint32_t draw_roulette(uint32_t w) { return 64u + 64u * w; }
__device__ __forceinline__ uint32_t draw_bounce(uint32_t w) { return 65u + 64u * w; }

struct PhotonParams {
  float3 lc;
  float lsize;
  uint32_t n;      // photons in this batch
  uint32_t path0;  // path id of the batch's first photon
  uint32_t seed, max_bounces;
  float albedo, emit_offset, bounce_offset, shadow_offset, skip_offset;
  int split;       // 1: bounce 0 -> store 0 (direct), later -> store 1 (indirect)
};

// A photon store: 3 floats per photon each, and an optional tag per photon
// (path id << 4 | shadow << 3 | min(bounce, 7)).
struct PhotonStore {
  float* pos;
  float* nrm;
  float* pw;
  uint32_t* tag;
  uint32_t cap;
};

// counters: [0], [1] photons offered to store 0 / 1; [2] next wave's rays;
// [3] next shadow wave's rays; [4] shadow rays dropped at the step limit.
__device__ __forceinline__ void store_photon(const PhotonStore& S, uint32_t* counter, float3 p,
                                             float3 n, float power, uint32_t tag) {
  const uint32_t slot = atomicAdd(counter, 1u);
  if (slot >= S.cap) return;  // a full map drops the photon (PhotonMap::AddPhoton)
  const size_t k = 3 * (size_t)slot;
  S.pos[k] = p.x;
  S.pos[k + 1] = p.y;
  S.pos[k + 2] = p.z;
  S.nrm[k] = n.x;
  S.nrm[k + 1] = n.y;
  S.nrm[k + 2] = n.z;
  S.pw[k] = power;
  S.pw[k + 1] = power;
  S.pw[k + 2] = power;
  if (S.tag) S.tag[slot] = tag;
}

// RectangleLight::EmitPhoton (RectangleLight.cpp:172-185): a point on the
// square light facing -y and a direction in its cut cosine lobe
// (randDirectionN, e1 >= 0.01); TracePhoton starts the path 0.01 (scaled:
// emit_offset) along it (PhotonMapperCPU.cpp:618).
__global__ void photon_emit_kernel(PhotonParams P, float* rays, uint32_t* path) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
    const uint32_t id = P.path0 + i;
    const float3 o = make_float3(fa(P.lc.x, fm(fs(rnd(P.seed, id, 0), 0.5f), P.lsize)), P.lc.y,
                                 fa(P.lc.z, fm(fs(rnd(P.seed, id, 1), 0.5f), P.lsize)));
    const float3 d = lobe_dir(make_float3(0.f, -1.f, 0.f), 0.01f, P.seed, id, kDrawEmitLobe);
    put_ray(rays, i,
            make_float3(fa(o.x, fm(d.x, P.emit_offset)), fa(o.y, fm(d.y, P.emit_offset)),
                        fa(o.z, fm(d.z, P.emit_offset))),
            0.f, d, INFINITY);
    path[i] = id;
  }
}

// One wave of TracePhoton (PhotonMapperCPU.cpp:614-674) with diffuse
// surfaces: every hit stores a photon (ReflectPhotonDiffusely, :701-745:
// bounce 0 into the direct map, later bounces into the indirect map); at
// bounce 0 a shadow photon ray continues through the surface
// (EmitShadowPhoton, :776-798); the path goes on with probability albedo
// (E < pD) and while bounces <= max_bounces, in randDirectionSuperN's lobe
// about the stored normal, 0.001 (scaled: bounce_offset) along it.
__global__ void photon_bounce_kernel(PhotonParams P, TriView tv, uint32_t wave, const float4* rays,
                                     const int4* hits, const uint32_t* path, uint32_t n,
                                     PhotonStore s0, PhotonStore s1, uint32_t* counters,
                                     float* next_rays, uint32_t* next_path, float* shadow_rays,
                                     uint32_t* shadow_path) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 p, nn, e1, e2;
    if (!hit_surface(tv, hits[i], p, nn, e1, e2)) continue;
    const uint32_t id = path[i];
    const uint32_t tag = (id << 4) | (wave < 7 ? wave : 7u);
    if (P.split && wave > 0) store_photon(s1, counters + 1, p, nn, 1.0f, tag);
    else store_photon(s0, counters + 0, p, nn, 1.0f, tag);
    if (wave == 0 && P.shadow_offset > 0.0f) {
      // shadowPhotonPath: from hitPoint + dir * 2 (scaled: shadow_offset) on
      const float4 r1 = rays[2 * (size_t)i + 1];
      const float3 d = make_float3(r1.x, r1.y, r1.z);
      const uint32_t k = atomicAdd(counters + 3, 1u);
      put_ray(shadow_rays, k,
              make_float3(fa(p.x, fm(d.x, P.shadow_offset)), fa(p.y, fm(d.y, P.shadow_offset)),
                          fa(p.z, fm(d.z, P.shadow_offset))),
              0.f, d, INFINITY);
      shadow_path[k] = id;
    }
    if (wave >= P.max_bounces) continue;
    if (!(rnd(P.seed, id, draw_roulette(wave)) < P.albedo)) continue;  // absorbed
    const float3 d = lobe_dir(nn, 0.001f, P.seed, id, draw_bounce(wave));
    if (!(d.x == d.x) || !(d.y == d.y) || !(d.z == d.z)) continue;  // zero normal: no direction
    const uint32_t k = atomicAdd(counters + 2, 1u);
    put_ray(next_rays, k,
            make_float3(fa(p.x, fm(d.x, P.bounce_offset)), fa(p.y, fm(d.y, P.bounce_offset)),
                        fa(p.z, fm(d.z, P.bounce_offset))),
            0.f, d, INFINITY);
    next_path[k] = id;
  }
}

// One step of EmitShadowPhoton's loop (PhotonMapperCPU.cpp:780-793): a hit
// on a surface the ray leaves (not isEntering: Dot(dir, hitNormal) >= 0)
// moves the origin 0.01 (scaled: skip_offset) past it and traces again; the
// first hit on a surface it enters stores a shadow photon there, with
// negative power and that surface's normal, in the direct map; a miss stores
// nothing.
__global__ void photon_shadow_kernel(PhotonParams P, TriView tv, const float4* rays,
                                     const int4* hits, const uint32_t* path, uint32_t n,
                                     PhotonStore s0, uint32_t* counters, float* next_rays,
                                     uint32_t* next_path, int last_step) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 p, nn, e1, e2;
    if (!hit_surface(tv, hits[i], p, nn, e1, e2)) continue;
    const float4 r1 = rays[2 * (size_t)i + 1];
    const float3 d = make_float3(r1.x, r1.y, r1.z);
    const float dn = fa(fa(fm(d.x, nn.x), fm(d.y, nn.y)), fm(d.z, nn.z));
    const uint32_t id = path[i];
    if (dn < 0.0f) {
      store_photon(s0, counters + 0, p, nn, -1.0f, (id << 4) | 8u);
      continue;
    }
    if (last_step) {
      atomicAdd(counters + 4, 1u);
      continue;
    }
    const uint32_t k = atomicAdd(counters + 3, 1u);
    put_ray(next_rays, k,
            make_float3(fa(p.x, fm(d.x, P.skip_offset)), fa(p.y, fm(d.y, P.skip_offset)),
                        fa(p.z, fm(d.z, P.skip_offset))),
            0.f, d, INFINITY);
    next_path[k] = id;
  }
}

// PhotonMap::ScalePhotons: every stored photon's power times `scale`
// (power 1 per photon at storage, so the light's total power 1 is split
// evenly over the photons emitted).
__global__ void photon_scale_kernel(PhotonStore S, uint32_t n, float scale) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x)
    S.pw[i] = fm(S.pw[i], scale);
}

int grid_for(size_t n, int block) {
  size_t g = (n + block - 1) / block;
  const size_t cap = (size_t)device_sm_count(0) * 32;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

TriView tri_view(const DevAccel& a) {
  return TriView{reinterpret_cast<const float4*>(a.d_tris), a.d_tri_pos, a.ntris};
}

// Host restatement of the camera basis in the reference's FP32 operations,
// identical to the Python generator's (scenes.camera_rays).
float clampf(float x) { return (-0.001 < x && x < 0.001) ? 0.0f : x; }
void crossf(const float* a, const float* b, float* o) {
  float x = a[1] * b[2] - a[2] * b[1];
  float y = -(a[0] * b[2] - a[2] * b[0]);
  float z = a[0] * b[1] - a[1] * b[0];
  o[0] = clampf(x);
  o[1] = clampf(y);
  o[2] = clampf(z);
}
void normf(float* v) {
  volatile float m2 = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
  float m = (float)std::sqrt((double)m2);
  for (int i = 0; i < 3; ++i) v[i] = clampf(v[i] / m);
}

}  // namespace
}  // namespace enc

using namespace enc;

extern "C" {

enc_status enc_camera_rays_device(const enc_camera* cam, float* d_rays, enc_stream stream) {
  if (!cam || !d_rays || cam->width == 0 || cam->height == 0) {
    set_error("enc_camera_rays_device: bad argument");
    return ENC_ERR_INVALID_ARG;
  }
  float n[3], u[3], v[3];
  for (int i = 0; i < 3; ++i) n[i] = cam->eye[i] - cam->look[i];
  crossf(cam->up, n, u);
  normf(n);
  normf(u);
  crossf(n, u, v);
  CamParams c;
  c.eye = make_float3(cam->eye[0], cam->eye[1], cam->eye[2]);
  c.u = make_float3(u[0], u[1], u[2]);
  c.v = make_float3(v[0], v[1], v[2]);
  const float near = 1.0f;
  c.dn = make_float3(n[0] * -near, n[1] * -near, n[2] * -near);
  c.H = (float)(1.0 * std::tan((double)cam->fov_deg * ((double)3.14159f / 360.0)));
  c.W = c.H * (float)((double)cam->width / (double)cam->height);
  c.width = cam->width;
  c.height = cam->height;
  c.seed = cam->jitter_seed;
  const size_t n_rays = (size_t)cam->width * cam->height;
  camera_kernel<<<grid_for(n_rays, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(c, d_rays);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("enc_camera_rays_device: ") + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  return ENC_OK;
}

enc_status enc_hit_surface_device(enc_accel accel, const enc_hit* d_hits, size_t n, float* d_pos,
                                  float* d_nrm, enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || (n && (!d_hits || !d_pos || !d_nrm))) return ENC_ERR_INVALID_ARG;
  if (n == 0) return ENC_OK;
  surface_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      tri_view(*a), reinterpret_cast<const int4*>(d_hits), n, d_pos, d_nrm);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("enc_hit_surface_device: ") + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  return ENC_OK;
}

enc_status enc_diffuse_rays_device(enc_accel accel, const float* d_rays, const enc_hit* d_hits,
                                   size_t n, uint32_t per_hit, uint32_t seed, float offset,
                                   float* d_out, enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || (n && (!d_rays || !d_hits || !d_out)) || per_hit == 0 || per_hit > 64)
    return ENC_ERR_INVALID_ARG;
  if (n == 0) return ENC_OK;
  diffuse_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      tri_view(*a), reinterpret_cast<const float4*>(d_rays), reinterpret_cast<const int4*>(d_hits), n,
      per_hit, seed, offset, d_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("enc_diffuse_rays_device: ") + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  return ENC_OK;
}

}  // extern "C"

namespace enc {
namespace {

// The photon tracer behind both entry points: batches of opts->nphotons
// emitted until `fill` says stop, each traced wave by wave (and its bounce-0
// shadow photons step by step), then every stored photon's power scaled by
// 1 / photons emitted.
constexpr uint32_t kMaxBatches = 64;
constexpr int kShadowSteps = 32;

enc_status trace_photons(enc_accel accel, const enc_photon_opts* o, int split, float shadow_offset,
                         int fill, PhotonStore s0, PhotonStore s1, uint32_t stored[2],
                         uint32_t* emitted_out, cudaStream_t s, const char* what) {
  const DevAccel* a = accel_device_view(accel);
  if (a->kind != ENC_ACCEL_WBVH) {
    set_error(std::string(what) + ": wide-BVH accelerators only");
    return ENC_ERR_UNSUPPORTED;
  }
  if (o->max_bounces > 30 || !(o->albedo >= 0.0f) || !(shadow_offset >= 0.0f)) {
    set_error(std::string(what) + ": max_bounces <= 30, albedo >= 0, shadow_offset >= 0");
    return ENC_ERR_INVALID_ARG;
  }
  const uint64_t max_paths = fill ? (uint64_t)o->nphotons * kMaxBatches : o->nphotons;
  if (max_paths >= (1ull << 28)) {
    set_error(std::string(what) + ": at most 2^28 photon paths (tags hold the path id in 28 bits)");
    return ENC_ERR_INVALID_ARG;
  }
  stored[0] = stored[1] = 0;
  if (emitted_out) *emitted_out = 0;
  if (o->nphotons == 0) return ENC_OK;
  PhotonParams P;
  P.lc = make_float3(o->light_center[0], o->light_center[1], o->light_center[2]);
  P.lsize = o->light_size;
  P.seed = o->seed ? o->seed : 1u;
  P.max_bounces = o->max_bounces;
  P.albedo = o->albedo;
  P.emit_offset = o->emit_offset;
  P.bounce_offset = o->bounce_offset;
  P.shadow_offset = shadow_offset;
  P.skip_offset = o->emit_offset;  // EmitShadowPhoton steps 0.01, TracePhoton's emission offset
  P.split = split;
  const size_t n = o->nphotons;
  WaveScratch& w = *accel_wave_scratch(accel);
  std::lock_guard<std::mutex> lk(w.mu);
  cudaError_t e = cudaSuccess;
  if (w.cap < n || (shadow_offset > 0.0f && !w.srays[0])) {
    // grow the kept scratch (no allocation once it is large enough)
    free_wave_scratch(&w);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
      e = cudaMalloc((void**)&w.rays[i], n * 32);
      if (e == cudaSuccess) e = cudaMalloc((void**)&w.path[i], n * 4);
      if (e == cudaSuccess) e = cudaMalloc((void**)&w.srays[i], n * 32);
      if (e == cudaSuccess) e = cudaMalloc((void**)&w.spath[i], n * 4);
    }
    if (e == cudaSuccess) e = cudaMalloc(&w.hits, n * 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&w.counters, 32);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&w.h_counts, 32);
    if (e != cudaSuccess) {
      free_wave_scratch(&w);
      set_error(std::string(what) + ": " + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? ENC_ERR_OUT_OF_MEMORY : ENC_ERR_CUDA;
    }
    w.cap = n;
  }
  int4* hits = static_cast<int4*>(w.hits);
  uint32_t* counters = w.counters;
  uint32_t* hc = w.h_counts;
  const TriView tv = tri_view(*a);
  Launch L = resolve_launch(nullptr, a->kind, a->width);
  e = cudaMemsetAsync(counters, 0, 32, s);
  uint64_t emitted = 0;
  uint32_t batches = 0;
  auto read_counts = [&]() {
    cudaError_t r = cudaMemcpyAsync(hc, counters, 20, cudaMemcpyDeviceToHost, s);
    if (r == cudaSuccess) r = cudaStreamSynchronize(s);
    return r;
  };
  while (e == cudaSuccess) {
    P.n = o->nphotons;
    P.path0 = (uint32_t)emitted;
    photon_emit_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, w.rays[0], w.path[0]);
    e = cudaGetLastError();
    uint32_t count = P.n;
    int cur = 0;
    for (uint32_t wave = 0; e == cudaSuccess && count > 0 && wave <= o->max_bounces; ++wave) {
      int le = launch_closest(*a, w.rays[cur], count, reinterpret_cast<enc_hit*>(hits), L, s,
                              nullptr);
      if (le) {
        e = (cudaError_t)le;
        break;
      }
      e = cudaMemsetAsync(counters + 2, 0, 8, s);
      if (e != cudaSuccess) break;
      photon_bounce_kernel<<<grid_for(count, 256), 256, 0, s>>>(
          P, tv, wave, reinterpret_cast<const float4*>(w.rays[cur]), hits, w.path[cur], count, s0,
          s1, counters, w.rays[cur ^ 1], w.path[cur ^ 1], w.srays[0], w.spath[0]);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = read_counts();
      if (e != cudaSuccess) break;
      count = hc[2];
      // the bounce-0 hits' shadow photons, step by step
      uint32_t scount = wave == 0 ? hc[3] : 0u;
      int sc = 0;
      for (int step = 0; e == cudaSuccess && scount > 0 && step < kShadowSteps; ++step) {
        int le2 = launch_closest(*a, w.srays[sc], scount, reinterpret_cast<enc_hit*>(hits), L, s,
                                 nullptr);
        if (le2) {
          e = (cudaError_t)le2;
          break;
        }
        e = cudaMemsetAsync(counters + 3, 0, 4, s);
        if (e != cudaSuccess) break;
        photon_shadow_kernel<<<grid_for(scount, 256), 256, 0, s>>>(
            P, tv, reinterpret_cast<const float4*>(w.srays[sc]), hits, w.spath[sc], scount, s0,
            counters, w.srays[sc ^ 1], w.spath[sc ^ 1], step == kShadowSteps - 1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = read_counts();
        scount = hc[3];
        sc ^= 1;
      }
      cur ^= 1;
    }
    emitted += P.n;
    ++batches;
    if (e != cudaSuccess) break;
    if (e == cudaSuccess) e = read_counts();
    if (e != cudaSuccess) break;
    if (!fill || hc[1] >= s1.cap || batches >= kMaxBatches) break;
  }
  if (e == cudaSuccess) e = read_counts();
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  stored[0] = hc[0] < s0.cap ? hc[0] : s0.cap;
  stored[1] = split ? (hc[1] < s1.cap ? hc[1] : s1.cap) : 0u;
  const float scale = (float)(1.0 / (double)emitted);
  if (stored[0]) photon_scale_kernel<<<grid_for(3 * (size_t)stored[0], 256), 256, 0, s>>>(s0, stored[0], scale);
  if (stored[1]) photon_scale_kernel<<<grid_for(3 * (size_t)stored[1], 256), 256, 0, s>>>(s1, stored[1], scale);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  if (emitted_out) *emitted_out = (uint32_t)emitted;
  if (hc[4] != 0) {
    set_error(std::string(what) + ": a shadow photon ray left more than 32 surfaces");
    return ENC_ERR_WATCHDOG;
  }
  return ENC_OK;
}

}  // namespace
}  // namespace enc

extern "C" {

enc_status enc_photons_trace_device(enc_accel accel, const enc_photon_opts* o, float* d_pos,
                                    float* d_nrm, float* d_pow, uint32_t capacity,
                                    uint32_t* stored, enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || !o || !stored || (capacity && (!d_pos || !d_nrm || !d_pow))) return ENC_ERR_INVALID_ARG;
  PhotonStore s0{d_pos, d_nrm, d_pow, nullptr, capacity};
  PhotonStore s1{nullptr, nullptr, nullptr, nullptr, 0};
  uint32_t st[2] = {0, 0};
  enc_status r = trace_photons(accel, o, 0, 0.0f, 0, s0, s1, st, nullptr,
                               static_cast<cudaStream_t>(stream), "enc_photons_trace_device");
  *stored = st[0];
  return r;
}

enc_status enc_photons_trace_maps_device(enc_accel accel, const enc_photon_opts* o,
                                         float shadow_offset, int32_t fill_indirect,
                                         const enc_photon_store* direct,
                                         const enc_photon_store* indirect, uint32_t stored[2],
                                         uint32_t* emitted, enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || !o || !stored || !direct || !indirect) return ENC_ERR_INVALID_ARG;
  for (const enc_photon_store* m : {direct, indirect}) {
    if (m->capacity && (!m->d_pos || !m->d_nrm || !m->d_pow)) {
      set_error("enc_photons_trace_maps_device: a store with capacity needs its arrays");
      return ENC_ERR_INVALID_ARG;
    }
  }
  PhotonStore s0{direct->d_pos, direct->d_nrm, direct->d_pow, direct->d_tag, direct->capacity};
  PhotonStore s1{indirect->d_pos, indirect->d_nrm, indirect->d_pow, indirect->d_tag,
                 indirect->capacity};
  return trace_photons(accel, o, 1, shadow_offset, fill_indirect ? 1 : 0, s0, s1, stored, emitted,
                       static_cast<cudaStream_t>(stream), "enc_photons_trace_maps_device");
}

enc_status enc_photons_trace_maps(enc_accel accel, const enc_photon_opts* o, float shadow_offset,
                                  int32_t fill_indirect, const enc_photon_store* direct,
                                  const enc_photon_store* indirect, uint32_t stored[2],
                                  uint32_t* emitted, enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || !o || !stored || !direct || !indirect) return ENC_ERR_INVALID_ARG;
  const enc_photon_store* hs[2] = {direct, indirect};
  for (const enc_photon_store* m : hs) {
    if (m->capacity && (!m->d_pos || !m->d_nrm || !m->d_pow)) {
      set_error("enc_photons_trace_maps: a store with capacity needs its arrays");
      return ENC_ERR_INVALID_ARG;
    }
  }
  // device stores for the call, copied back and freed at its end
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != a->device) cudaSetDevice(a->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PhotonStore ds[2];
  void* blocks[2] = {nullptr, nullptr};
  cudaError_t e = cudaSuccess;
  for (int m = 0; m < 2 && e == cudaSuccess; ++m) {
    const size_t cap = hs[m]->capacity;
    const size_t bytes = cap * (36 + (hs[m]->d_tag ? 4 : 0)) + 16;
    e = cudaMalloc(&blocks[m], bytes);
    float* base = static_cast<float*>(blocks[m]);
    ds[m] = PhotonStore{base, base + 3 * cap, base + 6 * cap,
                        hs[m]->d_tag ? reinterpret_cast<uint32_t*>(base + 9 * cap) : nullptr,
                        hs[m]->capacity};
  }
  enc_status st = ENC_OK;
  if (e == cudaSuccess) {
    st = trace_photons(accel, o, 1, shadow_offset, fill_indirect ? 1 : 0, ds[0], ds[1], stored,
                       emitted, s, "enc_photons_trace_maps");
    for (int m = 0; m < 2 && st == ENC_OK && e == cudaSuccess; ++m) {
      const size_t n = stored[m];
      if (!n) continue;
      e = cudaMemcpyAsync(hs[m]->d_pos, ds[m].pos, n * 12, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(hs[m]->d_nrm, ds[m].nrm, n * 12, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(hs[m]->d_pow, ds[m].pw, n * 12, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && ds[m].tag)
        e = cudaMemcpyAsync(hs[m]->d_tag, ds[m].tag, n * 4, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  cudaFree(blocks[0]);
  cudaFree(blocks[1]);
  if (prev >= 0 && prev != a->device) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_error(std::string("enc_photons_trace_maps: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? ENC_ERR_OUT_OF_MEMORY : ENC_ERR_CUDA;
  }
  return st;
}

}  // extern "C"
