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

// Cosine lobe about unit n: cos(theta) = sqrt(e1), phi = 2 pi e2, e1 drawn
// from [lo, 1) as randDirectionN/SuperN cut the grazing tip (Common.cpp:96,
// 156).  The frame is any orthonormal basis around n; the distribution is the
// same as the reference's rotation of +z onto n.
__device__ __forceinline__ float3 cosine_dir(float3 n, float lo, float u1, float u2) {
  const float e1 = lo + (1.0f - lo) * u1;
  const float ct = sqrtf(e1), st = sqrtf(fmaxf(0.f, 1.0f - e1));
  float sp, cp;
  sincospif(2.0f * u2, &sp, &cp);
  const float3 a = fabsf(n.x) > 0.9f ? make_float3(0.f, 1.f, 0.f) : make_float3(1.f, 0.f, 0.f);
  float3 t = make_float3(a.y * n.z - a.z * n.y, a.z * n.x - a.x * n.z, a.x * n.y - a.y * n.x);
  const float tl = rsqrtf(t.x * t.x + t.y * t.y + t.z * t.z);
  t = make_float3(t.x * tl, t.y * tl, t.z * tl);
  const float3 b = make_float3(n.y * t.z - n.z * t.y, n.z * t.x - n.x * t.z, n.x * t.y - n.y * t.x);
  return make_float3(st * cp * t.x + st * sp * b.x + ct * n.x, st * cp * t.y + st * sp * b.y + ct * n.y,
                     st * cp * t.z + st * sp * b.z + ct * n.z);
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
      const float3 d = cosine_dir(f, 0.0f, rnd(seed, (uint32_t)o, 0), rnd(seed, (uint32_t)o, 1));
      put_ray(out, o, make_float3(p.x + offset * f.x, p.y + offset * f.y, p.z + offset * f.z), 0.f,
              d, INFINITY);
    }
  }
}

struct PhotonParams {
  float3 lc;
  float lsize;
  uint32_t n, seed, max_bounces;
  float albedo, power, emit_offset, bounce_offset;
};

__global__ void photon_emit_kernel(PhotonParams P, float* rays, uint32_t* path) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
    const float3 o = make_float3(P.lc.x + (rnd(P.seed, i, 0) - 0.5f) * P.lsize, P.lc.y,
                                 P.lc.z + (rnd(P.seed, i, 1) - 0.5f) * P.lsize);
    const float3 d = cosine_dir(make_float3(0.f, -1.f, 0.f), 0.01f, rnd(P.seed, i, 2), rnd(P.seed, i, 3));
    put_ray(rays, i,
            make_float3(o.x + d.x * P.emit_offset, o.y + d.y * P.emit_offset, o.z + d.z * P.emit_offset),
            0.f, d, INFINITY);
    path[i] = i;
  }
}

// One wave: store a photon at every hit; survivors of the roulette (and of
// the bounce limit) spawn the next wave's rays.
__global__ void photon_bounce_kernel(PhotonParams P, TriView tv, uint32_t wave, const int4* hits,
                                     const uint32_t* path, uint32_t n, float* pos, float* nrm,
                                     float* pw, uint32_t capacity, uint32_t* counters,
                                     float* next_rays, uint32_t* next_path) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 p, nn, e1, e2;
    if (!hit_surface(tv, hits[i], p, nn, e1, e2)) continue;
    const uint32_t slot = atomicAdd(counters, 1u);
    if (slot < capacity) {
      pos[3 * (size_t)slot] = p.x;
      pos[3 * (size_t)slot + 1] = p.y;
      pos[3 * (size_t)slot + 2] = p.z;
      nrm[3 * (size_t)slot] = nn.x;
      nrm[3 * (size_t)slot + 1] = nn.y;
      nrm[3 * (size_t)slot + 2] = nn.z;
      pw[3 * (size_t)slot] = P.power;
      pw[3 * (size_t)slot + 1] = P.power;
      pw[3 * (size_t)slot + 2] = P.power;
    }
    const uint32_t id = path[i];
    if (wave >= P.max_bounces) continue;
    if (rnd(P.seed, id, 8 + 4 * wave) >= P.albedo) continue;  // absorbed
    // ReflectPhotonDiffusely bounces about the stored hit normal as is
    // (randDirectionSuperN(hitNormal)); a zero normal (degenerate triangle
    // under the clamp) ends the path.
    const float l2 = nn.x * nn.x + nn.y * nn.y + nn.z * nn.z;
    if (!(l2 > 0.f)) continue;
    const float il = rsqrtf(l2);
    const float3 un = make_float3(nn.x * il, nn.y * il, nn.z * il);
    const float3 d = cosine_dir(un, 0.001f, rnd(P.seed, id, 9 + 4 * wave), rnd(P.seed, id, 10 + 4 * wave));
    const uint32_t k = atomicAdd(counters + 1, 1u);
    put_ray(next_rays, k,
            make_float3(p.x + d.x * P.bounce_offset, p.y + d.y * P.bounce_offset, p.z + d.z * P.bounce_offset),
            0.f, d, INFINITY);
    next_path[k] = id;
  }
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

enc_status enc_photons_trace_device(enc_accel accel, const enc_photon_opts* o, float* d_pos,
                                    float* d_nrm, float* d_pow, uint32_t capacity,
                                    uint32_t* stored, enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || !o || !stored || (capacity && (!d_pos || !d_nrm || !d_pow))) return ENC_ERR_INVALID_ARG;
  if (a->kind != ENC_ACCEL_WBVH) {
    set_error("enc_photons_trace_device: wide-BVH accelerators only");
    return ENC_ERR_UNSUPPORTED;
  }
  *stored = 0;
  if (o->nphotons == 0) return ENC_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PhotonParams P;
  P.lc = make_float3(o->light_center[0], o->light_center[1], o->light_center[2]);
  P.lsize = o->light_size;
  P.n = o->nphotons;
  P.seed = o->seed ? o->seed : 1u;
  P.max_bounces = o->max_bounces;
  P.albedo = o->albedo;
  P.power = 1.0f / (float)o->nphotons;
  P.emit_offset = o->emit_offset;
  P.bounce_offset = o->bounce_offset;
  const size_t n = o->nphotons;
  WaveScratch& w = *accel_wave_scratch(accel);
  std::lock_guard<std::mutex> lk(w.mu);
  cudaError_t e = cudaSuccess;
  if (w.cap < n) {  // grow the kept scratch (no allocation once it is large enough)
    free_wave_scratch(&w);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
      e = cudaMalloc((void**)&w.rays[i], n * 32);
      if (e == cudaSuccess) e = cudaMalloc((void**)&w.path[i], n * 4);
    }
    if (e == cudaSuccess) e = cudaMalloc(&w.hits, n * 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&w.counters, 16);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&w.h_counts, 16);
    if (e != cudaSuccess) {
      free_wave_scratch(&w);
      set_error(std::string("enc_photons_trace_device: ") + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? ENC_ERR_OUT_OF_MEMORY : ENC_ERR_CUDA;
    }
    w.cap = n;
  }
  float* const* rays = w.rays;
  uint32_t* const* path = w.path;
  int4* hits = static_cast<int4*>(w.hits);
  uint32_t* counters = w.counters;
  e = cudaMemsetAsync(counters, 0, 16, s);
  Launch L = resolve_launch(nullptr, a->kind, a->width);
  uint32_t count = o->nphotons;
  int cur = 0;
  if (e == cudaSuccess) {
    photon_emit_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, rays[0], path[0]);
    e = cudaGetLastError();
  }
  for (uint32_t wave = 0; e == cudaSuccess && count > 0 && wave <= o->max_bounces; ++wave) {
    int le = launch_closest(*a, rays[cur], count, reinterpret_cast<enc_hit*>(hits), L, s, nullptr);
    if (le) {
      e = (cudaError_t)le;
      break;
    }
    e = cudaMemsetAsync(counters + 1, 0, 4, s);
    if (e != cudaSuccess) break;
    photon_bounce_kernel<<<grid_for(count, 256), 256, 0, s>>>(
        P, tri_view(*a), wave, hits, path[cur], count, d_pos, d_nrm, d_pow, capacity, counters,
        rays[cur ^ 1], path[cur ^ 1]);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(w.h_counts, counters, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    count = w.h_counts[1];
    cur ^= 1;
  }
  uint32_t total = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(w.h_counts, counters, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) total = w.h_counts[0];
  if (e != cudaSuccess) {
    set_error(std::string("enc_photons_trace_device: ") + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  *stored = total < capacity ? total : capacity;
  return ENC_OK;
}

}  // extern "C"
