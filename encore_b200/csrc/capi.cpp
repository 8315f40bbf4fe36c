// C ABI of the ray-query engine: handle management, device upload, launches
// and status checks.  Everything the reference's callers reach through
// AccelerationStructure / PhotonMap enters here.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.h"
#include "photon.h"
#include "scene.h"

struct enc_accel_s {
  enc::DevAccel dev;
  enc::WaveScratch wave;  // photon tracer scratch
  enc::WBVHHost host;  // wide BVH kept on the host for refits
  std::mutex mu;  // serialises the host-buffer forms (shared staging buffers)
  void* d_stage_in = nullptr;
  void* d_stage_out = nullptr;
  void* d_stage_od = nullptr;  // rays of 6 floats, before widening (enc_intersect_closest_od)
  size_t stage_in_bytes = 0, stage_out_bytes = 0, stage_od_bytes = 0;
  // host-form pipeline: copy-in, trace, copy-out, ray-widening and second
  // trace streams, and per-chunk events (copy-in done, trace done, widening
  // done)
  cudaStream_t pipe[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> ev_in, ev_trace, ev_wide;
  cudaEvent_t pipe_start = nullptr, pipe_done = nullptr;
};

struct enc_photonmap_s {
  enc::DevPhotonMap dev;
  std::mutex mu;
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
};

namespace enc {

namespace {
thread_local std::string g_err;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Makes `device` current for the scope and restores the caller's device.
struct DeviceScope {
  int prev = -1;
  bool ok = true;
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device) ok = cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

enc_status cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? ENC_ERR_OUT_OF_MEMORY : ENC_ERR_CUDA;
}

#define ENC_CUDA(call, what)                 \
  do {                                       \
    cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

template <class T>
cudaError_t upload(T** dst, const T* src, size_t count) {
  *dst = nullptr;
  if (count == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc((void**)dst, count * sizeof(T));
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
}

void free_dev(DevAccel& a) {
  cudaFree(a.d_nodes);
  cudaFree(a.d_tris);
  cudaFree(a.d_kd);
  cudaFree(a.d_kd_items);
  cudaFree(a.d_tri_pos);
  a.d_tri_pos = nullptr;
  cudaFree(a.d_status);
  cudaFree(a.d_counter);
  a.d_nodes = nullptr;
  a.d_tris = nullptr;
  a.d_kd = nullptr;
  a.d_kd_items = nullptr;
  a.d_status = nullptr;
  a.d_counter = nullptr;
}

enc_status grow(void** p, size_t* cap, size_t need) {
  if (*cap >= need) return ENC_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  size_t n = need + need / 4;
  cudaError_t e = cudaMalloc(p, n);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(staging)");
  *cap = n;
  return ENC_OK;
}

enc_status read_status(enc_accel a, cudaStream_t s) {
  ENC_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  uint32_t st = 0;
  ENC_CUDA(cudaMemcpy(&st, a->dev.d_status, sizeof(st), cudaMemcpyDeviceToHost), "read status");
  if (st != 0) {
    cudaMemset(a->dev.d_status, 0, sizeof(uint32_t));
    set_error("kernel stopped at a loop bound (status bits " + std::to_string(st) +
              ": 1 = step limit, 2 = stack depth, 4 = index out of range)");
    return ENC_ERR_WATCHDOG;
  }
  return ENC_OK;
}

}  // namespace

void set_error(const std::string& msg) { g_err = msg; }

const DevAccel* accel_device_view(enc_accel a) { return a ? &a->dev : nullptr; }

WaveScratch* accel_wave_scratch(enc_accel a) { return a ? &a->wave : nullptr; }

void free_wave_scratch(WaveScratch* w) {
  for (int i = 0; i < 2; ++i) {
    cudaFree(w->rays[i]);
    cudaFree(w->path[i]);
    cudaFree(w->srays[i]);
    cudaFree(w->spath[i]);
    w->rays[i] = nullptr;
    w->path[i] = nullptr;
    w->srays[i] = nullptr;
    w->spath[i] = nullptr;
  }
  cudaFree(w->hits);
  cudaFree(w->counters);
  cudaFreeHost(w->h_counts);
  w->hits = nullptr;
  w->counters = nullptr;
  w->h_counts = nullptr;
  w->cap = 0;
}

Launch resolve_launch(const enc_launch_opts* o, int kind, int width) {
  (void)kind;
  Launch L;
  L.block = 128;
  L.blocks_per_sm = 0;  // 0: each traversal kernel's own resident-block target
  L.chunk = 32;
  L.stack = 0;  // 0 = the tree's depth, which always suffices
  if (o) {
    if (o->block_threads > 0) L.block = o->block_threads;
    if (o->blocks_per_sm > 0) L.blocks_per_sm = o->blocks_per_sm;
    if (o->chunk > 0) L.chunk = o->chunk;
    if (o->stack_depth > 0) L.stack = o->stack_depth;
  }
  return L;
}

}  // namespace enc

using namespace enc;

extern "C" {

int32_t enc_abi_version(void) { return ENC_ABI_VERSION; }

const char* enc_last_error(void) { return g_err.c_str(); }

enc_status enc_device_count(int32_t* count) {
  if (!count) return ENC_ERR_INVALID_ARG;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    *count = 0;
    return cuda_fail(e, "cudaGetDeviceCount");
  }
  *count = n;
  return ENC_OK;
}

enc_status enc_scene_create(const float* tri_verts, uint32_t ntris, enc_scene* out) {
  if (!out || (!tri_verts && ntris)) {
    set_error("enc_scene_create: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  enc_scene s = new (std::nothrow) enc_scene_s();
  if (!s) return ENC_ERR_OUT_OF_MEMORY;
  try {
    s->verts.assign(tri_verts, tri_verts + 9 * (size_t)ntris);
  } catch (const std::bad_alloc&) {
    delete s;
    return ENC_ERR_OUT_OF_MEMORY;
  }
  s->ntris = ntris;
  s->desc.ntris = ntris;
  s->desc.nprims = ntris;
  *out = s;
  return ENC_OK;
}

enc_status enc_scene_destroy(enc_scene scene) {
  delete scene;
  return ENC_OK;
}

enc_status enc_accel_build(enc_scene scene, const enc_build_opts* opts, int32_t device,
                           enc_accel* out) {
  if (!scene || !out) {
    set_error("enc_accel_build: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  if (scene->ntris == 0) {
    set_error("enc_accel_build: scene has no triangles");
    return ENC_ERR_INVALID_ARG;
  }
  enc_build_opts o = {ENC_ACCEL_WBVH, 8, 3, ENC_PRED_REFERENCE};
  if (opts) o = *opts;
  if (o.width == 0) o.width = 8;
  if (o.max_leaf_tris == 0) o.max_leaf_tris = 3;
  if (o.kind != ENC_ACCEL_WBVH && o.kind != ENC_ACCEL_KDTREE) {
    set_error("enc_accel_build: unknown kind");
    return ENC_ERR_INVALID_ARG;
  }
  if (o.width != 2 && o.width != 4 && o.width != 8) {
    set_error("enc_accel_build: width must be 2, 4 or 8");
    return ENC_ERR_INVALID_ARG;
  }
  if (o.max_leaf_tris < 1 || o.max_leaf_tris > 4) {
    set_error("enc_accel_build: max_leaf_tris must be 1..4");
    return ENC_ERR_INVALID_ARG;
  }
  if (o.predicate != ENC_PRED_REFERENCE && o.predicate != ENC_PRED_NOCLAMP) {
    set_error("enc_accel_build: unknown predicate");
    return ENC_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_error("enc_accel_build: no such CUDA device");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(device);
  if (!ds.ok) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
  enc_accel a = new (std::nothrow) enc_accel_s();
  if (!a) return ENC_ERR_OUT_OF_MEMORY;
  DevAccel& d = a->dev;
  d.kind = o.kind;
  d.width = o.width;
  d.predicate = o.predicate;
  d.ntris = scene->ntris;
  d.device = device;
  double t0 = now_s();
  cudaError_t e = cudaSuccess;
  try {
    if (o.kind == ENC_ACCEL_WBVH) {
      WBVHHost h;
      build_wbvh(scene->verts.data(), scene->ntris, o.width, o.max_leaf_tris, &h);
      d.nnodes = h.nnodes;
      d.tree_depth = h.depth;
      if (h.depth > 64) throw std::runtime_error("wide BVH deeper than 64 levels");
      for (int i = 0; i < 3; ++i) {
        d.lo[i] = h.lo[i];
        d.hi[i] = h.hi[i];
      }
      uint8_t* dn = nullptr;
      e = upload(&dn, h.nodes.data(), h.nodes.size());
      d.d_nodes = dn;
      if (e == cudaSuccess) e = upload(&d.d_tris, h.tris.data(), h.tris.size());
      if (e == cudaSuccess) e = upload(&d.d_tri_pos, h.tri_pos.data(), h.tri_pos.size());
      d.node_bytes = h.nodes.size();
      d.tri_bytes = h.tris.size() * sizeof(DevTri);
      // keep the tree for refits (not the triangle records: refit rewrites them)
      h.tris.clear();
      h.tris.shrink_to_fit();
      a->host = std::move(h);
    } else {
      KdHost h;
      build_kd_reference(scene->verts.data(), scene->ntris, &h);
      std::vector<DevTri> tris(scene->ntris);
      make_dev_tris(scene->verts.data(), scene->ntris, nullptr, tris.data());
      d.nnodes = (uint32_t)h.nodes.size();
      d.kd_nitems = (uint32_t)h.items.size();
      d.tree_depth = h.max_depth + 1;  // levels below the root: one deferred child each
      for (int i = 0; i < 3; ++i) {
        d.kd_root_lo[i] = h.root_lo[i];
        d.kd_root_hi[i] = h.root_hi[i];
        d.lo[i] = h.root_lo[i];
        d.hi[i] = h.root_hi[i];
      }
      e = upload(&d.d_kd, h.nodes.data(), h.nodes.size());
      if (e == cudaSuccess) e = upload(&d.d_kd_items, h.items.data(), h.items.size());
      if (e == cudaSuccess) e = upload(&d.d_tris, tris.data(), tris.size());
      d.node_bytes = h.nodes.size() * sizeof(KdNode) + h.items.size() * sizeof(uint32_t);
      d.tri_bytes = tris.size() * sizeof(DevTri);
    }
  } catch (const std::bad_alloc&) {
    free_dev(d);
    delete a;
    set_error("enc_accel_build: host out of memory");
    return ENC_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& ex) {
    free_dev(d);
    delete a;
    set_error(std::string("enc_accel_build: ") + ex.what());
    return ENC_ERR_INVALID_ARG;
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_status, 16);
  if (e == cudaSuccess) e = cudaMemset(d.d_status, 0, 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_counter, kQueueSlots * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(d.d_counter, 0, kQueueSlots * sizeof(uint32_t));
  if (e != cudaSuccess) {
    free_dev(d);
    delete a;
    return cuda_fail(e, "enc_accel_build: upload");
  }
  d.device_bytes = d.node_bytes + d.tri_bytes + (d.d_tri_pos ? 4ull * d.ntris : 0) +
                   kQueueSlots * sizeof(uint32_t) + 16;
  // The no-allocation query entry point's fixed scratch on this device: its
  // address is looked up now, while allocating is allowed (the look-up makes
  // the runtime create the array).
  const int pe = noalloc_prepare(d);
  if (pe != 0) {
    free_dev(d);
    delete a;
    return cuda_fail((cudaError_t)pe, "enc_accel_build: fixed query scratch");
  }
  d.build_seconds = now_s() - t0;
  *out = a;
  return ENC_OK;
}

enc_status enc_accel_refit(enc_accel a, const float* tri_verts, uint32_t ntris) {
  if (!a || !tri_verts) {
    set_error("enc_accel_refit: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  DevAccel& d = a->dev;
  if (ntris != d.ntris) {
    set_error("enc_accel_refit: the triangle count must stay the same");
    return ENC_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(a->mu);
  DeviceScope ds(d.device);
  double t0 = now_s();
  try {
    if (d.kind == ENC_ACCEL_WBVH) {
      refit_wbvh(&a->host, tri_verts, ntris);
      ENC_CUDA(cudaMemcpy(d.d_nodes, a->host.nodes.data(), a->host.nodes.size(), cudaMemcpyHostToDevice),
               "refit upload");
      ENC_CUDA(cudaMemcpy(d.d_tris, a->host.tris.data(), a->host.tris.size() * sizeof(DevTri),
                          cudaMemcpyHostToDevice),
               "refit upload");
      for (int i = 0; i < 3; ++i) {
        d.lo[i] = a->host.lo[i];
        d.hi[i] = a->host.hi[i];
      }
      a->host.tris.clear();
      a->host.tris.shrink_to_fit();
    } else {
      // Kdtree::update rebuilds (Kdtree.h:138); so does the kd layout here
      KdHost h;
      build_kd_reference(tri_verts, ntris, &h);
      std::vector<DevTri> tris(ntris);
      make_dev_tris(tri_verts, ntris, nullptr, tris.data());
      KdNode* nodes = nullptr;
      uint32_t* items = nullptr;
      cudaError_t e = upload(&nodes, h.nodes.data(), h.nodes.size());
      if (e == cudaSuccess) e = upload(&items, h.items.data(), h.items.size());
      if (e == cudaSuccess)
        e = cudaMemcpy(d.d_tris, tris.data(), tris.size() * sizeof(DevTri), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        cudaFree(nodes);
        cudaFree(items);
        return cuda_fail(e, "refit upload");
      }
      cudaFree(d.d_kd);
      cudaFree(d.d_kd_items);
      d.d_kd = nodes;
      d.d_kd_items = items;
      d.nnodes = (uint32_t)h.nodes.size();
      d.kd_nitems = (uint32_t)h.items.size();
      d.tree_depth = h.max_depth + 1;
      d.node_bytes = h.nodes.size() * sizeof(KdNode) + h.items.size() * sizeof(uint32_t);
      for (int i = 0; i < 3; ++i) {
        d.kd_root_lo[i] = h.root_lo[i];
        d.kd_root_hi[i] = h.root_hi[i];
        d.lo[i] = h.root_lo[i];
        d.hi[i] = h.root_hi[i];
      }
    }
  } catch (const std::exception& ex) {
    set_error(std::string("enc_accel_refit: ") + ex.what());
    return ENC_ERR_INVALID_ARG;
  }
  d.build_seconds = now_s() - t0;
  return ENC_OK;
}

namespace {

// Serialised accelerator: a fixed header, then the sections it sizes.
struct AccelFileHeader {
  char magic[8];
  uint32_t version;
  int32_t kind, width, predicate;
  uint32_t ntris, nnodes, depth, kd_nitems;
  float lo[3], hi[3], kd_lo[3], kd_hi[3];
  uint64_t node_bytes, tri_bytes, order_bytes, items_bytes;
};
constexpr char kAccelMagic[8] = {'E', 'N', 'C', 'A', 'C', 'C', '0', '1'};
constexpr uint32_t kAccelVersion = 1;

size_t wbvh_node_bytes(int width) {
  return width == 2 ? WNodeLayout<2>::kBytes : width == 4 ? WNodeLayout<4>::kBytes
                                                          : WNodeLayout<8>::kBytes;
}

}  // namespace

enc_status enc_accel_serialize(enc_accel a, void* buf, size_t cap, size_t* size) {
  if (!a || !size) {
    set_error("enc_accel_serialize: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  const DevAccel& d = a->dev;
  AccelFileHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kAccelMagic, 8);
  h.version = kAccelVersion;
  h.kind = d.kind;
  h.width = d.width;
  h.predicate = d.predicate;
  h.ntris = d.ntris;
  h.nnodes = d.nnodes;
  h.depth = (uint32_t)d.tree_depth;
  h.kd_nitems = d.kd_nitems;
  for (int i = 0; i < 3; ++i) {
    h.lo[i] = d.lo[i];
    h.hi[i] = d.hi[i];
    h.kd_lo[i] = d.kd_root_lo[i];
    h.kd_hi[i] = d.kd_root_hi[i];
  }
  if (d.kind == ENC_ACCEL_WBVH) {
    h.node_bytes = (uint64_t)d.nnodes * wbvh_node_bytes(d.width);
    h.order_bytes = (uint64_t)a->host.tri_order.size() * 4;
  } else {
    h.node_bytes = (uint64_t)d.nnodes * sizeof(KdNode);
    h.items_bytes = (uint64_t)d.kd_nitems * 4;
  }
  h.tri_bytes = (uint64_t)d.ntris * sizeof(DevTri);
  const size_t total = sizeof(h) + h.node_bytes + h.tri_bytes + h.order_bytes + h.items_bytes;
  *size = total;
  if (!buf) return ENC_OK;  // size query
  if (cap < total) {
    set_error("enc_accel_serialize: buffer smaller than the size the call reports");
    return ENC_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(a->mu);
  DeviceScope ds(d.device);
  char* p = static_cast<char*>(buf);
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  if (d.kind == ENC_ACCEL_WBVH) {
    ENC_CUDA(cudaMemcpy(p, d.d_nodes, h.node_bytes, cudaMemcpyDeviceToHost), "read nodes");
  } else {
    ENC_CUDA(cudaMemcpy(p, d.d_kd, h.node_bytes, cudaMemcpyDeviceToHost), "read kd nodes");
  }
  p += h.node_bytes;
  ENC_CUDA(cudaMemcpy(p, d.d_tris, h.tri_bytes, cudaMemcpyDeviceToHost), "read triangles");
  p += h.tri_bytes;
  if (h.order_bytes) std::memcpy(p, a->host.tri_order.data(), h.order_bytes);
  p += h.order_bytes;
  if (h.items_bytes)
    ENC_CUDA(cudaMemcpy(p, d.d_kd_items, h.items_bytes, cudaMemcpyDeviceToHost), "read kd items");
  return ENC_OK;
}

enc_status enc_accel_deserialize(const void* buf, size_t size, int32_t device, enc_accel* out) {
  if (!buf || !out) {
    set_error("enc_accel_deserialize: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  AccelFileHeader h;
  if (size < sizeof(h)) {
    set_error("enc_accel_deserialize: shorter than the header");
    return ENC_ERR_INVALID_ARG;
  }
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, kAccelMagic, 8) != 0 || h.version != kAccelVersion) {
    set_error("enc_accel_deserialize: not a serialised accelerator of this version");
    return ENC_ERR_INVALID_ARG;
  }
  const bool wbvh = h.kind == ENC_ACCEL_WBVH;
  if ((h.kind != ENC_ACCEL_WBVH && h.kind != ENC_ACCEL_KDTREE) ||
      (wbvh && h.width != 2 && h.width != 4 && h.width != 8) ||
      (h.predicate != ENC_PRED_REFERENCE && h.predicate != ENC_PRED_NOCLAMP) || h.ntris == 0 ||
      h.nnodes == 0 || h.depth > 64 ||
      h.node_bytes != (uint64_t)h.nnodes * (wbvh ? wbvh_node_bytes(h.width) : sizeof(KdNode)) ||
      h.tri_bytes != (uint64_t)h.ntris * sizeof(DevTri) ||
      h.order_bytes != (wbvh ? (uint64_t)h.ntris * 4 : 0) ||
      h.items_bytes != (wbvh ? 0 : (uint64_t)h.kd_nitems * 4) ||
      size != sizeof(h) + h.node_bytes + h.tri_bytes + h.order_bytes + h.items_bytes) {
    set_error("enc_accel_deserialize: header and sizes do not agree");
    return ENC_ERR_INVALID_ARG;
  }
  const char* p = static_cast<const char*>(buf) + sizeof(h);
  const char* nodes = p;
  const DevTri* tris = reinterpret_cast<const DevTri*>(p + h.node_bytes);
  const char* sec3 = p + h.node_bytes + h.tri_bytes;
  std::vector<uint32_t> order;
  if (wbvh) {
    order.resize(h.ntris);
    std::memcpy(order.data(), sec3, h.order_bytes);
    std::vector<uint8_t> seen(h.ntris, 0);
    for (uint32_t v : order) {
      if (v >= h.ntris || seen[v]) {
        set_error("enc_accel_deserialize: the triangle order is not a permutation");
        return ENC_ERR_INVALID_ARG;
      }
      seen[v] = 1;
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_error("enc_accel_deserialize: no such CUDA device");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(device);
  if (!ds.ok) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
  enc_accel a = new (std::nothrow) enc_accel_s();
  if (!a) return ENC_ERR_OUT_OF_MEMORY;
  DevAccel& d = a->dev;
  d.kind = h.kind;
  d.width = wbvh ? h.width : 8;
  d.predicate = h.predicate;
  d.ntris = h.ntris;
  d.nnodes = h.nnodes;
  d.tree_depth = (int)h.depth;
  d.kd_nitems = h.kd_nitems;
  d.device = device;
  for (int i = 0; i < 3; ++i) {
    d.lo[i] = h.lo[i];
    d.hi[i] = h.hi[i];
    d.kd_root_lo[i] = h.kd_lo[i];
    d.kd_root_hi[i] = h.kd_hi[i];
  }
  const double t0 = now_s();
  cudaError_t e = cudaSuccess;
  try {
    if (wbvh) {
      WBVHHost& hh = a->host;
      hh.width = h.width;
      hh.nnodes = h.nnodes;
      hh.depth = (int)h.depth;
      hh.nodes.assign(nodes, nodes + h.node_bytes);
      hh.tri_order = order;
      hh.tri_pos.assign(h.ntris, 0);
      for (uint32_t i = 0; i < h.ntris; ++i) hh.tri_pos[order[i]] = i;
      for (int i = 0; i < 3; ++i) {
        hh.lo[i] = h.lo[i];
        hh.hi[i] = h.hi[i];
      }
      uint8_t* dn = nullptr;
      e = upload(&dn, hh.nodes.data(), hh.nodes.size());
      d.d_nodes = dn;
      if (e == cudaSuccess) e = upload(&d.d_tris, tris, h.ntris);
      if (e == cudaSuccess) e = upload(&d.d_tri_pos, hh.tri_pos.data(), hh.tri_pos.size());
    } else {
      e = upload(&d.d_kd, reinterpret_cast<const KdNode*>(nodes), h.nnodes);
      if (e == cudaSuccess && h.kd_nitems)
        e = upload(&d.d_kd_items, reinterpret_cast<const uint32_t*>(sec3), h.kd_nitems);
      if (e == cudaSuccess) e = upload(&d.d_tris, tris, h.ntris);
    }
  } catch (const std::bad_alloc&) {
    free_dev(d);
    delete a;
    set_error("enc_accel_deserialize: host out of memory");
    return ENC_ERR_OUT_OF_MEMORY;
  }
  d.node_bytes = wbvh ? h.node_bytes : h.node_bytes + h.items_bytes;
  d.tri_bytes = h.tri_bytes;
  if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_status, 16);
  if (e == cudaSuccess) e = cudaMemset(d.d_status, 0, 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_counter, kQueueSlots * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(d.d_counter, 0, kQueueSlots * sizeof(uint32_t));
  if (e != cudaSuccess) {
    free_dev(d);
    delete a;
    return cuda_fail(e, "enc_accel_deserialize: upload");
  }
  d.device_bytes = d.node_bytes + d.tri_bytes + (d.d_tri_pos ? 4ull * d.ntris : 0) +
                   kQueueSlots * sizeof(uint32_t) + 16;
  const int pe = noalloc_prepare(d);
  if (pe != 0) {
    free_dev(d);
    delete a;
    return cuda_fail((cudaError_t)pe, "enc_accel_deserialize: fixed query scratch");
  }
  d.build_seconds = now_s() - t0;
  *out = a;
  return ENC_OK;
}

enc_status enc_accel_destroy(enc_accel a) {
  if (!a) return ENC_OK;
  DeviceScope ds(a->dev.device);
  free_dev(a->dev);
  free_wave_scratch(&a->wave);
  cudaFree(a->d_stage_in);
  cudaFree(a->d_stage_od);
  cudaFree(a->d_stage_out);
  for (int i = 0; i < 5; ++i)
    if (a->pipe[i]) cudaStreamDestroy(a->pipe[i]);
  for (cudaEvent_t e : a->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : a->ev_trace) cudaEventDestroy(e);
  for (cudaEvent_t e : a->ev_wide) cudaEventDestroy(e);
  if (a->pipe_start) cudaEventDestroy(a->pipe_start);
  if (a->pipe_done) cudaEventDestroy(a->pipe_done);
  delete a;
  return ENC_OK;
}

enc_status enc_accel_info_get(enc_accel a, enc_accel_info* info) {
  if (!a || !info) return ENC_ERR_INVALID_ARG;
  const DevAccel& d = a->dev;
  info->kind = d.kind;
  info->width = d.width;
  info->predicate = d.predicate;
  info->ntris = d.ntris;
  info->nnodes = d.nnodes;
  info->node_bytes = d.node_bytes;
  info->tri_bytes = d.tri_bytes;
  info->device_bytes = d.device_bytes;
  info->build_seconds = d.build_seconds;
  for (int i = 0; i < 3; ++i) {
    info->scene_lo[i] = d.lo[i];
    info->scene_hi[i] = d.hi[i];
  }
  return ENC_OK;
}

enc_status enc_intersect_closest_device(enc_accel a, const float* d_rays, size_t nrays,
                                        enc_hit* d_hits, const enc_launch_opts* launch,
                                        enc_stream stream) {
  if (!a || (nrays && (!d_rays || !d_hits))) {
    set_error("enc_intersect_closest_device: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays > 0xffffffffull / 2) {
    set_error("enc_intersect_closest_device: too many rays in one call");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(a->dev.device);
  Launch L = resolve_launch(launch, a->dev.kind, a->dev.width);
  if (L.block % 32 != 0 || L.block > 128 || (L.stack != 0 && L.stack < 2) || L.stack > 64 || L.chunk < 1) {
    set_error("enc_intersect: launch options out of range (block multiple of 32 <= 128, stack 0 or 2..64)");
    return ENC_ERR_INVALID_ARG;
  }
  int e = launch_closest(a->dev, d_rays, nrays, d_hits, L, stream, nullptr);
  if (e != 0) return cuda_fail((cudaError_t)e, "closest-hit launch");
  return ENC_OK;
}

namespace {

// Default key: 16 bits, 10 of the origin cell and 6 of the direction.
constexpr int kBinOriginBits = 10;
constexpr int kBinDirBits = 6;

bool resolve_bin(const enc_bin_opts* o, int* ob, int* db, float* probe) {
  *ob = kBinOriginBits;
  *db = kBinDirBits;
  *probe = 0.0f;
  if (o) {
    if (o->origin_bits < 0 || o->dir_bits < 0 || !(o->probe_frac >= 0.0f) ||
        o->probe_frac > 16.0f)
      return false;
    if (o->origin_bits != 0 || o->dir_bits != 0) {
      *ob = o->origin_bits;
      *db = o->dir_bits;
    }
    *probe = o->probe_frac;
  }
  return *ob + *db >= 1 && *ob + *db <= kBinMaxKeyBits && *db <= 2 * kBinMaxDimBits &&
         *ob <= 3 * kBinMaxDimBits;
}

}  // namespace

enc_status enc_bin_scratch_bytes(size_t nrays, const enc_bin_opts* bin, size_t* bytes) {
  if (!bytes) return ENC_ERR_INVALID_ARG;
  int ob, db;
  float pf;
  if (!resolve_bin(bin, &ob, &db, &pf)) {
    set_error("enc_bin_scratch_bytes: origin_bits + dir_bits must be 1..20");
    return ENC_ERR_INVALID_ARG;
  }
  *bytes = bin_scratch_bytes(nrays, ob + db);
  return ENC_OK;
}

enc_status enc_bin_rays(enc_accel a, const float* d_rays, size_t nrays, void* d_scratch,
                        size_t scratch_bytes, const enc_bin_opts* bin, uint32_t** d_order,
                        enc_stream stream) {
  if (!a || !d_order || (nrays && (!d_rays || !d_scratch))) {
    set_error("enc_bin_rays: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *d_order = nullptr;
  if (nrays > 0xffffffffull / 2) {
    set_error("enc_bin_rays: too many rays in one call");
    return ENC_ERR_INVALID_ARG;
  }
  int ob, db;
  float pf;
  if (!resolve_bin(bin, &ob, &db, &pf)) {
    set_error("enc_bin_rays: origin_bits + dir_bits must be 1..20");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays == 0) return ENC_OK;
  if (scratch_bytes < bin_scratch_bytes(nrays, ob + db) ||
      (reinterpret_cast<uintptr_t>(d_scratch) & 255u) != 0) {
    set_error("enc_bin_rays: scratch smaller than enc_bin_scratch_bytes or not 256-byte aligned");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(a->dev.device);
  const BinSpec spec = make_bin_spec(a->dev.lo, a->dev.hi, ob + db, db, pf);
  int e = launch_bin(d_rays, nrays, spec, d_scratch, d_order, a->dev.device, stream);
  if (e != 0) return cuda_fail((cudaError_t)e, "binning launch");
  return ENC_OK;
}

enc_status enc_intersect_closest_device_ordered(enc_accel a, const float* d_rays, size_t nrays,
                                                const uint32_t* d_order, enc_hit* d_hits,
                                                const enc_launch_opts* launch, enc_stream stream) {
  if (!a || (nrays && (!d_rays || !d_hits || !d_order))) {
    set_error("enc_intersect_closest_device_ordered: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays > 0xffffffffull / 2) {
    set_error("enc_intersect_closest_device_ordered: too many rays in one call");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(a->dev.device);
  Launch L = resolve_launch(launch, a->dev.kind, a->dev.width);
  if (L.block % 32 != 0 || L.block > 128 || (L.stack != 0 && L.stack < 2) || L.stack > 64 || L.chunk < 1) {
    set_error("enc_intersect: launch options out of range (block multiple of 32 <= 128, stack 0 or 2..64)");
    return ENC_ERR_INVALID_ARG;
  }
  int e = launch_closest(a->dev, d_rays, nrays, d_hits, L, stream, nullptr, d_order);
  if (e != 0) return cuda_fail((cudaError_t)e, "closest-hit launch");
  return ENC_OK;
}

enc_status enc_intersect_closest_device_binned(enc_accel a, const float* d_rays, size_t nrays,
                                               enc_hit* d_hits, void* d_scratch,
                                               size_t scratch_bytes, const enc_bin_opts* bin,
                                               const enc_launch_opts* launch,
                                               enc_stream stream) {
  if (!a || (nrays && (!d_rays || !d_hits || !d_scratch))) {
    set_error("enc_intersect_closest_device_binned: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays > 0xffffffffull / 2) {
    set_error("enc_intersect_closest_device_binned: too many rays in one call");
    return ENC_ERR_INVALID_ARG;
  }
  int ob, db;
  float pf;
  if (!resolve_bin(bin, &ob, &db, &pf)) {
    set_error("enc_intersect_closest_device_binned: origin_bits + dir_bits must be 1..20");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays == 0) return ENC_OK;
  if (scratch_bytes < bin_scratch_bytes(nrays, ob + db) ||
      (reinterpret_cast<uintptr_t>(d_scratch) & 255u) != 0) {
    set_error("enc_intersect_closest_device_binned: scratch smaller than enc_bin_scratch_bytes "
              "or not 256-byte aligned");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(a->dev.device);
  Launch L = resolve_launch(launch, a->dev.kind, a->dev.width);
  if (L.block % 32 != 0 || L.block > 128 || (L.stack != 0 && L.stack < 2) || L.stack > 64 || L.chunk < 1) {
    set_error("enc_intersect: launch options out of range (block multiple of 32 <= 128, stack 0 or 2..64)");
    return ENC_ERR_INVALID_ARG;
  }
  const BinSpec spec = make_bin_spec(a->dev.lo, a->dev.hi, ob + db, db, pf);
  uint32_t* order = nullptr;
  int e = launch_bin(d_rays, nrays, spec, d_scratch, &order, a->dev.device, stream);
  if (e != 0) return cuda_fail((cudaError_t)e, "binning launch");
  e = launch_closest(a->dev, d_rays, nrays, d_hits, L, stream, nullptr, order);
  if (e != 0) return cuda_fail((cudaError_t)e, "closest-hit launch");
  return ENC_OK;
}

enc_status enc_intersect_any_device(enc_accel a, const float* d_rays, size_t nrays,
                                    uint8_t* d_occ, const enc_launch_opts* launch,
                                    enc_stream stream) {
  if (!a || (nrays && (!d_rays || !d_occ))) {
    set_error("enc_intersect_any_device: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays > 0xffffffffull / 2) {
    set_error("enc_intersect_any_device: too many rays in one call");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(a->dev.device);
  Launch L = resolve_launch(launch, a->dev.kind, a->dev.width);
  if (L.block % 32 != 0 || L.block > 128 || (L.stack != 0 && L.stack < 2) || L.stack > 64 || L.chunk < 1) {
    set_error("enc_intersect: launch options out of range (block multiple of 32 <= 128, stack 0 or 2..64)");
    return ENC_ERR_INVALID_ARG;
  }
  int e = launch_any(a->dev, d_rays, nrays, d_occ, L, stream);
  if (e != 0) return cuda_fail((cudaError_t)e, "any-hit launch");
  return ENC_OK;
}

namespace {

// Host-buffer form shared by closest and any hit.  Large batches are split
// into chunks over three internal streams: every copy in is queued back to
// back on one stream, each trace waits for its chunk's copy, and each copy
// out waits for its chunk's trace, so the host-to-device engine never idles
// behind a trace or a copy out, and the two copy directions overlap.  A
// batch then takes its copy in plus the trace and copy out of the last
// chunk.  (Measured on the 4.18M-ray bench batch: 512K-ray chunks beat 256K,
// 1M and 2M; the earlier two-stream form, whose copy in of chunk i+2 queued
// behind chunk i's copy out, was 15 % slower.)  Ordering with the caller's
// stream is kept with events; the call returns after the results are in
// `out`.  ray_floats = 8: rays in the traversal's layout; 6 (closest hit
// only): origin and direction, copied in at 24 bytes per ray and widened on a
// fourth stream ahead of each chunk's trace, with the traces alternating
// between two streams.
enc_status host_form(enc_accel a, const float* rays, size_t nrays, void* out, size_t out_bytes,
                     bool any, int ray_floats, const enc_launch_opts* launch, enc_stream stream,
                     const char* what) {
  if (!a || (nrays && (!rays || !out))) {
    set_error(std::string(what) + ": null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays == 0) return ENC_OK;
  if (nrays > 0xffffffffull / 2) {
    set_error(std::string(what) + ": too many rays in one call");
    return ENC_ERR_INVALID_ARG;
  }
  Launch L = resolve_launch(launch, a->dev.kind, a->dev.width);
  if (L.block % 32 != 0 || L.block > 128 || (L.stack != 0 && L.stack < 2) || L.stack > 64 ||
      L.chunk < 1) {
    set_error(std::string(what) + ": launch options out of range");
    return ENC_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(a->mu);
  DeviceScope ds(a->dev.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool od = ray_floats == 6;
  const size_t rb = (size_t)ray_floats * sizeof(float);  // bytes per ray in `rays`
  enc_status st = grow(&a->d_stage_in, &a->stage_in_bytes, nrays * 32);
  if (st) return st;
  st = grow(&a->d_stage_out, &a->stage_out_bytes, nrays * out_bytes);
  if (st) return st;
  if (od) {
    st = grow(&a->d_stage_od, &a->stage_od_bytes, nrays * rb);
    if (st) return st;
  }
  const size_t kChunk = (size_t)1 << 19;
  const size_t nchunks = nrays <= 2 * kChunk ? 1 : (nrays + kChunk - 1) / kChunk;
  char* din = static_cast<char*>(a->d_stage_in);
  char* dout = static_cast<char*>(a->d_stage_out);
  // where a chunk's rays land: the traversal layout, or the 6-float staging
  char* dcopy = od ? static_cast<char*>(a->d_stage_od) : din;
  if (nchunks == 1) {
    ENC_CUDA(cudaMemcpyAsync(dcopy, rays, nrays * rb, cudaMemcpyHostToDevice, s), "H2D rays");
    if (od) {
      const int e = launch_widen_rays((const float*)dcopy, nrays, (float*)din, a->dev.device, s);
      if (e) return cuda_fail((cudaError_t)e, "ray widen launch");
    }
    int e = any ? launch_any(a->dev, (const float*)din, nrays, (uint8_t*)dout, L, s)
                : launch_closest(a->dev, (const float*)din, nrays, (enc_hit*)dout, L, s, nullptr);
    if (e) return cuda_fail((cudaError_t)e, "trace launch");
    ENC_CUDA(cudaMemcpyAsync(out, dout, nrays * out_bytes, cudaMemcpyDeviceToHost, s), "D2H results");
    return read_status(a, s);
  }
  if (!a->pipe[0]) {
    for (int i = 0; i < 5; ++i)
      ENC_CUDA(cudaStreamCreateWithFlags(&a->pipe[i], cudaStreamNonBlocking), "stream create");
    ENC_CUDA(cudaEventCreateWithFlags(&a->pipe_start, cudaEventDisableTiming), "event create");
    ENC_CUDA(cudaEventCreateWithFlags(&a->pipe_done, cudaEventDisableTiming), "event create");
  }
  // chunk c covers rays [bound[c], bound[c + 1])
  std::vector<size_t> bound;
  for (size_t c = 0; c < nchunks; ++c) bound.push_back(c * kChunk);
  // A short final chunk: the call ends with the last chunk's trace and copy
  // out, so 64K rays there instead of up to 512K shorten it (+2.5 % on the
  // 4.18M-ray bench batch, four back-to-back passes).
  const size_t kTail = (size_t)1 << 16;
  if (nrays - bound.back() > kTail) bound.push_back(nrays - kTail);
  bound.push_back(nrays);
  const size_t nch = bound.size() - 1;
  while (a->ev_in.size() < nch) {
    cudaEvent_t e1 = nullptr, e2 = nullptr, e3 = nullptr;
    ENC_CUDA(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming), "event create");
    cudaError_t e = cudaEventCreateWithFlags(&e2, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e3, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      cudaEventDestroy(e1);
      if (e2) cudaEventDestroy(e2);
      return cuda_fail(e, "event create");
    }
    a->ev_in.push_back(e1);
    a->ev_trace.push_back(e2);
    a->ev_wide.push_back(e3);
  }
  cudaStream_t cin = a->pipe[0], ctr = a->pipe[1], cout = a->pipe[2], cwd = a->pipe[3];
  ENC_CUDA(cudaEventRecord(a->pipe_start, s), "event record");
  for (int i = 0; i < 5; ++i) ENC_CUDA(cudaStreamWaitEvent(a->pipe[i], a->pipe_start, 0), "wait");
  for (size_t c = 0; c < nch; ++c) {
    const size_t b = bound[c], n = bound[c + 1] - b;
    ENC_CUDA(cudaMemcpyAsync(dcopy + b * rb, rays + (size_t)ray_floats * b, n * rb,
                             cudaMemcpyHostToDevice, cin),
             "H2D rays");
    ENC_CUDA(cudaEventRecord(a->ev_in[c], cin), "event record");
    if (od) {
      // widened on a stream of its own, so the trace stream runs its traces
      // back to back (+2 % on the bench batch against widening on the trace
      // stream)
      ENC_CUDA(cudaStreamWaitEvent(cwd, a->ev_in[c], 0), "wait");
      const int e = launch_widen_rays((const float*)(dcopy + b * rb), n, (float*)(din + b * 32),
                                      a->dev.device, cwd);
      if (e) return cuda_fail((cudaError_t)e, "ray widen launch");
      ENC_CUDA(cudaEventRecord(a->ev_wide[c], cwd), "event record");
    }
  }
  for (size_t c = 0; c < nch; ++c) {
    const size_t b = bound[c], n = bound[c + 1] - b;
    // 24-byte rays: consecutive chunks alternate between two trace streams,
    // so a chunk's persistent launch starts while the previous one drains
    // its last rays (1,798 against 1,724 Mrays/s on the bench batch, five
    // interleaved passes on one box).
    cudaStream_t ctr_c = (od && (c & 1)) ? a->pipe[4] : ctr;
    ENC_CUDA(cudaStreamWaitEvent(ctr_c, od ? a->ev_wide[c] : a->ev_in[c], 0), "wait");
    // The chunks' traces run beside the copies.  With 32-byte rays the copy
    // in is the bottleneck: the per-lane closest-hit kernel (10 blocks per
    // SM) slows the copies less than the faster warp-cooperative one (the
    // whole call ran 4-9 % faster with it on the 4.18M-ray bench batch), and
    // only the last chunk, which has no copy in beside it, runs the
    // cooperative kernel to shorten the call's tail (+1.4 %).  With 24-byte
    // rays a chunk's copy in is shorter than its per-lane trace, so every
    // chunk runs the cooperative kernel (1,693 against 1,428 Mrays/s on the
    // bench batch, four passes each).
    L.per_lane = !od && c + 1 < nch;
    int e = any ? launch_any(a->dev, (const float*)(din + b * 32), n, (uint8_t*)(dout + b), L, ctr_c)
                : launch_closest(a->dev, (const float*)(din + b * 32), n,
                                 (enc_hit*)(dout + b * sizeof(enc_hit)), L, ctr_c, nullptr);
    if (e) return cuda_fail((cudaError_t)e, "trace launch");
    ENC_CUDA(cudaEventRecord(a->ev_trace[c], ctr_c), "event record");
    ENC_CUDA(cudaStreamWaitEvent(cout, a->ev_trace[c], 0), "wait");
    ENC_CUDA(cudaMemcpyAsync(static_cast<char*>(out) + b * out_bytes, dout + b * out_bytes,
                             n * out_bytes, cudaMemcpyDeviceToHost, cout),
             "D2H results");
  }
  ENC_CUDA(cudaEventRecord(a->pipe_done, cout), "event record");
  ENC_CUDA(cudaStreamWaitEvent(s, a->pipe_done, 0), "wait");
  return read_status(a, s);
}

}  // namespace

enc_status enc_intersect_closest(enc_accel a, const float* rays, size_t nrays, enc_hit* hits,
                                 const enc_launch_opts* launch, enc_stream stream) {
  return host_form(a, rays, nrays, hits, sizeof(enc_hit), false, 8, launch, stream,
                   "enc_intersect_closest");
}

enc_status enc_intersect_closest_od(enc_accel a, const float* rays, size_t nrays, enc_hit* hits,
                                    const enc_launch_opts* launch, enc_stream stream) {
  return host_form(a, rays, nrays, hits, sizeof(enc_hit), false, 6, launch, stream,
                   "enc_intersect_closest_od");
}

enc_status enc_intersect_any(enc_accel a, const float* rays, size_t nrays, uint8_t* occ,
                             const enc_launch_opts* launch, enc_stream stream) {
  return host_form(a, rays, nrays, occ, 1, true, 8, launch, stream, "enc_intersect_any");
}

enc_status enc_accel_check(enc_accel a, enc_stream stream) {
  if (!a) return ENC_ERR_INVALID_ARG;
  DeviceScope ds(a->dev.device);
  return read_status(a, static_cast<cudaStream_t>(stream));
}

enc_status enc_accel_count_visits(enc_accel a, const float* d_rays, size_t nrays,
                                  uint32_t* d_visits, enc_stream stream) {
  if (!a || (nrays && (!d_rays || !d_visits))) return ENC_ERR_INVALID_ARG;
  if (a->dev.kind != ENC_ACCEL_WBVH) {
    set_error("enc_accel_count_visits: wide BVH only");
    return ENC_ERR_UNSUPPORTED;
  }
  if (nrays == 0) return ENC_OK;
  std::lock_guard<std::mutex> lk(a->mu);
  DeviceScope ds(a->dev.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  enc_status st = grow(&a->d_stage_out, &a->stage_out_bytes, nrays * sizeof(enc_hit));
  if (st) return st;
  Launch L = resolve_launch(nullptr, a->dev.kind, a->dev.width);
  int e = launch_closest(a->dev, d_rays, nrays, (enc_hit*)a->d_stage_out, L, stream, d_visits);
  if (e != 0) return cuda_fail((cudaError_t)e, "count launch");
  return read_status(a, s);
}

// ---------------------------------------------------------------------------
// PhotonMap

enc_status enc_photonmap_create(const float* pos, const float* normal, const float* power,
                                size_t n, int32_t caustic, int32_t device, enc_photonmap* out) {
  if (!out || (n && (!pos || !normal || !power))) {
    set_error("enc_photonmap_create: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  if (n > 0x7fffffffull) {
    set_error("enc_photonmap_create: too many photons");
    return ENC_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_error("enc_photonmap_create: no such CUDA device");
    return ENC_ERR_INVALID_ARG;
  }
  DeviceScope ds(device);
  enc_photonmap m = new (std::nothrow) enc_photonmap_s();
  if (!m) return ENC_ERR_OUT_OF_MEMORY;
  DevPhotonMap& d = m->dev;
  d.caustic = caustic ? 1 : 0;
  d.device = device;
  d.n = (uint32_t)n;
  cudaError_t e = cudaSuccess;
  try {
    PhotonHost h;
    build_photon_tree(pos, normal, power, n, &h);
    d.nnodes = (uint32_t)h.nodes.size();
    d.depth = h.depth;
    d.nlevels = h.nlevels;
    for (int l = 0; l < kPhotonMaxLevels; ++l) {
      d.lvl_count[l] = h.lvl_count[l];
      d.lvl_off[l] = h.lvl_off[l];
      d.lvl_pad[l] = h.lvl_pad[l];
    }
    d.box_floats = h.box.size();
    d.leaf_words = h.leaf.size();
    e = upload(&d.d_box, h.box.data(), h.box.size());
    if (e == cudaSuccess) e = upload(&d.d_leaf, h.leaf.data(), h.leaf.size());
    if (e == cudaSuccess) e = upload(&d.d_pos4, h.pos4.data(), h.pos4.size());
    if (e == cudaSuccess) e = upload(&d.d_nrm4, h.nrm4.data(), h.nrm4.size());
    if (e == cudaSuccess) e = upload(&d.d_pow4, h.pow4.data(), h.pow4.size());
    if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_status, 16);
    if (e == cudaSuccess) e = cudaMemset(d.d_status, 0, 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_counter, kGatherSlots * sizeof(uint32_t));
  } catch (const std::exception& ex) {
    set_error(std::string("enc_photonmap_create: ") + ex.what());
    e = cudaErrorMemoryAllocation;
  }
  if (e != cudaSuccess) {
    cudaFree(d.d_box);
    cudaFree(d.d_leaf);
    cudaFree(d.d_pos4);
    cudaFree(d.d_nrm4);
    cudaFree(d.d_pow4);
    cudaFree(d.d_status);
    cudaFree(d.d_counter);
    delete m;
    return cuda_fail(e, "enc_photonmap_create");
  }
  *out = m;
  return ENC_OK;
}

enc_status enc_photonmap_create_device(const float* d_pos, const float* d_nrm, const float* d_pow,
                                       size_t n, int32_t caustic, int32_t device,
                                       enc_photonmap* out) {
  if (!out || (n && (!d_pos || !d_nrm || !d_pow))) {
    set_error("enc_photonmap_create_device: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  std::vector<float> pos(3 * n), nrm(3 * n), pw(3 * n);
  {
    DeviceScope ds(device);
    if (n) {
      ENC_CUDA(cudaMemcpy(pos.data(), d_pos, 12 * n, cudaMemcpyDeviceToHost), "D2H photons");
      ENC_CUDA(cudaMemcpy(nrm.data(), d_nrm, 12 * n, cudaMemcpyDeviceToHost), "D2H photons");
      ENC_CUDA(cudaMemcpy(pw.data(), d_pow, 12 * n, cudaMemcpyDeviceToHost), "D2H photons");
    }
  }
  return enc_photonmap_create(pos.data(), nrm.data(), pw.data(), n, caustic, device, out);
}

namespace {

struct PhotonFileHeader {
  char magic[8];
  uint32_t version;
  int32_t caustic;
  uint32_t n, nnodes;
  int32_t depth, nlevels;
  uint32_t lvl_count[kPhotonMaxLevels], lvl_off[kPhotonMaxLevels], lvl_pad[kPhotonMaxLevels];
  uint64_t box_floats, leaf_words;
};
constexpr char kPhotonMagic[8] = {'E', 'N', 'C', 'P', 'H', 'M', '0', '1'};

}  // namespace

enc_status enc_photonmap_serialize(enc_photonmap m, void* buf, size_t cap, size_t* size) {
  if (!m || !size) {
    set_error("enc_photonmap_serialize: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  const DevPhotonMap& d = m->dev;
  PhotonFileHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kPhotonMagic, 8);
  h.version = 1;
  h.caustic = d.caustic;
  h.n = d.n;
  h.nnodes = d.nnodes;
  h.depth = d.depth;
  h.nlevels = d.nlevels;
  for (int l = 0; l < kPhotonMaxLevels; ++l) {
    h.lvl_count[l] = d.lvl_count[l];
    h.lvl_off[l] = d.lvl_off[l];
    h.lvl_pad[l] = d.lvl_pad[l];
  }
  h.box_floats = d.box_floats;
  h.leaf_words = d.leaf_words;
  const size_t body = 4 * h.box_floats + 4 * h.leaf_words + 3 * 16 * (size_t)h.n;
  *size = sizeof(h) + body;
  if (!buf) return ENC_OK;
  if (cap < *size) {
    set_error("enc_photonmap_serialize: buffer smaller than the size the call reports");
    return ENC_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(m->mu);
  DeviceScope ds(d.device);
  char* p = static_cast<char*>(buf);
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  const void* src[5] = {d.d_box, d.d_leaf, d.d_pos4, d.d_nrm4, d.d_pow4};
  const size_t bytes[5] = {4 * h.box_floats, 4 * h.leaf_words, 16 * (size_t)h.n,
                           16 * (size_t)h.n, 16 * (size_t)h.n};
  for (int i = 0; i < 5; ++i) {
    if (bytes[i]) ENC_CUDA(cudaMemcpy(p, src[i], bytes[i], cudaMemcpyDeviceToHost), "read photon map");
    p += bytes[i];
  }
  return ENC_OK;
}

enc_status enc_photonmap_deserialize(const void* buf, size_t size, int32_t device,
                                     enc_photonmap* out) {
  if (!buf || !out) {
    set_error("enc_photonmap_deserialize: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  PhotonFileHeader h;
  if (size < sizeof(h)) {
    set_error("enc_photonmap_deserialize: shorter than the header");
    return ENC_ERR_INVALID_ARG;
  }
  std::memcpy(&h, buf, sizeof(h));
  auto bad = [](const char* why) {
    set_error(std::string("enc_photonmap_deserialize: ") + why);
    return ENC_ERR_INVALID_ARG;
  };
  if (std::memcmp(h.magic, kPhotonMagic, 8) != 0 || h.version != 1)
    return bad("not a serialised photon map of this version");
  if (h.nlevels < 0 || h.nlevels > kPhotonMaxLevels || h.n > 0x7fffffffu ||
      (h.n > 0 && h.nlevels < 1))
    return bad("level count or photon count out of range");
  const size_t body = 4 * h.box_floats + 4 * h.leaf_words + 3 * 16 * (size_t)h.n;
  if (size != sizeof(h) + body) return bad("sizes do not agree");
  for (int l = 0; l < h.nlevels; ++l) {
    if (h.lvl_count[l] > h.lvl_pad[l] || (uint64_t)h.lvl_off[l] + 6ull * h.lvl_pad[l] > h.box_floats)
      return bad("a box level lies outside the box array");
  }
  if (h.nlevels > 0 && h.leaf_words != 2ull * h.lvl_count[0]) return bad("leaf table size");
  // every leaf's photon range must lie inside the photon arrays, at most a
  // warp's 32 photons: the gather reads photons by these ranges
  const uint32_t* leaf = reinterpret_cast<const uint32_t*>(static_cast<const char*>(buf) +
                                                           sizeof(h) + 4 * h.box_floats);
  for (uint64_t i = 0; i < h.leaf_words / 2; ++i) {
    uint32_t b, e;
    std::memcpy(&b, leaf + 2 * i, 4);
    std::memcpy(&e, leaf + 2 * i + 1, 4);
    if (b > e || e > h.n || e - b > 32) return bad("a leaf's photon range is out of bounds");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return bad("no such CUDA device");
  DeviceScope ds(device);
  enc_photonmap m = new (std::nothrow) enc_photonmap_s();
  if (!m) return ENC_ERR_OUT_OF_MEMORY;
  DevPhotonMap& d = m->dev;
  d.caustic = h.caustic ? 1 : 0;
  d.device = device;
  d.n = h.n;
  d.nnodes = h.nnodes;
  d.depth = h.depth;
  d.nlevels = h.nlevels;
  for (int l = 0; l < kPhotonMaxLevels; ++l) {
    d.lvl_count[l] = h.lvl_count[l];
    d.lvl_off[l] = h.lvl_off[l];
    d.lvl_pad[l] = h.lvl_pad[l];
  }
  d.box_floats = h.box_floats;
  d.leaf_words = h.leaf_words;
  const char* p = static_cast<const char*>(buf) + sizeof(h);
  const float* fp = reinterpret_cast<const float*>(p);
  cudaError_t e = upload(&d.d_box, fp, h.box_floats);
  p += 4 * h.box_floats;
  if (e == cudaSuccess) e = upload(&d.d_leaf, reinterpret_cast<const uint32_t*>(p), h.leaf_words);
  p += 4 * h.leaf_words;
  float** dst[3] = {&d.d_pos4, &d.d_nrm4, &d.d_pow4};
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
    e = upload(dst[i], reinterpret_cast<const float*>(p), 4 * (size_t)h.n);
    p += 16 * (size_t)h.n;
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_status, 16);
  if (e == cudaSuccess) e = cudaMemset(d.d_status, 0, 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d.d_counter, kGatherSlots * sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaFree(d.d_box);
    cudaFree(d.d_leaf);
    cudaFree(d.d_pos4);
    cudaFree(d.d_nrm4);
    cudaFree(d.d_pow4);
    cudaFree(d.d_status);
    cudaFree(d.d_counter);
    delete m;
    return cuda_fail(e, "enc_photonmap_deserialize");
  }
  *out = m;
  return ENC_OK;
}

enc_status enc_photonmap_destroy(enc_photonmap m) {
  if (!m) return ENC_OK;
  DeviceScope ds(m->dev.device);
  cudaFree(m->dev.d_box);
  cudaFree(m->dev.d_leaf);
  cudaFree(m->dev.d_pos4);
  cudaFree(m->dev.d_nrm4);
  cudaFree(m->dev.d_pow4);
  cudaFree(m->dev.d_status);
  cudaFree(m->dev.d_counter);
  cudaFree(m->d_stage);
  delete m;
  return ENC_OK;
}

namespace {
enc_status gather_args(enc_photonmap m, size_t nq, int32_t k, float max_dist, const void* a,
                       const void* b, const void* c, const char* where) {
  if (!m || (nq && (!a || !b || !c))) {
    set_error(std::string(where) + ": null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (k < 0 || !(max_dist >= 0.0f) || nq > 0x7fffffffull) {
    set_error(std::string(where) + ": k must be >= 0, max_dist >= 0");
    return ENC_ERR_INVALID_ARG;
  }
  if (k > 256) {
    set_error(std::string(where) + ": k > 256 is not built");
    return ENC_ERR_UNSUPPORTED;
  }
  return ENC_OK;
}

enc_status pmap_status(enc_photonmap m, cudaStream_t s) {
  ENC_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  uint32_t st = 0;
  ENC_CUDA(cudaMemcpy(&st, m->dev.d_status, 4, cudaMemcpyDeviceToHost), "read status");
  if (st) {
    cudaMemset(m->dev.d_status, 0, 4);
    set_error("gather stopped at a loop bound");
    return ENC_ERR_WATCHDOG;
  }
  return ENC_OK;
}
}  // namespace

enc_status enc_photonmap_check(enc_photonmap m, enc_stream stream) {
  if (!m) return ENC_ERR_INVALID_ARG;
  DeviceScope ds(m->dev.device);
  return pmap_status(m, static_cast<cudaStream_t>(stream));
}

enc_status enc_photonmap_radiance_device(enc_photonmap m, const float* d_qpos, const float* d_qnrm,
                                         size_t nq, int32_t k, float max_dist, int32_t flags,
                                         float* d_rgb, enc_stream stream) {
  enc_status st = gather_args(m, nq, k, max_dist, d_qpos, d_qnrm, d_rgb, "enc_photonmap_radiance_device");
  if (st) return st;
  DeviceScope ds(m->dev.device);
  int e = launch_radiance(m->dev, d_qpos, d_qnrm, nq, k, max_dist, flags, d_rgb, stream);
  if (e) return cuda_fail((cudaError_t)e, "gather launch");
  return ENC_OK;
}

enc_status enc_photonmap_count_visits(enc_photonmap m, const float* d_qpos, const float* d_qnrm,
                                      size_t nq, int32_t k, float max_dist, int32_t flags,
                                      float* d_rgb, uint32_t* d_visits, enc_stream stream) {
  enc_status st = gather_args(m, nq, k, max_dist, d_qpos, d_qnrm, d_rgb, "enc_photonmap_count_visits");
  if (st) return st;
  if (nq && !d_visits) return ENC_ERR_INVALID_ARG;
  DeviceScope ds(m->dev.device);
  int e = launch_radiance_counted(m->dev, d_qpos, d_qnrm, nq, k, max_dist, flags, d_rgb, d_visits,
                                  stream);
  if (e) return cuda_fail((cudaError_t)e, "gather launch");
  return pmap_status(m, static_cast<cudaStream_t>(stream));
}

enc_status enc_photonmap_radiance(enc_photonmap m, const float* qpos, const float* qnrm, size_t nq,
                                  int32_t k, float max_dist, int32_t flags, float* rgb,
                                  enc_stream stream) {
  enc_status st = gather_args(m, nq, k, max_dist, qpos, qnrm, rgb, "enc_photonmap_radiance");
  if (st || nq == 0) return st;
  std::lock_guard<std::mutex> lk(m->mu);
  DeviceScope ds(m->dev.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t b3 = nq * 3 * sizeof(float);
  st = grow(&m->d_stage, &m->stage_bytes, 3 * b3);
  if (st) return st;
  float* dq = (float*)m->d_stage;
  float* dn = dq + 3 * nq;
  float* dr = dn + 3 * nq;
  ENC_CUDA(cudaMemcpyAsync(dq, qpos, b3, cudaMemcpyHostToDevice, s), "H2D queries");
  ENC_CUDA(cudaMemcpyAsync(dn, qnrm, b3, cudaMemcpyHostToDevice, s), "H2D normals");
  int e = launch_radiance(m->dev, dq, dn, nq, k, max_dist, flags, dr, stream);
  if (e) return cuda_fail((cudaError_t)e, "gather launch");
  ENC_CUDA(cudaMemcpyAsync(rgb, dr, b3, cudaMemcpyDeviceToHost, s), "D2H radiance");
  return pmap_status(m, s);
}

enc_status enc_photonmap_nearest(enc_photonmap m, const float* qpos, const float* qnrm, size_t nq,
                                 int32_t k, float max_dist, int32_t flags, int32_t* idx, float* d2,
                                 int32_t* count, enc_stream stream) {
  enc_status st = gather_args(m, nq, k, max_dist, qpos, qnrm, idx, "enc_photonmap_nearest");
  if (st || nq == 0) return st;
  if (!d2 || !count) return ENC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  DeviceScope ds(m->dev.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t b3 = nq * 3 * sizeof(float);
  const size_t bk = nq * (size_t)k * 4;
  st = grow(&m->d_stage, &m->stage_bytes, 2 * b3 + 2 * bk + nq * 4);
  if (st) return st;
  char* base = (char*)m->d_stage;
  float* dq = (float*)base;
  float* dn = (float*)(base + b3);
  int32_t* di = (int32_t*)(base + 2 * b3);
  float* dd = (float*)(base + 2 * b3 + bk);
  int32_t* dc = (int32_t*)(base + 2 * b3 + 2 * bk);
  ENC_CUDA(cudaMemcpyAsync(dq, qpos, b3, cudaMemcpyHostToDevice, s), "H2D queries");
  ENC_CUDA(cudaMemcpyAsync(dn, qnrm, b3, cudaMemcpyHostToDevice, s), "H2D normals");
  int e = launch_nearest(m->dev, dq, dn, nq, k, max_dist, flags, di, dd, dc, stream);
  if (e) return cuda_fail((cudaError_t)e, "gather launch");
  if (bk) {
    ENC_CUDA(cudaMemcpyAsync(idx, di, bk, cudaMemcpyDeviceToHost, s), "D2H idx");
    ENC_CUDA(cudaMemcpyAsync(d2, dd, bk, cudaMemcpyDeviceToHost, s), "D2H d2");
  }
  ENC_CUDA(cudaMemcpyAsync(count, dc, nq * 4, cudaMemcpyDeviceToHost, s), "D2H count");
  return pmap_status(m, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Multi-scene batched launch

struct enc_batch_s {
  enc::MultiLaunch m;
  enc::Launch L;
  SceneDesc* d_scenes = nullptr;
  BatchDesc* d_batches = nullptr;
  uint32_t* d_starts = nullptr;
  uint32_t* d_words = nullptr;  // queue head, status
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::mutex mu;
};

namespace {
void batch_free(enc_batch b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  cudaFree(b->d_scenes);
  cudaFree(b->d_batches);
  cudaFree(b->d_starts);
  cudaFree(b->d_words);
  delete b;
}
}  // namespace

extern "C" {

enc_status enc_batch_create(const enc_batch_item* items, uint32_t nitems,
                            const enc_launch_opts* launch, enc_batch* out) {
  if (!out || (nitems && !items)) {
    set_error("enc_batch_create: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  if (nitems == 0) {
    set_error("enc_batch_create: no batches");
    return ENC_ERR_INVALID_ARG;
  }
  const DevAccel* first = accel_device_view(items[0].accel);
  if (!first) {
    set_error("enc_batch_create: null accelerator");
    return ENC_ERR_INVALID_ARG;
  }
  Launch L = resolve_launch(launch, ENC_ACCEL_WBVH, first->width);
  if (L.block % 32 != 0 || L.block > 128 || (L.stack != 0 && L.stack < 2) || L.stack > 64 ||
      L.chunk < 1) {
    set_error("enc_batch_create: launch options out of range");
    return ENC_ERR_INVALID_ARG;
  }
  std::vector<SceneDesc> scenes;
  std::vector<const DevAccel*> uniq;
  std::vector<BatchDesc> batches(nitems);
  std::vector<uint32_t> starts(nitems + 1);
  uint64_t pos = 0;
  int depth = 8;
  for (uint32_t i = 0; i < nitems; ++i) {
    const DevAccel* a = accel_device_view(items[i].accel);
    if (!a || (items[i].nrays && (!items[i].d_rays || !items[i].d_hits))) {
      set_error("enc_batch_create: item " + std::to_string(i) + " has a null accelerator or buffer");
      return ENC_ERR_INVALID_ARG;
    }
    if (a->kind != ENC_ACCEL_WBVH || a->width != first->width ||
        a->predicate != first->predicate || a->device != first->device) {
      set_error("enc_batch_create: every item needs a wide BVH of the same width, predicate and device");
      return ENC_ERR_INVALID_ARG;
    }
    uint32_t si = 0;
    while (si < uniq.size() && uniq[si] != a) ++si;
    if (si == uniq.size()) {
      uniq.push_back(a);
      scenes.push_back(SceneDesc{static_cast<const uint8_t*>(a->d_nodes), a->d_tris, a->nnodes,
                                 a->ntris});
      depth = std::max(depth, a->tree_depth);
    }
    batches[i] = BatchDesc{items[i].d_rays, items[i].d_hits, si, items[i].nrays, (uint32_t)pos, 0};
    starts[i] = (uint32_t)pos;
    pos += ((uint64_t)items[i].nrays + L.chunk - 1) / L.chunk * L.chunk;
    if (pos > 0x7fffffffull) {
      set_error("enc_batch_create: more than 2^31 rays in one batch table");
      return ENC_ERR_INVALID_ARG;
    }
  }
  starts[nitems] = (uint32_t)pos;
  DeviceScope ds(first->device);
  enc_batch b = new (std::nothrow) enc_batch_s();
  if (!b) return ENC_ERR_OUT_OF_MEMORY;
  cudaError_t e = upload(&b->d_scenes, scenes.data(), scenes.size());
  if (e == cudaSuccess) e = upload(&b->d_batches, batches.data(), batches.size());
  if (e == cudaSuccess) e = upload(&b->d_starts, starts.data(), starts.size());
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_words, 16);
  if (e == cudaSuccess) e = cudaMemset(b->d_words, 0, 16);
  if (e != cudaSuccess) {
    batch_free(b);
    return cuda_fail(e, "enc_batch_create");
  }
  b->L = L;
  MultiLaunch& m = b->m;
  m.d_scenes = b->d_scenes;
  m.d_batches = b->d_batches;
  m.d_starts = b->d_starts;
  m.nbatches = nitems;
  m.total = (uint32_t)pos;
  m.width = first->width;
  m.predicate = first->predicate;
  m.device = first->device;
  m.stack_depth = depth;
  m.d_counter = b->d_words;
  m.d_status = b->d_words + 1;
  *out = b;
  return ENC_OK;
}

enc_status enc_batch_launch(enc_batch b, enc_stream stream) {
  if (!b) return ENC_ERR_INVALID_ARG;
  DeviceScope ds(b->m.device);
  int e = launch_multi_closest(b->m, b->L, stream);
  if (e) return cuda_fail((cudaError_t)e, "enc_batch_launch");
  return ENC_OK;
}

enc_status enc_batch_launch_graph(enc_batch b, enc_stream stream) {
  if (!b) return ENC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceScope ds(b->m.device);
  if (!b->exec) {
    ENC_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "stream create");
    ENC_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed), "begin capture");
    int le = launch_multi_closest(b->m, b->L, b->cap);
    cudaGraph_t g = nullptr;
    cudaError_t ee = cudaStreamEndCapture(b->cap, &g);
    if (le) {
      if (g) cudaGraphDestroy(g);
      return cuda_fail((cudaError_t)le, "enc_batch_launch_graph: capture");
    }
    if (ee != cudaSuccess) return cuda_fail(ee, "enc_batch_launch_graph: end capture");
    b->graph = g;
    ENC_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
  }
  ENC_CUDA(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)), "graph launch");
  return ENC_OK;
}

enc_status enc_batch_check(enc_batch b, enc_stream stream) {
  if (!b) return ENC_ERR_INVALID_ARG;
  DeviceScope ds(b->m.device);
  ENC_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "cudaStreamSynchronize");
  uint32_t st = 0;
  ENC_CUDA(cudaMemcpy(&st, b->m.d_status, 4, cudaMemcpyDeviceToHost), "read status");
  if (st) {
    cudaMemset(b->m.d_status, 0, 4);
    set_error("batched launch stopped a ray at a loop bound (status bits " + std::to_string(st) + ")");
    return ENC_ERR_WATCHDOG;
  }
  return ENC_OK;
}

enc_status enc_batch_destroy(enc_batch b) {
  if (!b) return ENC_OK;
  DeviceScope ds(b->m.device);
  batch_free(b);
  return ENC_OK;
}

}  // extern "C"
