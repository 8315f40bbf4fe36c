// enc_intersect_closest_noalloc: closest hit from host buffers without any
// device allocation.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree at query
// time.  A host application whose framework already owns the device memory
// (a caching allocator has reserved the pool, so a raw cudaMalloc fails or
// fragments it), or a frame loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree may cause, can build the accelerator
// once at start-up and then answer queries through this call, which touches
// no allocator.  enc_intersect_closest grows staging buffers with cudaMalloc
// on demand and so cannot serve them.
//
// The rays in, the hits out, the work-queue head and the status word live in
// one file-scope __device__ array of fixed size (about 3 MiB, held by every
// GPU that loads this library until the process exits).  A batch may hold at
// most ENC_NOALLOC_MAX_RAYS rays; larger batches are rejected.  The device
// address of the array is looked up with cudaGetSymbolAddress once per
// device, on the first call made for that device, with that device current;
// make that first call before any stream capture.  All calls share the one
// array, which keeps the contents of the last call: the queue head and the
// status word are cleared on every call.  Calls from this process are
// serialised by a mutex and each returns only after its stream has drained;
// calls that overlap on the GPU (for instance from stream captures replayed
// concurrently) would race on the array.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"

namespace enc {
namespace {

constexpr size_t kMaxRays = ENC_NOALLOC_MAX_RAYS;
constexpr size_t kRaysOff = 256;  // words 0 and 1: queue head, status
constexpr size_t kHitsOff = kRaysOff + kMaxRays * 32;
constexpr size_t kScratchBytes = kHitsOff + kMaxRays * sizeof(enc_hit);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
unsigned char* g_noalloc_ptr[kMaxDevices] = {nullptr};

}  // namespace
}  // namespace enc

using namespace enc;

extern "C" enc_status enc_intersect_closest_noalloc(enc_accel accel, const float* rays,
                                                    size_t nrays, enc_hit* hits,
                                                    enc_stream stream) {
  const DevAccel* a = accel_device_view(accel);
  if (!a || (nrays && (!rays || !hits))) {
    set_error("enc_intersect_closest_noalloc: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays > kMaxRays) {
    set_error("enc_intersect_closest_noalloc: " + std::to_string(nrays) +
              " rays exceed the fixed scratch of ENC_NOALLOC_MAX_RAYS = " +
              std::to_string(kMaxRays) + " rays; split the batch or use enc_intersect_closest");
    return ENC_ERR_INVALID_ARG;
  }
  if (a->kind != ENC_ACCEL_WBVH) {
    set_error("enc_intersect_closest_noalloc: wide-BVH accelerators only");
    return ENC_ERR_UNSUPPORTED;
  }
  if (a->device < 0 || a->device >= kMaxDevices) {
    set_error("enc_intersect_closest_noalloc: device ordinal out of range");
    return ENC_ERR_INVALID_ARG;
  }
  if (nrays == 0) return ENC_OK;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != a->device && cudaSetDevice(a->device) != cudaSuccess) {
    set_error("enc_intersect_closest_noalloc: cudaSetDevice failed");
    return ENC_ERR_CUDA;
  }
  enc_status st = ENC_OK;
  cudaError_t e = cudaSuccess;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* base = g_noalloc_ptr[a->device];
  if (!base) {
    // Host code cannot use g_noalloc_scratch's address directly (it names a
    // host-side stand-in); ask the runtime for the device address.
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&base), g_noalloc_scratch);
    if (e == cudaSuccess) g_noalloc_ptr[a->device] = base;
  }
  uint32_t status = 0;
  if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, 2 * sizeof(uint32_t), s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + kRaysOff, rays, nrays * 32, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    Launch L = resolve_launch(nullptr, a->kind, a->width);
    int le = launch_closest_external_scratch(
        *a, reinterpret_cast<const float*>(base + kRaysOff), nrays,
        reinterpret_cast<enc_hit*>(base + kHitsOff), L, stream,
        reinterpret_cast<uint32_t*>(base), reinterpret_cast<uint32_t*>(base) + 1);
    e = (cudaError_t)le;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hits, base + kHitsOff, nrays * sizeof(enc_hit), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&status, base + sizeof(uint32_t), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(std::string("enc_intersect_closest_noalloc: ") + cudaGetErrorString(e));
    st = ENC_ERR_CUDA;
  } else if (status != 0) {
    set_error("enc_intersect_closest_noalloc: kernel stopped at a loop bound (status bits " +
              std::to_string(status) + ")");
    st = ENC_ERR_WATCHDOG;
  }
  if (prev >= 0 && prev != a->device) cudaSetDevice(prev);
  return st;
}
