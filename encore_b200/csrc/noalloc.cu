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
// most ENC_NOALLOC_MAX_RAYS rays; larger batches are rejected.
//
// The runtime creates the array when this file's module is loaded on a
// device, and modules load lazily: the first cudaGetSymbolAddress on the
// array does it, and that allocates device memory.  So the look-up happens
// in noalloc_prepare, which enc_accel_build calls for the accelerator's
// device (with that device current), where allocation is allowed.  It also
// launches the traversal kernel this call uses once over an empty batch, so
// that kernel's module is loaded and the context's local memory is sized for
// it before any query.  A query call only reads the address found then, and
// fails if there is none.
//
// All calls share the one array, which keeps the contents of the last call:
// the queue head and the status word are cleared on every call.  Calls that
// overlapped on the GPU would race on the array, so this entry point
// serialises its calls with a process-wide mutex, and each call returns only
// after its stream has drained (it copies the status word back and waits).
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
// Per device, the traversal kernel variants already run once: bit
// (width index) * 2 + predicate, width index 0, 1, 2 for widths 2, 4, 8.
uint32_t g_noalloc_warm[kMaxDevices] = {0};

}  // namespace

int noalloc_prepare(const DevAccel& a) {
  if (a.kind != ENC_ACCEL_WBVH || a.device < 0 || a.device >= kMaxDevices) return 0;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  unsigned char* base = g_noalloc_ptr[a.device];
  if (!base) {
    // Host code cannot use g_noalloc_scratch's address directly (it names a
    // host-side stand-in); ask the runtime for the device address.  The
    // caller has made a.device current.
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&base), g_noalloc_scratch);
    if (e != cudaSuccess) return (int)e;
  }
  const int wi = a.width == 2 ? 0 : (a.width == 4 ? 1 : 2);
  const uint32_t bit = 1u << (wi * 2 + (a.predicate == ENC_PRED_REFERENCE ? 0 : 1));
  if (!(g_noalloc_warm[a.device] & bit)) {
    const int e = warm_closest_kernel(a, reinterpret_cast<uint32_t*>(base),
                                      reinterpret_cast<uint32_t*>(base) + 1);
    if (e != 0) return e;
    g_noalloc_warm[a.device] |= bit;
  }
  g_noalloc_ptr[a.device] = base;
  return 0;
}

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
    // set up by enc_accel_build; looking it up now could allocate
    if (prev >= 0 && prev != a->device) cudaSetDevice(prev);
    set_error("enc_intersect_closest_noalloc: the fixed scratch of this device was not set up "
              "when the accelerator was built");
    return ENC_ERR_CUDA;
  }
  uint32_t status = 0;
  e = cudaMemsetAsync(base, 0, 2 * sizeof(uint32_t), s);
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
