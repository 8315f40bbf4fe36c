// Serving loop: resident scene pool, admission by slot capacity and HBM
// budget, continuous batching into fused multi-scene launches.
//
// Threads.  submit() only queues: a request is split into pieces of at most
// a slot's ray capacity, so a request larger than one slot runs over several
// rounds.  The scheduler thread waits for a free slot and queued pieces,
// admits pieces in arrival order while they fit the slot's ray capacity, and
// enqueues on the slot's stream: the rays' copies in, the batch tables, one
// multi-scene closest-hit launch and one any-hit launch, the result copies
// out, one status word per piece, and an event.  It then goes back for the
// next group at once, so requests that arrive while a group is on the GPU
// form the next group and run alongside it on another stream.  The
// completion thread polls the in-flight events, stamps each piece's request
// (done once its last piece is; failed if any piece failed) and frees the
// slot.  Waiters block on a condition variable.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace enc {
namespace {

constexpr uint32_t kMaxScenes = 4096;
constexpr uint32_t kMaxReqPerSlot = 1024;

double steady_now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  uint64_t id = 0;
  uint32_t scene = 0;
  int kind = ENC_REQ_CLOSEST;
  const float* rays = nullptr;
  uint64_t n = 0;
  void* out = nullptr;
  double t_submit = 0, t_start = 0, t_done = 0;
  int status = ENC_OK;
  uint32_t pieces_left = 0;  // pieces not finished yet
  bool running = false;      // some piece has been admitted
  bool done = false;
};

// A contiguous range of a request's rays that fits one slot.
struct Piece {
  Request* r = nullptr;
  uint64_t off = 0;
  uint64_t n = 0;
};

struct Slot {
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  char* d_rays = nullptr;    // capacity * 32 bytes
  char* d_out = nullptr;     // capacity * 16 bytes
  BatchDesc* d_tab = nullptr;  // closest table, then any table (kMaxReqPerSlot each)
  uint32_t* d_starts = nullptr;
  uint32_t* d_words = nullptr;  // queue head closest, queue head any
  uint32_t* d_bstat = nullptr;  // per-piece status: closest pieces, then any pieces
  BatchDesc* h_tab = nullptr;   // pinned staging of the tables
  uint32_t* h_starts = nullptr;
  uint32_t* h_bstat = nullptr;  // pinned copy of the per-piece status words
  bool failed = false;          // the round could not be enqueued
  std::vector<Piece> pieces;
  std::vector<uint32_t> piece_word;  // each piece's index into h_bstat
  bool busy = false;
};

// Scene-table facts a round needs, read under the server lock when the
// round is formed (enc_server_add_scene writes them under the same lock).
struct RoundView {
  int width = 8, predicate = 0, depth = 8;
};

}  // namespace
}  // namespace enc

using namespace enc;

struct enc_server_s {
  enc_server_opts o{};
  Launch L;
  int device = 0;
  uint64_t capacity = 0;
  std::vector<const DevAccel*> scenes;
  SceneDesc* d_scenes = nullptr;
  uint64_t scene_bytes = 0, slot_bytes = 0;
  int width = 0, predicate = 0, depth = 8;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<Piece> pending;
  std::deque<int> inflight;
  std::unordered_map<uint64_t, Request*> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread sched, comp;
};

namespace {

cudaError_t enqueue_round(enc_server S, Slot& sl, const RoundView& v) {
  const uint32_t chunk = (uint32_t)S->L.chunk;
  uint64_t off = 0;
  uint32_t nc = 0, na = 0;
  uint64_t qc = 0, qa = 0;
  BatchDesc* tc = sl.h_tab;
  BatchDesc* ta = sl.h_tab + kMaxReqPerSlot;
  uint32_t* sc = sl.h_starts;
  uint32_t* sa = sl.h_starts + kMaxReqPerSlot + 1;
  cudaError_t e = cudaSuccess;
  sl.piece_word.clear();
  for (const Piece& pc : sl.pieces) {
    const Request* r = pc.r;
    e = cudaMemcpyAsync(sl.d_rays + off * 32, r->rays + 8 * pc.off, pc.n * 32,
                        cudaMemcpyHostToDevice, sl.s);
    if (e != cudaSuccess) return e;
    BatchDesc d{reinterpret_cast<const float*>(sl.d_rays + off * 32), sl.d_out + off * 16,
                r->scene, (uint32_t)pc.n, 0, (uint32_t)r->kind};
    if (r->kind == ENC_REQ_CLOSEST) {
      d.start = (uint32_t)qc;
      sc[nc] = (uint32_t)qc;
      sl.piece_word.push_back(nc);
      tc[nc++] = d;
      qc += (pc.n + chunk - 1) / chunk * chunk;
    } else {
      d.start = (uint32_t)qa;
      sa[na] = (uint32_t)qa;
      sl.piece_word.push_back(kMaxReqPerSlot + na);
      ta[na++] = d;
      qa += (pc.n + chunk - 1) / chunk * chunk;
    }
    off += pc.n;
  }
  sc[nc] = (uint32_t)qc;
  sa[na] = (uint32_t)qa;
  e = cudaMemcpyAsync(sl.d_tab, sl.h_tab, 2 * kMaxReqPerSlot * sizeof(BatchDesc),
                      cudaMemcpyHostToDevice, sl.s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sl.d_starts, sl.h_starts, 2 * (kMaxReqPerSlot + 1) * sizeof(uint32_t),
                        cudaMemcpyHostToDevice, sl.s);
  if (e == cudaSuccess) e = cudaMemsetAsync(sl.d_bstat, 0, 2 * kMaxReqPerSlot * 4, sl.s);
  if (e != cudaSuccess) return e;
  MultiLaunch m;
  m.d_scenes = S->d_scenes;
  m.width = v.width;
  m.predicate = v.predicate;
  m.device = S->device;
  m.stack_depth = v.depth;
  m.d_status = sl.d_words + 2;
  if (nc) {
    m.d_batches = sl.d_tab;
    m.d_starts = sl.d_starts;
    m.nbatches = nc;
    m.total = (uint32_t)qc;
    m.d_counter = sl.d_words;
    m.d_batch_status = sl.d_bstat;
    int le = launch_multi_closest(m, S->L, sl.s);
    if (le) return (cudaError_t)le;
  }
  if (na) {
    m.d_batches = sl.d_tab + kMaxReqPerSlot;
    m.d_starts = sl.d_starts + kMaxReqPerSlot + 1;
    m.nbatches = na;
    m.total = (uint32_t)qa;
    m.d_counter = sl.d_words + 1;
    m.d_batch_status = sl.d_bstat + kMaxReqPerSlot;
    int le = launch_multi_any(m, S->L, sl.s);
    if (le) return (cudaError_t)le;
  }
  off = 0;
  for (const Piece& pc : sl.pieces) {
    const Request* r = pc.r;
    const size_t rec = r->kind == ENC_REQ_CLOSEST ? sizeof(enc_hit) : 1;
    e = cudaMemcpyAsync(static_cast<char*>(r->out) + pc.off * rec, sl.d_out + off * 16,
                        pc.n * rec, cudaMemcpyDeviceToHost, sl.s);
    if (e != cudaSuccess) return e;
    off += pc.n;
  }
  e = cudaMemcpyAsync(sl.h_bstat, sl.d_bstat, 2 * kMaxReqPerSlot * 4, cudaMemcpyDeviceToHost, sl.s);
  if (e == cudaSuccess) e = cudaEventRecord(sl.ev, sl.s);
  return e;
}

void sched_loop(enc_server S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    int si = -1;
    S->cv_sched.wait(lk, [&] {
      if (S->stop) return true;
      if (S->pending.empty()) return false;
      for (size_t i = 0; i < S->slots.size(); ++i)
        if (!S->slots[i].busy) {
          si = (int)i;
          return true;
        }
      return false;
    });
    if (S->stop) return;
    Slot& sl = S->slots[si];
    sl.pieces.clear();
    sl.failed = false;
    uint64_t used = 0;
    const double t = steady_now();
    while (!S->pending.empty() && sl.pieces.size() < kMaxReqPerSlot) {
      const Piece pc = S->pending.front();
      if (used + pc.n > S->capacity) break;  // next group; arrival order is kept
      S->pending.pop_front();
      if (!pc.r->running) {
        pc.r->running = true;
        pc.r->t_start = t;
      }
      sl.pieces.push_back(pc);
      used += pc.n;
    }
    if (sl.pieces.empty()) continue;
    const RoundView v{S->width, S->predicate, S->depth};
    sl.busy = true;
    lk.unlock();
    cudaError_t e = enqueue_round(S, sl, v);
    lk.lock();
    if (e != cudaSuccess) {
      set_error(std::string("server round: ") + cudaGetErrorString(e));
      // let the completion thread finish these pieces with an error once
      // whatever was enqueued has drained
      sl.failed = true;
      cudaEventRecord(sl.ev, sl.s);
    }
    S->inflight.push_back(si);
    S->cv_done.notify_all();
  }
}

void comp_loop(enc_server S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    S->cv_done.wait(lk, [&] { return S->stop || !S->inflight.empty(); });
    if (S->inflight.empty() && S->stop) return;
    std::vector<int> live(S->inflight.begin(), S->inflight.end());
    lk.unlock();
    std::vector<std::pair<int, cudaError_t>> finished;
    for (int si : live) {
      cudaError_t q = cudaEventQuery(S->slots[si].ev);
      if (q != cudaErrorNotReady) finished.push_back({si, q});
    }
    const double t = steady_now();
    if (finished.empty()) std::this_thread::sleep_for(std::chrono::microseconds(20));
    lk.lock();
    for (auto& f : finished) {
      Slot& sl = S->slots[f.first];
      for (size_t i = 0; i < sl.pieces.size(); ++i) {
        Request* r = sl.pieces[i].r;
        int st = ENC_OK;
        if (f.second != cudaSuccess || sl.failed) st = ENC_ERR_CUDA;
        else if (i < sl.piece_word.size() && sl.h_bstat[sl.piece_word[i]]) st = ENC_ERR_WATCHDOG;
        if (st != ENC_OK && r->status == ENC_OK) r->status = st;
        if (--r->pieces_left == 0) {
          r->t_done = t;
          r->done = true;
        }
      }
      sl.pieces.clear();
      sl.busy = false;
      S->inflight.erase(std::find(S->inflight.begin(), S->inflight.end(), f.first));
    }
    if (!finished.empty()) {
      S->cv_done.notify_all();
      S->cv_sched.notify_all();
    }
  }
}

void free_slots(enc_server S) {
  for (Slot& sl : S->slots) {
    if (sl.s) cudaStreamDestroy(sl.s);
    if (sl.ev) cudaEventDestroy(sl.ev);
    cudaFree(sl.d_rays);
    cudaFree(sl.d_out);
    cudaFree(sl.d_tab);
    cudaFree(sl.d_starts);
    cudaFree(sl.d_words);
    cudaFree(sl.d_bstat);
    cudaFreeHost(sl.h_tab);
    cudaFreeHost(sl.h_starts);
    cudaFreeHost(sl.h_bstat);
  }
  S->slots.clear();
  cudaFree(S->d_scenes);
  S->d_scenes = nullptr;
}

}  // namespace

extern "C" {

double enc_server_now(void) { return steady_now(); }

enc_status enc_server_create(const enc_server_opts* opts, enc_server* out) {
  if (!out) return ENC_ERR_INVALID_ARG;
  *out = nullptr;
  enc_server_opts o{};
  if (opts) o = *opts;
  if (o.slots == 0) o.slots = 6;
  if (o.slot_rays == 0) o.slot_rays = 4ull << 20;
  if (o.budget_bytes == 0) o.budget_bytes = 120ull * 1000 * 1000 * 1000;
  if (o.slots > 16 || o.slot_rays > (1ull << 30)) {
    set_error("enc_server_create: slots <= 16 and slot_rays <= 2^30");
    return ENC_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || o.device < 0 || o.device >= ndev) {
    set_error("enc_server_create: no such CUDA device");
    return ENC_ERR_INVALID_ARG;
  }
  enc_server S = new (std::nothrow) enc_server_s();
  if (!S) return ENC_ERR_OUT_OF_MEMORY;
  S->o = o;
  S->device = o.device;
  S->capacity = o.slot_rays;
  S->L = resolve_launch(&o.launch, ENC_ACCEL_WBVH, 8);
  if (S->L.block % 32 != 0 || S->L.block > 128 || S->L.stack > 64 || S->L.chunk < 1) {
    delete S;
    set_error("enc_server_create: launch options out of range");
    return ENC_ERR_INVALID_ARG;
  }
  const uint64_t per_slot = o.slot_rays * 48 + 2 * kMaxReqPerSlot * (sizeof(BatchDesc) + 8) + 64;
  S->slot_bytes = per_slot * o.slots + kMaxScenes * sizeof(SceneDesc);
  if (S->slot_bytes > o.budget_bytes) {
    delete S;
    set_error("enc_server_create: slot buffers alone exceed the HBM budget");
    return ENC_ERR_BUDGET;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(o.device);
  cudaError_t e = cudaMalloc((void**)&S->d_scenes, kMaxScenes * sizeof(SceneDesc));
  S->slots.resize(o.slots);
  for (Slot& sl : S->slots) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_rays, o.slot_rays * 32);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_out, o.slot_rays * 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_tab, 2 * kMaxReqPerSlot * sizeof(BatchDesc));
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_starts, 2 * (kMaxReqPerSlot + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_words, 16);
    if (e == cudaSuccess) e = cudaMemset(sl.d_words, 0, 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_bstat, 2 * kMaxReqPerSlot * 4);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&sl.h_tab, 2 * kMaxReqPerSlot * sizeof(BatchDesc));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&sl.h_starts, 2 * (kMaxReqPerSlot + 1) * 4);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&sl.h_bstat, 2 * kMaxReqPerSlot * 4);
  }
  if (e != cudaSuccess) {
    set_error(std::string("enc_server_create: ") + cudaGetErrorString(e));
    free_slots(S);
    delete S;
    if (prev >= 0) cudaSetDevice(prev);
    return e == cudaErrorMemoryAllocation ? ENC_ERR_OUT_OF_MEMORY : ENC_ERR_CUDA;
  }
  if (prev >= 0) cudaSetDevice(prev);
  S->sched = std::thread(sched_loop, S);
  S->comp = std::thread(comp_loop, S);
  *out = S;
  return ENC_OK;
}

enc_status enc_server_add_scene(enc_server S, enc_accel accel, uint32_t* scene_id) {
  const DevAccel* a = accel_device_view(accel);
  if (!S || !a || !scene_id) return ENC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  if (a->kind != ENC_ACCEL_WBVH || a->device != S->device) {
    set_error("enc_server_add_scene: needs a wide BVH on the server's device");
    return ENC_ERR_INVALID_ARG;
  }
  if (!S->scenes.empty() && (a->width != S->width || a->predicate != S->predicate)) {
    set_error("enc_server_add_scene: all scenes need the same width and predicate");
    return ENC_ERR_INVALID_ARG;
  }
  if (S->scenes.size() >= kMaxScenes) {
    set_error("enc_server_add_scene: scene table full");
    return ENC_ERR_BUDGET;
  }
  if (S->scene_bytes + a->device_bytes + S->slot_bytes > S->o.budget_bytes) {
    set_error("enc_server_add_scene: scene does not fit the HBM budget");
    return ENC_ERR_BUDGET;
  }
  SceneDesc d{static_cast<const uint8_t*>(a->d_nodes), a->d_tris, a->nnodes, a->ntris};
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  cudaError_t e = cudaMemcpy(S->d_scenes + S->scenes.size(), &d, sizeof(d), cudaMemcpyHostToDevice);
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_error(std::string("enc_server_add_scene: ") + cudaGetErrorString(e));
    return ENC_ERR_CUDA;
  }
  if (S->scenes.empty()) {
    S->width = a->width;
    S->predicate = a->predicate;
  }
  S->depth = std::max(S->depth, a->tree_depth);
  *scene_id = (uint32_t)S->scenes.size();
  S->scenes.push_back(a);
  S->scene_bytes += a->device_bytes;
  return ENC_OK;
}

enc_status enc_server_submit(enc_server S, uint32_t scene_id, int32_t kind, const float* rays,
                             uint64_t nrays, void* out, uint64_t* request_id) {
  if (!S || !request_id || (nrays && (!rays || !out))) return ENC_ERR_INVALID_ARG;
  if (kind != ENC_REQ_CLOSEST && kind != ENC_REQ_ANY) return ENC_ERR_INVALID_ARG;
  Request* r = new (std::nothrow) Request();
  if (!r) return ENC_ERR_OUT_OF_MEMORY;
  r->scene = scene_id;
  r->kind = kind;
  r->rays = rays;
  r->n = nrays;
  r->out = out;
  r->t_submit = steady_now();
  std::lock_guard<std::mutex> lk(S->mu);
  if (scene_id >= S->scenes.size()) {
    delete r;
    set_error("enc_server_submit: unknown scene");
    return ENC_ERR_INVALID_ARG;
  }
  r->id = S->next_id++;
  S->reqs[r->id] = r;
  *request_id = r->id;
  if (nrays == 0) {
    r->done = true;
    r->t_start = r->t_done = r->t_submit;
    S->cv_done.notify_all();
    return ENC_OK;
  }
  // pieces of at most one slot's capacity, queued back to back
  for (uint64_t off = 0; off < nrays; off += S->capacity) {
    Piece pc;
    pc.r = r;
    pc.off = off;
    pc.n = std::min<uint64_t>(S->capacity, nrays - off);
    S->pending.push_back(pc);
    ++r->pieces_left;
  }
  S->cv_sched.notify_all();
  return ENC_OK;
}

enc_status enc_server_wait(enc_server S, uint64_t id, double timeout_s, enc_request_info* info) {
  if (!S) return ENC_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) {
    set_error("enc_server_wait: unknown request");
    return ENC_ERR_INVALID_ARG;
  }
  Request* r = it->second;
  if (timeout_s < 0) {
    S->cv_done.wait(lk, [&] { return r->done; });
  } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                  [&] { return r->done; })) {
    return ENC_ERR_NOT_READY;
  }
  if (info) {
    info->submit_s = r->t_submit;
    info->start_s = r->t_start;
    info->done_s = r->t_done;
    info->nrays = r->n;
    info->status = r->status;
    info->kind = r->kind;
  }
  const int st = r->status;
  S->reqs.erase(it);
  delete r;
  if (st != ENC_OK) set_error("request failed");
  return st;
}

enc_status enc_server_cancel(enc_server S, uint64_t id) {
  if (!S) return ENC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return ENC_ERR_INVALID_ARG;
  Request* r = it->second;
  if (r->done) return ENC_OK;
  if (r->running) return ENC_ERR_NOT_READY;
  S->pending.erase(std::remove_if(S->pending.begin(), S->pending.end(),
                                  [&](const Piece& pc) { return pc.r == r; }),
                   S->pending.end());
  r->pieces_left = 0;
  r->status = ENC_ERR_CANCELLED;
  r->done = true;
  r->t_start = r->t_done = steady_now();
  S->cv_done.notify_all();
  return ENC_OK;
}

enc_status enc_server_destroy(enc_server S) {
  if (!S) return ENC_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_sched.notify_all();
  S->cv_done.notify_all();
  S->sched.join();
  // drain launches already enqueued before the completion thread exits
  for (Slot& sl : S->slots)
    if (sl.s) cudaStreamSynchronize(sl.s);
  S->comp.join();
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  free_slots(S);
  if (prev >= 0) cudaSetDevice(prev);
  for (auto& kv : S->reqs) delete kv.second;
  delete S;
  return ENC_OK;
}

}  // extern "C"
