/*
 * encore_b200 — C ABI of the B200 ray-query engine.
 *
 * The engine replaces the reference's CPU query path:
 *   - AccelerationStructure::build / intersect
 *       (ENCORE/src/accelerators/AccelerationStructure.h:47, :63)
 *     as implemented by Kdtree (ENCORE/src/accelerators/Kdtree.cpp:84-200, 682-784)
 *     and Bvh (ENCORE/src/accelerators/BVH.cpp:123-187, 778-884);
 *   - the shadow test PhotonMapperCPU::IsInShadow
 *       (ENCORE/src/renderers/PhotonMapperCPU.cpp:1192-1207);
 *   - PhotonMap::AddPhoton / BalanceAndConstruct / GetNearestNPhotons /
 *     GetRadianceEstimate (ENCORE/src/renderers/PhotonMap.cpp:46-53, 167-221,
 *     76-94 + 224-297, 121-164).
 *
 * Every entry point returns an enc_status; nothing throws across the ABI.
 * Handles are thread-safe for concurrent queries on distinct streams; build
 * and destroy calls must not race with queries on the same handle.
 *
 * Data formats (all FP32, little endian):
 *   triangle soup : 9 floats per triangle (v0, v1, v2); the index in this
 *                   array is the triangle ID (primitive-list order,
 *                   ENCORE/src/scene/Model.cpp:255-264).
 *   ray           : 8 floats (ox, oy, oz, tmin, dx, dy, dz, tmax), 32 bytes.
 *                   A hit must satisfy tmin < t < tmax; the reference's own
 *                   rays are tmin = 0, tmax = +inf (TrianglePrim.cpp:223-224).
 *   hit           : enc_hit, 16 bytes; tri = -1 for a miss.
 *   photon        : position (3 floats), surface normal (3), RGB power (3).
 */
#ifndef ENCORE_B200_H
#define ENCORE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ENC_ABI_VERSION 1

typedef int32_t enc_status;
enum {
  ENC_OK = 0,
  ENC_ERR_INVALID_ARG = 1,   /* null handle/pointer, bad size, bad option */
  ENC_ERR_CUDA = 2,          /* a CUDA runtime call failed (see enc_last_error) */
  ENC_ERR_OUT_OF_MEMORY = 3, /* device or host allocation failed */
  ENC_ERR_WATCHDOG = 4,      /* a kernel hit its bounded-loop limit and stopped */
  ENC_ERR_BUDGET = 5,        /* serving: request larger than the memory budget */
  ENC_ERR_NOT_READY = 6,     /* serving: result not complete yet */
  ENC_ERR_CANCELLED = 7,     /* serving: request cancelled or timed out */
  ENC_ERR_UNSUPPORTED = 8    /* option combination not built */
};

typedef struct enc_hit {
  int32_t tri; /* triangle ID, -1 = miss */
  float t;     /* hit distance as the FP32 predicate computes it */
  float u;     /* alpha (barycentric of v1), TrianglePrim.cpp:219 */
  float v;     /* beta  (barycentric of v2), TrianglePrim.cpp:220 */
} enc_hit;

typedef struct enc_scene_s* enc_scene;
typedef struct enc_accel_s* enc_accel;
typedef struct enc_photonmap_s* enc_photonmap;
typedef void* enc_stream; /* a cudaStream_t; NULL = legacy default stream */

/* Accelerator kinds. */
enum {
  /* Flattened wide BVH, binned-SAH build, child boxes quantised to 8 bits and
   * rounded outward.  The throughput path. */
  ENC_ACCEL_WBVH = 0,
  /* Flattened kd-tree built by the reference's own rules (spatial median,
   * axis depth%3, box-overlap distribution, Kdtree.cpp:299-680) and walked in
   * the reference's traversal order (Kdtree.cpp:682-784).  Bit-exact with the
   * reference's Kdtree at any scene scale, including its degenerate cases. */
  ENC_ACCEL_KDTREE = 1
};

/* Predicate modes. */
enum {
  /* The reference's triangle test op for op: FP32, no FMA contraction, IEEE
   * division, Cross() components with |c| < 0.001 clamped to 0
   * (ENCORE/src/math/Vector3.h:148-161, Vector3.cpp:126-140). */
  ENC_PRED_REFERENCE = 0,
  /* The same FP32 operation order without the clamp (geometric mode). */
  ENC_PRED_NOCLAMP = 1
};

typedef struct enc_build_opts {
  int32_t kind;          /* ENC_ACCEL_* */
  int32_t width;         /* WBVH branching factor: 2, 4 or 8 (0 = 8) */
  int32_t max_leaf_tris; /* WBVH triangles per leaf, 1..4 (0 = 3) */
  int32_t predicate;     /* ENC_PRED_* */
} enc_build_opts;

typedef struct enc_launch_opts {
  int32_t block_threads; /* threads per block, multiple of 32 (0 = tuned default) */
  int32_t blocks_per_sm; /* persistent CTAs per SM (0 = tuned default) */
  int32_t chunk;         /* rays a warp takes from the queue per refill (0 = 32) */
  int32_t stack_depth;   /* traversal stack entries per ray (0 = the tree depth, which
                            always suffices; max 64) */
} enc_launch_opts;

typedef struct enc_accel_info {
  int32_t kind, width, predicate;
  uint32_t ntris;
  uint32_t nnodes;
  uint64_t node_bytes;
  uint64_t tri_bytes;
  uint64_t device_bytes; /* total device memory held by the accelerator */
  double build_seconds;  /* host build + upload wall time */
  float scene_lo[3], scene_hi[3];
} enc_accel_info;

/* Library / device. */
int32_t enc_abi_version(void);
const char* enc_last_error(void); /* thread-local message of the last failure */
enc_status enc_device_count(int32_t* count);

/* Scene: a triangle soup copied to host memory owned by the handle.
 * Replaces the IModel primitive lists that build() walks (Kdtree.cpp:99-114). */
enc_status enc_scene_create(const float* tri_verts, uint32_t ntris, enc_scene* out);
enc_status enc_scene_destroy(enc_scene scene);

/* Scene front-end: the reference's model and scene-file loaders.
 *
 * enc_scene_load_ply = Model::Model(filename, ...) for a .ply file: the mesh
 * read as Model::loadPLY reads it (Model.cpp:396-482; ascii, each face's
 * first three indices), then moved by Model::centerModel (Model.cpp:109-173:
 * scaled so its longest side is `size`, centred on `center`, rotated by
 * `angle_deg` about `axis`) in the reference's float operation order.  Binary
 * little/big-endian PLY files are read too (an extension; same face rule).
 *
 * enc_scene_load_file = Scene::load + Scene::HandleSceneVariable
 * (Scene.cpp:78-209): MODEL lines load PLY meshes, RECT_LIGHT adds the fixed
 * two-triangle ceiling light of RectangleLight (RectangleLight.cpp), SPHERE
 * takes a primitive index but no triangles (the engine traces triangles
 * only), CAMERA / MATERIAL / POINT_LIGHT / BACKGROUND_COLOR are recorded, a
 * token starting with '*' comments out the rest of its line.  Triangles are
 * in primitive-list order; enc_scene_prims gives, per triangle, the
 * reference's primitive index (a RECT_LIGHT's two triangles share one) and
 * material index.  Relative model paths resolve against `model_dir` (NULL =
 * the working directory, as the reference opens them). */
typedef struct enc_model_xform {
  float center[3];
  float size;
  float angle_deg;
  float axis[3];
} enc_model_xform;

typedef struct enc_scene_desc {
  uint32_t ntris, nprims, nmodels, nmaterials, nlights, nspheres, nunknown;
  int32_t has_camera;
  float cam_eye[3], cam_look[3], cam_up[3];
  float cam_fov_deg, cam_aspect, cam_near, cam_far;
  float background[4];
} enc_scene_desc;

#define ENC_LIGHT_RECT 0
#define ENC_LIGHT_POINT 1
typedef struct enc_scene_light {
  int32_t kind;
  float center[3];  /* RECT: the quad's centre; POINT: the position */
  float size;       /* RECT: side length (square in the xz plane); POINT: 0 */
  float color[3];
} enc_scene_light;

enc_status enc_scene_load_ply(const char* path, const enc_model_xform* xform, enc_scene* out);
enc_status enc_scene_load_file(const char* path, const char* model_dir, enc_scene* out);
enc_status enc_scene_desc_get(enc_scene scene, enc_scene_desc* desc);
/* Copies up to `cap` triangles (9 floats each); *ntris = the scene's count. */
enc_status enc_scene_tris(enc_scene scene, float* tri_verts, uint32_t cap, uint32_t* ntris);
/* Per triangle: primitive index and material index (-1 = default material);
 * either pointer may be NULL.  Writes min(cap, ntris) entries. */
enc_status enc_scene_prims(enc_scene scene, int32_t* prim_of_tri, int32_t* material_of_tri,
                           uint32_t cap);
/* Materials as MATERIAL lists them: diffuse rgb, specular rgb, ambient rgb,
 * reflectivity, transparency, refraction index, transmittance (13 floats). */
enc_status enc_scene_materials(enc_scene scene, float* out13, uint32_t cap, uint32_t* n);
enc_status enc_scene_lights(enc_scene scene, enc_scene_light* out, uint32_t cap, uint32_t* n);

/* AccelerationStructure::build (AccelerationStructure.h:47).  Builds on the
 * host, uploads to `device`, returns an accelerator resident in HBM.  The
 * scene may be destroyed afterwards. */
enc_status enc_accel_build(enc_scene scene, const enc_build_opts* opts, int32_t device,
                           enc_accel* out);
enc_status enc_accel_destroy(enc_accel accel);
/* AccelerationStructure::update (AccelerationStructure.h:51; Bvh::update,
 * BVH.cpp:52-121): the same triangles (same count and IDs) at new positions.
 * A wide BVH keeps its tree shape and gets its boxes recomputed bottom-up and
 * re-quantised; a kd layout is rebuilt, as Kdtree::update rebuilds
 * (Kdtree.h:138).  Must not run concurrently with queries on the handle. */
enc_status enc_accel_refit(enc_accel accel, const float* tri_verts, uint32_t ntris);
enc_status enc_accel_info_get(enc_accel accel, enc_accel_info* info);

/* Saving a built accelerator and loading it again without the host build
 * (the reference rebuilds its trees on every run, PhotonMapperCPU.cpp:222-255;
 * a 2M-triangle wide BVH takes over a second to build, a load only its
 * upload).  enc_accel_serialize writes a self-contained byte image (header,
 * nodes, triangle records, leaf order or kd item lists) into `buf`; with
 * buf = NULL it only sets *size.  enc_accel_deserialize checks the header
 * and every section size (ENC_ERR_INVALID_ARG on any mismatch) and uploads
 * the image to `device`; the result answers every query exactly as the saved
 * accelerator did and can be refitted.  The image is host-endian and tied to
 * this library's layout version. */
enc_status enc_accel_serialize(enc_accel accel, void* buf, size_t cap, size_t* size);
enc_status enc_accel_deserialize(const void* buf, size_t size, int32_t device, enc_accel* out);

/* AccelerationStructure::intersect (AccelerationStructure.h:63), batched.
 * Host-buffer form: copies rays in, traces, copies hits out, synchronises
 * `stream` before returning. */
enc_status enc_intersect_closest(enc_accel accel, const float* rays, size_t nrays, enc_hit* hits,
                                 const enc_launch_opts* launch, enc_stream stream);
/* AccelerationStructure::intersect (AccelerationStructure.h:63), batched, on
 * the reference's own ray payload: 6 floats per ray (ox, oy, oz, dx, dy, dz),
 * a Ray's m_Origin and m_Direction (Ray.h:44-45), which carries no distance
 * bounds (a hit needs t > 0 only, TrianglePrim.cpp:222-223).  Host buffers,
 * as enc_intersect_closest; the hits equal that call's on the same rays with
 * tmin = 0 and tmax = +inf, bit for bit.  24 bytes per ray cross PCIe instead
 * of 32; each chunk is widened to the 8-float layout in device memory ahead
 * of its trace. */
enc_status enc_intersect_closest_od(enc_accel accel, const float* rays, size_t nrays,
                                    enc_hit* hits, const enc_launch_opts* launch,
                                    enc_stream stream);
/* Device-buffer form: rays and hits already in device memory; asynchronous
 * on `stream`.  Kernel status is read by enc_accel_check.  Each launch on an
 * accelerator takes the next of its 256 work-queue heads, so at most 256
 * launches on one accelerator may be in flight together; a launch captured
 * into a CUDA graph keeps the head it was captured with. */
enc_status enc_intersect_closest_device(enc_accel accel, const float* d_rays, size_t nrays,
                                        enc_hit* d_hits, const enc_launch_opts* launch,
                                        enc_stream stream);

/* Binned closest hit, device buffers.  The same results as
 * enc_intersect_closest_device, bit for bit; the batch is first binned by a
 * key of each ray's origin cell and direction cell (a counting sort into a
 * permutation in `d_scratch`), and the traversal takes its rays in that
 * order, so the rays of a warp walk similar paths through the tree.  Hits are
 * written at each ray's own index.  Pays for incoherent batches (shuffled
 * bounces); the binning costs three streaming passes over the rays.
 *
 * The key interleaves `origin_bits` bits of the origin cell (over the scene
 * box; bits go to the axis with the widest cells first) with `dir_bits` bits
 * of the direction's octahedral coordinates.  origin_bits + dir_bits <= 20;
 * both 0 = the tuned default.  probe_frac > 0 bins the point
 * o + probe_frac * |scene diagonal| * d instead of the origin.
 *
 * d_scratch: device memory of at least enc_bin_scratch_bytes() bytes,
 * 256-byte aligned, owned by the caller and used on `stream` only until the
 * launch completes (calls that share one scratch buffer must be ordered on
 * one stream).  Both accelerator kinds: the kd-tree parity mode, which
 * walks one ray per thread, gains most from coherent warps.  No counterpart
 * in the reference (one ray per call). */
typedef struct enc_bin_opts {
  int32_t origin_bits;
  int32_t dir_bits;
  float probe_frac;
} enc_bin_opts;
enc_status enc_bin_scratch_bytes(size_t nrays, const enc_bin_opts* bin, size_t* bytes);
/* The two halves of the binned call, for callers that time them apart or
 * trace one binned batch more than once.  enc_bin_rays enqueues the binning
 * on `stream` and sets *d_order to the permutation inside d_scratch (valid
 * until the scratch is reused).  enc_intersect_closest_device_ordered traces
 * ray d_order[q] as the q-th ray of the queue and writes each hit at its
 * ray's index; d_order should be a permutation of 0..nrays-1 (an entry
 * >= nrays is skipped and reported by enc_accel_check as an index out of
 * range). */
enc_status enc_bin_rays(enc_accel accel, const float* d_rays, size_t nrays, void* d_scratch,
                        size_t scratch_bytes, const enc_bin_opts* bin, uint32_t** d_order,
                        enc_stream stream);
enc_status enc_intersect_closest_device_ordered(enc_accel accel, const float* d_rays,
                                                size_t nrays, const uint32_t* d_order,
                                                enc_hit* d_hits, const enc_launch_opts* launch,
                                                enc_stream stream);
enc_status enc_intersect_closest_device_binned(enc_accel accel, const float* d_rays,
                                               size_t nrays, enc_hit* d_hits, void* d_scratch,
                                               size_t scratch_bytes, const enc_bin_opts* bin,
                                               const enc_launch_opts* launch, enc_stream stream);

/* Shadow / any-hit: occluded[i] = 1 iff some triangle is hit with
 * tmin < t < tmax.  This is the boolean PhotonMapperCPU::IsInShadow
 * computes as closest-hit && hitTime < distToLight (PhotonMapperCPU.cpp:1204),
 * answered with an early exit. */
enc_status enc_intersect_any(enc_accel accel, const float* rays, size_t nrays, uint8_t* occluded,
                             const enc_launch_opts* launch, enc_stream stream);
enc_status enc_intersect_any_device(enc_accel accel, const float* d_rays, size_t nrays,
                                    uint8_t* d_occluded, const enc_launch_opts* launch,
                                    enc_stream stream);

/* Waits for `stream` and reports ENC_ERR_WATCHDOG if any kernel this library
 * launched on this accelerator stopped at its loop bound since the last check. */
enc_status enc_accel_check(enc_accel accel, enc_stream stream);

/* Per-ray traversal counters of the last enc_accel_count_visits call:
 * visits[2*i] = nodes visited, visits[2*i+1] = triangles tested. Used for the
 * bytes-per-ray roofline (device buffers, closest-hit traversal). */
enc_status enc_accel_count_visits(enc_accel accel, const float* d_rays, size_t nrays,
                                  uint32_t* d_visits, enc_stream stream);

/* Closest hit from host buffers with no device allocation.  This entry point
 * has no counterpart in the reference.  It is for callers that must not call
 * cudaMalloc/cudaFree while answering queries: code whose host framework
 * already owns the device memory, or frame loops that cannot take the
 * device-wide synchronisation an allocation can cause.  Results equal
 * enc_intersect_closest's.  Scratch (rays in, hits out, queue head, status)
 * is one fixed __device__ array inside this library, about 3 MiB per GPU that
 * loads it, held until exit; a batch may hold at most ENC_NOALLOC_MAX_RAYS
 * rays (more is ENC_ERR_INVALID_ARG).  enc_accel_build sets the array up on
 * the accelerator's device (it looks up its device address, which makes the
 * runtime create it, and runs this call's kernel once over an empty batch),
 * so queries allocate nothing.  Calls share the array, which keeps the last
 * call's contents; calls that overlapped on the GPU would race on it, so
 * calls are serialised by a process-wide mutex and each returns only after
 * its stream has drained.  Wide-BVH accelerators only. */
#define ENC_NOALLOC_MAX_RAYS 65536
enc_status enc_intersect_closest_noalloc(enc_accel accel, const float* rays, size_t nrays,
                                         enc_hit* hits, enc_stream stream);

/* ---- Multi-scene batched launch ------------------------------------------
 * No counterpart in the reference (it traces one ray per call).  Ray batches
 * of many scenes are traced by one persistent launch: warps take chunks of
 * rays from one queue that spans every batch, so small batches share the GPU
 * with large ones instead of each paying a launch and a tail.  The launch can
 * be recorded once into a CUDA graph and replayed. */
typedef struct enc_batch_s* enc_batch;
typedef struct enc_batch_item {
  enc_accel accel;     /* wide BVH; all items: same device, width, predicate */
  const float* d_rays; /* device memory, 8 floats per ray */
  enc_hit* d_hits;     /* device memory, one enc_hit per ray */
  uint32_t nrays;
  uint32_t reserved;   /* 0 */
} enc_batch_item;
enc_status enc_batch_create(const enc_batch_item* items, uint32_t nitems,
                            const enc_launch_opts* launch, enc_batch* out);
/* One launch over every batch; asynchronous on `stream`. */
enc_status enc_batch_launch(enc_batch batch, enc_stream stream);
/* The same launch, captured into a CUDA graph on first use and replayed. */
enc_status enc_batch_launch_graph(enc_batch batch, enc_stream stream);
/* Waits for `stream`; ENC_ERR_WATCHDOG if a ray stopped at a loop bound. */
enc_status enc_batch_check(enc_batch batch, enc_stream stream);
enc_status enc_batch_destroy(enc_batch batch);

/* ---- Serving ---------------------------------------------------------------
 * No counterpart in the reference.  A server keeps a pool of accelerators
 * resident in HBM and answers ray-batch requests with continuous batching: a
 * scheduler thread admits queued requests, in arrival order, into launch
 * slots as slots and slot memory free up; every admitted group is traced by
 * one fused multi-scene launch (plus one for any-hit requests) whose copies
 * run on the slot's own stream, so requests that arrive while others are on
 * the GPU overlap with them.  Resident scenes and slot buffers are counted
 * against an HBM budget. */
typedef struct enc_server_s* enc_server;
typedef struct enc_server_opts {
  int32_t device;
  uint32_t slots;          /* launches in flight at once (0 = 6) */
  uint64_t slot_rays;      /* ray capacity of one slot (0 = 4,194,304); a larger
                              request is split into pieces of at most this many rays,
                              traced over several rounds.  Smaller slots make more,
                              smaller rounds whose copies overlap other rounds'
                              traces: 6 x 4M served 1.52x plain on a mixed 13M-ray
                              pool, 3 x 8M only 1.15x. */
  uint64_t budget_bytes;   /* HBM budget: resident scenes + slot buffers (0 = 120 GB) */
  enc_launch_opts launch;  /* kernel launch shape (zeros = defaults) */
} enc_server_opts;
enum { ENC_REQ_CLOSEST = 0, ENC_REQ_ANY = 1 };
typedef struct enc_request_info {
  double submit_s;   /* steady-clock seconds at submit */
  double start_s;    /* when its slot's copies were enqueued */
  double done_s;     /* when its results were in host memory */
  uint64_t nrays;
  int32_t status;    /* enc_status of the request */
  int32_t kind;
} enc_request_info;

enc_status enc_server_create(const enc_server_opts* opts, enc_server* out);
/* Adds a resident scene (a wide BVH built on the server's device); the
 * server does not take ownership.  ENC_ERR_BUDGET if it does not fit. */
enc_status enc_server_add_scene(enc_server server, enc_accel accel, uint32_t* scene_id);
/* Queues a request.  rays: host memory, 8 floats per ray (pinned memory lets
 * the copies overlap); out: host memory, enc_hit per ray (closest) or one
 * byte per ray (any); both must stay valid until the request completes.  A
 * request of more than slot_rays rays is split into slot-sized pieces; it is
 * done when its last piece is.  Its status is its own: a kernel that stops
 * at a loop bound on one piece fails only that piece's request. */
enc_status enc_server_submit(enc_server server, uint32_t scene_id, int32_t kind,
                             const float* rays, uint64_t nrays, void* out, uint64_t* request_id);
/* Waits up to timeout_s (< 0: forever) for a request; ENC_ERR_NOT_READY on
 * timeout.  info may be NULL.  A finished request is forgotten after it has
 * been waited for. */
enc_status enc_server_wait(enc_server server, uint64_t request_id, double timeout_s,
                           enc_request_info* info);
/* Cancels a request that has not been admitted yet (ENC_ERR_NOT_READY if it
 * already runs). */
enc_status enc_server_cancel(enc_server server, uint64_t request_id);
/* Steady-clock seconds (the clock of enc_request_info). */
double enc_server_now(void);
enc_status enc_server_destroy(enc_server server);

/* ---- Ray and photon generation on the device ------------------------------ */
typedef struct enc_camera {
  float eye[3], look[3], up[3];
  float fov_deg;         /* vertical field of view */
  uint32_t width, height;
  uint32_t jitter_seed;  /* 0: pixel centres; otherwise a seeded random point per pixel */
} enc_camera;
/* One eye ray per pixel, row-major from the bottom row, formed as
 * RayTracer::CalcEyeRaySamples does (RayTracer.cpp:489-525) with the basis of
 * Camera::CalcCamVectors (Camera.cpp:157-166): FP32, clamping Cross and
 * Normalize, near plane 1.  d_rays: width*height rays. */
enc_status enc_camera_rays_device(const enc_camera* cam, float* d_rays, enc_stream stream);
/* Hit point v0 + (v1-v0)*alpha + (v2-v0)*beta and the normal
 * Normalize(Cross(edge1, edge2)) that TrianglePrim::intersect stores
 * (TrianglePrim.cpp:236-239), 3 floats each per hit; NaN for misses. */
enc_status enc_hit_surface_device(enc_accel accel, const enc_hit* d_hits, size_t n, float* d_pos,
                                  float* d_nrm, enc_stream stream);
/* per_hit cosine-weighted diffuse rays from each closest hit, drawn as
 * randDirectionSuperN draws them (Common.cpp:144-182: cos^2(theta) uniform
 * on [0.001, 1), azimuth uniform) about the geometric normal facing the
 * incoming ray, origin pushed `offset` along that normal; output ray
 * i*per_hit+k belongs to hit i, misses give empty rays (tmax = 0).  Seeded,
 * independent of the launch shape. */
enc_status enc_diffuse_rays_device(enc_accel accel, const float* d_rays, const enc_hit* d_hits,
                                   size_t n, uint32_t per_hit, uint32_t seed, float offset,
                                   float* d_out, enc_stream stream);
typedef struct enc_photon_opts {
  float light_center[3];
  float light_size;      /* square light facing -y, side length */
  uint32_t nphotons;     /* photons emitted; each carries power 1/nphotons per channel */
  uint32_t max_bounces;  /* m_cMaxBounces: a path makes at most max_bounces + 1 hits */
  float albedo;          /* diffuse reflectance = Russian roulette survival */
  uint32_t seed;
  float emit_offset;     /* origin offset along the direction at emission (0.01 at unit scale) */
  float bounce_offset;   /* ... after a diffuse bounce (0.001 at unit scale) */
} enc_photon_opts;
/* Photon emission and tracing (PhotonMapperCPU::EmitPhotons / TracePhoton /
 * ReflectPhotonDiffusely, PhotonMapperCPU.cpp:503-745): photons leave the
 * light in a cosine lobe (RectangleLight::EmitPhoton, RectangleLight.cpp:172-185),
 * a photon is stored at every surface hit with the hit's stored normal, and
 * the path continues with probability albedo in a cosine lobe about that
 * normal.  Stores into the capacity-sized arrays (3 floats per photon);
 * *stored = photons stored (those past capacity are dropped, as AddPhoton
 * drops photons into a full map).  Synchronises `stream`. */
enc_status enc_photons_trace_device(enc_accel accel, const enc_photon_opts* opts, float* d_pos,
                                    float* d_nrm, float* d_pow, uint32_t capacity,
                                    uint32_t* stored, enc_stream stream);
/* The reference's map split (PhotonMapperCPU.cpp:516-528, 701-745, 776-798):
 * photons traced as enc_photons_trace_device traces them, each stored hit
 * routed by ReflectPhotonDiffusely's rule -- the first hit of a path
 * (bounce 0) into `direct`, later hits into `indirect` -- and, when
 * shadow_offset > 0, a shadow photon for every bounce-0 hit: a ray from
 * hitPoint + shadow_offset * dir along the same direction (the reference's
 * offset is 2 at unit scale) that passes the surfaces it leaves (stepping
 * emit_offset past each) and stores, at the first surface it enters, a photon
 * with negative power and that surface's normal in `direct`.  There are no
 * specular surfaces on this path, so no caustic map is filled.
 *
 * Photons are emitted in batches of opts->nphotons (path ids 0, 1, ...);
 * with fill_indirect != 0, batches continue until `indirect` is full
 * (EmitPhotons' while (!m_IndirectPhotonMap->Full()), :538-554), at most 64
 * batches; otherwise one batch.  A full store drops further photons
 * (PhotonMap::AddPhoton).  Every stored photon's power is then 1 / photons
 * emitted (the light's unit power split evenly, as ScalePhotons scales it).
 * d_tag (optional, may be NULL): per stored photon,
 * path id << 4 | shadow << 3 | min(bounce, 7).  stored[0], stored[1]:
 * photons in each store; *emitted (may be NULL): paths emitted.  Synchronises
 * `stream`.  Paths of one call: at most 2^28. */
typedef struct enc_photon_store {
  float* d_pos;     /* 3 floats per photon */
  float* d_nrm;     /* 3 floats per photon */
  float* d_pow;     /* 3 floats per photon */
  uint32_t* d_tag;  /* 1 word per photon, or NULL */
  uint32_t capacity;
} enc_photon_store;
enc_status enc_photons_trace_maps_device(enc_accel accel, const enc_photon_opts* opts,
                                         float shadow_offset, int32_t fill_indirect,
                                         const enc_photon_store* direct,
                                         const enc_photon_store* indirect, uint32_t stored[2],
                                         uint32_t* emitted, enc_stream stream);
/* The same with host stores (the pointers of enc_photon_store in host
 * memory): device stores are allocated for the call, copied back and freed.
 * GpuPhotonMap's GpuEmitPhotons fills a direct and an indirect map with it. */
enc_status enc_photons_trace_maps(enc_accel accel, const enc_photon_opts* opts,
                                  float shadow_offset, int32_t fill_indirect,
                                  const enc_photon_store* direct,
                                  const enc_photon_store* indirect, uint32_t stored[2],
                                  uint32_t* emitted, enc_stream stream);
/* PhotonMap over photon arrays in device memory (3 floats each per photon). */
enc_status enc_photonmap_create_device(const float* d_pos, const float* d_nrm, const float* d_pow,
                                       size_t nphotons, int32_t caustic, int32_t device,
                                       enc_photonmap* out);

/* PhotonMap: AddPhoton x n followed by BalanceAndConstruct
 * (PhotonMap.cpp:46-53, 167-221).  caustic != 0 selects the caustic-map
 * estimate (cone weight and N/(pi r^2), PhotonMap.cpp:147, 157). */
enc_status enc_photonmap_create(const float* pos, const float* normal, const float* power,
                                size_t nphotons, int32_t caustic, int32_t device,
                                enc_photonmap* out);
enc_status enc_photonmap_destroy(enc_photonmap map);
/* A balanced photon map saved as a byte image and loaded without the host
 * balance (enc_accel_serialize's counterpart for photon maps; buf = NULL
 * only sets *size).  Loading checks the header, the section sizes, the box
 * levels and every leaf's photon range (ENC_ERR_INVALID_ARG on a mismatch). */
enc_status enc_photonmap_serialize(enc_photonmap map, void* buf, size_t cap, size_t* size);
enc_status enc_photonmap_deserialize(const void* buf, size_t size, int32_t device,
                                     enc_photonmap* out);

/* Gather flags. */
enum {
  /* Accept photons regardless of normal (IGNORE_NORMAL = true, PhotonMap.cpp:23).
   * Default: a photon counts only if its stored surface normal equals the
   * query normal exactly (PhotonMap.cpp:244). */
  ENC_GATHER_IGNORE_NORMAL = 1
};

/* GetRadianceEstimate (PhotonMap.cpp:121-164) for nq query points
 * (position + normal, 3 floats each); rgb gets 3 floats per query.
 * nq < 2^31 and k <= 256 (ENC_ERR_INVALID_ARG / ENC_ERR_UNSUPPORTED beyond).
 * The _device form is asynchronous on `stream` and does not read the
 * kernel's status: call enc_photonmap_check after it.  Calls on one map from
 * different streams may run at once: each launch takes the next of 256
 * work-queue heads per map, in turn, so at most 256 launches on one map may
 * be in flight together (the 257th would share the first one's head).  A
 * launch captured into a CUDA graph keeps the head it was captured with;
 * replays of it count against the same bound as eager launches. */
enc_status enc_photonmap_radiance(enc_photonmap map, const float* qpos, const float* qnrm,
                                  size_t nq, int32_t k, float max_dist, int32_t flags,
                                  float* rgb, enc_stream stream);
/* Waits for `stream` and reports ENC_ERR_WATCHDOG if any gather on this map
 * stopped at its loop bound since the last check or synchronous call (the
 * map's launches share one status word). */
enc_status enc_photonmap_check(enc_photonmap map, enc_stream stream);
enc_status enc_photonmap_radiance_device(enc_photonmap map, const float* d_qpos,
                                         const float* d_qnrm, size_t nq, int32_t k,
                                         float max_dist, int32_t flags, float* d_rgb,
                                         enc_stream stream);
/* enc_photonmap_radiance_device that also writes, per query, the work
 * behind the gather's bytes-per-query roofline into d_visits (4 words per
 * query): child boxes tested (24 bytes each), photons tested (a 16-byte
 * position each), normals read (16 bytes each), photons found (their 16-byte
 * power).  Synchronises `stream`. */
enc_status enc_photonmap_count_visits(enc_photonmap map, const float* d_qpos,
                                      const float* d_qnrm, size_t nq, int32_t k, float max_dist,
                                      int32_t flags, float* d_rgb, uint32_t* d_visits,
                                      enc_stream stream);
/* GetNearestNPhotons (PhotonMap.cpp:76-94): for each query the indices (into
 * the arrays given to enc_photonmap_create) and squared distances of the k
 * nearest accepted photons, ascending by distance, padded with -1; count[i]
 * is how many were found. */
enc_status enc_photonmap_nearest(enc_photonmap map, const float* qpos, const float* qnrm,
                                 size_t nq, int32_t k, float max_dist, int32_t flags,
                                 int32_t* idx, float* d2, int32_t* count, enc_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* ENCORE_B200_H */
