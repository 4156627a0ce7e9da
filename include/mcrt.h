/*
 * libmcrt: the C ABI of the B200 ray tracer.
 *
 * An mcrt_executor is one GPU tile executor: the device-side counterpart of
 * the reference's worker (createTileHandler, src/protocol.ts:55-110, behind
 * the TileExecutor interface of src/executors.ts:4-14). It keeps the latest
 * geometry and shading it was sent, by version, and texture pixels by id, all
 * resident in HBM, and renders tiles or whole images from them. A Node-API
 * addon (or any FFI) binds these functions one to one.
 *
 * Conventions: every function returns MCRT_OK (0) or an error code, and
 * mcrt_last_error() then returns the message (per thread). Host pointers are
 * borrowed for the duration of the call. Calls on one executor must not run
 * concurrently; separate executors are independent.
 */
#ifndef MCRT_H
#define MCRT_H

#include <stdint.h>

#include "mcrt_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MCRT_OK 0
#define MCRT_ERR_INVALID 1   /* bad argument or malformed scene data */
#define MCRT_ERR_CUDA 2      /* a CUDA call failed */
#define MCRT_ERR_NO_SCENE 3  /* geometry / shading version not received */
#define MCRT_ERR_TEXTURE 4   /* a texture id was not sent */
#define MCRT_ERR_LIMIT 5     /* beyond a documented limit */
#define MCRT_ERR_WALK 6      /* a BVH walk reached one of its bounds (mcrt_stats.status
                                bits), so the result may differ from the reference's */

typedef struct mcrt_executor mcrt_executor;

/* Work and device time of the renders since the last reset. */
typedef struct mcrt_stats {
  uint64_t closest_rays;  /* closest-hit BVH queries (camera and bounce rays) */
  uint64_t any_rays;      /* any-hit BVH queries (shadow rays) */
  uint64_t samples;       /* paths started */
  uint64_t launches;      /* kernels launched */
  double ms_total;        /* device time of whole render calls */
  double ms_raygen, ms_extend, ms_shade, ms_shadow, ms_resolve, ms_accumulate;
  uint64_t n_raygen, n_extend, n_shade, n_shadow, n_resolve, n_accumulate;
  uint64_t path_bytes;    /* HBM held for path state */
  uint64_t scene_bytes;   /* HBM held for the resident scene */
  uint32_t status;        /* bounds BVH walks reached (each also fails its call with
                             MCRT_ERR_WALK): 1 traversal stack deeper than 104 entries,
                             2 more than 64 distinct see-through hits on one shadow ray,
                             4 a query's step budget, 8 a leaf past the last triangle */
  uint32_t pad_;
} mcrt_stats;

/* Message of the last failed call on this thread (empty after success). */
const char* mcrt_last_error(void);

/* ABI version: 1. */
int32_t mcrt_version(void);

/* Number of CUDA devices visible. */
int32_t mcrt_device_count(int32_t* count);

/* new WorkerExecutor(...) / createTileHandler(), src/executors.ts:54-94,
 * src/protocol.ts:55: an executor on `device`. */
int32_t mcrt_executor_create(int32_t device, mcrt_executor** out);

/* TileExecutor.dispose, src/executors.ts:89-93. */
int32_t mcrt_executor_destroy(mcrt_executor* executor);

/* RequestMessage 'geometry', src/protocol.ts:30 and 64-67: replaces the
 * resident geometry (CompiledGeometry with its BVH, src/types.ts:137-167). */
int32_t mcrt_send_geometry(mcrt_executor* executor, int32_t version, const mcrt_geometry* geometry);

/* RequestMessage 'textures', src/protocol.ts:31 and 68-70: texture pixels
 * keyed by mcrt_texture.id, kept until the executor is destroyed. */
int32_t mcrt_send_textures(mcrt_executor* executor, int32_t count, const mcrt_texture* items);

/* RequestMessage 'shading', src/protocol.ts:32 and 71-74: materials, lights,
 * environments, background and fog. A texture whose `data` is NULL refers
 * to pixels sent before under its id. */
int32_t mcrt_send_shading(mcrt_executor* executor, int32_t version, const mcrt_shading* shading);

/* RequestMessage 'tile' answered by Tracer.renderTile (src/protocol.ts:75-104,
 * src/tracer.ts:62-89): one pass of a tile, premultiplied RGBA floats,
 * tile->width * tile->height * 4, row by row. Fails with MCRT_ERR_NO_SCENE
 * when the versions are not the resident ones. */
int32_t mcrt_render_tile(mcrt_executor* executor, int32_t geometry_version, int32_t shading_version,
                         const mcrt_camera* camera, const mcrt_settings* settings, const mcrt_tile* tile,
                         int32_t width, int32_t height, int32_t pass, int32_t block, float* out);

/* raytraceCompiled, src/raytrace.ts:69-82, on the resident scene: `samples`
 * passes, Float32 accumulation and RGBA8 encode on the device; out_rgba is a
 * host buffer of width * height * 4 bytes, top row first, straight alpha. */
int32_t mcrt_raytrace(mcrt_executor* executor, int32_t geometry_version, int32_t shading_version,
                      const mcrt_camera* camera, const mcrt_settings* settings, int32_t width, int32_t height,
                      int32_t samples, int32_t srgb, uint8_t* out_rgba);

/* As mcrt_raytrace, writing into device memory (a CUDA device pointer of
 * width * height * 4 bytes on the executor's device). */
int32_t mcrt_raytrace_device(mcrt_executor* executor, int32_t geometry_version, int32_t shading_version,
                             const mcrt_camera* camera, const mcrt_settings* settings, int32_t width,
                             int32_t height, int32_t samples, int32_t srgb, void* device_rgba);

/* raytraceCompiled restricted to listed pixels (each pixel is independent):
 * out_rgba gets 4 bytes and out_sum (may be NULL) the 4 running-sum floats
 * per listed pixel. */
int32_t mcrt_render_pixels(mcrt_executor* executor, int32_t geometry_version, int32_t shading_version,
                           const mcrt_camera* camera, const mcrt_settings* settings, int32_t width,
                           int32_t height, int32_t samples, int32_t srgb, int32_t count, const int32_t* px,
                           const int32_t* py, uint8_t* out_rgba, float* out_sum);

/* The first closest-hit query of each listed pixel's sample for one pass:
 * triangle index in BVH order (-1 for a miss), distance t and front flag. */
int32_t mcrt_trace_primary(mcrt_executor* executor, int32_t geometry_version, const mcrt_camera* camera,
                           int32_t width, int32_t height, int32_t pass, uint32_t seed, int32_t count,
                           const int32_t* px, const int32_t* py, int32_t* triangle, float* t, int32_t* front);

/* intersectClosest, src/bvh.ts:202-282, for `count` rays given as 8 floats
 * each (origin xyz, -, direction xyz, -), culling by side when `cull`. */
int32_t mcrt_intersect_closest(mcrt_executor* executor, int32_t geometry_version, int32_t count,
                               const float* rays, int32_t cull, int32_t* triangle, float* t, float* u,
                               int32_t* front);

/* mcrt_intersect_closest without allocating: the same query, arguments and
 * results, for callers that must not allocate device memory during the call,
 * such as a picking query issued between frames while renders run on other
 * streams (cudaFree waits for all work on the device, and cudaMalloc may), or
 * a process whose device memory is already handed to another allocator (a
 * framework's caching pool), where a new allocation would fail. It has no
 * counterpart in the reference.
 *
 * Its working memory (staged rays, hits, counters) is one fixed array per
 * device, 4 MiB + 256 B, held by every GPU that loads this library until the
 * process exits. At most 65,536 rays per call; a longer list is rejected
 * with MCRT_ERR_LIMIT. The first call on each device looks up that device's
 * array (a call with count 0 does only this); make it before any stream
 * capture. All calls share the array, which keeps the last call's contents:
 * overlapping calls on one device, from any executors or threads, race and
 * must be serialised by the caller. The resident scene is the one uploaded
 * earlier by mcrt_send_geometry. */
int32_t mcrt_intersect_closest_noalloc(mcrt_executor* executor, int32_t geometry_version, int32_t count,
                                       const float* rays, int32_t cull, int32_t* triangle, float* t, float* u,
                                       int32_t* front);

/* intersectAny, src/bvh.ts:289-332, with a counting visitor: the number of
 * triangles each ray hits between 0 and its limit (rays as above, the 4th
 * float a positive t limit or 0 for none). */
int32_t mcrt_intersect_any_count(mcrt_executor* executor, int32_t geometry_version, int32_t count,
                                 const float* rays, int32_t* counts);

/* buildBvh, src/bvh.ts:16-178, on the GPU: binned SAH with 16 bins, leaves of
 * at most 4 triangles (SAH leaves up to 16), depth at most 100. `bounds`
 * and `nodes` hold max(1, 2 count - 1) nodes; *node_count receives the count. */
int32_t mcrt_build_bvh(mcrt_executor* executor, const float* triangles, int32_t count, float* bounds,
                       int32_t* nodes, uint32_t* order, int32_t* node_count);

/* compileGeometry after the flatten, src/compile.ts:359-403, on the GPU:
 * float32 rounding of world-space triangles, BVH, reorder into BVH order,
 * tangents (writeTangent, src/compile.ts:406-432) and epsilon. Inputs and
 * outputs as the reference's sink and CompiledGeometry (see oracle.h's
 * oracle_compile_geometry for the same shapes). */
int32_t mcrt_compile_geometry(mcrt_executor* executor, int32_t count, const double* p, const double* n,
                              const double* uv, const double* colors, const uint8_t* has_color,
                              const uint32_t* materials, const uint8_t* flags, const uint8_t* sides,
                              float* triangles_out, float* normals_out, float* uvs_out, float* tangents_out,
                              float* colors_out, uint32_t* materials_out, uint8_t* flags_out, uint8_t* sides_out,
                              float* bounds_out, int32_t* nodes_out, uint32_t* order_out, int32_t* node_count_out,
                              double* epsilon_out, int32_t* any_colors);

/* ------------------------------------------------------------------------
 * Instanced geometry compiled on the device. The reference flattens meshes
 * on the host (addMesh, src/compile.ts:212-306) and ships the result; here
 * the meshes are uploaded once and every rebuild (a frame whose instances
 * moved) runs the flatten, the BVH build, the reorder, tangents and epsilon
 * on the GPU, leaving the geometry resident with no host round trip.
 * ------------------------------------------------------------------------ */
typedef struct mcrt_mesh {
  int32_t vertex_count;
  int32_t index_count;      /* 0: not indexed (vertex_count a multiple of 3) */
  const float* position;    /* 3 floats per vertex */
  const float* normal;      /* 3 floats per vertex, or NULL: face normals */
  const float* uv;          /* 2 floats per vertex, or NULL: zeros */
  const uint32_t* index;    /* index_count entries, or NULL */
} mcrt_mesh;

typedef struct mcrt_instance {
  double world[16];         /* column-major world matrix (matrixWorld, times instanceMatrix) */
  int32_t mesh;             /* index into the uploaded meshes */
  uint32_t material;        /* material index of all its triangles */
  uint8_t flags;            /* TRI_OPAQUE | TRI_CAST_SHADOW | TRI_RECEIVE_SHADOW */
  uint8_t side;             /* FrontSide 0, BackSide 1, DoubleSide 2 */
  uint8_t flat_shading;     /* 1: face normals */
  uint8_t pad_[5];
} mcrt_instance;

typedef struct mcrt_build_info {
  double flatten_ms, build_ms, finish_ms, total_ms;  /* device times: flatten, BVH, reorder + tangents, all */
  int32_t triangle_count, node_count, levels, bins;
  uint64_t geometry_bytes;  /* HBM of the resident geometry */
  uint64_t build_bytes;     /* HBM the builder keeps between builds */
} mcrt_build_info;

/* Host arrays sized for the triangle count n (and 2n - 1 nodes) that
 * receive the compiled geometry in the CompiledGeometry layout; any pointer
 * may be NULL. The counts and epsilon are written back. */
typedef struct mcrt_compiled_out {
  float* triangles;
  float* normals;
  float* uvs;
  float* tangents;
  uint32_t* materials;
  uint8_t* flags;
  uint8_t* sides;
  float* bounds;
  int32_t* nodes;
  uint32_t* order;
  double epsilon;
  int32_t triangle_count;
  int32_t node_count;
} mcrt_compiled_out;

/* Uploads the meshes that instances refer to, replacing earlier ones. No
 * counterpart in the reference (it reads three.js buffers directly). */
int32_t mcrt_upload_meshes(mcrt_executor* executor, int32_t count, const mcrt_mesh* meshes);

/* compileGeometry (src/compile.ts:327-432) of `count` instances on the GPU,
 * meshes in instance order and triangles in index order as addMesh emits
 * them, with a binned-SAH BVH of `bins` bins per axis (buildBvh's 16 keeps
 * the reference's tree; up to 32). The result becomes the resident geometry
 * under `version`, as after mcrt_send_geometry. `info` (or NULL) receives
 * times and memory; `out` (or NULL) the compiled arrays. Vertex colours and
 * geometry groups are not part of this path. */
int32_t mcrt_compile_instances(mcrt_executor* executor, int32_t version, int32_t count,
                               const mcrt_instance* instances, int32_t bins, mcrt_build_info* info,
                               mcrt_compiled_out* out);

/* Kernel timing with CUDA events on the executor's stream (adds a sync per
 * kernel; for profiling only). */
int32_t mcrt_set_timing(mcrt_executor* executor, int32_t enabled);

/* Path-state capacity (paths in flight per launch); the autotuner sets it. */
int32_t mcrt_set_capacity(mcrt_executor* executor, int32_t paths);

/* The traversal kernel variants compiled into the library: up to `max`
 * (threads per block, shared-memory short-stack entries per thread) pairs,
 * and *count = how many there are. Variant 0, (128, 4), is the default. No
 * counterpart in the reference (its traversal is one JavaScript loop). */
int32_t mcrt_traversal_variants(int32_t max, int32_t* blocks, int32_t* stacks, int32_t* count);

/* Chooses the closest-hit and shadow traversal kernels of an executor by
 * block size and short-stack depth (one of mcrt_traversal_variants); the
 * autotuner sets it. Results do not depend on the choice. */
int32_t mcrt_set_traversal(mcrt_executor* executor, int32_t block, int32_t stack);

int32_t mcrt_get_stats(mcrt_executor* executor, mcrt_stats* out);
/* Test and debugging hook: caps the node visits plus leaves one BVH query may
 * take (a walk of a well-formed tree of N triangles takes fewer than 2N + 64,
 * the default, restored by 0). A query that reaches the cap ends, sets status
 * bit 4 and its call fails with MCRT_ERR_WALK. */
int32_t mcrt_set_step_limit(mcrt_executor* executor, int32_t steps);
int32_t mcrt_reset_stats(mcrt_executor* executor);

/* ------------------------------------------------------------------------
 * Batched and served rendering. No counterpart in the reference, whose
 * ProgressiveRenderer (src/progressive.ts:177-282) schedules one render at a
 * time over tile executors: here many progressive renders (scenes, cameras,
 * sizes, sample counts) share one wavefront. Each request follows
 * ProgressiveRenderer.render for a whole-image tile: an optional block preview
 * written straight into the image, then `samples` passes accumulated in pass
 * order, so the final image equals mcrt_raytrace's for the same inputs.
 * ------------------------------------------------------------------------ */
typedef struct mcrt_batch mcrt_batch;

typedef struct mcrt_request {
  mcrt_executor* scene;     /* executor whose resident scene is rendered (same device; keep it alive
                               and unchanged while the request runs) */
  int32_t geometry_version; /* versions the executor must hold (MCRT_ERR_NO_SCENE otherwise) */
  int32_t shading_version;
  mcrt_camera camera;
  mcrt_settings settings;
  int32_t width, height;
  int32_t samples;          /* passes to accumulate (>= 1) */
  int32_t preview_block;    /* > 1: a block preview first (ProgressiveOptions.previewBlock) */
  int32_t srgb;             /* encode sRGB output */
  uint8_t* image;           /* host RGBA8, width * height * 4, for the final image; or NULL */
  uint8_t* preview_image;   /* host RGBA8 for the block preview; or NULL */
  uint8_t* progress_image;  /* host RGBA8 refreshed after every chunk that completes a pass short of the
                               last (ProgressiveFrame with samples < maxSamples); or NULL. Given, the
                               request's passes are scheduled one pass (or as many whole passes as a
                               chunk holds) at a time; NULL, in groups of up to 16 passes per pixel,
                               which trace faster (a warp's rays are passes of one or two pixels) */
} mcrt_request;

/* PREVIEW: preview_image holds the block preview. PROGRESS: `samples` passes
 * are accumulated (progress_image holds them, if given); without a
 * progress_image these come at the ends of pass groups. DONE: image holds
 * the final image. */
enum { MCRT_EVENT_PREVIEW = 1, MCRT_EVENT_DONE = 2, MCRT_EVENT_PROGRESS = 3 };

typedef struct mcrt_batch_event {
  int64_t id;
  int32_t kind;     /* MCRT_EVENT_*: preview_image / image (if given) hold the result */
  int32_t samples;  /* passes accumulated */
} mcrt_batch_event;

typedef struct mcrt_batch_stats {
  uint64_t closest_rays, any_rays, samples, chunks, graph_launches;
  double gpu_ms;        /* device time of the chunks, overlapping chunks counted once */
  uint64_t arena_bytes; /* budget for request buffers (sums and images) */
  uint64_t arena_used;
  uint64_t path_bytes;  /* path pool */
  uint32_t status;      /* kernel-reported limits hit (as mcrt_stats) */
  uint32_t pad_;
} mcrt_batch_stats;

/* A batch renderer on `device`: a pool of `capacity` (at least 2) paths that
 * two chunks in flight share half and half (one chunk's last, slowest paths
 * overlap the other's work), `arena_bytes` of device memory for admitted
 * requests' sums and images (admission waits for room), `use_graph` 1 to run
 * each chunk's bounce loop as one CUDA graph with a while node, 0 for a
 * host-driven loop. */
int32_t mcrt_batch_create(int32_t device, int32_t capacity, int64_t arena_bytes, int32_t use_graph,
                          mcrt_batch** out);
int32_t mcrt_batch_destroy(mcrt_batch* batch);
/* Paths per chunk (at most half the pool; 0: half the pool); smaller chunks
 * bound preview latency. */
int32_t mcrt_batch_set_chunk(mcrt_batch* batch, int32_t paths);
/* As mcrt_set_traversal, for the batch's kernels. */
int32_t mcrt_batch_set_traversal(mcrt_batch* batch, int32_t block, int32_t stack);
/* Queues a request; *id identifies it in events. */
int32_t mcrt_batch_submit(mcrt_batch* batch, const mcrt_request* request, int64_t* id);
/* Stops a request (a camera move restarts it as a new request). */
int32_t mcrt_batch_cancel(mcrt_batch* batch, int64_t id);
/* Launches the next chunk, waits for the previous one and returns up to
 * max_events events; *idle is 1 when nothing is queued or in flight. */
int32_t mcrt_batch_step(mcrt_batch* batch, mcrt_batch_event* events, int32_t max_events, int32_t* n_events,
                        int32_t* idle);
/* Submits `count` requests and runs until all are done. When nothing else is
 * queued, every request fits the arena at once and none asks for a
 * preview_image or progress_image, the whole batch runs as one CUDA graph
 * launch (every chunk planned ahead, the requests split between the two
 * halves of the pool, each half's chunks run in a device-driven loop);
 * otherwise chunk by chunk as mcrt_batch_step runs them. Images are the
 * same either way. */
int32_t mcrt_batch_render(mcrt_batch* batch, int32_t count, const mcrt_request* requests);
int32_t mcrt_batch_get_stats(mcrt_batch* batch, mcrt_batch_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* MCRT_H */
