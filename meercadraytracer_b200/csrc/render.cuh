// Host-side interface of the wavefront renderer (render.cu) and the device
// path-state layout its kernels share.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "device_scene.cuh"

namespace mcrt {

// Per-path flag bits.
constexpr uint32_t kFlagSeen = 1u;       // surfaceSeen, tracer.ts:102
constexpr uint32_t kFlagToneMap = 2u;    // toneMapped, tracer.ts:103
constexpr uint32_t kFlagCull = 4u;       // cull, tracer.ts:109
constexpr uint32_t kFlagDone = 8u;       // the path loop ended; finalize after this bounce's shadows
constexpr uint32_t kFlagDirect = 16u;    // the sample was written directly (a background)
MCRT_HD uint32_t flag_passes(uint32_t f) { return (f >> 8) & 0xffu; }
MCRT_HD uint32_t flag_bounce(uint32_t f) { return (f >> 16) & 0xffu; }
MCRT_HD int flag_last_env(uint32_t f) { return static_cast<int>(f >> 24) - 1; }

// Camera, image, sample mapping and settings of one launch series.
struct FrameParams {
  double proj_inv[16];
  double world[16];
  float cam_forward[3];
  float cam_position[3];
  int width, height;
  int pass0;       // pass of the first slice of paths
  int npix;        // paths per pass in this launch series: pixels, blocks, or listed pixels
  int pix0;        // index of the first of them in the tile / block grid / pixel list
  int mode;        // 0: tile grid (with block), 1: pixel list
  int tile_x, tile_y, tile_w, tile_h, block, nbx;
  const int* list_x;
  const int* list_y;
  uint32_t seed;
  int max_bounces, shadows, gi, tone_mapping;
  float exposure;
  float clear_color[3], clear_alpha;
  int slot_count;  // shadow slots per path: lights + 1
  int capacity;    // path-state capacity
  int path_base;   // path id of this launch series' first path (0 unless batched)
  int npass;       // > 0: the series' passes, pixel-major (path k: pixel k / npass, pass k % npass); 0: pass-major
};


// Structure-of-arrays path state, indexed by path id.
struct PathState {
  float4* ray_o;   // origin, -
  float4* ray_d;   // direction, -
  float4* hit;     // t, u, v, bits((front << 31) | (triangle + 1)); 0 = miss
  float4* thr;     // throughput rgb, fog factor
  float4* rad;     // radiance rgb, last environment scale
  float4* med;     // absorption rgb of the volume the ray is in, -
  uint32_t* rng;
  uint32_t* flags;
  unsigned long long* smask;  // shadow slots written this bounce
  float4* sample;  // finished sample: premultiplied, tone mapped RGBA
  float4* slots;   // [slot][capacity] shadow contributions
  int* queue[2];
  int* binned;           // the queue in shading order
  uint8_t* cls;          // shading class of each queue position (sort scratch)
  unsigned int* bins;    // class counts and cursors of that order
  float4* shadow_queue;  // 3 float4 per shadow ray
  int* seg;              // batched renders: the segment each path belongs to
};

struct Counters {
  unsigned int next_count;
  unsigned int shadow_count;
  unsigned int status;
  unsigned int fetch;         // next query a closest-hit traversal warp takes
  unsigned int fetch_shadow;  // the same for the any-hit (shadow) traversal
};

// Work and time of the kernels of one render, for benchmarks.
struct RenderStats {
  unsigned long long closest_rays = 0;
  unsigned long long any_rays = 0;
  unsigned long long samples = 0;
  unsigned long long launches = 0;
  double ms_raygen = 0, ms_extend = 0, ms_shade = 0, ms_shadow = 0, ms_resolve = 0, ms_accumulate = 0;
  unsigned long long n_raygen = 0, n_extend = 0, n_shade = 0, n_shadow = 0, n_resolve = 0, n_accumulate = 0;
  unsigned int status = 0;
};

// Device buffers of the path state, grown on demand.
class PathBuffers {
 public:
  ~PathBuffers();
  // Makes room for `capacity` paths with `slots` shadow slots each.
  cudaError_t reserve(int capacity, int slots);
  PathState state() const { return st_; }
  int capacity() const { return capacity_; }
  int slots() const { return slots_; }
  size_t bytes() const { return bytes_; }
  Counters* counters() const { return counters_; }
  Counters* host_counters() const { return host_counters_; }
  // A second stream and two events (made on first use, kept until destruction)
  // for running a bounce's shadow rays beside the next bounce's closest hits.
  cudaError_t side_stream(cudaStream_t* side, cudaEvent_t* fork, cudaEvent_t* join);

 private:
  void release();
  cudaStream_t side_ = nullptr;
  cudaEvent_t fork_ = nullptr, join_ = nullptr;
  PathState st_{};
  Counters* counters_ = nullptr;
  Counters* host_counters_ = nullptr;
  std::vector<void*> allocations_;
  int capacity_ = 0;
  int slots_ = 0;
  size_t bytes_ = 0;
};

// Traces `passes` passes over `npix` paths per pass (pixels, blocks or listed
// pixels as `fp` maps them), in chunks of at most the buffers' capacity,
// calling `on_chunk(first_pass, pass_count)` after each chunk so the caller
// can consume the samples. Returns a CUDA error, or cudaSuccess.
class Wavefront {
 public:
  int variant = 0;  // traversal variant (see traversal_variant_info)
  bool sort_shading = true;  // shade each bounce's paths grouped by what they hit
  bool packet_first = true;  // camera rays walk warp-coherent (traverse_packet)
  cudaError_t run(const DScene& scene, FrameParams fp, int passes, PathBuffers& buffers, cudaStream_t stream,
                  RenderStats* stats, bool timed,
                  cudaError_t (*on_chunk)(void* ctx, int first_pass, int pass_count), void* ctx);
};

// Camera rays of one pass over fp.npix paths and their closest hits, left in
// the path state's `hit` array.
cudaError_t primary_hits(const DScene& scene, FrameParams fp, PathBuffers& buffers, cudaStream_t stream);

// ----------------------------------------------------------- batched renders
// Many requests (cameras, scenes, sizes, sample counts) share one path pool.
// A chunk is a list of segments, each one request's passes [pass0, pass0 +
// passes) over its pixels (or preview blocks) [pix0, pix0 + npix), at most one
// segment per request, grouped by scene: the paths of scene s hold the ids
// [base, base + paths), and its queue entries and shadow rays use the
// matching ranges of the queues, so every stage runs once per scene.
constexpr int kMaxBatchScenes = 8;
// Shading classes of the hit-class sort: a miss, or a material model,
// transmissive or not (render.cu shade_class). The sort's bins hold two
// counters per class and scene.
constexpr int kShadeClasses = 16;
constexpr int kMaxSegments = 256;
constexpr unsigned kStatusIterationLimit = 16u;  // a chunk still had paths after max_iterations

struct SceneQueues {
  unsigned base;          // first path id of the scene in this chunk
  unsigned paths;
  unsigned count;         // paths queued for this iteration's closest hits
  unsigned next_count;    // paths this iteration's shade step continued
  unsigned shadow_count;  // shadow rays of this iteration
  unsigned fetch;         // work counters of the persistent traversals
  unsigned fetch_shadow;
  unsigned pad;
};

// Where a segment's samples go.
struct SegmentOut {
  float4* sum;      // the request's Float32 running sums, one per pixel
  uint8_t* image;   // the request's RGBA8 image
  int passes;       // passes in this segment
  int done_after;   // passes accumulated once this segment is in
  int preview;      // a block preview: written straight into the image
  int srgb;
};

// Everything a chunk's kernels read, uploaded once per chunk.
struct BatchTables {
  int segments;
  int paths;
  int iteration;       // wavefront iteration (queue parity)
  int max_iterations;
  int seg_base[kMaxSegments + 1];  // first path of each segment; [segments] = paths
  int pix_base[kMaxSegments + 1];  // first accumulate item of each segment; [segments] = total
  SceneQueues scenes[kMaxBatchScenes];
  SegmentOut out[kMaxSegments];
  FrameParams fp[kMaxSegments];    // per segment; path_base = seg_base[j]
};

// Device totals that outlive the per-chunk uploads.
struct BatchCounters {
  unsigned long long closest;  // closest-hit queries traced
  unsigned long long any;      // shadow queries traced
  unsigned long long samples;
  unsigned status;
  unsigned more;               // set by the iteration step when paths remain (host-driven loop)
};

// Grid sizes of the batched kernels on the current device, for a traversal variant.
struct BatchGrids {
  int raygen, extend, shade, shadow, resolve, accumulate, sort;
  int variant, block;
};

cudaError_t batch_grids(BatchGrids* g, int variant, int capacity);

// Traversal variants: the closest-hit and shadow kernels compiled for several
// (threads per block, shared-memory short-stack entries per thread) pairs.
// Variant 0 is the default (128, 16).
int traversal_variant_count();
void traversal_variant_info(int variant, int* block, int* stack);
int find_traversal_variant(int block, int stack);  // -1 when not compiled
// Camera rays of every segment of the chunk.
cudaError_t launch_batch_raygen(const BatchTables* t, const PathState& ps, const BatchGrids& g, cudaStream_t s);
// One wavefront iteration over every scene: closest hits, shading, shadow
// rays, resolve, then the queue swap. `graph`: the swap sets conditional
// `handle` (the loop runs as a graph's while node); otherwise it sets
// counters->more for a host-driven loop.
// Streams and events that run each scene's stages as a parallel branch of a
// captured iteration (fork from the iteration's stream, join before advance).
struct SceneLanes {
  cudaStream_t stream[kMaxBatchScenes];
  cudaEvent_t fork;
  cudaEvent_t join[kMaxBatchScenes];
};

cudaError_t launch_batch_iteration(const DScene* scenes, int nscenes, BatchTables* t, const PathState& ps,
                                   int capacity, int slots, BatchCounters* counters, const BatchGrids& g, bool graph,
                                   cudaGraphConditionalHandle handle, cudaStream_t s,
                                   const SceneLanes* lanes = nullptr);
// Accumulates (or, for previews, writes) every segment's samples and encodes
// the requests' images.
cudaError_t launch_batch_accumulate(const BatchTables* t, const PathState& ps, const BatchGrids& g, cudaStream_t s);

// A whole batch planned ahead for one half of the pool: its chunks' tables in
// order (sizeof(BatchTables) apart, at least one, an empty table when the half
// has no work) and the chunk that runs now.
struct BatchPlan {
  const BatchTables* tables;
  int count;
  int index;
};
// Copies the current chunk's table into `dst`, where the chunk's kernels read
// it, and opens the bounce loop (`inner` = 1).
cudaError_t launch_batch_load_chunk(const BatchPlan* plan, BatchTables* dst, cudaGraphConditionalHandle inner,
                                    cudaStream_t s);
// Moves to the next chunk; `outer` = 1 while chunks remain.
cudaError_t launch_batch_next_chunk(BatchPlan* plan, cudaGraphConditionalHandle outer, cudaStream_t s);

// Kernel launchers used by the executor.
cudaError_t launch_accumulate(const float4* samples, int npix, int passes_in_chunk, float4* sum, int total_passes,
                              int last_chunk, uint8_t* image, const FrameParams& fp, int srgb, cudaStream_t s);
cudaError_t launch_tile_output(const float4* samples, const FrameParams& fp, float* out, cudaStream_t s);
// `fetch` is a device counter the persistent traversal uses (reset here);
// fetch[1] collects the walk status bits (the caller clears it).
cudaError_t launch_trace_rays(const DScene& scene, const float4* rays, int count, int cull, int4* hits,
                              unsigned* fetch, cudaStream_t s);
cudaError_t launch_count_hits(const DScene& scene, const float4* rays, int count, int* counts, unsigned* fetch,
                              cudaStream_t s);

}  // namespace mcrt
