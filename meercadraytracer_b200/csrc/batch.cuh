// Batched and served rendering: many progressive render requests (scenes,
// cameras, sizes, sample counts) traced together in one wavefront over a
// shared path pool, with admission by a device-memory budget.
//
// A request follows ProgressiveRenderer.render (src/progressive.ts:189-282)
// for a whole-image tile: an optional block preview written straight into the
// image, then `samples` passes accumulated in pass order into a Float32 running
// sum, the image re-encoded after each chunk (writeTile, progressive.ts:288-313).
// Each pass traces exactly the paths raytraceCompiled (src/raytrace.ts:69-82)
// traces, so a request's image is the same alone and in any mix.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "render.cuh"

namespace mcrt {

// First-fit allocator over one device allocation (request sums and images), so
// admitting and retiring requests never calls cudaMalloc or cudaFree, which
// would synchronise the device.
class DeviceArena {
 public:
  ~DeviceArena();
  cudaError_t init(size_t bytes);
  // Offset-aligned block of `bytes`, or nullptr when it does not fit now.
  void* alloc(size_t bytes);
  void free(void* p);
  size_t capacity() const { return size_; }
  size_t used() const { return used_; }

 private:
  char* base_ = nullptr;
  size_t size_ = 0, used_ = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  std::map<size_t, size_t> live_;  // offset -> length
};

struct BatchRequestDesc {
  int scene = 0;          // scene slot
  FrameParams fp{};       // camera, settings and image size; mode 0, whole image
  int samples = 1;        // passes to accumulate
  int preview_block = 0;  // > 1: a block preview first (ProgressiveOptions.previewBlock)
  int srgb = 1;
};

enum BatchEventKind { kEventPreview = 1, kEventDone = 2, kEventProgress = 3 };

struct BatchEvent {
  long long id;
  int kind;
  int samples;  // passes accumulated when the event was raised
};

struct BatchTotals {
  unsigned long long closest = 0, any = 0, samples = 0, chunks = 0, graph_launches = 0;
  unsigned status = 0;
  double gpu_ms = 0;  // device time of the chunks (events around each chunk)
};

class BatchEngine {
 public:
  BatchEngine() = default;
  ~BatchEngine();
  BatchEngine(const BatchEngine&) = delete;
  BatchEngine& operator=(const BatchEngine&) = delete;

  // `capacity`: paths in the pool, which two chunks share half and half;
  // `arena_bytes`: budget for the requests' sums and images; `use_graph`: run
  // each chunk's bounce loop as a CUDA graph with a while node (else a
  // host-driven loop, one sync per bounce).
  cudaError_t init(int device, int capacity, size_t arena_bytes, bool use_graph);
  // Puts a scene into `slot` (< kMaxBatchScenes) with `lights` lights. Fails
  // while requests on the slot are unfinished.
  cudaError_t set_scene(int slot, const DScene& scene, int lights);
  bool scene_busy(int slot) const;
  // Queues a request; its buffers are taken from the arena when it is admitted.
  // `host_progress` (or nullptr) receives the image after every chunk that
  // completes a pass short of the last.
  long long submit(const BatchRequestDesc& d, uint8_t* host_image, uint8_t* host_preview,
                   uint8_t* host_progress = nullptr);
  // Stops a request; its buffers return to the arena once no chunk uses them.
  bool cancel(long long id);
  // Launches the next chunk (if any request has work), then waits for the
  // chunk before it and appends the events it completed. *idle: nothing is
  // queued, active or in flight. *progressed (if given): a chunk was launched
  // or finished; a step that does neither while not idle is a scheduling
  // fault, which callers report instead of stepping again.
  cudaError_t step(std::vector<BatchEvent>& events, bool* idle, bool* progressed = nullptr);
  // Renders every queued request to completion as one graph launch: the
  // requests are split between the two halves of the pool, each half's
  // chunks are planned ahead and uploaded at once, and each half runs its
  // chunks in order in a device-driven loop (raygen, the bounce loop,
  // accumulation), the two halves side by side. Appends a done event (and a
  // preview event for a request with a block preview) per request.
  // *rendered is false, and nothing is launched, when a chunk is in flight,
  // graphs are off, a request wants its block preview or progress images
  // delivered while it runs, or the arena cannot hold every request at once;
  // step() then renders them.
  cudaError_t render_whole(std::vector<BatchEvent>& events, bool* rendered);
  BatchTotals totals() const { return totals_; }
  int capacity() const { return capacity_; }
  // The most paths one chunk holds: half the pool (two chunks run at once).
  int max_chunk_paths() const { return half_; }
  size_t path_bytes() const { return paths_.bytes(); }
  const DeviceArena& arena() const { return arena_; }
  // Limits a chunk to `paths` paths (<= max_chunk_paths): smaller chunks bound
  // the latency of a new request's preview under load.
  void set_chunk_paths(int paths) { chunk_paths_ = paths; }
  // Traversal kernel variant (traversal_variant_info); waits for chunks in
  // flight and rebuilds the graphs on the next launch.
  cudaError_t set_variant(int variant);
  int variant() const { return grids_.variant; }

 private:
  // Two chunks run at once, each in its own half of the path pool with its
  // own stream, tables, counters, shading-order bins and graph, so one
  // chunk's bounce tails (the last, slowest paths of each stage) overlap the
  // other's work. Accumulation stays in chunk order (an event chain), so a
  // request's pixels still add their passes in pass order.
  static constexpr int kSlots = 2;

  struct Request {
    long long id;
    BatchRequestDesc d;
    uint8_t* host_image = nullptr;    // final image
    uint8_t* host_preview = nullptr;  // block preview
    uint8_t* host_progress = nullptr; // intermediate images
    float4* sum = nullptr;
    uint8_t* image = nullptr;
    bool admitted = false, cancelled = false, finished = false;
    int preview = 0;          // 0 none, 1 to schedule, 2 scheduled
    int next_pass = 0;        // first pass not yet scheduled
    int next_pix = 0;         // first pixel of the pass group at next_pass not yet scheduled
    int group = 0;            // passes of that group while it is split by pixel range
    int branch = -1;          // half of the pool a whole-batch render gives it (render_whole)
    int inflight = 0;         // chunks in flight that hold a segment of this request
    int copying = 0;          // chunks in flight copying this request's image to the host
    long long pixels() const { return static_cast<long long>(d.fp.width) * d.fp.height; }
  };
  struct SegmentPlan {
    Request* r;
    int preview;
    int pass0, passes, pix0, npix, done_after;
  };
  struct Chunk {
    int slot;  // half of the pool, stream, tables and graph
    std::vector<SegmentPlan> segs;
    cudaEvent_t start = nullptr, done = nullptr, copied = nullptr;
    bool copies = false;
    // Per segment: the pass count its image holds when the chunk ends, if
    // the chunk completes a pass of the request (else 0).
    std::vector<int> passes_done;
  };

  PathState slot_state(int slot) const;
  cudaError_t ensure_graph(int slot);
  cudaError_t ensure_whole_graph();
  void destroy_graphs();
  bool admit(Request& r);
  void plan(Chunk& c);
  // The chunk's tables as its kernels read them (host copy).
  void fill_tables(const Chunk& c, BatchTables* T);
  cudaError_t launch(Chunk& c);
  cudaError_t finish(Chunk& c, std::vector<BatchEvent>& events);
  void release(Request& r);

  int device_ = 0;
  int capacity_ = 0, half_ = 0, chunk_paths_ = 0;
  int slots_ = 1;
  bool use_graph_ = true;
  cudaStream_t stream_[kSlots] = {};
  cudaStream_t copy_stream_ = nullptr;
  SceneLanes lanes_{};  // per-scene branches of the captured bounce iteration
  PathBuffers paths_;
  unsigned int* bins1_ = nullptr;  // slot 1's shading-order bins (slot 0 uses the pool's)
  DeviceArena arena_;
  BatchTables* tables_dev_[kSlots] = {};
  BatchTables* tables_host_[kSlots] = {};
  BatchCounters* counters_dev_[kSlots] = {};
  BatchCounters* counters_host_[kSlots] = {};
  BatchCounters slot_totals_[kSlots] = {};  // each slot's counters after its last finished chunk
  BatchGrids grids_{};
  DScene scenes_[kMaxBatchScenes]{};
  int lights_[kMaxBatchScenes]{};
  bool scene_set_[kMaxBatchScenes]{};
  int nscenes_ = 0;
  cudaGraph_t graph_[kSlots] = {};
  cudaGraphExec_t exec_[kSlots] = {};
  bool graph_valid_[kSlots] = {};
  // Whole-batch renders: per half, the planned chunks' tables and the loop
  // state, and one graph running both halves' chunk loops.
  int plan_branch_ = -1;  // plan() takes only this half's requests (>= 0)
  BatchTables* plan_tables_dev_[kSlots] = {};
  size_t plan_tables_cap_[kSlots] = {};  // tables the allocation holds
  BatchPlan* plan_dev_[kSlots] = {};
  cudaGraph_t whole_graph_ = nullptr;
  cudaGraphExec_t whole_exec_ = nullptr;
  bool whole_valid_ = false;
  long long next_id_ = 1;
  std::deque<std::unique_ptr<Request>> requests_;  // submission order
  std::deque<Chunk> inflight_;
  // Copy-stream event of the last chunk that copied images to the host: a
  // chunk's accumulation waits for it before rewriting an image being copied.
  cudaEvent_t last_copy_ = nullptr;
  bool copy_pending_ = false;
  // Recorded after each chunk's accumulation; the next chunk's waits for it.
  cudaEvent_t accumulated_ = nullptr;
  bool accumulated_pending_ = false;
  // Done event of the chunk finished last, kept to count overlapped time once.
  cudaEvent_t held_done_ = nullptr;
  int next_slot_ = 0;
  BatchTotals totals_;
};

}  // namespace mcrt
