// Batched and served rendering (batch.cuh): chunk planning, admission, the
// per-chunk CUDA graph and completion events.
#include "batch.cuh"

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <iterator>

namespace mcrt {

// ------------------------------------------------------------------ arena
DeviceArena::~DeviceArena() {
  if (base_) cudaFree(base_);
}

cudaError_t DeviceArena::init(size_t bytes) {
  bytes = std::max<size_t>(bytes, 256) & ~static_cast<size_t>(255);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&base_), bytes);
  if (e != cudaSuccess) {
    base_ = nullptr;
    return e;
  }
  size_ = bytes;
  free_.clear();
  live_.clear();
  free_[0] = bytes;
  used_ = 0;
  return cudaSuccess;
}

void* DeviceArena::alloc(size_t bytes) {
  bytes = (std::max<size_t>(bytes, 1) + 255) & ~static_cast<size_t>(255);
  for (auto it = free_.begin(); it != free_.end(); ++it) {
    if (it->second < bytes) continue;
    const size_t off = it->first, len = it->second;
    free_.erase(it);
    if (len > bytes) free_[off + bytes] = len - bytes;
    live_[off] = bytes;
    used_ += bytes;
    return base_ + off;
  }
  return nullptr;
}

void DeviceArena::free(void* p) {
  if (!p) return;
  const size_t off = static_cast<size_t>(static_cast<char*>(p) - base_);
  auto it = live_.find(off);
  if (it == live_.end()) return;
  size_t start = off, len = it->second;
  used_ -= len;
  live_.erase(it);
  auto next = free_.lower_bound(start);
  if (next != free_.end() && next->first == start + len) {  // merge with the block after
    len += next->second;
    next = free_.erase(next);
  }
  if (next != free_.begin()) {  // and with the block before
    auto prev = std::prev(next);
    if (prev->first + prev->second == start) {
      start = prev->first;
      len += prev->second;
      free_.erase(prev);
    }
  }
  free_[start] = len;
}

// ----------------------------------------------------------------- engine
BatchEngine::~BatchEngine() {
  cudaSetDevice(device_);
  for (cudaStream_t st : stream_)
    if (st) cudaStreamSynchronize(st);
  if (copy_stream_) cudaStreamSynchronize(copy_stream_);
  for (Chunk& c : inflight_) {
    if (c.start) cudaEventDestroy(c.start);
    if (c.done) cudaEventDestroy(c.done);
    if (c.copied) cudaEventDestroy(c.copied);
  }
  if (held_done_) cudaEventDestroy(held_done_);
  if (last_copy_) cudaEventDestroy(last_copy_);
  if (accumulated_) cudaEventDestroy(accumulated_);
  for (int i = 0; i < kMaxBatchScenes; i++) {
    if (lanes_.stream[i]) cudaStreamDestroy(lanes_.stream[i]);
    if (lanes_.join[i]) cudaEventDestroy(lanes_.join[i]);
  }
  if (lanes_.fork) cudaEventDestroy(lanes_.fork);
  destroy_graphs();
  for (int k = 0; k < kSlots; k++) {
    if (plan_tables_dev_[k]) cudaFree(plan_tables_dev_[k]);
    if (plan_dev_[k]) cudaFree(plan_dev_[k]);
    if (tables_dev_[k]) cudaFree(tables_dev_[k]);
    if (tables_host_[k]) cudaFreeHost(tables_host_[k]);
    if (counters_dev_[k]) cudaFree(counters_dev_[k]);
    if (counters_host_[k]) cudaFreeHost(counters_host_[k]);
    if (stream_[k]) cudaStreamDestroy(stream_[k]);
  }
  if (bins1_) cudaFree(bins1_);
  if (copy_stream_) cudaStreamDestroy(copy_stream_);
}

cudaError_t BatchEngine::init(int device, int capacity, size_t arena_bytes, bool use_graph) {
  device_ = device;
  capacity_ = std::max(capacity, 2);
  half_ = capacity_ / 2;
  use_graph_ = use_graph;
  cudaError_t e = cudaSetDevice(device);
  for (int k = 0; k < kSlots && e == cudaSuccess; k++) e = cudaStreamCreateWithFlags(&stream_[k], cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&last_copy_, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&accumulated_, cudaEventDisableTiming);
  for (int i = 0; i < kMaxBatchScenes && e == cudaSuccess; i++) {
    e = cudaStreamCreateWithFlags(&lanes_.stream[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&lanes_.join[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&lanes_.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = arena_.init(arena_bytes);
  for (int k = 0; k < kSlots && e == cudaSuccess; k++) {
    e = cudaMalloc(reinterpret_cast<void**>(&tables_dev_[k]), sizeof(BatchTables));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&tables_host_[k]), sizeof(BatchTables));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&counters_dev_[k]), sizeof(BatchCounters));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&counters_host_[k]), sizeof(BatchCounters));
    if (e == cudaSuccess) e = cudaMemset(counters_dev_[k], 0, sizeof(BatchCounters));
    if (e == cudaSuccess) e = cudaMemset(tables_dev_[k], 0, sizeof(BatchTables));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&plan_dev_[k]), sizeof(BatchPlan));
  }
  const size_t bin_bytes = sizeof(unsigned int) * 2 * kShadeClasses * kMaxBatchScenes;
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&bins1_), bin_bytes);
  if (e == cudaSuccess) e = cudaMemset(bins1_, 0, bin_bytes);
  if (e == cudaSuccess) e = paths_.reserve(capacity_, slots_);
  if (e == cudaSuccess) e = batch_grids(&grids_, 0, half_);
  return e;
}

// The path state of one half of the pool: every per-path array from the
// half's first path, the shadow queue from its first entry. Shadow slots keep
// the whole pool's stride (FrameParams.capacity), so they are offset by the
// half's first path only.
PathState BatchEngine::slot_state(int slot) const {
  PathState ps = paths_.state();
  if (slot == 0) return ps;
  const size_t off = static_cast<size_t>(half_);
  ps.ray_o += off;
  ps.ray_d += off;
  ps.hit += off;
  ps.thr += off;
  ps.rad += off;
  ps.med += off;
  ps.rng += off;
  ps.flags += off;
  ps.smask += off;
  ps.sample += off;
  ps.slots += off;
  ps.queue[0] += off;
  ps.queue[1] += off;
  ps.binned += off;
  ps.cls += off;
  ps.shadow_queue += 3 * off * static_cast<size_t>(paths_.slots());
  ps.seg += off;
  ps.bins = bins1_;
  return ps;
}

bool BatchEngine::scene_busy(int slot) const {
  for (const auto& r : requests_)
    if (r->d.scene == slot && (!r->finished || r->inflight > 0) && !(r->cancelled && r->inflight == 0)) return true;
  return false;
}

cudaError_t BatchEngine::set_scene(int slot, const DScene& scene, int lights) {
  if (slot < 0 || slot >= kMaxBatchScenes || lights < 0) return cudaErrorInvalidValue;
  if (scene_busy(slot)) return cudaErrorNotReady;
  cudaSetDevice(device_);
  // Chunks in flight keep the old graphs and path state: wait for them.
  for (cudaStream_t st : stream_) {
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
  }
  scenes_[slot] = scene;
  lights_[slot] = lights;
  scene_set_[slot] = true;
  nscenes_ = std::max(nscenes_, slot + 1);
  int slots = 1;
  for (int i = 0; i < nscenes_; i++)
    if (scene_set_[i]) slots = std::max(slots, lights_[i] + 1);
  if (slots > paths_.slots()) {
    const cudaError_t e = paths_.reserve(capacity_, slots);
    if (e != cudaSuccess) return e;
  }
  slots_ = std::max(slots_, slots);
  graph_valid_[0] = graph_valid_[1] = false;
  whole_valid_ = false;
  return cudaSuccess;
}

cudaError_t BatchEngine::set_variant(int variant) {
  if (variant == grids_.variant) return cudaSuccess;
  cudaSetDevice(device_);
  cudaError_t e = cudaSuccess;
  for (cudaStream_t st : stream_)
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = batch_grids(&grids_, variant, half_);
  graph_valid_[0] = graph_valid_[1] = false;
  whole_valid_ = false;
  return e;
}

void BatchEngine::destroy_graphs() {
  for (int k = 0; k < kSlots; k++) {
    if (exec_[k]) cudaGraphExecDestroy(exec_[k]);
    if (graph_[k]) cudaGraphDestroy(graph_[k]);
    exec_[k] = nullptr;
    graph_[k] = nullptr;
    graph_valid_[k] = false;
  }
  if (whole_exec_) cudaGraphExecDestroy(whole_exec_);
  if (whole_graph_) cudaGraphDestroy(whole_graph_);
  whole_exec_ = nullptr;
  whole_graph_ = nullptr;
  whole_valid_ = false;
}

// One graph per half of the pool and scene set: raygen, then a while node
// around the bounce iteration (its last kernel sets the condition). Every
// kernel reads the chunk from the half's device tables, so the graph is
// reused by every chunk of that half. Accumulation runs after the graph, in
// chunk order (launch()).
cudaError_t BatchEngine::ensure_graph(int slot) {
  if (!use_graph_ || graph_valid_[slot]) return cudaSuccess;
  if (exec_[slot]) cudaGraphExecDestroy(exec_[slot]);
  if (graph_[slot]) cudaGraphDestroy(graph_[slot]);
  exec_[slot] = nullptr;
  graph_[slot] = nullptr;
  const PathState ps = slot_state(slot);
  cudaStream_t st = stream_[slot];
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  cudaGraph_t& graph = graph_[slot];
  cudaError_t e = cudaGraphCreate(&graph, 0);
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0, mode);
  if (e != cudaSuccess) return e;
  cudaError_t le = launch_batch_raygen(tables_dev_[slot], ps, grids_, st);
  e = cudaStreamEndCapture(st, &graph);
  if (e == cudaSuccess) e = le;
  if (e != cudaSuccess) return e;
  size_t n = 0;
  e = cudaGraphGetNodes(graph, nullptr, &n);
  if (e != cudaSuccess) return e;
  std::vector<cudaGraphNode_t> roots(n);
  if (n > 0) e = cudaGraphGetNodes(graph, roots.data(), &n);
  cudaGraphConditionalHandle handle = 0;
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = handle;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t loop = nullptr;
  e = cudaGraphAddNode(&loop, graph, roots.data(), n, &p);
  if (e != cudaSuccess) return e;
  cudaGraph_t body = p.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode);
  if (e != cudaSuccess) return e;
  le = launch_batch_iteration(scenes_, nscenes_, tables_dev_[slot], ps, paths_.capacity(), paths_.slots(),
                              counters_dev_[slot], grids_, true, handle, st, &lanes_);
  e = cudaStreamEndCapture(st, &body);
  if (e == cudaSuccess) e = le;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec_[slot], graph, 0);
  if (e == cudaSuccess) graph_valid_[slot] = true;
  return e;
}

// One graph for whole-batch renders: per half of the pool, a while node over
// its planned chunks whose body loads the chunk's table, generates its rays,
// runs the bounce loop (a nested while node around the same captured
// iteration as ensure_graph's), accumulates, and moves to the next chunk. The
// halves' loops are independent roots, so they run side by side; each half
// accumulates only its own requests, in chunk order.
cudaError_t BatchEngine::ensure_whole_graph() {
  if (whole_valid_) return cudaSuccess;
  if (whole_exec_) cudaGraphExecDestroy(whole_exec_);
  if (whole_graph_) cudaGraphDestroy(whole_graph_);
  whole_exec_ = nullptr;
  whole_graph_ = nullptr;
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  cudaError_t e = cudaGraphCreate(&whole_graph_, 0);
  for (int k = 0; k < kSlots && e == cudaSuccess; k++) {
    const PathState ps = slot_state(k);
    cudaStream_t st = stream_[k];
    cudaGraphConditionalHandle outer = 0, inner = 0;
    e = cudaGraphConditionalHandleCreate(&outer, whole_graph_, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) break;
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = outer;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t outer_node = nullptr;
    e = cudaGraphAddNode(&outer_node, whole_graph_, nullptr, 0, &p);
    if (e != cudaSuccess) break;
    cudaGraph_t body = p.conditional.phGraph_out[0];
    // The bounce loop's condition is set by the chunk's table load.
    e = cudaGraphConditionalHandleCreate(&inner, body, 0, 0);
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode);
    if (e != cudaSuccess) break;
    cudaError_t le = launch_batch_load_chunk(plan_dev_[k], tables_dev_[k], inner, st);
    if (le == cudaSuccess) le = launch_batch_raygen(tables_dev_[k], ps, grids_, st);
    e = cudaStreamEndCapture(st, &body);
    if (e == cudaSuccess) e = le;
    if (e != cudaSuccess) break;
    size_t n = 0;
    e = cudaGraphGetNodes(body, nullptr, &n);
    std::vector<cudaGraphNode_t> head(n);
    if (e == cudaSuccess && n > 0) e = cudaGraphGetNodes(body, head.data(), &n);
    if (e != cudaSuccess) break;
    cudaGraphNodeParams q{};
    q.type = cudaGraphNodeTypeConditional;
    q.conditional.handle = inner;
    q.conditional.type = cudaGraphCondTypeWhile;
    q.conditional.size = 1;
    cudaGraphNode_t inner_node = nullptr;
    e = cudaGraphAddNode(&inner_node, body, head.data(), n, &q);
    if (e != cudaSuccess) break;
    cudaGraph_t loop = q.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(st, loop, nullptr, nullptr, 0, mode);
    if (e != cudaSuccess) break;
    le = launch_batch_iteration(scenes_, nscenes_, tables_dev_[k], ps, paths_.capacity(), paths_.slots(),
                                counters_dev_[k], grids_, true, inner, st, &lanes_);
    e = cudaStreamEndCapture(st, &loop);
    if (e == cudaSuccess) e = le;
    if (e != cudaSuccess) break;
    e = cudaStreamBeginCaptureToGraph(st, body, &inner_node, nullptr, 1, mode);
    if (e != cudaSuccess) break;
    le = launch_batch_accumulate(tables_dev_[k], ps, grids_, st);
    if (le == cudaSuccess) le = launch_batch_next_chunk(plan_dev_[k], outer, st);
    e = cudaStreamEndCapture(st, &body);
    if (e == cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&whole_exec_, whole_graph_, 0);
  if (e == cudaSuccess) whole_valid_ = true;
  return e;
}

long long BatchEngine::submit(const BatchRequestDesc& d, uint8_t* host_image, uint8_t* host_preview,
                              uint8_t* host_progress) {
  if (d.scene < 0 || d.scene >= kMaxBatchScenes || !scene_set_[d.scene]) return -1;
  if (d.fp.width <= 0 || d.fp.height <= 0 || d.samples < 1) return -1;
  auto r = std::make_unique<Request>();
  r->id = next_id_++;
  r->d = d;
  r->host_image = host_image;
  r->host_preview = host_preview;
  r->host_progress = host_progress;
  r->preview = d.preview_block > 1 ? 1 : 0;
  const long long id = r->id;
  requests_.push_back(std::move(r));
  return id;
}

bool BatchEngine::cancel(long long id) {
  for (auto it = requests_.begin(); it != requests_.end(); ++it) {
    Request& r = **it;
    if (r.id != id || r.cancelled || r.finished) continue;
    r.cancelled = true;
    if (r.inflight == 0) {
      release(r);
      requests_.erase(it);
    }
    return true;
  }
  return false;
}

void BatchEngine::release(Request& r) {
  if (r.sum) arena_.free(r.sum);
  r.sum = nullptr;
  r.image = nullptr;
}

bool BatchEngine::admit(Request& r) {
  const size_t pix = static_cast<size_t>(r.pixels());
  const size_t sum_bytes = (pix * sizeof(float4) + 255) & ~static_cast<size_t>(255);
  void* p = arena_.alloc(sum_bytes + pix * 4);
  if (!p) return false;
  r.sum = static_cast<float4*>(p);
  r.image = static_cast<uint8_t*>(p) + sum_bytes;
  // No clearing: a pixel's first pass starts its sum from zero (k_batch_accumulate).
  r.admitted = true;
  return true;
}

// Chooses the chunk's segments: admissions in submission order while the
// arena has room, previews first, then passes of the admitted requests in
// submission order, each request at most once: whole passes where a group of
// kGroupPasses of them (or all that are left) fits, else a pixel range of such
// a group that fills the room. A segment's paths run pixel-major, so a warp
// holds passes of one or two pixels: coherent camera and shadow rays. A
// request that asked for progress images goes by groups of one pass, so its
// client sees every pass that a chunk completes.
constexpr int kMinFragment = 1 << 16;
constexpr int kGroupPasses = 16;
void BatchEngine::plan(Chunk& c) {
  long long room = chunk_paths_ > 0 ? std::min(chunk_paths_, half_) : half_;
  for (auto& rp : requests_) {
    Request& r = *rp;
    if (r.admitted || r.cancelled) continue;
    if (!admit(r)) break;  // no overtaking: later requests wait too
  }
  std::vector<Request*> used;
  auto take = [&](Request& r, int preview, int pass0, int passes, int pix0, int npix) {
    SegmentPlan s{&r, preview, pass0, passes, pix0, npix, preview ? 0 : pass0 + passes};
    c.segs.push_back(s);
    used.push_back(&r);
    room -= static_cast<long long>(npix) * passes;
  };
  auto active = [](const Request& r) { return r.admitted && !r.cancelled && !r.finished; };
  for (auto& rp : requests_) {
    Request& r = *rp;
    if (!active(r) || r.preview != 1 || static_cast<int>(c.segs.size()) >= kMaxSegments) continue;
    if (plan_branch_ >= 0 && r.branch != plan_branch_) continue;
    const int b = r.d.preview_block;
    const long long blocks = static_cast<long long>((r.d.fp.width + b - 1) / b) * ((r.d.fp.height + b - 1) / b);
    // A preview larger than the chunk size (never than half the pool:
    // submission checks) goes alone into an empty chunk.
    if (blocks > room && !(c.segs.empty() && blocks <= half_)) continue;
    take(r, 1, 0, 1, 0, static_cast<int>(blocks));
    r.preview = 2;
  }
  for (auto& rp : requests_) {
    Request& r = *rp;
    if (!active(r) || r.preview == 1 || static_cast<int>(c.segs.size()) >= kMaxSegments) continue;
    if (plan_branch_ >= 0 && r.branch != plan_branch_) continue;
    if (std::find(used.begin(), used.end(), &r) != used.end()) continue;
    if (r.next_pass >= r.d.samples || room <= 0) continue;
    const long long P = r.pixels();
    const int left = r.d.samples - r.next_pass;
    const int unit = r.host_progress ? 1 : std::min(left, kGroupPasses);
    if (r.next_pix == 0 && P * unit <= room) {
      const int k = static_cast<int>(std::min<long long>(left, room / P));
      take(r, 0, r.next_pass, k, 0, static_cast<int>(P));
      r.next_pass += k;
      continue;
    }
    // A pass group larger than the room left in this chunk, or one already
    // split: its next pixel range, so chunks run full. A group has at most
    // half the pool's paths per pixel, so one pixel always fits an empty
    // chunk. A range of fewer than kMinFragment paths that does not end the
    // group waits for the next chunk, unless nothing else is in this one (a
    // chunk smaller than kMinFragment still makes progress).
    if (r.next_pix == 0) r.group = std::min(unit, std::max(half_, 1));
    const int g = r.group;
    long long n = std::min<long long>(room / g, P - r.next_pix);
    if (n <= 0 && c.segs.empty()) n = 1;
    if (n <= 0 || (n * g < kMinFragment && n < P - r.next_pix && !c.segs.empty())) continue;
    take(r, 0, r.next_pass, g, r.next_pix, static_cast<int>(n));
    r.next_pix += static_cast<int>(n);
    if (r.next_pix >= P) {
      r.next_pix = 0;
      r.next_pass += g;
    }
  }
  // Scene-major order: each scene's paths form one range.
  std::stable_sort(c.segs.begin(), c.segs.end(),
                   [](const SegmentPlan& a, const SegmentPlan& b) { return a.r->d.scene < b.r->d.scene; });
  for (SegmentPlan& s : c.segs) s.r->inflight++;
}

void BatchEngine::fill_tables(const Chunk& c, BatchTables* T) {
  const int nseg = static_cast<int>(c.segs.size());
  T->segments = nseg;
  T->iteration = 0;
  int max_bounces = 0;
  std::memset(T->scenes, 0, sizeof(T->scenes));
  int paths = 0, items = 0;
  for (int j = 0; j < nseg; j++) {
    const SegmentPlan& s = c.segs[j];
    const Request& r = *s.r;
    FrameParams fp = r.d.fp;
    fp.mode = 0;
    fp.tile_x = fp.tile_y = 0;
    fp.tile_w = fp.width;
    fp.tile_h = fp.height;
    fp.block = s.preview ? r.d.preview_block : 1;
    fp.nbx = (fp.width + fp.block - 1) / fp.block;
    fp.pass0 = s.pass0;
    fp.pix0 = s.pix0;
    fp.npix = s.npix;
    fp.npass = s.passes;  // pixel-major, as the plain wavefront runs its chunks
    fp.path_base = paths;
    fp.capacity = paths_.capacity();
    fp.slot_count = paths_.slots();
    T->fp[j] = fp;
    T->seg_base[j] = paths;
    T->pix_base[j] = items;
    SegmentOut& o = T->out[j];
    o.sum = r.sum;
    o.image = r.image;
    o.passes = s.passes;
    o.done_after = s.done_after;
    o.preview = s.preview;
    o.srgb = r.d.srgb;
    SceneQueues& q = T->scenes[r.d.scene];
    if (q.paths == 0) q.base = static_cast<unsigned>(paths);
    q.paths += static_cast<unsigned>(s.npix * s.passes);
    paths += s.npix * s.passes;
    items += s.npix;
    max_bounces = std::max(max_bounces, fp.max_bounces);
    totals_.samples += static_cast<unsigned long long>(s.npix) * s.passes;
  }
  for (int i = 0; i < kMaxBatchScenes; i++) T->scenes[i].count = T->scenes[i].paths;
  T->seg_base[nseg] = paths;
  T->pix_base[nseg] = items;
  T->paths = paths;
  // Paths end by bounce count or after kMaxPassThrough pass-throughs per bounce.
  T->max_iterations = (max_bounces + 1) * (kMaxPassThrough + 1) + 2;
}

cudaError_t BatchEngine::launch(Chunk& c) {
  const int k = c.slot;
  cudaStream_t st = stream_[k];
  BatchTables* T = tables_host_[k];
  fill_tables(c, T);
  const size_t bytes = offsetof(BatchTables, fp) + sizeof(FrameParams) * static_cast<size_t>(T->segments);

  cudaError_t e = cudaSuccess;
  if (!c.start) e = cudaEventCreate(&c.start);
  if (e == cudaSuccess && !c.done) e = cudaEventCreate(&c.done);
  if (e == cudaSuccess && !c.copied) e = cudaEventCreateWithFlags(&c.copied, cudaEventDisableTiming);
  if (e == cudaSuccess) e = ensure_graph(k);
  if (e == cudaSuccess) e = cudaEventRecord(c.start, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tables_dev_[k], T, bytes, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  const PathState ps = slot_state(k);
  if (use_graph_) {
    e = cudaGraphLaunch(exec_[k], st);
    totals_.graph_launches++;
  } else {
    e = launch_batch_raygen(tables_dev_[k], ps, grids_, st);
    for (int it = 0; e == cudaSuccess && it < T->max_iterations; it++) {
      e = launch_batch_iteration(scenes_, nscenes_, tables_dev_[k], ps, paths_.capacity(), paths_.slots(),
                                 counters_dev_[k], grids_, false, 0, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(counters_host_[k], counters_dev_[k], sizeof(BatchCounters), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e == cudaSuccess && !counters_host_[k]->more) break;
    }
  }
  // Accumulation in chunk order: after the previous chunk's (the other half
  // may still be tracing it), and after any copy to the host of an image this
  // chunk rewrites.
  bool wait_copy = false;
  for (const SegmentPlan& s : c.segs) wait_copy = wait_copy || s.r->copying > 0;
  if (e == cudaSuccess && wait_copy && copy_pending_) e = cudaStreamWaitEvent(st, last_copy_, 0);
  if (e == cudaSuccess && accumulated_pending_) e = cudaStreamWaitEvent(st, accumulated_, 0);
  if (e == cudaSuccess) e = launch_batch_accumulate(tables_dev_[k], ps, grids_, st);
  if (e == cudaSuccess) e = cudaEventRecord(accumulated_, st);
  if (e == cudaSuccess) accumulated_pending_ = true;
  if (e == cudaSuccess) e = cudaEventRecord(c.done, st);
  if (e != cudaSuccess) return e;
  totals_.chunks++;
  // Images a request's client is waiting for: its preview, the image after
  // each completed pass (when asked for), and the final image.
  c.copies = false;
  c.passes_done.assign(c.segs.size(), 0);
  for (size_t j = 0; j < c.segs.size(); j++) {
    const SegmentPlan& s = c.segs[j];
    Request& r = *s.r;
    const bool pass_end = !s.preview && s.pix0 + s.npix == r.pixels();
    const bool last = pass_end && s.pass0 + s.passes == r.d.samples;
    if (pass_end) c.passes_done[j] = s.pass0 + s.passes;
    uint8_t* dst = s.preview ? r.host_preview : (last ? r.host_image : (pass_end ? r.host_progress : nullptr));
    if (!dst) continue;
    if (!c.copies) e = cudaStreamWaitEvent(copy_stream_, c.done, 0);
    c.copies = true;
    r.copying++;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dst, r.image, static_cast<size_t>(r.pixels()) * 4, cudaMemcpyDeviceToHost, copy_stream_);
  }
  if (e == cudaSuccess && c.copies) e = cudaEventRecord(c.copied, copy_stream_);
  if (e == cudaSuccess && c.copies) e = cudaEventRecord(last_copy_, copy_stream_);
  if (c.copies) copy_pending_ = true;
  return e;
}

cudaError_t BatchEngine::finish(Chunk& c, std::vector<BatchEvent>& events) {
  cudaError_t e = cudaEventSynchronize(c.done);
  if (e == cudaSuccess && c.copies) e = cudaEventSynchronize(c.copied);
  if (e != cudaSuccess) return e;
  // Device time once: the part of this chunk after the chunk finished
  // before it (the two halves overlap).
  float ms = 0;
  if (cudaEventElapsedTime(&ms, c.start, c.done) == cudaSuccess) {
    float since = 0;
    if (held_done_ && cudaEventElapsedTime(&since, held_done_, c.done) == cudaSuccess) ms = std::min(ms, std::max(since, 0.0f));
    totals_.gpu_ms += ms;
  }
  const int k = c.slot;
  e = cudaMemcpy(counters_host_[k], counters_dev_[k], sizeof(BatchCounters), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  slot_totals_[k] = *counters_host_[k];
  totals_.closest = slot_totals_[0].closest + slot_totals_[1].closest;
  totals_.any = slot_totals_[0].any + slot_totals_[1].any;
  totals_.status |= slot_totals_[k].status;
  for (size_t j = 0; j < c.segs.size(); j++) {
    const SegmentPlan& s = c.segs[j];
    Request& r = *s.r;
    r.inflight--;
    const bool copied = s.preview ? r.host_preview != nullptr
                                  : (c.passes_done[j] > 0 && (c.passes_done[j] == r.d.samples ? r.host_image != nullptr
                                                                                               : r.host_progress != nullptr));
    if (copied) r.copying--;
    if (r.cancelled) continue;
    if (s.preview) {
      events.push_back(BatchEvent{r.id, kEventPreview, 0});
    } else if (c.passes_done[j] == r.d.samples) {
      r.finished = true;
      events.push_back(BatchEvent{r.id, kEventDone, r.d.samples});
    } else if (c.passes_done[j] > 0) {
      events.push_back(BatchEvent{r.id, kEventProgress, c.passes_done[j]});
    }
  }
  if (inflight_.size() <= 1) copy_pending_ = false;  // this chunk's copies were the last enqueued
  for (auto it = requests_.begin(); it != requests_.end();) {
    Request& r = **it;
    if ((r.finished || r.cancelled) && r.inflight == 0) {
      release(r);
      it = requests_.erase(it);
    } else {
      ++it;
    }
  }
  return cudaSuccess;
}

cudaError_t BatchEngine::step(std::vector<BatchEvent>& events, bool* idle, bool* progressed) {
  cudaError_t e = cudaSetDevice(device_);
  if (e != cudaSuccess) return e;
  bool launched = false;
  if (progressed) *progressed = !inflight_.empty();  // a chunk in flight is finished below
  if (inflight_.size() < 2) {
    Chunk c;
    c.slot = next_slot_;
    plan(c);
    if (!c.segs.empty()) {
      next_slot_ ^= 1;
      inflight_.push_back(std::move(c));
      e = launch(inflight_.back());
      if (e != cudaSuccess) return e;
      launched = true;
      if (progressed) *progressed = true;
    }
  }
  if (!inflight_.empty() && (inflight_.size() == 2 || !launched)) {
    e = finish(inflight_.front(), events);
    Chunk& done = inflight_.front();
    if (done.start) cudaEventDestroy(done.start);
    if (held_done_) cudaEventDestroy(held_done_);
    held_done_ = done.done;  // the next chunk's device time counts from here
    if (done.copied) cudaEventDestroy(done.copied);
    inflight_.pop_front();
    if (e != cudaSuccess) return e;
  }
  bool pending = false;
  for (const auto& r : requests_)
    if (!r->cancelled && !r->finished) pending = true;
  if (idle) *idle = !pending && inflight_.empty();
  return cudaSuccess;
}

// The most chunks a whole-batch render plans per half before it calls the
// plan a scheduling fault.
constexpr size_t kMaxPlannedChunks = 1 << 16;

cudaError_t BatchEngine::render_whole(std::vector<BatchEvent>& events, bool* rendered) {
  *rendered = false;
  cudaError_t e = cudaSetDevice(device_);
  if (e != cudaSuccess) return e;
  if (!use_graph_ || !inflight_.empty()) return cudaSuccess;
  std::vector<Request*> todo;
  for (auto& rp : requests_) {
    Request& r = *rp;
    if (r.cancelled || r.finished) continue;
    const bool started = r.next_pass > 0 || r.next_pix > 0 || r.preview == 2 || r.inflight > 0;
    if (started || r.host_progress || (r.host_preview && r.d.preview_block > 1)) return cudaSuccess;
    todo.push_back(&r);
  }
  if (todo.empty()) return cudaSuccess;
  for (Request* r : todo)
    if (!r->admitted && !admit(*r)) return cudaSuccess;  // step() admits the rest as room frees up

  // The halves take the requests by samples (pixels x passes), largest first,
  // each to the half with fewer so far.
  std::vector<Request*> order = todo;
  auto work = [](const Request* r) { return r->pixels() * std::max(1, r->d.samples); };
  std::stable_sort(order.begin(), order.end(), [&](const Request* a, const Request* b) { return work(a) > work(b); });
  long long load[kSlots] = {};
  for (Request* r : order) {
    const int b = load[0] <= load[1] ? 0 : 1;
    r->branch = b;
    load[b] += work(r);
  }
  std::vector<Chunk> chunks[kSlots];
  for (int b = 0; b < kSlots; b++) {
    plan_branch_ = b;
    for (;;) {
      Chunk c;
      c.slot = b;
      plan(c);
      if (c.segs.empty()) break;
      chunks[b].push_back(std::move(c));
      if (chunks[b].size() > kMaxPlannedChunks) break;
    }
  }
  plan_branch_ = -1;
  // After planning, a failure drops these requests (their passes are taken):
  // the caller gets the error and their buffers return to the arena.
  auto abandon = [&](cudaError_t err) {
    for (Request* r : todo) {
      r->cancelled = true;
      r->inflight = 0;
      r->branch = -1;
    }
    for (auto it = requests_.begin(); it != requests_.end();) {
      if ((*it)->cancelled) {
        release(**it);
        it = requests_.erase(it);
      } else {
        ++it;
      }
    }
    return err;
  };
  for (Request* r : todo)
    if (r->next_pass < r->d.samples || r->preview == 1) return abandon(cudaErrorInvalidValue);  // a stalled plan

  // Every table of each half in one upload, then one graph launch.
  for (int b = 0; b < kSlots && e == cudaSuccess; b++) {
    const size_t n = std::max<size_t>(1, chunks[b].size());
    if (plan_tables_cap_[b] < n) {
      if (plan_tables_dev_[b]) cudaFree(plan_tables_dev_[b]);
      plan_tables_dev_[b] = nullptr;
      plan_tables_cap_[b] = 0;
      e = cudaMalloc(reinterpret_cast<void**>(&plan_tables_dev_[b]), n * sizeof(BatchTables));
      if (e != cudaSuccess) break;
      plan_tables_cap_[b] = n;
    }
    std::vector<BatchTables> host(n);  // zeroed: an empty table when the half has no chunk
    for (size_t i = 0; i < chunks[b].size(); i++) fill_tables(chunks[b][i], &host[i]);
    e = cudaMemcpy(plan_tables_dev_[b], host.data(), n * sizeof(BatchTables), cudaMemcpyHostToDevice);
    const BatchPlan pl{plan_tables_dev_[b], static_cast<int>(n), 0};
    if (e == cudaSuccess) e = cudaMemcpy(plan_dev_[b], &pl, sizeof(BatchPlan), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = ensure_whole_graph();
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ev1);
  cudaStream_t st = stream_[0];
  if (e == cudaSuccess) e = cudaEventRecord(ev0, st);
  if (e == cudaSuccess) e = cudaGraphLaunch(whole_exec_, st);
  if (e == cudaSuccess) e = cudaEventRecord(ev1, st);
  for (Request* r : todo)
    if (e == cudaSuccess && r->host_image)
      e = cudaMemcpyAsync(r->host_image, r->image, static_cast<size_t>(r->pixels()) * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float ms = 0;
  if (e == cudaSuccess && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) totals_.gpu_ms += ms;
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (e != cudaSuccess) return abandon(e);
  totals_.graph_launches++;
  totals_.chunks += chunks[0].size() + chunks[1].size();
  for (int k = 0; k < kSlots; k++) {
    e = cudaMemcpy(counters_host_[k], counters_dev_[k], sizeof(BatchCounters), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    slot_totals_[k] = *counters_host_[k];
    totals_.status |= slot_totals_[k].status;
  }
  totals_.closest = slot_totals_[0].closest + slot_totals_[1].closest;
  totals_.any = slot_totals_[0].any + slot_totals_[1].any;
  for (Request* r : todo) {
    if (r->preview == 2) events.push_back(BatchEvent{r->id, kEventPreview, 0});
    events.push_back(BatchEvent{r->id, kEventDone, r->d.samples});
    r->finished = true;
    r->inflight = 0;
    r->branch = -1;
  }
  for (auto it = requests_.begin(); it != requests_.end();) {
    Request& r = **it;
    if ((r.finished || r.cancelled) && r.inflight == 0) {
      release(r);
      it = requests_.erase(it);
    } else {
      ++it;
    }
  }
  *rendered = true;
  return cudaSuccess;
}

}  // namespace mcrt
