// The C ABI (include/mcrt.h): executors, scene upload into the device
// layout, and render orchestration on the executor's stream.
//
// Scene data arrives in the reference's compiled format (src/types.ts) and is
// validated on the host before anything is uploaded, so that no kernel can
// read outside its buffers: BVH node references, triangle ranges, material,
// texture and environment indices are all checked here.
#include <cuda_runtime.h>


#include <algorithm>
#include <climits>
#include <cmath>
#include <deque>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "dfg_lut.h"
#include "mcrt.h"
#include "render.cuh"
#include "scene_build.cuh"
#include "traverse.cuh"

namespace mcrt {
namespace {

thread_local std::string g_error;

struct Error {
  int32_t code;
  std::string message;
};

[[noreturn]] void fail(int32_t code, const std::string& message) { throw Error{code, message}; }

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(MCRT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int32_t guard(F&& f) {
  try {
    f();
    g_error.clear();
    return MCRT_OK;
  } catch (const Error& e) {
    g_error = e.message;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_error = "out of host memory";
    return MCRT_ERR_LIMIT;
  } catch (const std::exception& e) {
    g_error = e.what();
    return MCRT_ERR_INVALID;
  }
}

// ------------------------------------------------------------ conversions
// tris: v0, v1 = v0 + e1, v2 = v0 + e2 (sums in double, rounded once), with
// flags | side << 8 and the material index in the w lanes.
__global__ void k_pack_tris(const float* __restrict__ t9, const uint32_t* __restrict__ mats,
                            const uint8_t* __restrict__ flags, const uint8_t* __restrict__ sides, int n,
                            float4* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float* t = t9 + 9 * static_cast<size_t>(k);
  float v1[3], v2[3];
  for (int a = 0; a < 3; a++) {
    v1[a] = static_cast<float>(static_cast<double>(t[a]) + static_cast<double>(t[3 + a]));
    v2[a] = static_cast<float>(static_cast<double>(t[a]) + static_cast<double>(t[6 + a]));
  }
  const int word = static_cast<int>(flags[k]) | (static_cast<int>(sides[k]) << 8);
  out[3 * static_cast<size_t>(k)] = make_float4(t[0], t[1], t[2], __int_as_float(word));
  out[3 * static_cast<size_t>(k) + 1] = make_float4(v1[0], v1[1], v1[2], __int_as_float(static_cast<int>(mats[k])));
  out[3 * static_cast<size_t>(k) + 2] = make_float4(v2[0], v2[1], v2[2], 0.0f);
}

// attrs: the 9 normal floats then the 6 uv floats of a triangle, padded to 16.
__global__ void k_pack_attrs(const float* __restrict__ normals, const float* __restrict__ uvs, int n,
                             float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  float* o = out + 16 * static_cast<size_t>(k);
  for (int i = 0; i < 9; i++) o[i] = normals[9 * static_cast<size_t>(k) + i];
  for (int i = 0; i < 6; i++) o[9 + i] = uvs[6 * static_cast<size_t>(k) + i];
  o[15] = 0.0f;
}

__global__ void k_inner_flags(const int* __restrict__ nodes, int m, int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) flags[i] = nodes[3 * i + 1] == 0 ? 1 : 0;
}

// One DNode per inner node of the reference layout (first, count, axis with
// children at first and first + 1), numbered in order by `index`.
__global__ void k_pack_nodes(const float* __restrict__ bounds, const int* __restrict__ nodes,
                             const int* __restrict__ index, int m, DNode* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || nodes[3 * i + 1] != 0 || index[i] < 0) return;  // a leaf, or unreachable from the root
  const int l = nodes[3 * i], r = l + 1;
  const float* bl = bounds + 6 * static_cast<size_t>(l);
  const float* br = bounds + 6 * static_cast<size_t>(r);
  DNode d;
  d.lxy = make_float4(bl[0], bl[3], bl[1], bl[4]);
  d.rxy = make_float4(br[0], br[3], br[1], br[4]);
  d.lrz = make_float4(bl[2], bl[5], br[2], br[5]);
  // Child references: an inner node's index, or ~first for a leaf.
  const int lc = nodes[3 * l + 1], rc = nodes[3 * r + 1];
  d.kids = make_int4(lc > 0 ? ~nodes[3 * l] : index[l], rc > 0 ? ~nodes[3 * r] : index[r], lc, rc);
  out[index[i]] = d;
}

// Flags the last triangle of every leaf (kLeafEnd), which ends the leaf's
// triangle loop during traversal.
__global__ void k_mark_leaf_ends(const int* __restrict__ nodes, int m, float4* __restrict__ tris) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int first = nodes[3 * i], count = nodes[3 * i + 1];
  if (count <= 0) return;
  float4* t = tris + 3 * static_cast<size_t>(first + count - 1);
  t->w = __int_as_float(__float_as_int(t->w) | kLeafEnd);
}

int blocks(long long n, int b) { return static_cast<int>((n + b - 1) / b); }

// ---------------------------------------------------------------- buffers
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  void* ensure(size_t bytes) {
    if (bytes <= n_ && p_) return p_;
    reset();
    cuda_check(cudaMalloc(&p_, std::max<size_t>(bytes, 16)), "cudaMalloc");
    n_ = std::max<size_t>(bytes, 16);
    return p_;
  }
  void* upload(const void* host, size_t bytes, cudaStream_t s) {
    ensure(bytes);
    if (bytes) cuda_check(cudaMemcpyAsync(p_, host, bytes, cudaMemcpyHostToDevice, s), "upload");
    return p_;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p_);
  }
  size_t size() const { return n_; }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
};

struct GeometryGpu {
  DevBuf nodes, tris, attrs, tangents, colors;
  int tri_count = 0, root_count = 0, node_count = 0;
  float eps = 1e-7f;
  int64_t max_material = -1;
  bool has_colors = false;
  size_t bytes() const { return nodes.size() + tris.size() + attrs.size() + tangents.size() + colors.size(); }
};

struct TextureGpu {
  DevBuf texels;
  int width = 0, height = 0, format = 0;
};

struct ShadingGpu {
  DevBuf materials, lights, envs, textures;
  int material_count = 0, light_count = 0, env_count = 0, texture_count = 0;
  DBackground background{};
  DFog fog{};
  int environment = -1;
  std::vector<int> texture_ids;
};

}  // namespace
}  // namespace mcrt

using namespace mcrt;

struct mcrt_executor {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool have_geometry = false, have_shading = false;
  int32_t geometry_version = 0, shading_version = 0;
  GeometryGpu geo;
  ShadingGpu sh;
  std::unordered_map<int, std::unique_ptr<TextureGpu>> textures;
  PathBuffers paths;
  int capacity = 1 << 25;  // paths in flight: 32M, about 17 GB of path state with 5 lights
  int variant = 0;         // traversal kernels' (block, short stack) variant
  int step_limit = 0;      // > 0: a query's step budget (mcrt_set_step_limit)
  bool timed = false;
  RenderStats stats;
  double ms_total = 0;
  DevBuf sum, image, list_x, list_y, out_tile, rays, hits, scratch;
  DevBuf pack_flag, pack_index, pack_temp;  // node packing of device-compiled geometry, kept across rebuilds
  DevBuf dfg_buf, srgb_lut;
  cudaTextureObject_t dfg_tex = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  SceneBuilder builder;
};

namespace {

// Copies device -> host on the executor's stream and waits: the stream is
// non-blocking, so a plain cudaMemcpy would not be ordered after its kernels.
void download(mcrt_executor* ex, void* host, const void* dev, size_t bytes, const char* what) {
  cuda_check(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ex->stream), what);
  cuda_check(cudaStreamSynchronize(ex->stream), what);
}

// Fails the call with MCRT_ERR_WALK when its BVH walks reached a bound: the
// reference's walks have none (src/bvh.ts:202-332, src/tracer.ts:515-594), so
// the result may differ from the reference's and is not handed back as valid,
// as the reference's worker reports any failure ({type: 'error'},
// src/protocol.ts:101-104).
void check_walk(unsigned status) {
  status &= kStatusStackOverflow | kStatusShadowListOverflow | kStatusStepLimit | kStatusLeafRange;
  if (!status) return;
  std::string m = "a BVH walk reached a bound, so the result may differ from the reference's:";
  if (status & kStatusStackOverflow) m += " traversal stack deeper than " + std::to_string(kStackMax) + " entries;";
  if (status & kStatusShadowListOverflow) m += " more than 64 distinct see-through hits on one shadow ray;";
  if (status & kStatusStepLimit) m += " a query's step budget ran out;";
  if (status & kStatusLeafRange) m += " a leaf ran past the last triangle;";
  m.pop_back();
  fail(MCRT_ERR_WALK, m);
}

double half_to_double(unsigned h) {  // halfToFloat, src/color.ts:28-35
  const double sign = (h & 0x8000) ? -1.0 : 1.0;
  const int exponent = (h >> 10) & 0x1f;
  const int fraction = h & 0x3ff;
  if (exponent == 0) return sign * std::ldexp(fraction / 1024.0, -14);
  if (exponent == 31) return fraction ? NAN : sign * INFINITY;
  return sign * std::ldexp(1 + fraction / 1024.0, exponent - 15);
}

void set_device(mcrt_executor* ex) { cuda_check(cudaSetDevice(ex->device), "cudaSetDevice"); }

mcrt_executor* checked(mcrt_executor* ex) {
  if (!ex) fail(MCRT_ERR_INVALID, "executor is NULL");
  set_device(ex);
  return ex;
}

DScene make_scene(mcrt_executor* ex) {
  DScene s{};
  s.nodes = ex->geo.nodes.as<DNode>();
  s.tris = ex->geo.tris.as<float4>();
  s.attrs = ex->geo.attrs.as<float4>();
  s.tangents = ex->geo.tangents.as<float4>();
  s.colors = ex->geo.has_colors ? ex->geo.colors.as<float4>() : nullptr;
  s.tri_count = ex->geo.tri_count;
  s.root_count = ex->geo.root_count;
  s.eps = ex->geo.eps;
  s.node_count = ex->geo.node_count;
  s.materials = ex->sh.materials.as<DMaterial>();
  s.lights = ex->sh.lights.as<DLight>();
  s.envs = ex->sh.envs.as<DEnvironment>();
  s.textures = ex->sh.textures.as<DTexture>();
  s.srgb_lut = ex->srgb_lut.as<float>();
  s.dfg = ex->dfg_tex;
  s.light_count = ex->sh.light_count;
  s.environment = ex->sh.environment;
  s.step_limit = ex->step_limit;
  s.background = ex->sh.background;
  s.fog = ex->sh.fog;
  return s;
}

void require_scene(mcrt_executor* ex, int32_t gv, int32_t sv, bool need_shading) {
  // createTileHandler's check, src/protocol.ts:77-79.
  if (!ex->have_geometry || ex->geometry_version != gv || (need_shading && (!ex->have_shading || ex->shading_version != sv)))
    fail(MCRT_ERR_NO_SCENE, "the tile refers to a scene this worker has not received");
  if (need_shading && ex->geo.max_material >= ex->sh.material_count && ex->geo.tri_count > 0)
    fail(MCRT_ERR_INVALID, "a triangle refers to a material the shading does not have");
}

FrameParams frame_params(const mcrt_camera* cam, const mcrt_settings* st, int width, int height) {
  if (!cam) fail(MCRT_ERR_INVALID, "camera is NULL");
  if (width <= 0 || height <= 0) fail(MCRT_ERR_INVALID, "width and height must be positive");
  FrameParams fp{};
  std::memcpy(fp.proj_inv, cam->projection_inverse, sizeof(fp.proj_inv));
  std::memcpy(fp.world, cam->world, sizeof(fp.world));
  for (int i = 0; i < 3; i++) {
    fp.cam_forward[i] = static_cast<float>(cam->forward[i]);
    fp.cam_position[i] = static_cast<float>(cam->position[i]);
  }
  fp.width = width;
  fp.height = height;
  fp.block = 1;
  if (st) {
    fp.seed = st->seed;
    fp.max_bounces = std::max(0, st->max_bounces);
    fp.shadows = st->shadows;
    fp.gi = st->global_illumination ? 1 : 0;
    fp.tone_mapping = st->tone_mapping;
    fp.exposure = static_cast<float>(st->tone_mapping_exposure);
    for (int i = 0; i < 3; i++) fp.clear_color[i] = static_cast<float>(st->clear_color[i]);
    fp.clear_alpha = static_cast<float>(st->clear_alpha);
    if (fp.shadows < 0 || fp.shadows > 2) fail(MCRT_ERR_INVALID, "unknown shadows mode");
  }
  return fp;
}

// Grows the path state to hold `paths` paths (capped by the capacity setting).
int reserve_paths(mcrt_executor* ex, long long paths) {
  const long long want = std::max(1LL, std::min<long long>(paths, ex->capacity));
  cuda_check(ex->paths.reserve(static_cast<int>(want), ex->sh.light_count + 1), "path state allocation");
  return ex->paths.capacity();
}

struct ChunkCtx {
  mcrt_executor* ex;
  FrameParams fp;
  int total_passes;
  int srgb;
  uint8_t* image;
  float4* sum;
  float* tile_out;
};

cudaError_t accumulate_chunk(void* p, int first, int count) {
  ChunkCtx* c = static_cast<ChunkCtx*>(p);
  PathState ps = c->ex->paths.state();
  const bool last = first + count == c->total_passes;
  return launch_accumulate(ps.sample, c->fp.npix, count, c->sum, c->total_passes, last ? 1 : 0, c->image, c->fp,
                           c->srgb, c->ex->stream);
}

cudaError_t tile_chunk(void* p, int, int) {
  ChunkCtx* c = static_cast<ChunkCtx*>(p);
  return launch_tile_output(c->ex->paths.state().sample, c->fp, c->tile_out, c->ex->stream);
}

// Runs `passes` passes over `total` paths per pass in pixel chunks that fit
// the path state, calling `chunk` after each pass chunk. A chunk takes every
// pass of as many pixels as fit, so a warp's paths are passes of one or two
// pixels (the wavefront runs them pixel-major): near-identical camera rays,
// and shadow rays from near-identical points. Fewer pixels than passes fit
// only in a pool smaller than the pass count; the wavefront then splits the
// passes. Each pixel's passes still reach its sum in pass order.
void run_frame(mcrt_executor* ex, FrameParams fp, int total, int passes, ChunkCtx& ctx,
               cudaError_t (*chunk)(void*, int, int)) {
  const int cap = reserve_paths(ex, static_cast<long long>(total) * passes);
  const int span = std::max(1, std::min(total, cap / passes));
  const DScene scene = make_scene(ex);
  cuda_check(cudaEventRecord(ex->ev0, ex->stream), "cudaEventRecord");
  // This call's walk status alone, merged into the running stats afterwards.
  const unsigned earlier = ex->stats.status;
  ex->stats.status = 0;
  cudaError_t e = cudaSuccess;
  for (int p0 = 0; p0 < total && e == cudaSuccess; p0 += span) {
    fp.pix0 = p0;
    fp.npix = std::min(span, total - p0);
    ctx.fp = fp;
    Wavefront wf;
    wf.variant = ex->variant;
    e = wf.run(scene, fp, passes, ex->paths, ex->stream, &ex->stats, ex->timed, chunk, &ctx);
  }
  const unsigned walk = ex->stats.status;
  ex->stats.status |= earlier;
  cuda_check(e, "render");
  cuda_check(cudaEventRecord(ex->ev1, ex->stream), "cudaEventRecord");
  cuda_check(cudaEventSynchronize(ex->ev1), "render");
  float ms = 0;
  cudaEventElapsedTime(&ms, ex->ev0, ex->ev1);
  ex->ms_total += ms;
  check_walk(walk);
}

void raytrace_impl(mcrt_executor* ex, int32_t gv, int32_t sv, const mcrt_camera* cam, const mcrt_settings* st,
                   int32_t width, int32_t height, int32_t samples, int32_t srgb, uint8_t* device_image) {
  require_scene(ex, gv, sv, true);
  FrameParams fp = frame_params(cam, st, width, height);
  if (samples < 1) samples = 1;
  const long long total = static_cast<long long>(width) * height;
  if (total > INT_MAX / 4) fail(MCRT_ERR_LIMIT, "image too large");
  fp.mode = 0;
  fp.tile_w = width;
  fp.tile_h = height;
  fp.nbx = width;
  fp.pass0 = 0;
  float4* sum = static_cast<float4*>(ex->sum.ensure(sizeof(float4) * total));
  cuda_check(cudaMemsetAsync(sum, 0, sizeof(float4) * total, ex->stream), "cudaMemset");
  ChunkCtx ctx{ex, fp, samples, srgb ? 1 : 0, device_image, sum, nullptr};
  run_frame(ex, fp, static_cast<int>(total), samples, ctx, accumulate_chunk);
}

// -------------------------------------------------------------- validation
void validate_geometry(const mcrt_geometry* g) {
  if (!g) fail(MCRT_ERR_INVALID, "geometry is NULL");
  const int n = g->triangle_count, m = g->node_count;
  if (n < 0 || m < 0) fail(MCRT_ERR_INVALID, "negative triangle or node count");
  if (n == 0) return;
  if (!g->triangles || !g->normals || !g->uvs || !g->tangents || !g->materials || !g->flags || !g->sides)
    fail(MCRT_ERR_INVALID, "geometry arrays missing");
  if (m == 0 || !g->bvh_bounds || !g->bvh_nodes) fail(MCRT_ERR_INVALID, "geometry has triangles but no BVH");
  for (int i = 0; i < m; i++) {
    const int first = g->bvh_nodes[3 * i], count = g->bvh_nodes[3 * i + 1];
    if (count < 0) fail(MCRT_ERR_INVALID, "BVH node with a negative count");
    if (count > 0) {
      if (first < 0 || static_cast<long long>(first) + count > n) fail(MCRT_ERR_INVALID, "BVH leaf outside the triangles");
    } else if (first <= i || first + 1 >= m) {
      fail(MCRT_ERR_INVALID, "BVH inner node whose children are not after it");
    }
  }
  if (g->bvh_nodes[1] > 0 && (g->bvh_nodes[0] != 0 || g->bvh_nodes[1] != n))
    fail(MCRT_ERR_INVALID, "a root leaf must cover every triangle");
}

void check_index(int v, int count, const char* what) {
  if (v < -1 || v >= count) fail(MCRT_ERR_INVALID, std::string(what) + " index out of range");
}

}  // namespace

// ------------------------------------------------ statically held scratch
// Working memory of mcrt_intersect_closest_noalloc, which allocates nothing:
// one fixed array per device, created when the library's device code is
// loaded there and held until the process exits. Offsets in bytes:
//   [0, 256)           counters: work counter, walk status
//   kNoAllocRaysAt     staged rays, 32 B each
//   kNoAllocHitsAt     packed hits (triangle, t, u, front | tests << 8), 16 B each
//   kNoAllocFieldsAt   the hits split per field: triangle, t, u, front, 4 B each
// with room for kNoAllocMaxRays rays in every region (4 MiB + 256 B in all).
static constexpr int kNoAllocMaxRays = 1 << 16;
static constexpr size_t kNoAllocRaysAt = 256;
static constexpr size_t kNoAllocHitsAt = kNoAllocRaysAt + 32 * static_cast<size_t>(kNoAllocMaxRays);
static constexpr size_t kNoAllocFieldsAt = kNoAllocHitsAt + 16 * static_cast<size_t>(kNoAllocMaxRays);
static constexpr size_t kNoAllocBytes = kNoAllocFieldsAt + 16 * static_cast<size_t>(kNoAllocMaxRays);

static __device__ __align__(256) unsigned char g_query_scratch[kNoAllocBytes];

namespace mcrt {
namespace {

// Splits packed closest hits into one array per field, so each field can be
// copied straight into the caller's array.
__global__ void k_split_hits(const int4* __restrict__ hits, int n, int* __restrict__ tri, float* __restrict__ t,
                             float* __restrict__ u, int* __restrict__ front) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 h = hits[i];
  tri[i] = h.x;
  t[i] = __int_as_float(h.y);
  u[i] = __int_as_float(h.z);
  front[i] = h.w & 1;
}

// Device address of g_query_scratch on `device`, which must be current. In
// host code the array's name stands for the variable, not for a device
// address, so the address is asked of the runtime once per device (the
// first call there) and kept.
unsigned char* query_scratch(int device) {
  constexpr int kDevices = 64;
  static std::mutex mu;
  static unsigned char* addr[kDevices] = {};
  if (device < 0 || device >= kDevices) fail(MCRT_ERR_INVALID, "device index beyond the scratch table");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    cuda_check(cudaGetSymbolAddress(&p, g_query_scratch), "cudaGetSymbolAddress (query scratch)");
    addr[device] = static_cast<unsigned char*>(p);
  }
  return addr[device];
}

}  // namespace
}  // namespace mcrt

// ====================================================================== ABI
extern "C" {

const char* mcrt_last_error(void) { return g_error.c_str(); }

int32_t mcrt_version(void) { return 1; }

int32_t mcrt_device_count(int32_t* count) {
  return guard([&] {
    int c = 0;
    cuda_check(cudaGetDeviceCount(&c), "cudaGetDeviceCount");
    if (count) *count = c;
  });
}

int32_t mcrt_executor_create(int32_t device, mcrt_executor** out) {
  return guard([&] {
    if (!out) fail(MCRT_ERR_INVALID, "out is NULL");
    int c = 0;
    cuda_check(cudaGetDeviceCount(&c), "cudaGetDeviceCount");
    if (device < 0 || device >= c) fail(MCRT_ERR_INVALID, "no such CUDA device");
    std::unique_ptr<mcrt_executor> ex(new mcrt_executor());
    ex->device = device;
    set_device(ex.get());
    cuda_check(cudaStreamCreateWithFlags(&ex->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaEventCreate(&ex->ev0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&ex->ev1), "cudaEventCreate");
    // DFG table as floats (brdf.ts:8-12) behind a texture object; sRGB levels (color.ts:21-25).
    float dfg[512];
    for (int i = 0; i < 512; i++) dfg[i] = static_cast<float>(half_to_double(MCRT_DFG_LUT_HALF[i]));
    ex->dfg_buf.upload(dfg, sizeof(dfg), ex->stream);
    float lut[256];
    for (int i = 0; i < 256; i++) {
      const double c8 = i / 255.0;
      lut[i] = static_cast<float>(c8 < 0.04045 ? c8 * 0.0773993808 : std::pow(c8 * 0.9478672986 + 0.0521327014, 2.4));
    }
    ex->srgb_lut.upload(lut, sizeof(lut), ex->stream);
    cudaResourceDesc res{};
    res.resType = cudaResourceTypeLinear;
    res.res.linear.devPtr = ex->dfg_buf.as<void>();
    res.res.linear.desc = cudaCreateChannelDesc<float>();
    res.res.linear.sizeInBytes = sizeof(dfg);
    cudaTextureDesc td{};
    td.readMode = cudaReadModeElementType;
    td.filterMode = cudaFilterModePoint;
    td.addressMode[0] = cudaAddressModeClamp;
    cuda_check(cudaCreateTextureObject(&ex->dfg_tex, &res, &td, nullptr), "cudaCreateTextureObject");
    cuda_check(cudaStreamSynchronize(ex->stream), "executor setup");
    *out = ex.release();
  });
}

int32_t mcrt_executor_destroy(mcrt_executor* ex) {
  return guard([&] {
    if (!ex) return;
    cudaSetDevice(ex->device);
    cudaStreamSynchronize(ex->stream);
    if (ex->dfg_tex) cudaDestroyTextureObject(ex->dfg_tex);
    if (ex->ev0) cudaEventDestroy(ex->ev0);
    if (ex->ev1) cudaEventDestroy(ex->ev1);
    cudaStream_t s = ex->stream;
    delete ex;
    if (s) cudaStreamDestroy(s);
  });
}

int32_t mcrt_send_geometry(mcrt_executor* ex, int32_t version, const mcrt_geometry* g) {
  return guard([&] {
    checked(ex);
    validate_geometry(g);
    ex->have_geometry = false;
    GeometryGpu& G = ex->geo;
    const int n = g->triangle_count;
    const int m = n > 0 ? g->node_count : 0;
    G.tri_count = n;
    G.node_count = m;
    G.eps = static_cast<float>(g->epsilon);
    G.root_count = (m > 0 && g->bvh_nodes[1] > 0) ? g->bvh_nodes[1] : 0;
    G.max_material = -1;
    for (int k = 0; k < n; k++) G.max_material = std::max<int64_t>(G.max_material, g->materials[k]);
    cudaStream_t s = ex->stream;
    if (n > 0) {
      DevBuf t9, mats, flags, sides, nrm, uvs;
      t9.upload(g->triangles, sizeof(float) * 9 * n, s);
      mats.upload(g->materials, sizeof(uint32_t) * n, s);
      flags.upload(g->flags, n, s);
      sides.upload(g->sides, n, s);
      G.tris.ensure(sizeof(float4) * 3 * n);
      k_pack_tris<<<blocks(n, 256), 256, 0, s>>>(t9.as<float>(), mats.as<uint32_t>(), flags.as<uint8_t>(),
                                                 sides.as<uint8_t>(), n, G.tris.as<float4>());
      nrm.upload(g->normals, sizeof(float) * 9 * n, s);
      uvs.upload(g->uvs, sizeof(float) * 6 * n, s);
      G.attrs.ensure(sizeof(float) * 16 * n);
      k_pack_attrs<<<blocks(n, 256), 256, 0, s>>>(nrm.as<float>(), uvs.as<float>(), n, G.attrs.as<float>());
      G.tangents.upload(g->tangents, sizeof(float) * 4 * n, s);
      G.has_colors = g->colors != nullptr;
      if (G.has_colors) G.colors.upload(g->colors, sizeof(float) * 12 * n, s);
      DevBuf nodes;
      nodes.upload(g->bvh_nodes, sizeof(int) * 3 * m, s);
      k_mark_leaf_ends<<<blocks(m, 256), 256, 0, s>>>(nodes.as<int>(), m, G.tris.as<float4>());
      if (G.root_count == 0) {
        // Inner nodes numbered depth first (preorder, left child first): a
        // node's left child follows it in memory, often in the same cache
        // line, and every subtree is one contiguous range.
        std::vector<int> order_index(m, -1);
        std::vector<int> todo;
        todo.reserve(256);
        todo.push_back(0);
        int inner = 0;
        while (!todo.empty()) {
          const int i = todo.back();
          todo.pop_back();
          if (g->bvh_nodes[3 * i + 1] != 0 || order_index[i] >= 0) continue;
          order_index[i] = inner++;
          const int first = g->bvh_nodes[3 * i];
          todo.push_back(first + 1);
          todo.push_back(first);
        }
        DevBuf bounds, index;
        bounds.upload(g->bvh_bounds, sizeof(float) * 6 * m, s);
        index.upload(order_index.data(), sizeof(int) * m, s);
        G.nodes.ensure(sizeof(DNode) * std::max(inner, 1));
        k_pack_nodes<<<blocks(m, 256), 256, 0, s>>>(bounds.as<float>(), nodes.as<int>(), index.as<int>(), m,
                                                    G.nodes.as<DNode>());
        cuda_check(cudaGetLastError(), "BVH conversion");
        cuda_check(cudaStreamSynchronize(s), "geometry upload");
      } else {
        cuda_check(cudaGetLastError(), "geometry conversion");
        cuda_check(cudaStreamSynchronize(s), "geometry upload");
      }
    }
    ex->geometry_version = version;
    ex->have_geometry = true;
  });
}

int32_t mcrt_send_textures(mcrt_executor* ex, int32_t count, const mcrt_texture* items) {
  return guard([&] {
    checked(ex);
    if (count < 0 || (count > 0 && !items)) fail(MCRT_ERR_INVALID, "bad texture list");
    for (int i = 0; i < count; i++) {
      const mcrt_texture& t = items[i];
      if (t.width <= 0 || t.height <= 0 || !t.data || (t.format != 0 && t.format != 1))
        fail(MCRT_ERR_INVALID, "bad texture");
      std::unique_ptr<TextureGpu> tex(new TextureGpu());
      tex->width = t.width;
      tex->height = t.height;
      tex->format = t.format;
      const size_t bytes = static_cast<size_t>(t.width) * t.height * 4 * (t.format == 1 ? 4 : 1);
      tex->texels.upload(t.data, bytes, ex->stream);
      ex->textures[t.id] = std::move(tex);
    }
    cuda_check(cudaStreamSynchronize(ex->stream), "texture upload");
  });
}

int32_t mcrt_send_shading(mcrt_executor* ex, int32_t version, const mcrt_shading* s) {
  return guard([&] {
    checked(ex);
    if (!s) fail(MCRT_ERR_INVALID, "shading is NULL");
    ex->have_shading = false;
    ShadingGpu& S = ex->sh;
    const int nt = s->texture_count, ne = s->environment_count, nm = s->material_count, nl = s->light_count;
    if (nt < 0 || ne < 0 || nm < 0 || nl < 0) fail(MCRT_ERR_INVALID, "negative counts");
    if (nl > kMaxLights) fail(MCRT_ERR_LIMIT, "at most 63 lights are supported");
    if (ne > 254) fail(MCRT_ERR_LIMIT, "at most 254 environments are supported");
    // Textures: pixels sent now or before, by id (createTileHandler, src/protocol.ts:82-87).
    std::vector<mcrt_texture> sent;
    for (int i = 0; i < nt; i++) {
      const mcrt_texture& t = s->textures[i];
      if (t.data) sent.push_back(t);
    }
    if (!sent.empty()) {
      const int32_t r = mcrt_send_textures(ex, static_cast<int32_t>(sent.size()), sent.data());
      if (r != MCRT_OK) fail(r, g_error);
    }
    std::vector<DTexture> tex(std::max(nt, 1));
    for (int i = 0; i < nt; i++) {
      const mcrt_texture& t = s->textures[i];
      auto it = ex->textures.find(t.id);
      if (it == ex->textures.end()) fail(MCRT_ERR_TEXTURE, "texture " + std::to_string(t.id) + " was not sent");
      const TextureGpu& g = *it->second;
      if (g.width != t.width || g.height != t.height || g.format != t.format)
        fail(MCRT_ERR_INVALID, "texture " + std::to_string(t.id) + " does not match the pixels sent");
      DTexture& d = tex[i];
      d = DTexture{};
      d.data = g.texels.as<uint8_t>();
      d.width = t.width;
      d.height = t.height;
      d.format = t.format;
      d.srgb = t.srgb ? 1 : 0;
      d.flip_y = t.flip_y ? 1 : 0;
      d.wrap_s = t.wrap_s;
      d.wrap_t = t.wrap_t;
      for (int k = 0; k < 9; k++) d.matrix[k] = static_cast<float>(t.matrix[k]);
    }
    std::vector<DEnvironment> envs(std::max(ne, 1));
    for (int i = 0; i < ne; i++) {
      const mcrt_environment& e = s->environments[i];
      DEnvironment& d = envs[i];
      d = DEnvironment{};
      d.kind = e.kind;
      if (e.kind == MCRT_ENV_EQUIRECT) {
        if (e.texture < 0 || e.texture >= nt) fail(MCRT_ERR_INVALID, "environment texture index out of range");
      } else if (e.kind == MCRT_ENV_CUBE) {
        for (int f = 0; f < 6; f++)
          if (e.faces[f] < 0 || e.faces[f] >= nt) fail(MCRT_ERR_INVALID, "cube face index out of range");
      } else {
        fail(MCRT_ERR_INVALID, "unknown environment kind");
      }
      d.texture = e.texture;
      d.flip_x = e.flip_x ? 1 : 0;
      for (int f = 0; f < 6; f++) d.faces[f] = e.faces[f];
      for (int k = 0; k < 9; k++) d.rotation[k] = static_cast<float>(e.rotation[k]);
      d.intensity = static_cast<float>(e.intensity);
    }
    std::vector<DMaterial> mats(std::max(nm, 1));
    for (int i = 0; i < nm; i++) {
      const mcrt_material& m = s->materials[i];
      if (m.model < 0 || m.model > 4) fail(MCRT_ERR_INVALID, "unknown material model");
      for (int idx : {m.map, m.alpha_map, m.emissive_map, m.normal_map, m.ao_map, m.roughness_map, m.metalness_map})
        check_index(idx, nt, "material texture");
      check_index(m.env_map, ne, "material environment");
      DMaterial& d = mats[i];
      d = DMaterial{};
      d.model = m.model;
      d.side = m.side;
      d.transparent = m.transparent ? 1 : 0;
      d.vertex_colors = m.vertex_colors ? 1 : 0;
      d.flat_shading = m.flat_shading ? 1 : 0;
      d.tone_mapped = m.tone_mapped ? 1 : 0;
      d.physical = m.physical ? 1 : 0;
      d.combine = m.combine;
      d.map = m.map;
      d.alpha_map = m.alpha_map;
      d.emissive_map = m.emissive_map;
      d.normal_map = m.normal_map;
      d.ao_map = m.ao_map;
      d.roughness_map = m.roughness_map;
      d.metalness_map = m.metalness_map;
      d.env_map = m.env_map;
      for (int k = 0; k < 3; k++) {
        d.color[k] = static_cast<float>(m.color[k]);
        d.emissive[k] = static_cast<float>(m.emissive[k]);
        d.specular_color[k] = static_cast<float>(m.specular_color[k]);
        d.attenuation[k] = static_cast<float>(m.attenuation[k]);
        d.specular[k] = static_cast<float>(m.specular[k]);
      }
      d.opacity = static_cast<float>(m.opacity);
      d.alpha_test = static_cast<float>(m.alpha_test);
      d.normal_scale[0] = static_cast<float>(m.normal_scale[0]);
      d.normal_scale[1] = static_cast<float>(m.normal_scale[1]);
      d.ao_map_intensity = static_cast<float>(m.ao_map_intensity);
      d.roughness = static_cast<float>(m.roughness);
      d.metalness = static_cast<float>(m.metalness);
      d.ior = static_cast<float>(m.ior);
      d.specular_intensity = static_cast<float>(m.specular_intensity);
      d.transmission = static_cast<float>(m.transmission);
      d.thickness = static_cast<float>(m.thickness);
      d.shininess = static_cast<float>(m.shininess);
      d.env_map_intensity = static_cast<float>(m.env_map_intensity);
      d.reflectivity = static_cast<float>(m.reflectivity);
    }
    std::vector<DLight> lights(std::max(nl, 1));
    for (int i = 0; i < nl; i++) {
      const mcrt_light& l = s->lights[i];
      if (l.type < 0 || l.type > 4) fail(MCRT_ERR_INVALID, "unknown light type");
      DLight& d = lights[i];
      d = DLight{};
      d.type = l.type;
      d.cast_shadow = l.cast_shadow ? 1 : 0;
      for (int k = 0; k < 3; k++) {
        d.color[k] = static_cast<float>(l.color[k]);
        d.ground[k] = static_cast<float>(l.ground_color[k]);
        d.direction[k] = static_cast<float>(l.direction[k]);
        d.position[k] = static_cast<float>(l.position[k]);
      }
      d.distance = static_cast<float>(l.distance);
      d.decay = static_cast<float>(l.decay);
      d.cone_cos = static_cast<float>(l.cone_cos);
      d.penumbra_cos = static_cast<float>(l.penumbra_cos);
    }
    const mcrt_background& b = s->background;
    DBackground bg{};
    bg.kind = b.kind;
    if (b.kind == MCRT_BACKGROUND_SCREEN && (b.texture < 0 || b.texture >= nt))
      fail(MCRT_ERR_INVALID, "background texture index out of range");
    if (b.kind == MCRT_BACKGROUND_ENVIRONMENT && (b.environment < 0 || b.environment >= ne))
      fail(MCRT_ERR_INVALID, "background environment index out of range");
    if (b.kind < 0 || b.kind > 3) fail(MCRT_ERR_INVALID, "unknown background kind");
    bg.texture = b.texture;
    bg.environment = b.environment;
    for (int k = 0; k < 3; k++) bg.color[k] = static_cast<float>(b.color[k]);
    bg.intensity = static_cast<float>(b.intensity);
    DFog fog{};
    fog.kind = s->fog.kind;
    for (int k = 0; k < 3; k++) fog.color[k] = static_cast<float>(s->fog.color[k]);
    fog.near_ = static_cast<float>(s->fog.near_);
    fog.far_ = static_cast<float>(s->fog.far_);
    fog.density = static_cast<float>(s->fog.density);
    check_index(s->environment, ne, "scene environment");
    S.textures.upload(tex.data(), sizeof(DTexture) * tex.size(), ex->stream);
    S.envs.upload(envs.data(), sizeof(DEnvironment) * envs.size(), ex->stream);
    S.materials.upload(mats.data(), sizeof(DMaterial) * mats.size(), ex->stream);
    S.lights.upload(lights.data(), sizeof(DLight) * lights.size(), ex->stream);
    cuda_check(cudaStreamSynchronize(ex->stream), "shading upload");
    S.material_count = nm;
    S.light_count = nl;
    S.env_count = ne;
    S.texture_count = nt;
    S.background = bg;
    S.fog = fog;
    S.environment = s->environment;
    ex->shading_version = version;
    ex->have_shading = true;
  });
}

int32_t mcrt_render_tile(mcrt_executor* ex, int32_t gv, int32_t sv, const mcrt_camera* cam, const mcrt_settings* st,
                         const mcrt_tile* tile, int32_t width, int32_t height, int32_t pass, int32_t block,
                         float* out) {
  return guard([&] {
    checked(ex);
    require_scene(ex, gv, sv, true);
    if (!tile || !out) fail(MCRT_ERR_INVALID, "tile or output is NULL");
    if (tile->x < 0 || tile->y < 0 || tile->width < 0 || tile->height < 0 || tile->x + tile->width > width ||
        tile->y + tile->height > height)
      fail(MCRT_ERR_INVALID, "tile outside the image");
    if (pass < 0) fail(MCRT_ERR_INVALID, "negative pass");
    const long long pixels = static_cast<long long>(tile->width) * tile->height;
    if (pixels == 0) return;
    FrameParams fp = frame_params(cam, st, width, height);
    fp.mode = 0;
    fp.tile_x = tile->x;
    fp.tile_y = tile->y;
    fp.tile_w = tile->width;
    fp.tile_h = tile->height;
    fp.block = std::max(1, block);
    fp.nbx = (tile->width + fp.block - 1) / fp.block;
    const int nby = (tile->height + fp.block - 1) / fp.block;
    fp.pass0 = pass;
    float* dout = static_cast<float*>(ex->out_tile.ensure(sizeof(float4) * pixels));
    ChunkCtx ctx{ex, fp, 1, 0, nullptr, nullptr, dout};
    run_frame(ex, fp, fp.nbx * nby, 1, ctx, tile_chunk);
    download(ex, out, dout, sizeof(float4) * pixels, "tile download");
  });
}

int32_t mcrt_raytrace(mcrt_executor* ex, int32_t gv, int32_t sv, const mcrt_camera* cam, const mcrt_settings* st,
                      int32_t width, int32_t height, int32_t samples, int32_t srgb, uint8_t* out_rgba) {
  return guard([&] {
    checked(ex);
    if (!out_rgba) fail(MCRT_ERR_INVALID, "output is NULL");
    const size_t bytes = static_cast<size_t>(std::max(width, 0)) * std::max(height, 0) * 4;
    uint8_t* img = static_cast<uint8_t*>(ex->image.ensure(bytes));
    raytrace_impl(ex, gv, sv, cam, st, width, height, samples, srgb, img);
    cuda_check(cudaMemcpyAsync(out_rgba, img, bytes, cudaMemcpyDeviceToHost, ex->stream), "image download");
    cuda_check(cudaStreamSynchronize(ex->stream), "image download");
  });
}

int32_t mcrt_raytrace_device(mcrt_executor* ex, int32_t gv, int32_t sv, const mcrt_camera* cam,
                             const mcrt_settings* st, int32_t width, int32_t height, int32_t samples, int32_t srgb,
                             void* device_rgba) {
  return guard([&] {
    checked(ex);
    if (!device_rgba) fail(MCRT_ERR_INVALID, "output is NULL");
    raytrace_impl(ex, gv, sv, cam, st, width, height, samples, srgb, static_cast<uint8_t*>(device_rgba));
  });
}

int32_t mcrt_render_pixels(mcrt_executor* ex, int32_t gv, int32_t sv, const mcrt_camera* cam, const mcrt_settings* st,
                           int32_t width, int32_t height, int32_t samples, int32_t srgb, int32_t count,
                           const int32_t* px, const int32_t* py, uint8_t* out_rgba, float* out_sum) {
  return guard([&] {
    checked(ex);
    require_scene(ex, gv, sv, true);
    if (count < 0 || (count > 0 && (!px || !py || !out_rgba))) fail(MCRT_ERR_INVALID, "bad pixel list");
    if (count == 0) return;
    for (int i = 0; i < count; i++)
      if (px[i] < 0 || py[i] < 0 || px[i] >= width || py[i] >= height) fail(MCRT_ERR_INVALID, "pixel outside the image");
    FrameParams fp = frame_params(cam, st, width, height);
    if (samples < 1) samples = 1;
    fp.mode = 1;
    fp.list_x = static_cast<int*>(ex->list_x.upload(px, sizeof(int) * count, ex->stream));
    fp.list_y = static_cast<int*>(ex->list_y.upload(py, sizeof(int) * count, ex->stream));
    float4* sum = static_cast<float4*>(ex->sum.ensure(sizeof(float4) * count));
    cuda_check(cudaMemsetAsync(sum, 0, sizeof(float4) * count, ex->stream), "cudaMemset");
    uint8_t* img = static_cast<uint8_t*>(ex->image.ensure(4 * static_cast<size_t>(count)));
    ChunkCtx ctx{ex, fp, samples, srgb ? 1 : 0, img, sum, nullptr};
    run_frame(ex, fp, count, samples, ctx, accumulate_chunk);
    download(ex, out_rgba, img, 4 * static_cast<size_t>(count), "download");
    if (out_sum) download(ex, out_sum, sum, sizeof(float4) * count, "download");
  });
}

int32_t mcrt_trace_primary(mcrt_executor* ex, int32_t gv, const mcrt_camera* cam, int32_t width, int32_t height,
                           int32_t pass, uint32_t seed, int32_t count, const int32_t* px, const int32_t* py,
                           int32_t* triangle, float* t, int32_t* front) {
  return guard([&] {
    checked(ex);
    require_scene(ex, gv, 0, false);
    if (count < 0 || (count > 0 && (!px || !py || !triangle || !t))) fail(MCRT_ERR_INVALID, "bad pixel list");
    if (count == 0) return;
    FrameParams fp = frame_params(cam, nullptr, width, height);
    fp.seed = seed;
    fp.mode = 1;
    fp.pass0 = pass;
    fp.list_x = static_cast<int*>(ex->list_x.upload(px, sizeof(int) * count, ex->stream));
    fp.list_y = static_cast<int*>(ex->list_y.upload(py, sizeof(int) * count, ex->stream));
    if (ex->paths.capacity() == 0) cuda_check(ex->paths.reserve(std::min(count, ex->capacity), 1), "path state");
    const int cap = std::max(ex->paths.capacity(), std::min(count, ex->capacity));
    cuda_check(ex->paths.reserve(cap, std::max(ex->paths.slots(), 1)), "path state");
    const DScene scene = make_scene(ex);
    std::vector<float4> hits(count);
    for (int p0 = 0; p0 < count; p0 += ex->paths.capacity()) {
      fp.pix0 = p0;
      fp.npix = std::min(ex->paths.capacity(), count - p0);
      cuda_check(primary_hits(scene, fp, ex->paths, ex->stream), "primary rays");
      cuda_check(cudaMemcpyAsync(hits.data() + p0, ex->paths.state().hit, sizeof(float4) * fp.npix,
                                 cudaMemcpyDeviceToHost, ex->stream),
                 "download");
      cuda_check(cudaStreamSynchronize(ex->stream), "primary rays");
    }
    for (int i = 0; i < count; i++) {
      unsigned w;
      std::memcpy(&w, &hits[i].w, 4);
      triangle[i] = static_cast<int>(w & 0x7fffffffu) - 1;
      t[i] = hits[i].x;
      if (front) front[i] = (w >> 31) ? 1 : 0;
    }
  });
}

int32_t mcrt_intersect_closest(mcrt_executor* ex, int32_t gv, int32_t count, const float* rays, int32_t cull,
                               int32_t* triangle, float* t, float* u, int32_t* front) {
  return guard([&] {
    checked(ex);
    require_scene(ex, gv, 0, false);
    if (count < 0 || (count > 0 && (!rays || !triangle))) fail(MCRT_ERR_INVALID, "bad ray list");
    if (count == 0) return;
    float4* r = static_cast<float4*>(ex->rays.upload(rays, sizeof(float) * 8 * count, ex->stream));
    int4* h = static_cast<int4*>(ex->hits.ensure(sizeof(int4) * count));
    unsigned* fetch = static_cast<unsigned*>(ex->scratch.ensure(2 * sizeof(unsigned)));
    cuda_check(cudaMemsetAsync(fetch + 1, 0, sizeof(unsigned), ex->stream), "memset");
    cuda_check(launch_trace_rays(make_scene(ex), r, count, cull, h, fetch, ex->stream), "trace");
    unsigned walk_status = 0;
    download(ex, &walk_status, fetch + 1, sizeof(unsigned), "download");
    ex->stats.status |= walk_status;
    check_walk(walk_status);
    std::vector<int4> out(count);
    download(ex, out.data(), h, sizeof(int4) * count, "download");
    for (int i = 0; i < count; i++) {
      triangle[i] = out[i].x;
      if (t) std::memcpy(&t[i], &out[i].y, 4);
      if (u) std::memcpy(&u[i], &out[i].z, 4);
      if (front) front[i] = out[i].w & 1;
    }
  });
}

int32_t mcrt_intersect_any_count(mcrt_executor* ex, int32_t gv, int32_t count, const float* rays, int32_t* counts) {
  return guard([&] {
    checked(ex);
    require_scene(ex, gv, 0, false);
    if (count < 0 || (count > 0 && (!rays || !counts))) fail(MCRT_ERR_INVALID, "bad ray list");
    if (count == 0) return;
    float4* r = static_cast<float4*>(ex->rays.upload(rays, sizeof(float) * 8 * count, ex->stream));
    int* c = static_cast<int*>(ex->hits.ensure(sizeof(int) * count));
    unsigned* fetch = static_cast<unsigned*>(ex->scratch.ensure(2 * sizeof(unsigned)));
    cuda_check(cudaMemsetAsync(fetch + 1, 0, sizeof(unsigned), ex->stream), "memset");
    cuda_check(launch_count_hits(make_scene(ex), r, count, c, fetch, ex->stream), "trace");
    unsigned walk_status = 0;
    download(ex, &walk_status, fetch + 1, sizeof(unsigned), "download");
    ex->stats.status |= walk_status;
    check_walk(walk_status);
    download(ex, counts, c, sizeof(int) * count, "download");
  });
}

int32_t mcrt_intersect_closest_noalloc(mcrt_executor* ex, int32_t gv, int32_t count, const float* rays,
                                       int32_t cull, int32_t* triangle, float* t, float* u, int32_t* front) {
  return guard([&] {
    checked(ex);
    require_scene(ex, gv, 0, false);
    if (count < 0 || (count > 0 && (!rays || !triangle))) fail(MCRT_ERR_INVALID, "bad ray list");
    if (count > kNoAllocMaxRays)
      fail(MCRT_ERR_LIMIT, "mcrt_intersect_closest_noalloc: " + std::to_string(count) +
                               " rays exceed its limit of " + std::to_string(kNoAllocMaxRays) +
                               " per call (split the list, or use mcrt_intersect_closest)");
    unsigned char* base = query_scratch(ex->device);  // set-up on the device's first call
    if (count == 0) return;
    unsigned* counters = reinterpret_cast<unsigned*>(base);
    float4* r = reinterpret_cast<float4*>(base + kNoAllocRaysAt);
    int4* h = reinterpret_cast<int4*>(base + kNoAllocHitsAt);
    int* f_tri = reinterpret_cast<int*>(base + kNoAllocFieldsAt);
    float* f_t = reinterpret_cast<float*>(f_tri + kNoAllocMaxRays);
    float* f_u = f_t + kNoAllocMaxRays;
    int* f_front = reinterpret_cast<int*>(f_u + kNoAllocMaxRays);
    const cudaStream_t s = ex->stream;
    cuda_check(cudaMemcpyAsync(r, rays, sizeof(float) * 8 * count, cudaMemcpyHostToDevice, s), "upload");
    // The array keeps the previous call's contents: the walk status starts
    // at zero here, the work counter inside launch_trace_rays.
    cuda_check(cudaMemsetAsync(counters + 1, 0, sizeof(unsigned), s), "memset");
    cuda_check(launch_trace_rays(make_scene(ex), r, count, cull, h, counters, s), "trace");
    k_split_hits<<<blocks(count, 256), 256, 0, s>>>(h, count, f_tri, f_t, f_u, f_front);
    cuda_check(cudaGetLastError(), "split hits");
    unsigned walk_status = 0;
    const cudaMemcpyKind d2h = cudaMemcpyDeviceToHost;
    cuda_check(cudaMemcpyAsync(&walk_status, counters + 1, sizeof(unsigned), d2h, s), "download");
    cuda_check(cudaMemcpyAsync(triangle, f_tri, sizeof(int32_t) * count, d2h, s), "download");
    if (t) cuda_check(cudaMemcpyAsync(t, f_t, sizeof(float) * count, d2h, s), "download");
    if (u) cuda_check(cudaMemcpyAsync(u, f_u, sizeof(float) * count, d2h, s), "download");
    if (front) cuda_check(cudaMemcpyAsync(front, f_front, sizeof(int32_t) * count, d2h, s), "download");
    cuda_check(cudaStreamSynchronize(s), "download");
    ex->stats.status |= walk_status;
    check_walk(walk_status);
  });
}

int32_t mcrt_build_bvh(mcrt_executor* ex, const float* triangles, int32_t count, float* bounds, int32_t* nodes,
                       uint32_t* order, int32_t* node_count) {
  return guard([&] {
    checked(ex);
    if (count < 0 || (count > 0 && (!triangles || !bounds || !nodes || !order)) || !node_count)
      fail(MCRT_ERR_INVALID, "bad BVH build arguments");
    *node_count = ex->builder.build_bvh_host(triangles, count, bounds, nodes, order, ex->stream);
  });
}

int32_t mcrt_compile_geometry(mcrt_executor* ex, int32_t count, const double* p, const double* n, const double* uv,
                              const double* colors, const uint8_t* has_color, const uint32_t* materials,
                              const uint8_t* flags, const uint8_t* sides, float* triangles_out, float* normals_out,
                              float* uvs_out, float* tangents_out, float* colors_out, uint32_t* materials_out,
                              uint8_t* flags_out, uint8_t* sides_out, float* bounds_out, int32_t* nodes_out,
                              uint32_t* order_out, int32_t* node_count_out, double* epsilon_out,
                              int32_t* any_colors) {
  return guard([&] {
    checked(ex);
    if (count < 0) fail(MCRT_ERR_INVALID, "negative triangle count");
    if (count > 0 && (!p || !n || !uv || !materials || !flags || !sides || !triangles_out || !normals_out ||
                      !uvs_out || !tangents_out || !materials_out || !flags_out || !sides_out || !bounds_out ||
                      !nodes_out || !order_out))
      fail(MCRT_ERR_INVALID, "compile arrays missing");
    if (!node_count_out || !epsilon_out || !any_colors) fail(MCRT_ERR_INVALID, "compile outputs missing");
    ex->builder.compile_host(count, p, n, uv, colors, has_color, materials, flags, sides, triangles_out, normals_out,
                             uvs_out, tangents_out, colors_out, materials_out, flags_out, sides_out, bounds_out,
                             nodes_out, order_out, node_count_out, epsilon_out, any_colors, ex->stream);
  });
}

int32_t mcrt_upload_meshes(mcrt_executor* ex, int32_t count, const mcrt_mesh* meshes) {
  return guard([&] {
    checked(ex);
    if (count < 0 || (count > 0 && !meshes)) fail(MCRT_ERR_INVALID, "bad mesh list");
    std::vector<MeshInput> in(count);
    for (int i = 0; i < count; i++) {
      const mcrt_mesh& m = meshes[i];
      if (m.vertex_count < 0 || (m.vertex_count > 0 && !m.position)) fail(MCRT_ERR_INVALID, "bad mesh positions");
      if (m.index_count < 0 || m.index_count % 3 != 0 || (m.index_count > 0 && !m.index))
        fail(MCRT_ERR_INVALID, "bad mesh index");
      if (m.index_count == 0 && m.vertex_count % 3 != 0) fail(MCRT_ERR_INVALID, "bad mesh vertex count");
      for (int k = 0; k < m.index_count; k++)
        if (m.index[k] >= static_cast<uint32_t>(m.vertex_count)) fail(MCRT_ERR_INVALID, "mesh index out of range");
      in[i] = MeshInput{m.vertex_count, m.position, m.normal, m.uv, m.index_count, m.index};
    }
    ex->builder.upload_meshes(count, in.data(), ex->stream);
  });
}

int32_t mcrt_compile_instances(mcrt_executor* ex, int32_t version, int32_t count, const mcrt_instance* instances,
                               int32_t bins, mcrt_build_info* info, mcrt_compiled_out* out) {
  return guard([&] {
    checked(ex);
    if (count < 0 || (count > 0 && !instances)) fail(MCRT_ERR_INVALID, "bad instance list");
    if (bins < 2 || bins > 32) fail(MCRT_ERR_INVALID, "bins must be 2 to 32");
    std::vector<InstanceInput> in(count);
    int64_t max_material = -1;
    for (int i = 0; i < count; i++) {
      const mcrt_instance& t = instances[i];
      InstanceInput d{};
      std::memcpy(d.world, t.world, sizeof(d.world));
      d.mesh = t.mesh;
      d.material = t.material;
      d.flags = t.flags & 7;
      d.side = t.side;
      d.flat_shading = t.flat_shading;
      in[i] = d;
      max_material = std::max<int64_t>(max_material, t.material);
    }
    const long long total = ex->builder.instance_triangles(count, in.data());
    if (total < 0) fail(MCRT_ERR_INVALID, "an instance names a mesh that was not uploaded");
    if (total > (1ll << 30)) fail(MCRT_ERR_LIMIT, "at most 2^30 triangles");
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    cuda_check(cudaEventRecord(e0, ex->stream), "event");
    ex->have_geometry = false;
    DeviceGeometry g{};
    float times[3] = {0, 0, 0};
    ex->builder.compile_instances(count, in.data(), bins, ex->stream, &g, times);
    // Make it resident as mcrt_send_geometry does, from device memory.
    GeometryGpu& G = ex->geo;
    cudaStream_t s = ex->stream;
    const int n = g.n, m = g.node_count;
    G.tri_count = n;
    G.node_count = m;
    G.eps = static_cast<float>(g.epsilon);
    G.root_count = g.root_count;
    G.max_material = n > 0 ? max_material : -1;
    G.has_colors = false;
    if (n > 0) {
      G.tris.ensure(sizeof(float4) * 3 * n);
      k_pack_tris<<<blocks(n, 256), 256, 0, s>>>(g.triangles, g.materials, g.flags, g.sides, n, G.tris.as<float4>());
      G.attrs.ensure(sizeof(float) * 16 * n);
      k_pack_attrs<<<blocks(n, 256), 256, 0, s>>>(g.normals, g.uvs, n, G.attrs.as<float>());
      G.tangents.ensure(sizeof(float) * 4 * n);
      cuda_check(cudaMemcpyAsync(G.tangents.as<float>(), g.tangents, sizeof(float) * 4 * n, cudaMemcpyDeviceToDevice, s),
                 "copy");
      k_mark_leaf_ends<<<blocks(m, 256), 256, 0, s>>>(g.nodes, m, G.tris.as<float4>());
      if (G.root_count == 0) {
        // A full binary tree of m nodes has (m - 1) / 2 inner nodes; buffers
        // are sized for the most any build of n triangles can make, so a
        // rebuild every frame allocates (and synchronises) nothing.
        DevBuf& flag = ex->pack_flag;
        DevBuf& index = ex->pack_index;
        DevBuf& temp = ex->pack_temp;
        const size_t m_cap = 2 * static_cast<size_t>(n);
        flag.ensure(sizeof(int) * m_cap);
        index.ensure(sizeof(int) * m_cap);
        k_inner_flags<<<blocks(m, 256), 256, 0, s>>>(g.nodes, m, flag.as<int>());
        temp.ensure(sizeof(int) * exclusive_scan_scratch());
        exclusive_scan(flag.as<int>(), index.as<int>(), m, temp.as<int>(), s);
        G.nodes.ensure(sizeof(DNode) * std::max(n - 1, 1));
        k_pack_nodes<<<blocks(m, 256), 256, 0, s>>>(g.bounds, g.nodes, index.as<int>(), m, G.nodes.as<DNode>());
        cuda_check(cudaGetLastError(), "BVH conversion");
        cuda_check(cudaStreamSynchronize(s), "geometry pack");
      }
    }
    cuda_check(cudaGetLastError(), "geometry pack");
    if (out) {
      // The CompiledGeometry arrays, for callers that check or keep them.
      auto down = [&](void* h, const void* d, size_t bytes) {
        if (h && bytes) cuda_check(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s), "download");
      };
      const size_t N = static_cast<size_t>(n);
      down(out->triangles, g.triangles, sizeof(float) * 9 * N);
      down(out->normals, g.normals, sizeof(float) * 9 * N);
      down(out->uvs, g.uvs, sizeof(float) * 6 * N);
      down(out->tangents, g.tangents, sizeof(float) * 4 * N);
      down(out->materials, g.materials, sizeof(uint32_t) * N);
      down(out->flags, g.flags, N);
      down(out->sides, g.sides, N);
      down(out->bounds, g.bounds, sizeof(float) * 6 * m);
      down(out->nodes, g.nodes, sizeof(int) * 3 * m);
      down(out->order, g.order, sizeof(uint32_t) * N);
      out->epsilon = g.epsilon;
      out->node_count = m;
      out->triangle_count = n;
    }
    cuda_check(cudaEventRecord(e1, s), "event");
    cuda_check(cudaEventSynchronize(e1), "compile");
    float total_ms = 0;
    cudaEventElapsedTime(&total_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ex->geometry_version = version;
    ex->have_geometry = true;
    if (info) {
      mcrt_build_info r{};
      r.flatten_ms = times[0];
      r.build_ms = times[1];
      r.finish_ms = times[2];
      r.total_ms = total_ms;
      r.triangle_count = n;
      r.node_count = m;
      r.levels = g.levels;
      r.bins = bins;
      r.geometry_bytes = G.bytes();
      r.build_bytes = ex->builder.device_bytes();
      *info = r;
    }
  });
}

int32_t mcrt_set_timing(mcrt_executor* ex, int32_t enabled) {
  return guard([&] {
    checked(ex);
    ex->timed = enabled != 0;
  });
}

int32_t mcrt_set_capacity(mcrt_executor* ex, int32_t paths) {
  return guard([&] {
    checked(ex);
    if (paths < 1024) fail(MCRT_ERR_INVALID, "capacity must be at least 1024 paths");
    ex->capacity = paths;
  });
}

int32_t mcrt_traversal_variants(int32_t max, int32_t* blocks, int32_t* stacks, int32_t* count) {
  return guard([&] {
    if (max < 0 || (max > 0 && (!blocks || !stacks))) fail(MCRT_ERR_INVALID, "bad output arrays");
    const int n = traversal_variant_count();
    for (int i = 0; i < n && i < max; i++) traversal_variant_info(i, &blocks[i], &stacks[i]);
    if (count) *count = n;
  });
}

int32_t mcrt_set_traversal(mcrt_executor* ex, int32_t block, int32_t stack) {
  return guard([&] {
    checked(ex);
    const int v = find_traversal_variant(block, stack);
    if (v < 0) fail(MCRT_ERR_INVALID, "no traversal kernels compiled for this block size and stack depth");
    ex->variant = v;
  });
}

int32_t mcrt_set_step_limit(mcrt_executor* ex, int32_t steps) {
  return guard([&] {
    checked(ex);
    if (steps < 0) fail(MCRT_ERR_INVALID, "negative step limit");
    ex->step_limit = steps;
  });
}

int32_t mcrt_get_stats(mcrt_executor* ex, mcrt_stats* out) {
  return guard([&] {
    checked(ex);
    if (!out) fail(MCRT_ERR_INVALID, "out is NULL");
    const RenderStats& s = ex->stats;
    mcrt_stats r{};
    r.closest_rays = s.closest_rays;
    r.any_rays = s.any_rays;
    r.samples = s.samples;
    r.launches = s.launches;
    r.ms_total = ex->ms_total;
    r.ms_raygen = s.ms_raygen;
    r.ms_extend = s.ms_extend;
    r.ms_shade = s.ms_shade;
    r.ms_shadow = s.ms_shadow;
    r.ms_resolve = s.ms_resolve;
    r.ms_accumulate = s.ms_accumulate;
    r.n_raygen = s.n_raygen;
    r.n_extend = s.n_extend;
    r.n_shade = s.n_shade;
    r.n_shadow = s.n_shadow;
    r.n_resolve = s.n_resolve;
    r.n_accumulate = s.n_accumulate;
    r.path_bytes = ex->paths.bytes();
    r.scene_bytes = ex->geo.bytes();
    r.status = s.status;
    *out = r;
  });
}

int32_t mcrt_reset_stats(mcrt_executor* ex) {
  return guard([&] {
    checked(ex);
    ex->stats = RenderStats{};
    ex->ms_total = 0;
  });
}

}  // extern "C"

// ------------------------------------------------------------ batch renders
// A batch renderer maps each (executor, geometry version, shading version)
// its requests name to one of the engine's scene slots.
struct mcrt_batch {
  int device = 0;
  BatchEngine engine;
  struct Slot {
    mcrt_executor* ex = nullptr;
    int32_t gv = 0, sv = 0;
    bool used = false;
  } slots[kMaxBatchScenes];
  std::deque<BatchEvent> pending;
};

namespace {

mcrt_batch* checked_batch(mcrt_batch* b) {
  if (!b) fail(MCRT_ERR_INVALID, "batch is NULL");
  cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
  return b;
}

// Fails when a slot's executor no longer holds the scene its unfinished
// requests were submitted for.
void check_slots(mcrt_batch* b) {
  for (int i = 0; i < kMaxBatchScenes; i++) {
    const auto& s = b->slots[i];
    if (!s.used || !b->engine.scene_busy(i)) continue;
    if (!s.ex->have_geometry || !s.ex->have_shading || s.ex->geometry_version != s.gv ||
        s.ex->shading_version != s.sv)
      fail(MCRT_ERR_NO_SCENE, "a batched request's executor changed its scene before the request finished");
  }
}

int scene_slot(mcrt_batch* b, const mcrt_request* r) {
  for (int i = 0; i < kMaxBatchScenes; i++) {
    const auto& s = b->slots[i];
    if (s.used && s.ex == r->scene && s.gv == r->geometry_version && s.sv == r->shading_version) return i;
  }
  int slot = -1;
  for (int i = 0; i < kMaxBatchScenes && slot < 0; i++)
    if (!b->slots[i].used) slot = i;
  for (int i = 0; i < kMaxBatchScenes && slot < 0; i++)
    if (!b->engine.scene_busy(i)) slot = i;
  if (slot < 0) fail(MCRT_ERR_LIMIT, "a batch holds at most 8 scenes with unfinished requests");
  cuda_check(b->engine.set_scene(slot, make_scene(r->scene), r->scene->sh.light_count), "batch scene");
  b->slots[slot] = mcrt_batch::Slot{r->scene, r->geometry_version, r->shading_version, true};
  return slot;
}

int64_t submit_request(mcrt_batch* b, const mcrt_request* r) {
  if (!r || !r->scene) fail(MCRT_ERR_INVALID, "request or its scene is NULL");
  if (r->scene->device != b->device) fail(MCRT_ERR_INVALID, "the request's executor is on another device");
  set_device(r->scene);
  require_scene(r->scene, r->geometry_version, r->shading_version, true);
  cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
  if (r->samples < 1) fail(MCRT_ERR_INVALID, "samples must be at least 1");
  if (static_cast<long long>(r->width) * r->height > INT_MAX / 4) fail(MCRT_ERR_LIMIT, "image too large");
  BatchRequestDesc d;
  d.fp = frame_params(&r->camera, &r->settings, r->width, r->height);
  d.samples = r->samples;
  d.preview_block = r->preview_block > 1 ? r->preview_block : 0;
  d.srgb = r->srgb ? 1 : 0;
  const size_t pix = static_cast<size_t>(r->width) * r->height;
  if (pix * 20 + 512 > b->engine.arena().capacity())
    fail(MCRT_ERR_LIMIT, "the request's buffers exceed the batch's memory budget");
  if (d.preview_block > 1) {
    const long long blocks = static_cast<long long>((r->width + d.preview_block - 1) / d.preview_block) *
                             ((r->height + d.preview_block - 1) / d.preview_block);
    if (blocks > b->engine.max_chunk_paths())
      fail(MCRT_ERR_LIMIT, "the block preview needs more paths than one chunk of the batch's pool holds (half the pool)");
  }
  d.scene = scene_slot(b, r);
  const long long id = b->engine.submit(d, r->image, r->preview_image, r->progress_image);
  if (id < 0) fail(MCRT_ERR_INVALID, "request rejected");
  return id;
}

}  // namespace

extern "C" {

int32_t mcrt_batch_create(int32_t device, int32_t capacity, int64_t arena_bytes, int32_t use_graph,
                          mcrt_batch** out) {
  return guard([&] {
    if (!out) fail(MCRT_ERR_INVALID, "out is NULL");
    int c = 0;
    cuda_check(cudaGetDeviceCount(&c), "cudaGetDeviceCount");
    if (device < 0 || device >= c) fail(MCRT_ERR_INVALID, "no such CUDA device");
    if (capacity < 2) fail(MCRT_ERR_INVALID, "capacity must be at least 2 (two chunks share the pool)");
    if (arena_bytes < 4096) fail(MCRT_ERR_INVALID, "memory budget too small");
    std::unique_ptr<mcrt_batch> b(new mcrt_batch());
    b->device = device;
    cuda_check(b->engine.init(device, capacity, static_cast<size_t>(arena_bytes), use_graph != 0), "batch setup");
    *out = b.release();
  });
}

int32_t mcrt_batch_destroy(mcrt_batch* b) {
  return guard([&] {
    if (!b) return;
    cudaSetDevice(b->device);
    delete b;
  });
}

int32_t mcrt_batch_set_chunk(mcrt_batch* b, int32_t paths) {
  return guard([&] {
    checked_batch(b);
    if (paths < 0) fail(MCRT_ERR_INVALID, "negative chunk size");
    b->engine.set_chunk_paths(paths);
  });
}

int32_t mcrt_batch_set_traversal(mcrt_batch* b, int32_t block, int32_t stack) {
  return guard([&] {
    checked_batch(b);
    const int v = find_traversal_variant(block, stack);
    if (v < 0) fail(MCRT_ERR_INVALID, "no traversal kernels compiled for this block size and stack depth");
    cuda_check(b->engine.set_variant(v), "batch traversal variant");
  });
}

int32_t mcrt_batch_submit(mcrt_batch* b, const mcrt_request* r, int64_t* id) {
  return guard([&] {
    checked_batch(b);
    const int64_t v = submit_request(b, r);
    if (id) *id = v;
  });
}

int32_t mcrt_batch_cancel(mcrt_batch* b, int64_t id) {
  return guard([&] {
    checked_batch(b);
    b->engine.cancel(id);
  });
}

int32_t mcrt_batch_step(mcrt_batch* b, mcrt_batch_event* events, int32_t max_events, int32_t* n_events,
                        int32_t* idle) {
  return guard([&] {
    checked_batch(b);
    if (max_events < 0 || (max_events > 0 && !events)) fail(MCRT_ERR_INVALID, "bad event buffer");
    check_slots(b);
    std::vector<BatchEvent> ev;
    bool is_idle = false, progressed = false;
    const unsigned earlier = b->engine.totals().status;
    cuda_check(b->engine.step(ev, &is_idle, &progressed), "batch step");
    if (!is_idle && !progressed) fail(MCRT_ERR_LIMIT, "the batch engine could not schedule a pending request");
    if (b->engine.totals().status & kStatusIterationLimit)
      fail(MCRT_ERR_CUDA, "a batched chunk did not finish within its iteration limit");
    check_walk(b->engine.totals().status & ~earlier);
    for (const BatchEvent& e : ev) b->pending.push_back(e);
    int n = 0;
    while (n < max_events && !b->pending.empty()) {
      const BatchEvent& e = b->pending.front();
      events[n++] = mcrt_batch_event{e.id, e.kind, e.samples};
      b->pending.pop_front();
    }
    if (n_events) *n_events = n;
    if (idle) *idle = is_idle && b->pending.empty() ? 1 : 0;
  });
}

int32_t mcrt_batch_render(mcrt_batch* b, int32_t count, const mcrt_request* requests) {
  return guard([&] {
    checked_batch(b);
    if (count < 0 || (count > 0 && !requests)) fail(MCRT_ERR_INVALID, "bad request list");
    for (int i = 0; i < count; i++) submit_request(b, requests + i);
    // The whole batch as one graph launch when no request needs host work
    // between chunks (BatchEngine::render_whole); otherwise, or for what is
    // left, chunk by chunk.
    {
      check_slots(b);
      std::vector<BatchEvent> ev;
      const unsigned earlier = b->engine.totals().status;
      bool rendered = false;
      cuda_check(b->engine.render_whole(ev, &rendered), "whole-batch render");
      if (b->engine.totals().status & kStatusIterationLimit)
        fail(MCRT_ERR_CUDA, "a batched chunk did not finish within its iteration limit");
      check_walk(b->engine.totals().status & ~earlier);
    }
    // Every step launches or finishes a chunk until the engine is idle, so
    // this loop ends; a step that does neither is a scheduling fault and fails
    // the call rather than spinning.
    bool idle = false;
    while (!idle) {
      check_slots(b);
      std::vector<BatchEvent> ev;
      const unsigned earlier = b->engine.totals().status;
      bool progressed = false;
      cuda_check(b->engine.step(ev, &idle, &progressed), "batch step");
      if (!idle && !progressed) fail(MCRT_ERR_LIMIT, "the batch engine could not schedule a pending request");
      if (b->engine.totals().status & kStatusIterationLimit)
        fail(MCRT_ERR_CUDA, "a batched chunk did not finish within its iteration limit");
      check_walk(b->engine.totals().status & ~earlier);
    }
  });
}

int32_t mcrt_batch_get_stats(mcrt_batch* b, mcrt_batch_stats* out) {
  return guard([&] {
    checked_batch(b);
    if (!out) fail(MCRT_ERR_INVALID, "out is NULL");
    const BatchTotals t = b->engine.totals();
    mcrt_batch_stats r{};
    r.closest_rays = t.closest;
    r.any_rays = t.any;
    r.samples = t.samples;
    r.chunks = t.chunks;
    r.graph_launches = t.graph_launches;
    r.gpu_ms = t.gpu_ms;
    r.arena_bytes = b->engine.arena().capacity();
    r.arena_used = b->engine.arena().used();
    r.path_bytes = b->engine.path_bytes();
    r.status = t.status;
    *out = r;
  });
}

}  // extern "C"
