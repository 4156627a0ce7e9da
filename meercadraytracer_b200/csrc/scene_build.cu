// GPU binned-SAH BVH build and geometry compile (src/bvh.ts:16-178,
// src/compile.ts:359-432).
//
// The build runs level by level, one thread block per node being split. It
// makes exactly the reference's decisions: per-triangle bounds and centroids
// are computed in double and rounded to float as the reference's Float32Array
// stores do; bins, areas and SAH costs are computed in double; this file is
// compiled without fused multiply-add contraction so every double operation
// rounds as JavaScript's does. Hence every node splits the same set of
// triangles as the reference, with the same 16 bins, leaves of at most 4
// (SAH leaves up to 16) and depth at most 100. Only the numbering of nodes
// (breadth first here) and the order of triangles inside a leaf may differ;
// partitions here are stable.
#include <cuda_runtime.h>

#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <vector>

#include "scene_build.cuh"

namespace mcrt {

namespace {

constexpr int kBins = 16;      // bvh.ts:3 (the default; a build may ask for up to kMaxBins)
constexpr int kMaxBins = 32;
static_assert(kBins <= kMaxBins, "the default bin count must fit the bin arrays");
constexpr int kMaxLeaf = 4;    // bvh.ts:4
constexpr int kBuildDepth = 100;  // bvh.ts:5
constexpr int kBuildBlock = 256;
// A node of at least kWideMin triangles is binned and partitioned by several
// blocks, kSegment triangles each; the results are combined with exact
// (order independent) atomics, so the decisions equal a single block's.
constexpr int kWideMin = 1 << 15;
constexpr int kSegment = 1 << 13;
// A node of at most kWarpMax triangles is split by one warp (8 per block):
// a whole block per node left most threads idle at the deep levels (512
// measured 5 % faster than 128 on an 83.9M-triangle build, 2048 no faster).
constexpr int kWarpMax = 512;
constexpr int kWarpsPerBlock = kBuildBlock / 32;
// A node of at most kTinyMax triangles is split by half a warp, one triangle
// per lane: its bins are never materialised (see k_split_tiny).
constexpr int kTinyMax = 16;

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  ~DevArray() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  T* ensure(size_t count) {
    if (count <= n && p) return p;
    reset();
    check(cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)), "cudaMalloc");
    n = std::max<size_t>(count, 1);
    return p;
  }
};

struct Slot {
  int node, first, count, depth;
};

// A resident mesh of instanced geometry.
struct DMeshRef {
  const float* pos;
  const float* nrm;      // or nullptr: face normals
  const float* uv;       // or nullptr: zeros
  const uint32_t* idx;   // or nullptr: not indexed
  int tri_count;
};

// An instance on the device: its world matrix, normal matrix (filled by
// k_instance_matrices), first output triangle and per-triangle words.
struct DInstance {
  double world[16];
  double nm[9];
  long long tri_base;
  int mesh, mirror, flags, side, flat;
  uint32_t material;
};

// mode: -1 leaf, 0 split at `bin` of `axis` (binned with lo and scale), 1
// split the run in half.
struct Split {
  int mode, axis, bin, nleft;
  double lo, scale;
};

// Accumulators of one wide node: bounds (node min xyz, -max xyz, centroid
// min xyz, -max xyz, all min-reduced), then bin counts and boxes.
struct WideAcc {
  float box[12];
  int cnt[3][kMaxBins];
  float bb[3][kMaxBins][6];
  unsigned done;
};

// Per level: blocks of each slot, where its blocks start, its wide index.
struct LevelPlan {
  const int* nb;     // blocks per slot
  const int* boff;   // first block of each slot
  const int* wid;    // index into the wide accumulators (valid when nb > 1)
  int active;        // slots
};

// Float min / max through integer atomics (exact, order independent).
__device__ __forceinline__ void atomic_min_f(float* a, float v) {
  if (__float_as_int(v) >= 0) {
    atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
  } else {
    atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
  }
}
__device__ __forceinline__ void atomic_max_f(float* a, float v) {
  if (__float_as_int(v) >= 0) {
    atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
  } else {
    atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
  }
}
__device__ __forceinline__ void atomic_min_d(double* a, double v) {
  long long b = __double_as_longlong(v);
  if (b >= 0) {
    atomicMin(reinterpret_cast<long long*>(a), b);
  } else {
    atomicMax(reinterpret_cast<unsigned long long*>(a), static_cast<unsigned long long>(b));
  }
}
__device__ __forceinline__ void atomic_max_d(double* a, double v) {
  long long b = __double_as_longlong(v);
  if (b >= 0) {
    atomicMax(reinterpret_cast<long long*>(a), b);
  } else {
    atomicMin(reinterpret_cast<unsigned long long*>(a), static_cast<unsigned long long>(b));
  }
}

__host__ __device__ inline double area(double x0, double y0, double z0, double x1, double y1, double z1) {
  const double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;  // bvh.ts:180-183
  return dx * dy + dy * dz + dz * dx;
}

// Math.hypot as V8 computes it: scaled by the largest magnitude, summed with
// Kahan compensation.
__host__ __device__ inline double js_hypot3(double a, double b, double c) {
  const double x[3] = {fabs(a), fabs(b), fabs(c)};
  double mx = 0;
  for (int i = 0; i < 3; i++) {
    if (isinf(x[i])) return INFINITY;
  }
  for (int i = 0; i < 3; i++) {
    if (isnan(x[i])) return NAN;
    if (x[i] > mx) mx = x[i];
  }
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (int i = 0; i < 3; i++) {
    const double n = x[i] / mx;
    const double summand = n * n - comp;
    const double prelim = sum + summand;
    comp = (prelim - sum) - summand;
    sum = prelim;
  }
  return sqrt(sum) * mx;
}

// Per-triangle box and centroid, bvh.ts:22-33.
__global__ void k_prepare(const float* __restrict__ tris, int n, float4* __restrict__ bmin, float4* __restrict__ bmax,
                          float4* __restrict__ cent, uint32_t* __restrict__ order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* o = tris + 9 * static_cast<size_t>(i);
  double lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    const double v0 = o[a], v1 = v0 + static_cast<double>(o[3 + a]), v2 = v0 + static_cast<double>(o[6 + a]);
    lo[a] = fmin(v0, fmin(v1, v2));
    hi[a] = fmax(v0, fmax(v1, v2));
  }
  bmin[i] = make_float4(static_cast<float>(lo[0]), static_cast<float>(lo[1]), static_cast<float>(lo[2]), 0.0f);
  bmax[i] = make_float4(static_cast<float>(hi[0]), static_cast<float>(hi[1]), static_cast<float>(hi[2]), 0.0f);
  cent[i] = make_float4(static_cast<float>((lo[0] + hi[0]) * 0.5), static_cast<float>((lo[1] + hi[1]) * 0.5),
                        static_cast<float>((lo[2] + hi[2]) * 0.5), 0.0f);
  order[i] = i;
}

__device__ __forceinline__ float comp4(float4 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

__device__ __forceinline__ int bin_of(float c, double lo, double scale, int bins) {
  return static_cast<int>(fmin(static_cast<double>(bins - 1), floor((static_cast<double>(c) - lo) * scale)));
}

// The slot whose blocks include block b: the last j with boff[j] <= b.
__device__ __forceinline__ int slot_of_block(const LevelPlan& lp, int b) {
  int lo = 0, hi = lp.active - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (lp.boff[mid] <= b) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

// Blocks of each slot (0 for a warp- or half-warp-sized node), its wide,
// small (one warp) and tiny (half a warp) flags.
__global__ void k_level_plan(const Slot* __restrict__ slots, int active, int* __restrict__ nb,
                             int* __restrict__ wide, int* __restrict__ small, int* __restrict__ tiny) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= active) return;
  const int c = slots[j].count;
  const int w = c >= kWideMin ? 1 : 0;
  const int ti = c <= kTinyMax ? 1 : 0;
  const int sm = !ti && c <= kWarpMax ? 1 : 0;
  nb[j] = w ? (c + kSegment - 1) / kSegment : (sm || ti ? 0 : 1);
  wide[j] = w;
  small[j] = sm;
  tiny[j] = ti;
}

__global__ void k_level_totals(const int* __restrict__ nb, const int* __restrict__ boff,
                               const int* __restrict__ wide, const int* __restrict__ wid,
                               const int* __restrict__ small, const int* __restrict__ spos,
                               const int* __restrict__ tiny, const int* __restrict__ tpos, int active,
                               int* __restrict__ out) {
  out[0] = boff[active - 1] + nb[active - 1];
  out[1] = wid[active - 1] + wide[active - 1];
  out[2] = spos[active - 1] + small[active - 1];
  out[3] = tpos[active - 1] + tiny[active - 1];
}

// The warp-sized slots of a level, listed, then the half-warp-sized ones
// (from totals[2] on).
__global__ void k_small_list(const int* __restrict__ small, const int* __restrict__ spos,
                             const int* __restrict__ tiny, const int* __restrict__ tpos, int active,
                             const int* __restrict__ totals, int* __restrict__ list) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= active) return;
  if (small[j]) list[spos[j]] = j;
  if (tiny[j]) list[totals[2] + tpos[j]] = j;
}

__global__ void k_wide_init(WideAcc* __restrict__ acc, int count) {
  const int i = blockIdx.x;
  if (i >= count) return;
  WideAcc& a = acc[i];
  for (int k = threadIdx.x; k < 12; k += blockDim.x) a.box[k] = INFINITY;
  for (int k = threadIdx.x; k < 3 * kMaxBins; k += blockDim.x) {
    const int ax = k / kMaxBins, b = k % kMaxBins;
    a.cnt[ax][b] = 0;
    for (int q = 0; q < 3; q++) {
      a.bb[ax][b][q] = INFINITY;
      a.bb[ax][b][3 + q] = -INFINITY;
    }
  }
  if (threadIdx.x == 0) a.done = 0;
}

// The 12 bounds of triangles order[first, end) reduced over the block into out[12].
__device__ void block_bounds(const uint32_t* __restrict__ order, int first, int end, const float4* __restrict__ bmin,
                             const float4* __restrict__ bmax, const float4* __restrict__ cent, float* out) {
  __shared__ float red[kBuildBlock / 32][12];
  const int tid = threadIdx.x;
  float m[12];
  for (int i = 0; i < 12; i++) m[i] = INFINITY;
  for (int k = first + tid; k < end; k += kBuildBlock) {
    const uint32_t t = order[k];
    const float4 a = bmin[t], b = bmax[t], c = cent[t];
    m[0] = fminf(m[0], a.x); m[1] = fminf(m[1], a.y); m[2] = fminf(m[2], a.z);
    m[3] = fminf(m[3], -b.x); m[4] = fminf(m[4], -b.y); m[5] = fminf(m[5], -b.z);
    m[6] = fminf(m[6], c.x); m[7] = fminf(m[7], c.y); m[8] = fminf(m[8], c.z);
    m[9] = fminf(m[9], -c.x); m[10] = fminf(m[10], -c.y); m[11] = fminf(m[11], -c.z);
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int i = 0; i < 12; i++) m[i] = fminf(m[i], __shfl_xor_sync(0xffffffffu, m[i], off));
  if ((tid & 31) == 0)
    for (int i = 0; i < 12; i++) red[tid >> 5][i] = m[i];
  __syncthreads();
  if (tid < 12) {
    float v = INFINITY;
    for (int w = 0; w < kBuildBlock / 32; w++) v = fminf(v, red[w][tid]);
    out[tid] = v;
  }
  __syncthreads();
}

// Partial bounds of each wide node, one segment per block.
__global__ void __launch_bounds__(kBuildBlock) k_bounds(LevelPlan lp, const Slot* __restrict__ slots,
                                                        const uint32_t* __restrict__ order,
                                                        const float4* __restrict__ bmin,
                                                        const float4* __restrict__ bmax,
                                                        const float4* __restrict__ cent, WideAcc* __restrict__ acc) {
  __shared__ int sj;
  if (threadIdx.x == 0) sj = slot_of_block(lp, blockIdx.x);
  __syncthreads();
  const int j = sj;
  if (lp.nb[j] <= 1) return;
  const Slot s = slots[j];
  const int seg = blockIdx.x - lp.boff[j];
  const int first = s.first + seg * kSegment;
  const int end = min(s.first + s.count, first + kSegment);
  __shared__ float part[12];
  block_bounds(order, first, end, bmin, bmax, cent, part);
  if (threadIdx.x < 12) atomic_min_f(&acc[lp.wid[j]].box[threadIdx.x], part[threadIdx.x]);
}

// The choice of a node (bvh.ts:137-163) from its cheapest split candidate
// (best_axis < 0: none): a SAH leaf, the binned split with `nleft` triangles
// on the left, or the median split when the bins put everything on one side.
__device__ void commit_choice(const Slot& s, const float* nb, double best_cost, int best_axis, int best_split,
                              int nleft, const double* lo, const double* scale, int j, int* nodes, Split* split,
                              int* is_split, bool wide, int* live_out) {
  Split d{1, 0, 0, s.count >> 1, 0.0, 0.0};
  bool leaf = false;
  if (best_axis >= 0) {
    const double parent_area = area(nb[0], nb[1], nb[2], -static_cast<double>(nb[3]), -static_cast<double>(nb[4]),
                                     -static_cast<double>(nb[5]));
    const double split_cost = 1 + (1 * best_cost) / fmax(parent_area, 1e-30);
    if (split_cost >= 1.0 * s.count && s.count <= 16) {
      leaf = true;
    } else {
      d = Split{0, best_axis, best_split, nleft, lo[best_axis], scale[best_axis]};
      if (nleft == 0 || nleft == s.count) d = Split{1, best_axis, 0, s.count >> 1, 0.0, 0.0};
    }
  }
  if (leaf) {
    int* nd = nodes + 3 * static_cast<size_t>(s.node);
    nd[0] = s.first; nd[1] = s.count; nd[2] = 0;
    split[j] = Split{-1, 0, 0, 0, 0.0, 0.0};
    is_split[j] = 0;
    live_out[j] = 0;
  } else {
    split[j] = d;
    is_split[j] = 1;
    // Children that will be leaves whatever the next level decides (few
    // enough triangles, or at the depth limit) are finished by this node's
    // scatter when one block partitions it; only the others go on.
    const bool last = s.depth + 1 >= kBuildDepth;
    const int small = wide ? 0 : (last || d.nleft <= kMaxLeaf ? 1 : 0) + (last || s.count - d.nleft <= kMaxLeaf ? 1 : 0);
    live_out[j] = 2 - small;
  }
}

// The SAH sweeps (bvh.ts:110-134) and the choice (bvh.ts:137-163) of one
// node from its bins, on one thread. nb: the node's 12 bounds as block_bounds
// gives them; lo / scale / live: the binning of each axis.
__device__ void decide(const Slot& s, const float* nb, const int (*cnt)[kMaxBins], const float (*bbox)[kMaxBins][6],
                       const double* lo, const double* scale, const bool* live, int bins, int j, int* nodes,
                       Split* split, int* is_split, bool wide, int* live_out) {
  // Called by the 32 lanes of one warp, lane i holding bin i. The right
  // sweep's unions and counts are suffix scans, the left sweep's prefix
  // scans (min, max and sums are exact in any order, and the areas and costs
  // are the same expressions, so every candidate cost equals the one-thread
  // sweep's); the first minimum in (axis, split) order wins, as there. The
  // unions are taken on the float bin bounds and widened to double for the
  // areas: min and max commute with the exact float-to-double conversion, so
  // the values are the reference's, for half the shuffles.
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  double best_cost = INFINITY;
  int best_axis = -1, best_split = -1;
  for (int a = 0; a < 3; a++) {
    if (!live[a]) continue;
    const bool in = lane < bins;
    const float* o = bbox[a][lane < kMaxBins ? lane : 0];
    int c = in ? cnt[a][lane] : 0;
    float b0 = in ? o[0] : INFINITY, b1 = in ? o[1] : INFINITY, b2 = in ? o[2] : INFINITY;
    float b3 = in ? o[3] : -INFINITY, b4 = in ? o[4] : -INFINITY, b5 = in ? o[5] : -INFINITY;
    // Suffix: bins [lane, bins).
    int rc = c;
    float r0 = b0, r1 = b1, r2 = b2, r3 = b3, r4 = b4, r5 = b5;
    for (int off = 1; off < 32; off <<= 1) {
      const int oc = __shfl_down_sync(full, rc, off);
      const float o0 = __shfl_down_sync(full, r0, off), o1 = __shfl_down_sync(full, r1, off);
      const float o2 = __shfl_down_sync(full, r2, off), o3 = __shfl_down_sync(full, r3, off);
      const float o4 = __shfl_down_sync(full, r4, off), o5 = __shfl_down_sync(full, r5, off);
      if (lane + off < 32) {
        rc += oc;
        r0 = fminf(r0, o0); r1 = fminf(r1, o1); r2 = fminf(r2, o2);
        r3 = fmaxf(r3, o3); r4 = fmaxf(r4, o4); r5 = fmaxf(r5, o5);
      }
    }
    const double right_area = rc > 0 ? area(r0, r1, r2, r3, r4, r5) : 0;
    // Prefix: bins [0, lane].
    int lc = c;
    float l0 = b0, l1 = b1, l2 = b2, l3 = b3, l4 = b4, l5 = b5;
    for (int off = 1; off < 32; off <<= 1) {
      const int oc = __shfl_up_sync(full, lc, off);
      const float o0 = __shfl_up_sync(full, l0, off), o1 = __shfl_up_sync(full, l1, off);
      const float o2 = __shfl_up_sync(full, l2, off), o3 = __shfl_up_sync(full, l3, off);
      const float o4 = __shfl_up_sync(full, l4, off), o5 = __shfl_up_sync(full, l5, off);
      if (lane >= off) {
        lc += oc;
        l0 = fminf(l0, o0); l1 = fminf(l1, o1); l2 = fminf(l2, o2);
        l3 = fmaxf(l3, o3); l4 = fmaxf(l4, o4); l5 = fmaxf(l5, o5);
      }
    }
    // Split after bin `lane`: the left union with the right union from lane + 1.
    const int rc2 = __shfl_down_sync(full, rc, 1);
    const double ra2 = __shfl_down_sync(full, right_area, 1);
    double cost = INFINITY;
    if (lane < bins - 1 && lc != 0 && rc2 != 0) {
      cost = lc * area(l0, l1, l2, l3, l4, l5) + rc2 * ra2;
      if (isnan(cost)) cost = INFINITY;
    }
    int at = lane;
    for (int off = 16; off > 0; off >>= 1) {
      const double oc = __shfl_xor_sync(full, cost, off);
      const int oi = __shfl_xor_sync(full, at, off);
      if (oc < cost || (oc == cost && oi < at)) {
        cost = oc;
        at = oi;
      }
    }
    if (cost < best_cost) {
      best_cost = cost;
      best_axis = a;
      best_split = at;
    }
  }
  if (lane != 0) return;
  int nleft = 0;
  if (best_axis >= 0)
    for (int i = 0; i <= best_split; i++) nleft += cnt[best_axis][i];
  commit_choice(s, nb, best_cost, best_axis, best_split, nleft, lo, scale, j, nodes, split, is_split, wide, live_out);
}

// Bounds, leaf test, binning and SAH choice of every node of a level
// (bvh.ts:55-144). A node of one block is handled by that block alone; the
// blocks of a wide node bin their segments into the node's accumulators
// (k_bounds has reduced its bounds) and the last block to finish decides.
__global__ void __launch_bounds__(kBuildBlock) k_split(LevelPlan lp, const Slot* __restrict__ slots,
                                                       const uint32_t* __restrict__ order,
                                                       const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                                                       const float4* __restrict__ cent, float* __restrict__ bounds,
                                                       int* __restrict__ nodes, Split* __restrict__ split,
                                                       int* __restrict__ is_split, WideAcc* __restrict__ acc,
                                                       int bins, int* __restrict__ live_children) {
  __shared__ int sj;
  __shared__ float nb[12];  // node min xyz, -max xyz, centroid min xyz, -max xyz
  __shared__ int cnt[3][kMaxBins];
  __shared__ float bbox[3][kMaxBins][6];
  __shared__ int last;
  const int tid = threadIdx.x;
  if (tid == 0) sj = slot_of_block(lp, blockIdx.x);
  __syncthreads();
  const int j = sj;
  const Slot s = slots[j];
  const int blocks = lp.nb[j];
  const bool wide = blocks > 1;
  const int seg = blockIdx.x - lp.boff[j];
  WideAcc* wa = wide ? acc + lp.wid[j] : nullptr;
  if (wide) {
    if (tid < 12) nb[tid] = __ldcg(&wa->box[tid]);
    __syncthreads();
  } else {
    block_bounds(order, s.first, s.first + s.count, bmin, bmax, cent, nb);
  }
  if (tid == 0 && seg == 0) {
    float* bo = bounds + 6 * static_cast<size_t>(s.node);
    bo[0] = nb[0]; bo[1] = nb[1]; bo[2] = nb[2];
    bo[3] = -nb[3]; bo[4] = -nb[4]; bo[5] = -nb[5];
  }
  if (s.count <= kMaxLeaf || s.depth >= kBuildDepth) {
    if (tid == 0 && seg == 0) {
      int* nd = nodes + 3 * static_cast<size_t>(s.node);
      nd[0] = s.first; nd[1] = s.count; nd[2] = 0;
      split[j] = Split{-1, 0, 0, 0, 0.0, 0.0};
      is_split[j] = 0;
      live_children[j] = 0;
    }
    return;
  }
  for (int i = tid; i < 3 * kMaxBins; i += kBuildBlock) {
    const int a = i / kMaxBins, b = i % kMaxBins;
    cnt[a][b] = 0;
    for (int q = 0; q < 3; q++) {
      bbox[a][b][q] = INFINITY;
      bbox[a][b][3 + q] = -INFINITY;
    }
  }
  // Bin the centroids along every axis with extent (bvh.ts:89-109).
  const double cmin[3] = {nb[6], nb[7], nb[8]};
  const double cmax[3] = {-nb[9], -nb[10], -nb[11]};
  double lo[3], scale[3];
  bool live[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = cmin[a];
    const double extent = cmax[a] - lo[a];
    live[a] = extent > 0;
    scale[a] = live[a] ? bins / extent : 0.0;
  }
  __syncthreads();
  const int first = wide ? s.first + seg * kSegment : s.first;
  const int end = wide ? min(s.first + s.count, first + kSegment) : s.first + s.count;
  for (int k = first + tid; k < end; k += kBuildBlock) {
    const uint32_t t = order[k];
    const float4 a4 = bmin[t], b4 = bmax[t], c4 = cent[t];
    for (int a = 0; a < 3; a++) {
      if (!live[a]) continue;
      const int b = bin_of(comp4(c4, a), lo[a], scale[a], bins);
      atomicAdd(&cnt[a][b], 1);
      atomic_min_f(&bbox[a][b][0], a4.x);
      atomic_min_f(&bbox[a][b][1], a4.y);
      atomic_min_f(&bbox[a][b][2], a4.z);
      atomic_max_f(&bbox[a][b][3], b4.x);
      atomic_max_f(&bbox[a][b][4], b4.y);
      atomic_max_f(&bbox[a][b][5], b4.z);
    }
  }
  __syncthreads();
  if (wide) {
    // Fold this segment's bins into the node's, then let the last block decide.
    for (int i = tid; i < 3 * bins; i += kBuildBlock) {
      const int a = i / bins, b = i % bins;
      if (!live[a] || cnt[a][b] == 0) continue;
      atomicAdd(&wa->cnt[a][b], cnt[a][b]);
      for (int q = 0; q < 3; q++) {
        atomic_min_f(&wa->bb[a][b][q], bbox[a][b][q]);
        atomic_max_f(&wa->bb[a][b][3 + q], bbox[a][b][3 + q]);
      }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(&wa->done, 1u) == static_cast<unsigned>(blocks - 1) ? 1 : 0;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int i = tid; i < 3 * bins; i += kBuildBlock) {
      const int a = i / bins, b = i % bins;
      cnt[a][b] = __ldcg(&wa->cnt[a][b]);
      for (int q = 0; q < 6; q++) bbox[a][b][q] = __ldcg(&wa->bb[a][b][q]);
    }
    __syncthreads();
  }
  if (tid < 32) decide(s, nb, cnt, bbox, lo, scale, live, bins, j, nodes, split, is_split, wide, live_children);
}

// k_split for warp-sized nodes: one warp per node, 8 per block, with the
// node's bounds reduced over shuffles and its bins in the warp's own shared
// memory; the same decisions as a block would take.
__global__ void __launch_bounds__(kBuildBlock) k_split_small(const int* __restrict__ list, int count,
                                                             const Slot* __restrict__ slots,
                                                             const uint32_t* __restrict__ order,
                                                             const float4* __restrict__ bmin,
                                                             const float4* __restrict__ bmax,
                                                             const float4* __restrict__ cent,
                                                             float* __restrict__ bounds, int* __restrict__ nodes,
                                                             Split* __restrict__ split, int* __restrict__ is_split,
                                                             int bins, int* __restrict__ live_children) {
  __shared__ int cnt_s[kWarpsPerBlock][3][kMaxBins];
  __shared__ float bbox_s[kWarpsPerBlock][3][kMaxBins][6];
  const unsigned full = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * kWarpsPerBlock + w;
  if (k >= count) return;  // the whole warp
  const int j = list[k];
  const Slot s = slots[j];
  float nb[12];
  for (int i = 0; i < 12; i++) nb[i] = INFINITY;
  for (int q = s.first + lane; q < s.first + s.count; q += 32) {
    const uint32_t t = order[q];
    const float4 a = bmin[t], b = bmax[t], c = cent[t];
    nb[0] = fminf(nb[0], a.x); nb[1] = fminf(nb[1], a.y); nb[2] = fminf(nb[2], a.z);
    nb[3] = fminf(nb[3], -b.x); nb[4] = fminf(nb[4], -b.y); nb[5] = fminf(nb[5], -b.z);
    nb[6] = fminf(nb[6], c.x); nb[7] = fminf(nb[7], c.y); nb[8] = fminf(nb[8], c.z);
    nb[9] = fminf(nb[9], -c.x); nb[10] = fminf(nb[10], -c.y); nb[11] = fminf(nb[11], -c.z);
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int i = 0; i < 12; i++) nb[i] = fminf(nb[i], __shfl_xor_sync(full, nb[i], off));
  if (lane == 0) {
    float* bo = bounds + 6 * static_cast<size_t>(s.node);
    bo[0] = nb[0]; bo[1] = nb[1]; bo[2] = nb[2];
    bo[3] = -nb[3]; bo[4] = -nb[4]; bo[5] = -nb[5];
  }
  if (s.count <= kMaxLeaf || s.depth >= kBuildDepth) {
    if (lane == 0) {
      int* nd = nodes + 3 * static_cast<size_t>(s.node);
      nd[0] = s.first; nd[1] = s.count; nd[2] = 0;
      split[j] = Split{-1, 0, 0, 0, 0.0, 0.0};
      is_split[j] = 0;
      live_children[j] = 0;
    }
    return;
  }
  int (*cnt)[kMaxBins] = cnt_s[w];
  float (*bbox)[kMaxBins][6] = bbox_s[w];
  for (int i = lane; i < 3 * kMaxBins; i += 32) {
    const int a = i / kMaxBins, b = i % kMaxBins;
    cnt[a][b] = 0;
    for (int q = 0; q < 3; q++) {
      bbox[a][b][q] = INFINITY;
      bbox[a][b][3 + q] = -INFINITY;
    }
  }
  const double cmin[3] = {nb[6], nb[7], nb[8]};
  const double cmax[3] = {-nb[9], -nb[10], -nb[11]};
  double lo[3], scale[3];
  bool live[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = cmin[a];
    const double extent = cmax[a] - lo[a];
    live[a] = extent > 0;
    scale[a] = live[a] ? bins / extent : 0.0;
  }
  __syncwarp();
  for (int q = s.first + lane; q < s.first + s.count; q += 32) {
    const uint32_t t = order[q];
    const float4 a4 = bmin[t], b4 = bmax[t], c4 = cent[t];
    for (int a = 0; a < 3; a++) {
      if (!live[a]) continue;
      const int b = bin_of(comp4(c4, a), lo[a], scale[a], bins);
      atomicAdd(&cnt[a][b], 1);
      atomic_min_f(&bbox[a][b][0], a4.x);
      atomic_min_f(&bbox[a][b][1], a4.y);
      atomic_min_f(&bbox[a][b][2], a4.z);
      atomic_max_f(&bbox[a][b][3], b4.x);
      atomic_max_f(&bbox[a][b][4], b4.y);
      atomic_max_f(&bbox[a][b][5], b4.z);
    }
  }
  __syncwarp();
  decide(s, nb, cnt, bbox, lo, scale, live, bins, j, nodes, split, is_split, false, live_children);
}

// k_split for nodes of at most kTinyMax triangles: half a warp per node, one
// triangle per lane, so two nodes per warp. Per axis the lanes sort their
// triangles by bin (a bitonic network on bin * 16 + lane), then prefix and
// suffix unions over the sorted order give, at the last triangle of each
// occupied bin b, the left set {bins <= b} and the right set {bins > b} of the
// split after b. Split positions between occupied bins have the same two sets
// and so the same cost as the occupied bin before them, and positions before
// the first or from the last occupied bin leave a side empty, so the first
// minimum over these candidates in (axis, split) order is the binned sweep's:
// the same costs from the same float unions, the same choice.
__global__ void __launch_bounds__(kBuildBlock) k_split_tiny(const int* __restrict__ list, int count,
                                                            const Slot* __restrict__ slots,
                                                            const uint32_t* __restrict__ order,
                                                            const float4* __restrict__ bmin,
                                                            const float4* __restrict__ bmax,
                                                            const float4* __restrict__ cent,
                                                            float* __restrict__ bounds, int* __restrict__ nodes,
                                                            Split* __restrict__ split, int* __restrict__ is_split,
                                                            int bins, int* __restrict__ live_children) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, i = lane & 15;
  const int pair = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (2 * pair >= count) return;  // the whole warp
  const int k = 2 * pair + (lane >> 4);
  const bool valid = k < count;  // this half holds a node (every lane still shuffles)
  const int j = valid ? list[k] : 0;
  const Slot s = valid ? slots[j] : Slot{0, 0, 0, 0};
  const int n = s.count;
  const bool has = i < n;
  float m[12];
  for (int q = 0; q < 12; q++) m[q] = INFINITY;
  float4 a4 = make_float4(INFINITY, INFINITY, INFINITY, 0.0f), b4 = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
  float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (has) {
    const uint32_t t = order[s.first + i];
    a4 = bmin[t];
    b4 = bmax[t];
    c4 = cent[t];
    m[0] = a4.x; m[1] = a4.y; m[2] = a4.z;
    m[3] = -b4.x; m[4] = -b4.y; m[5] = -b4.z;
    m[6] = c4.x; m[7] = c4.y; m[8] = c4.z;
    m[9] = -c4.x; m[10] = -c4.y; m[11] = -c4.z;
  }
  for (int off = 8; off > 0; off >>= 1)
    for (int q = 0; q < 12; q++) m[q] = fminf(m[q], __shfl_xor_sync(full, m[q], off, 16));
  const bool leafy = n <= kMaxLeaf || s.depth >= kBuildDepth;
  if (valid && i == 0) {
    float* bo = bounds + 6 * static_cast<size_t>(s.node);
    bo[0] = m[0]; bo[1] = m[1]; bo[2] = m[2];
    bo[3] = -m[3]; bo[4] = -m[4]; bo[5] = -m[5];
    if (leafy) {
      int* nd = nodes + 3 * static_cast<size_t>(s.node);
      nd[0] = s.first; nd[1] = s.count; nd[2] = 0;
      split[j] = Split{-1, 0, 0, 0, 0.0, 0.0};
      is_split[j] = 0;
      live_children[j] = 0;
    }
  }
  const bool work = valid && !leafy;
  double lo[3], scale[3];
  bool live[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = m[6 + a];
    const double extent = -static_cast<double>(m[9 + a]) - lo[a];
    live[a] = work && extent > 0;
    scale[a] = live[a] ? bins / extent : 0.0;
  }
  double best_cost = INFINITY;
  int best_axis = -1, best_split = -1, best_nleft = 0;
  for (int a = 0; a < 3; a++) {
    // Sort the half's triangles by bin; lanes without one sort last.
    const int bin = (has && live[a]) ? bin_of(comp4(c4, a), lo[a], scale[a], bins) : kMaxBins;
    int key = (bin << 4) | i;
    for (int kk = 2; kk <= 16; kk <<= 1) {
      for (int jj = kk >> 1; jj > 0; jj >>= 1) {
        const int other = __shfl_xor_sync(full, key, jj, 16);
        const bool keep_min = ((i & jj) == 0) == ((i & kk) == 0);
        key = keep_min ? min(key, other) : max(key, other);
      }
    }
    const int src = key & 15, sb = key >> 4;
    float l0 = __shfl_sync(full, a4.x, src, 16), l1 = __shfl_sync(full, a4.y, src, 16);
    float l2 = __shfl_sync(full, a4.z, src, 16), l3 = __shfl_sync(full, b4.x, src, 16);
    float l4 = __shfl_sync(full, b4.y, src, 16), l5 = __shfl_sync(full, b4.z, src, 16);
    float r0 = l0, r1 = l1, r2 = l2, r3 = l3, r4 = l4, r5 = l5;
    for (int off = 1; off < 16; off <<= 1) {
      const float o0 = __shfl_up_sync(full, l0, off, 16), o1 = __shfl_up_sync(full, l1, off, 16);
      const float o2 = __shfl_up_sync(full, l2, off, 16), o3 = __shfl_up_sync(full, l3, off, 16);
      const float o4 = __shfl_up_sync(full, l4, off, 16), o5 = __shfl_up_sync(full, l5, off, 16);
      if (i >= off) {
        l0 = fminf(l0, o0); l1 = fminf(l1, o1); l2 = fminf(l2, o2);
        l3 = fmaxf(l3, o3); l4 = fmaxf(l4, o4); l5 = fmaxf(l5, o5);
      }
      const float p0 = __shfl_down_sync(full, r0, off, 16), p1 = __shfl_down_sync(full, r1, off, 16);
      const float p2 = __shfl_down_sync(full, r2, off, 16), p3 = __shfl_down_sync(full, r3, off, 16);
      const float p4 = __shfl_down_sync(full, r4, off, 16), p5 = __shfl_down_sync(full, r5, off, 16);
      if (i + off < 16) {
        r0 = fminf(r0, p0); r1 = fminf(r1, p1); r2 = fminf(r2, p2);
        r3 = fmaxf(r3, p3); r4 = fmaxf(r4, p4); r5 = fmaxf(r5, p5);
      }
    }
    // Split after bin sb (this lane the last of its bin): positions [0, i] left, (i, n) right.
    const double right_here = i < n ? area(r0, r1, r2, r3, r4, r5) : 0;
    const double right_area = __shfl_down_sync(full, right_here, 1, 16);
    const int next_bin = __shfl_down_sync(full, sb, 1, 16);
    double cost = INFINITY;
    const int lc = i + 1, rc = n - i - 1;
    if (live[a] && i < n - 1 && sb != next_bin) {
      cost = lc * area(l0, l1, l2, l3, l4, l5) + rc * right_area;
      if (isnan(cost)) cost = INFINITY;
    }
    int at = sb, atl = lc;
    for (int off = 8; off > 0; off >>= 1) {
      const double oc = __shfl_xor_sync(full, cost, off, 16);
      const int oi = __shfl_xor_sync(full, at, off, 16);
      const int ol = __shfl_xor_sync(full, atl, off, 16);
      if (oc < cost || (oc == cost && oi < at)) {
        cost = oc;
        at = oi;
        atl = ol;
      }
    }
    if (cost < best_cost) {
      best_cost = cost;
      best_axis = a;
      best_split = at;
      best_nleft = atl;
    }
  }
  if (work && i == 0)
    commit_choice(s, m, best_cost, best_axis, best_split, best_nleft, lo, scale, j, nodes, split, is_split, false,
                  live_children);
}

// The first triangle of a block's share of its node, and the end.
__device__ __forceinline__ void block_range(const Slot& s, bool wide, int seg, int& first, int& end) {
  first = wide ? s.first + seg * kSegment : s.first;
  end = wide ? min(s.first + s.count, first + kSegment) : s.first + s.count;
}

__device__ __forceinline__ int goes_left(const Split& d, const Slot& s, int k, const float4* __restrict__ cent,
                                         const uint32_t* __restrict__ order, int bins) {
  return d.mode == 0 ? (bin_of(comp4(cent[order[k]], d.axis), d.lo, d.scale, bins) <= d.bin ? 1 : 0)
                     : (k - s.first < d.nleft ? 1 : 0);
}

// After a split node's partition: its node entry, and its children either
// queued for the next level (at live_pos[j]) or, when they must be leaves (at
// most 4 triangles, or at the depth limit; never for a wide parent), finished
// here: bounds (bvh.ts:55-72 on their triangles), node, and their triangles
// in both order buffers, since no later level copies them across.
__device__ void place_children(const Slot& s, const Split& d, bool wide, int j, const int* __restrict__ rank,
                               int child_base, int* __restrict__ nodes, Slot* __restrict__ next,
                               const int* __restrict__ live_pos, const uint32_t* order_out, uint32_t* order_keep,
                               const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                               float* __restrict__ bounds) {
  const int left = child_base + 2 * rank[j];
  int* nd = nodes + 3 * static_cast<size_t>(s.node);
  nd[0] = left; nd[1] = 0; nd[2] = d.axis;
  const Slot kids[2] = {Slot{left, s.first, d.nleft, s.depth + 1},
                        Slot{left + 1, s.first + d.nleft, s.count - d.nleft, s.depth + 1}};
  int at = live_pos[j];
  for (int c = 0; c < 2; c++) {
    const Slot& k = kids[c];
    const bool small = !wide && (k.count <= kMaxLeaf || k.depth >= kBuildDepth);
    if (!small) {
      next[at++] = k;
      continue;
    }
    float m[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int q = k.first; q < k.first + k.count; q++) {
      const uint32_t t = order_out[q];
      order_keep[q] = t;
      const float4 a = bmin[t], b = bmax[t];
      m[0] = fminf(m[0], a.x); m[1] = fminf(m[1], a.y); m[2] = fminf(m[2], a.z);
      m[3] = fmaxf(m[3], b.x); m[4] = fmaxf(m[4], b.y); m[5] = fmaxf(m[5], b.z);
    }
    float* bo = bounds + 6 * static_cast<size_t>(k.node);
    for (int a = 0; a < 6; a++) bo[a] = m[a];
    int* kn = nodes + 3 * static_cast<size_t>(k.node);
    kn[0] = k.first; kn[1] = k.count; kn[2] = 0;
  }
}

// Triangles going left in each block's segment of a wide split node; 0 for
// every other block.
__global__ void __launch_bounds__(kBuildBlock) k_count_left(LevelPlan lp, const Slot* __restrict__ slots,
                                                            const Split* __restrict__ split,
                                                            const uint32_t* __restrict__ order,
                                                            const float4* __restrict__ cent, int bins,
                                                            int* __restrict__ blk_left) {
  __shared__ int sj;
  __shared__ int part[kBuildBlock / 32];
  const int tid = threadIdx.x;
  if (tid == 0) sj = slot_of_block(lp, blockIdx.x);
  __syncthreads();
  const int j = sj;
  const Split d = split[j];
  if (lp.nb[j] <= 1 || d.mode < 0) {
    if (tid == 0) blk_left[blockIdx.x] = 0;
    return;
  }
  const Slot s = slots[j];
  int first, end;
  block_range(s, true, blockIdx.x - lp.boff[j], first, end);
  int c = 0;
  for (int k = first + tid; k < end; k += kBuildBlock) c += goes_left(d, s, k, cent, order, bins);
  for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
  if ((tid & 31) == 0) part[tid >> 5] = c;
  __syncthreads();
  if (tid == 0) {
    int t = 0;
    for (int w = 0; w < kBuildBlock / 32; w++) t += part[w];
    blk_left[blockIdx.x] = t;
  }
}

// Stable partition of each split node's run and its two children
// (bvh.ts:145-171); leaves copy their run unchanged. A wide node's blocks
// place their segments after the lefts and rights of the blocks before them
// (blk_pre: exclusive sums of k_count_left over all blocks).
__global__ void __launch_bounds__(kBuildBlock) k_scatter(LevelPlan lp, const Slot* __restrict__ slots,
                                                         const Split* __restrict__ split,
                                                         const int* __restrict__ rank, int child_base,
                                                         const uint32_t* order,
                                                         uint32_t* __restrict__ order_out,
                                                         const float4* __restrict__ cent, int* __restrict__ nodes,
                                                         Slot* __restrict__ next, const int* __restrict__ blk_pre,
                                                         int bins, const int* __restrict__ live_pos,
                                                         uint32_t* order_keep, const float4* __restrict__ bmin,
                                                         const float4* __restrict__ bmax, float* __restrict__ bounds) {
  using Scan = cub::BlockScan<int, kBuildBlock>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ int sj;
  const int tid = threadIdx.x;
  if (tid == 0) sj = slot_of_block(lp, blockIdx.x);
  __syncthreads();
  const int j = sj;
  const Slot s = slots[j];
  const Split d = split[j];
  const bool wide = lp.nb[j] > 1;
  const int seg = blockIdx.x - lp.boff[j];
  int first, end;
  block_range(s, wide, seg, first, end);
  if (d.mode < 0) {
    for (int k = first + tid; k < end; k += kBuildBlock) order_out[k] = order[k];
    return;
  }
  int left_off = wide ? blk_pre[blockIdx.x] - blk_pre[lp.boff[j]] : 0;
  int right_off = (first - s.first) - left_off;
  for (int base = first; base < end; base += kBuildBlock) {
    const int k = base + tid;
    int f = 0;
    uint32_t t = 0;
    if (k < end) {
      t = order[k];
      f = goes_left(d, s, k, cent, order, bins);
    }
    int pre = 0, total = 0;
    Scan(scan_tmp).ExclusiveSum(f, pre, total);
    if (k < end) {
      const int dst = f ? s.first + left_off + pre : s.first + d.nleft + right_off + (tid - pre);
      order_out[dst] = t;
    }
    const int in_chunk = min(kBuildBlock, end - base);
    left_off += total;
    right_off += in_chunk - total;
    __syncthreads();
  }
  if (seg != 0) return;
  if (!wide) __syncthreads();  // this block's order_out writes are visible to thread 0
  if (tid == 0)
    place_children(s, d, wide, j, rank, child_base, nodes, next, live_pos, order_out, order_keep, bmin, bmax, bounds);
}

// k_scatter for warp-sized nodes: one warp per node, a stable partition by
// ballots over 32-triangle chunks.
__global__ void __launch_bounds__(kBuildBlock) k_scatter_small(
    const int* __restrict__ list, int count, const Slot* __restrict__ slots, const Split* __restrict__ split,
    const int* __restrict__ rank, int child_base, const uint32_t* order, uint32_t* __restrict__ order_out,
    const float4* __restrict__ cent, int* __restrict__ nodes, Slot* __restrict__ next, int bins,
    const int* __restrict__ live_pos, uint32_t* order_keep, const float4* __restrict__ bmin,
    const float4* __restrict__ bmax, float* __restrict__ bounds) {
  const unsigned full = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = blockIdx.x * kWarpsPerBlock + w;
  if (k >= count) return;  // the whole warp
  const int j = list[k];
  const Slot s = slots[j];
  const Split d = split[j];
  const int end = s.first + s.count;
  if (d.mode < 0) {
    for (int q = s.first + lane; q < end; q += 32) order_out[q] = order[q];
    return;
  }
  int left_off = 0, right_off = 0;
  for (int base = s.first; base < end; base += 32) {
    const int q = base + lane;
    int f = 0;
    uint32_t t = 0;
    if (q < end) {
      t = order[q];
      f = goes_left(d, s, q, cent, order, bins);
    }
    const unsigned ballot = __ballot_sync(full, f);
    const int pre = __popc(ballot & ((1u << lane) - 1u));
    const int total = __popc(ballot);
    if (q < end) {
      const int dst = f ? s.first + left_off + pre : s.first + d.nleft + right_off + (lane - pre);
      order_out[dst] = t;
    }
    left_off += total;
    right_off += min(32, end - base) - total;
  }
  __syncwarp();  // the warp's order_out writes are visible to lane 0
  if (lane == 0)
    place_children(s, d, false, j, rank, child_base, nodes, next, live_pos, order_out, order_keep, bmin, bmax,
                   bounds);
}

// ---- compile (src/compile.ts:336-343 and 359-432)

// Float32 triangles from the sink's doubles, and the largest coordinate.
__global__ void k_sink_triangles(const double* __restrict__ p, int n, float* __restrict__ tris,
                                 unsigned long long* __restrict__ max_coord) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double mc = 0;
  if (i < n) {
    const double* q = p + 9 * static_cast<size_t>(i);
    float* t = tris + 9 * static_cast<size_t>(i);
    for (int a = 0; a < 3; a++) {
      t[a] = static_cast<float>(q[a]);
      t[3 + a] = static_cast<float>(q[3 + a] - q[a]);
      t[6 + a] = static_cast<float>(q[6 + a] - q[a]);
    }
    for (int k = 0; k < 9; k++) mc = fmax(mc, fabs(q[k]));
  }
  for (int off = 16; off > 0; off >>= 1) mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, off));
  if ((threadIdx.x & 31) == 0) atomicMax(max_coord, static_cast<unsigned long long>(__double_as_longlong(mc)));
}

// Everything in BVH order (compile.ts:364-377).
__global__ void k_reorder(const uint32_t* __restrict__ order, int n, const float* __restrict__ tris_in,
                          const double* __restrict__ nrm, const double* __restrict__ uv,
                          const double* __restrict__ colors, const uint8_t* __restrict__ has_color, int any_colors,
                          const uint32_t* __restrict__ mats, const uint8_t* __restrict__ flags,
                          const uint8_t* __restrict__ sides, float* __restrict__ tris_out,
                          float* __restrict__ nrm_out, float* __restrict__ uv_out, float* __restrict__ col_out,
                          uint32_t* __restrict__ mats_out, uint8_t* __restrict__ flags_out,
                          uint8_t* __restrict__ sides_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t s = order[i];
  for (int k = 0; k < 9; k++) tris_out[9 * static_cast<size_t>(i) + k] = tris_in[9 * s + k];
  for (int k = 0; k < 9; k++) nrm_out[9 * static_cast<size_t>(i) + k] = static_cast<float>(nrm[9 * s + k]);
  for (int k = 0; k < 6; k++) uv_out[6 * static_cast<size_t>(i) + k] = static_cast<float>(uv[6 * s + k]);
  if (any_colors) {
    for (int k = 0; k < 12; k++)
      col_out[12 * static_cast<size_t>(i) + k] = has_color[s] ? static_cast<float>(colors[12 * s + k]) : 1.0f;
  }
  mats_out[i] = mats[s];
  flags_out[i] = flags[s];
  sides_out[i] = sides[s];
}

// writeTangent (compile.ts:406-432) and the vertex bounding box (compile.ts:378-385).
__global__ void k_tangents(const float* __restrict__ tris, const float* __restrict__ uvs, int n,
                           float* __restrict__ tangents, double* __restrict__ box) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (i < n) {
    const float* o = tris + 9 * static_cast<size_t>(i);
    const float* u6 = uvs + 6 * static_cast<size_t>(i);
    for (int v = 0; v < 3; v++) {
      for (int a = 0; a < 3; a++) {
        const double x = static_cast<double>(o[a]) + (v == 1 ? o[3 + a] : v == 2 ? o[6 + a] : 0.0f);
        lo[a] = fmin(lo[a], x);
        hi[a] = fmax(hi[a], x);
      }
    }
    const double e1x = o[3], e1y = o[4], e1z = o[5], e2x = o[6], e2y = o[7], e2z = o[8];
    const double du1 = static_cast<double>(u6[2]) - u6[0], dv1 = static_cast<double>(u6[3]) - u6[1];
    const double du2 = static_cast<double>(u6[4]) - u6[0], dv2 = static_cast<double>(u6[5]) - u6[1];
    const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const double d = du1 * dv2 - du2 * dv1;
    double tx, ty, tz, sign = 1;
    if (fabs(d) > 1e-20) {
      const double r = 1 / d;
      tx = (e1x * dv2 - e2x * dv1) * r;
      ty = (e1y * dv2 - e2y * dv1) * r;
      tz = (e1z * dv2 - e2z * dv1) * r;
      const double bx = (e2x * du1 - e1x * du2) * r, by = (e2y * du1 - e1y * du2) * r, bz = (e2z * du1 - e1z * du2) * r;
      const double cx = ny * tz - nz * ty, cy = nz * tx - nx * tz, cz = nx * ty - ny * tx;
      sign = cx * bx + cy * by + cz * bz < 0 ? -1 : 1;
    } else if (fabs(nx) < 0.9 * js_hypot3(nx, ny, nz)) {
      tx = 0; ty = -nz; tz = ny;
    } else {
      tx = nz; ty = 0; tz = -nx;
    }
    double length = js_hypot3(tx, ty, tz);
    if (length == 0 || isnan(length)) length = 1;
    float* t = tangents + 4 * static_cast<size_t>(i);
    t[0] = static_cast<float>(tx / length);
    t[1] = static_cast<float>(ty / length);
    t[2] = static_cast<float>(tz / length);
    t[3] = static_cast<float>(sign);
  }
  for (int off = 16; off > 0; off >>= 1) {
    for (int a = 0; a < 3; a++) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
    }
  }
  if ((threadIdx.x & 31) == 0 && i - static_cast<int>(threadIdx.x & 31) < n) {
    for (int a = 0; a < 3; a++) {
      atomic_min_d(box + a, lo[a]);
      atomic_max_d(box + 3 + a, hi[a]);
    }
  }
}

int blocks_of(long long n, int b) { return static_cast<int>((n + b - 1) / b); }

// ---- instanced geometry on the device (addMesh, src/compile.ts:212-306)

// normalMatrix, src/compile.ts:192-205: cofactors divided by the determinant,
// evaluated in the reference's order (this file is compiled without FMA).
__global__ void k_instance_matrices(DInstance* __restrict__ inst, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  DInstance& d = inst[i];
  const double* m = d.world;
  const double a = m[0], b = m[4], c = m[8], dd = m[1], e = m[5], f = m[9], g = m[2], h = m[6], ii = m[10];
  const double A = e * ii - f * h, B = -(dd * ii - f * g), C = dd * h - e * g;
  const double det = a * A + b * B + c * C;
  const double sc = det != 0 ? 1 / det : 0;
  d.nm[0] = A * sc; d.nm[1] = (-(b * ii - c * h)) * sc; d.nm[2] = (b * f - c * e) * sc;
  d.nm[3] = B * sc; d.nm[4] = (a * ii - c * g) * sc; d.nm[5] = (-(a * f - c * dd)) * sc;
  d.nm[6] = C * sc; d.nm[7] = (-(a * h - b * g)) * sc; d.nm[8] = (a * e - b * dd) * sc;
  d.mirror = det < 0 ? 1 : 0;
}

// One thread per triangle of instance blockIdx.y: world-space positions in
// double, float32 v0 / e1 / e2 as the compile's Float32Array stores make them
// (compile.ts:337-343), normals through the normal matrix normalised with
// Math.hypot (or the face normal), uvs, material, flags, side; and the
// largest coordinate for the epsilon.
__global__ void k_flatten(const DInstance* __restrict__ inst, const DMeshRef* __restrict__ meshes,
                          float* __restrict__ tris, float* __restrict__ nrm, float* __restrict__ uvs,
                          uint32_t* __restrict__ mats, uint8_t* __restrict__ flags, uint8_t* __restrict__ sides,
                          unsigned long long* __restrict__ max_coord) {
  const DInstance& d = inst[blockIdx.y];
  const DMeshRef mr = meshes[d.mesh];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double mc = 0;
  if (k < mr.tri_count) {
    const size_t o = static_cast<size_t>(d.tri_base) + k;
    int ids[3] = {3 * k, 3 * k + 1, 3 * k + 2};
    if (mr.idx) {
      for (int v = 0; v < 3; v++) ids[v] = static_cast<int>(mr.idx[ids[v]]);
    }
    if (d.mirror) {  // a mirroring transform reverses the winding
      const int t = ids[1];
      ids[1] = ids[2];
      ids[2] = t;
    }
    const double* w = d.world;
    double p[9];
    for (int v = 0; v < 3; v++) {
      const float* q = mr.pos + 3 * static_cast<size_t>(ids[v]);
      const double x = q[0], y = q[1], z = q[2];
      p[3 * v] = w[0] * x + w[4] * y + w[8] * z + w[12];
      p[3 * v + 1] = w[1] * x + w[5] * y + w[9] * z + w[13];
      p[3 * v + 2] = w[2] * x + w[6] * y + w[10] * z + w[14];
    }
    float* t = tris + 9 * o;
    for (int a = 0; a < 3; a++) {
      t[a] = static_cast<float>(p[a]);
      t[3 + a] = static_cast<float>(p[3 + a] - p[a]);
      t[6 + a] = static_cast<float>(p[6 + a] - p[a]);
    }
    for (int q = 0; q < 9; q++) mc = fmax(mc, fabs(p[q]));
    float* nn = nrm + 9 * o;
    if (mr.nrm && !d.flat) {
      for (int v = 0; v < 3; v++) {
        const float* q = mr.nrm + 3 * static_cast<size_t>(ids[v]);
        const double x = q[0], y = q[1], z = q[2];
        const double nx = d.nm[0] * x + d.nm[3] * y + d.nm[6] * z;
        const double ny = d.nm[1] * x + d.nm[4] * y + d.nm[7] * z;
        const double nz = d.nm[2] * x + d.nm[5] * y + d.nm[8] * z;
        double len = js_hypot3(nx, ny, nz);
        if (!(len != 0) || isnan(len)) len = 1;  // Math.hypot(...) || 1
        nn[3 * v] = static_cast<float>(nx / len);
        nn[3 * v + 1] = static_cast<float>(ny / len);
        nn[3 * v + 2] = static_cast<float>(nz / len);
      }
    } else {
      const double ex = p[3] - p[0], ey = p[4] - p[1], ez = p[5] - p[2];
      const double fx = p[6] - p[0], fy = p[7] - p[1], fz = p[8] - p[2];
      const double cx = ey * fz - ez * fy, cy = ez * fx - ex * fz, cz = ex * fy - ey * fx;
      const double len = js_hypot3(cx, cy, cz);
      float f3[3] = {0.0f, 0.0f, 1.0f};
      if (len > 0) {
        f3[0] = static_cast<float>(cx / len);
        f3[1] = static_cast<float>(cy / len);
        f3[2] = static_cast<float>(cz / len);
      }
      for (int v = 0; v < 3; v++)
        for (int a = 0; a < 3; a++) nn[3 * v + a] = f3[a];
    }
    float* u = uvs + 6 * o;
    for (int v = 0; v < 3; v++) {
      u[2 * v] = mr.uv ? mr.uv[2 * static_cast<size_t>(ids[v])] : 0.0f;
      u[2 * v + 1] = mr.uv ? mr.uv[2 * static_cast<size_t>(ids[v]) + 1] : 0.0f;
    }
    mats[o] = d.material;
    flags[o] = static_cast<uint8_t>(d.flags);
    sides[o] = static_cast<uint8_t>(d.side);
  }
  for (int off = 16; off > 0; off >>= 1) mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, off));
  if ((threadIdx.x & 31) == 0) atomicMax(max_coord, static_cast<unsigned long long>(__double_as_longlong(mc)));
}

// Float32 arrays into BVH order (compile.ts:364-377, the float path).
__global__ void k_reorder_f32(const uint32_t* __restrict__ order, int n, const float* __restrict__ tris_in,
                              const float* __restrict__ nrm, const float* __restrict__ uv,
                              const uint32_t* __restrict__ mats, const uint8_t* __restrict__ flags,
                              const uint8_t* __restrict__ sides, float* __restrict__ tris_out,
                              float* __restrict__ nrm_out, float* __restrict__ uv_out, uint32_t* __restrict__ mats_out,
                              uint8_t* __restrict__ flags_out, uint8_t* __restrict__ sides_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t s = order[i];
  for (int k = 0; k < 9; k++) tris_out[9 * static_cast<size_t>(i) + k] = tris_in[9 * s + k];
  for (int k = 0; k < 9; k++) nrm_out[9 * static_cast<size_t>(i) + k] = nrm[9 * s + k];
  for (int k = 0; k < 6; k++) uv_out[6 * static_cast<size_t>(i) + k] = uv[6 * s + k];
  mats_out[i] = mats[s];
  flags_out[i] = flags[s];
  sides_out[i] = sides[s];
}

// Exclusive prefix sums of up to kScanMax int arrays of the same length n, in
// two launches over a fixed grid of kScanBlocks blocks, each owning one
// contiguous segment of every array: k_scan_sums adds up each block's
// segments; k_scan_write gives each block the sums of the blocks before it
// and scans its segments tile by tile. Integer sums are exact in any order,
// so the results are those of a sequential scan.
constexpr int kScanMax = 4;
constexpr int kScanBlocks = 4 * 148;
constexpr int kScanThreads = 256;

struct ScanArrays {
  const int* in[kScanMax];
  int* out[kScanMax];
  int count;
};

__device__ __forceinline__ void scan_segment(int n, int& lo, int& hi) {
  const int seg = (n + kScanBlocks - 1) / kScanBlocks;
  lo = min(n, static_cast<int>(blockIdx.x) * seg);
  hi = min(n, lo + seg);
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(ScanArrays a, int n, int* __restrict__ sums) {
  using Reduce = cub::BlockReduce<int, kScanThreads>;
  __shared__ typename Reduce::TempStorage tmp;
  int lo, hi;
  scan_segment(n, lo, hi);
  for (int k = 0; k < a.count; k++) {
    int v = 0;
    for (int i = lo + static_cast<int>(threadIdx.x); i < hi; i += kScanThreads) v += a.in[k][i];
    const int total = Reduce(tmp).Sum(v);
    if (threadIdx.x == 0) sums[k * kScanBlocks + blockIdx.x] = total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_write(ScanArrays a, int n, const int* __restrict__ sums) {
  using Reduce = cub::BlockReduce<int, kScanThreads>;
  using Scan = cub::BlockScan<int, kScanThreads>;
  __shared__ union {
    typename Reduce::TempStorage reduce;
    typename Scan::TempStorage scan;
  } tmp;
  __shared__ int base;
  int lo, hi;
  scan_segment(n, lo, hi);
  for (int k = 0; k < a.count; k++) {
    int before = 0;
    for (int b = static_cast<int>(threadIdx.x); b < static_cast<int>(blockIdx.x); b += kScanThreads)
      before += sums[k * kScanBlocks + b];
    const int offset = Reduce(tmp.reduce).Sum(before);
    if (threadIdx.x == 0) base = offset;
    __syncthreads();
    int running = base;
    for (int tile = lo; tile < hi; tile += kScanThreads) {
      const int i = tile + static_cast<int>(threadIdx.x);
      const int v = i < hi ? a.in[k][i] : 0;
      int ex = 0, total = 0;
      Scan(tmp.scan).ExclusiveSum(v, ex, total);
      if (i < hi) a.out[k][i] = running + ex;
      running += total;
      __syncthreads();
    }
    __syncthreads();  // every thread has read `base` before the next array rewrites it
  }
}

// Exclusive sums of in[k] into out[k] (k < count <= kScanMax), each of length
// n; `sums` holds kScanMax * kScanBlocks ints.
void scan_arrays(std::initializer_list<const int*> in, std::initializer_list<int*> out, int n, int* sums,
                 cudaStream_t s) {
  ScanArrays a{};
  a.count = static_cast<int>(in.size());
  if (a.count > kScanMax || out.size() != in.size()) throw std::runtime_error("scan_arrays: bad array count");
  int k = 0;
  for (const int* p : in) a.in[k++] = p;
  k = 0;
  for (int* p : out) a.out[k++] = p;
  if (n <= 0) return;
  k_scan_sums<<<kScanBlocks, kScanThreads, 0, s>>>(a, n, sums);
  k_scan_write<<<kScanBlocks, kScanThreads, 0, s>>>(a, n, sums);
}

}  // namespace

void exclusive_scan(const int* in, int* out, int n, int* sums, cudaStream_t s) {
  scan_arrays({in}, {out}, n, sums, s);
}

int exclusive_scan_scratch() { return kScanMax * kScanBlocks; }

struct BuildBuffers {
  DevArray<float4> bmin, bmax, cent;
  DevArray<uint32_t> order_tmp;
  DevArray<Slot> slots[2];
  DevArray<Split> split;
  DevArray<int> is_split, rank;
  DevArray<int> nb, boff, wide, wid, blk_left, blk_pre, totals, live, live_pos, small, spos, tiny, tpos, slist;
  DevArray<WideAcc> acc;
  DevArray<int> scan_sums;  // per-block sums of the level plan's prefix sums (scan_arrays)
  DevArray<int> host_pair;
  // compile
  DevArray<double> p, nrm, uv, colors, box;
  DevArray<uint8_t> has_color, flags, sides, flags_out, sides_out;
  DevArray<uint32_t> mats, mats_out, order;
  DevArray<float> tris, tris_out, nrm_out, uv_out, col_out, tan_out, bounds;
  DevArray<int> nodes;
  DevArray<unsigned long long> max_coord;
  // instanced geometry
  DevArray<DInstance> inst;
  DevArray<DMeshRef> mesh_refs;
  DevArray<float> flat_nrm, flat_uv;
  std::vector<DevArray<float>> mesh_pos, mesh_nrm, mesh_uv;
  std::vector<DevArray<uint32_t>> mesh_idx;
  std::vector<int> mesh_tris;
};

SceneBuilder::SceneBuilder() : b_(new BuildBuffers()) {}
SceneBuilder::~SceneBuilder() { delete b_; }

int SceneBuilder::build_device(const float* d_tris, int n, float* d_bounds, int* d_nodes, uint32_t* d_order,
                               cudaStream_t s, int bins) {
  last_levels_ = 0;
  if (n <= 0) return 0;
  if (bins < 2 || bins > kMaxBins) throw std::runtime_error("bin count out of range");
  BuildBuffers& B = *b_;
  float4* bmin = B.bmin.ensure(n);
  float4* bmax = B.bmax.ensure(n);
  float4* cent = B.cent.ensure(n);
  uint32_t* tmp = B.order_tmp.ensure(n);
  const int max_slots = std::max(1, n);
  // Blocks of a level: one per node, plus the extra segments of wide nodes.
  const int max_blocks = max_slots + n / kSegment + 1;
  Slot* slots[2] = {B.slots[0].ensure(max_slots), B.slots[1].ensure(max_slots)};
  Split* split = B.split.ensure(max_slots);
  int* is_split = B.is_split.ensure(max_slots);
  int* rank = B.rank.ensure(max_slots);
  int* live = B.live.ensure(max_slots);
  int* live_pos = B.live_pos.ensure(max_slots);
  int* small = B.small.ensure(max_slots);
  int* spos = B.spos.ensure(max_slots);
  int* tiny = B.tiny.ensure(max_slots);
  int* tpos = B.tpos.ensure(max_slots);
  int* slist = B.slist.ensure(max_slots);
  int* nbk = B.nb.ensure(max_slots);
  int* boff = B.boff.ensure(max_slots);
  int* wide = B.wide.ensure(max_slots);
  int* wid = B.wid.ensure(max_slots);
  int* blk_left = B.blk_left.ensure(max_blocks);
  int* blk_pre = B.blk_pre.ensure(max_blocks);
  int* totals = B.totals.ensure(4);
  WideAcc* acc = B.acc.ensure(n / kWideMin + 1);
  k_prepare<<<blocks_of(n, 256), 256, 0, s>>>(d_tris, n, bmin, bmax, cent, d_order);
  Slot root{0, 0, n, 0};
  check(cudaMemcpyAsync(slots[0], &root, sizeof(Slot), cudaMemcpyHostToDevice, s), "upload");
  int* scan_sums = B.scan_sums.ensure(kScanMax * kScanBlocks);
  int active = 1, total = 1, cur = 0;
  uint32_t* order_a = d_order;
  uint32_t* order_b = tmp;
  int pair[2], tot[4], lives[2];
  while (active > 0) {
    k_level_plan<<<blocks_of(active, 256), 256, 0, s>>>(slots[cur], active, nbk, wide, small, tiny);
    scan_arrays({nbk, wide, small, tiny}, {boff, wid, spos, tpos}, active, scan_sums, s);
    k_level_totals<<<1, 1, 0, s>>>(nbk, boff, wide, wid, small, spos, tiny, tpos, active, totals);
    k_small_list<<<blocks_of(active, 256), 256, 0, s>>>(small, spos, tiny, tpos, active, totals, slist);
    check(cudaMemcpyAsync(tot, totals, sizeof(tot), cudaMemcpyDeviceToHost, s), "download");
    check(cudaStreamSynchronize(s), "BVH level plan");
    const int nblocks = tot[0], nwide = tot[1], nsmall = tot[2], ntiny = tot[3];
    const int small_blocks = blocks_of(nsmall, kWarpsPerBlock);
    // Both lists share k_scatter_small, one warp per node.
    const int scatter_blocks = blocks_of(nsmall + ntiny, kWarpsPerBlock);
    const LevelPlan lp{nbk, boff, wid, active};
    if (nwide > 0) {
      k_wide_init<<<nwide, 128, 0, s>>>(acc, nwide);
      k_bounds<<<nblocks, kBuildBlock, 0, s>>>(lp, slots[cur], order_a, bmin, bmax, cent, acc);
    }
    if (nblocks > 0)
      k_split<<<nblocks, kBuildBlock, 0, s>>>(lp, slots[cur], order_a, bmin, bmax, cent, d_bounds, d_nodes, split,
                                              is_split, acc, bins, live);
    if (nsmall > 0)
      k_split_small<<<small_blocks, kBuildBlock, 0, s>>>(slist, nsmall, slots[cur], order_a, bmin, bmax, cent,
                                                         d_bounds, d_nodes, split, is_split, bins, live);
    if (ntiny > 0)
      k_split_tiny<<<blocks_of(ntiny, 2 * kWarpsPerBlock), kBuildBlock, 0, s>>>(
          slist + nsmall, ntiny, slots[cur], order_a, bmin, bmax, cent, d_bounds, d_nodes, split, is_split, bins, live);
    scan_arrays({is_split, live}, {rank, live_pos}, active, scan_sums, s);
    check(cudaMemcpyAsync(&pair[0], rank + active - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
    check(cudaMemcpyAsync(&pair[1], is_split + active - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
    check(cudaMemcpyAsync(&lives[0], live_pos + active - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
    check(cudaMemcpyAsync(&lives[1], live + active - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
    if (nwide > 0) {
      k_count_left<<<nblocks, kBuildBlock, 0, s>>>(lp, slots[cur], split, order_a, cent, bins, blk_left);
      scan_arrays({blk_left}, {blk_pre}, nblocks, scan_sums, s);
    }
    if (nblocks > 0)
      k_scatter<<<nblocks, kBuildBlock, 0, s>>>(lp, slots[cur], split, rank, total, order_a, order_b, cent, d_nodes,
                                                slots[cur ^ 1], blk_pre, bins, live_pos, order_a, bmin, bmax,
                                                d_bounds);
    if (nsmall + ntiny > 0)
      k_scatter_small<<<scatter_blocks, kBuildBlock, 0, s>>>(slist, nsmall + ntiny, slots[cur], split, rank, total, order_a,
                                                           order_b, cent, d_nodes, slots[cur ^ 1], bins, live_pos,
                                                           order_a, bmin, bmax, d_bounds);
    check(cudaStreamSynchronize(s), "BVH level");
    const int splits = pair[0] + pair[1];
    std::swap(order_a, order_b);
    total += 2 * splits;
    active = lives[0] + lives[1];
    cur ^= 1;
    last_levels_++;
  }
  if (order_a != d_order) {
    check(cudaMemcpyAsync(d_order, order_a, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s), "copy");
  }
  check(cudaGetLastError(), "BVH build");
  check(cudaStreamSynchronize(s), "BVH build");
  return total;
}

void SceneBuilder::upload_meshes(int count, const MeshInput* meshes, cudaStream_t s) {
  BuildBuffers& B = *b_;
  B.mesh_pos.clear();
  B.mesh_nrm.clear();
  B.mesh_uv.clear();
  B.mesh_idx.clear();
  B.mesh_tris.assign(count, 0);
  B.mesh_pos.resize(count);
  B.mesh_nrm.resize(count);
  B.mesh_uv.resize(count);
  B.mesh_idx.resize(count);
  std::vector<DMeshRef> refs(std::max(count, 1));
  auto up = [&](void* d, const void* h, size_t bytes) {
    check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s), "upload");
  };
  for (int i = 0; i < count; i++) {
    const MeshInput& m = meshes[i];
    const size_t v = static_cast<size_t>(m.vertex_count);
    DMeshRef r{};
    r.pos = B.mesh_pos[i].ensure(3 * v);
    up(const_cast<float*>(r.pos), m.position, sizeof(float) * 3 * v);
    if (m.normal) {
      r.nrm = B.mesh_nrm[i].ensure(3 * v);
      up(const_cast<float*>(r.nrm), m.normal, sizeof(float) * 3 * v);
    }
    if (m.uv) {
      r.uv = B.mesh_uv[i].ensure(2 * v);
      up(const_cast<float*>(r.uv), m.uv, sizeof(float) * 2 * v);
    }
    if (m.index_count > 0) {
      r.idx = B.mesh_idx[i].ensure(static_cast<size_t>(m.index_count));
      up(const_cast<uint32_t*>(r.idx), m.index, sizeof(uint32_t) * m.index_count);
    }
    r.tri_count = (m.index_count > 0 ? m.index_count : m.vertex_count) / 3;
    B.mesh_tris[i] = r.tri_count;
    refs[i] = r;
  }
  DMeshRef* d_refs = B.mesh_refs.ensure(refs.size());
  up(d_refs, refs.data(), sizeof(DMeshRef) * refs.size());
  check(cudaStreamSynchronize(s), "mesh upload");
}

long long SceneBuilder::instance_triangles(int count, const InstanceInput* inst) const {
  long long n = 0;
  for (int i = 0; i < count; i++) {
    const int m = inst[i].mesh;
    if (m < 0 || m >= static_cast<int>(b_->mesh_tris.size())) return -1;
    n += b_->mesh_tris[m];
  }
  return n;
}

void SceneBuilder::compile_instances(int count, const InstanceInput* inst, int bins, cudaStream_t s,
                                     DeviceGeometry* out, float* times_ms) {
  BuildBuffers& B = *b_;
  const long long total = instance_triangles(count, inst);
  if (total < 0) throw std::runtime_error("an instance names a mesh that was not uploaded");
  if (total > (1ll << 30)) throw std::runtime_error("too many triangles");
  const int n = static_cast<int>(total);
  const size_t N = static_cast<size_t>(std::max(n, 1));
  const size_t cap = std::max<size_t>(1, 2 * N - 1);
  cudaEvent_t ev[4];
  for (auto& e : ev) check(cudaEventCreate(&e), "event");
  check(cudaEventRecord(ev[0], s), "event");
  // Instance table: tri_base and words on the host, matrices on the device.
  std::vector<DInstance> h(std::max(count, 1));
  long long base = 0;
  int max_tris = 0;
  for (int i = 0; i < count; i++) {
    DInstance d{};
    std::memcpy(d.world, inst[i].world, sizeof(d.world));
    d.tri_base = base;
    d.mesh = inst[i].mesh;
    d.flags = inst[i].flags;
    d.side = inst[i].side;
    d.flat = inst[i].flat_shading;
    d.material = inst[i].material;
    base += B.mesh_tris[d.mesh];
    max_tris = std::max(max_tris, B.mesh_tris[d.mesh]);
    h[i] = d;
  }
  DInstance* d_inst = B.inst.ensure(h.size());
  check(cudaMemcpyAsync(d_inst, h.data(), sizeof(DInstance) * h.size(), cudaMemcpyHostToDevice, s), "upload");
  k_instance_matrices<<<blocks_of(count, 128), 128, 0, s>>>(d_inst, count);
  float* d_tris = B.tris.ensure(9 * N);
  float* d_n = B.flat_nrm.ensure(9 * N);
  float* d_uv = B.flat_uv.ensure(6 * N);
  uint32_t* d_m = B.mats.ensure(N);
  uint8_t* d_f = B.flags.ensure(N);
  uint8_t* d_s = B.sides.ensure(N);
  unsigned long long* d_mc = B.max_coord.ensure(1);
  check(cudaMemsetAsync(d_mc, 0, sizeof(unsigned long long), s), "memset");
  if (count > 0 && max_tris > 0) {
    const dim3 grid(blocks_of(max_tris, 256), count);
    k_flatten<<<grid, 256, 0, s>>>(d_inst, B.mesh_refs.p, d_tris, d_n, d_uv, d_m, d_f, d_s, d_mc);
  }
  check(cudaGetLastError(), "flatten");
  check(cudaEventRecord(ev[1], s), "event");
  float* d_bounds = B.bounds.ensure(6 * cap);
  int* d_nodes = B.nodes.ensure(3 * cap);
  uint32_t* d_order = B.order.ensure(N);
  const int m = build_device(d_tris, n, d_bounds, d_nodes, d_order, s, bins);
  check(cudaEventRecord(ev[2], s), "event");
  float* t_out = B.tris_out.ensure(9 * N);
  float* n_out = B.nrm_out.ensure(9 * N);
  float* uv_out = B.uv_out.ensure(6 * N);
  float* tg_out = B.tan_out.ensure(4 * N);
  uint32_t* m_out = B.mats_out.ensure(N);
  uint8_t* f_out = B.flags_out.ensure(N);
  uint8_t* s_out = B.sides_out.ensure(N);
  double box_init[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  double* d_box = B.box.ensure(6);
  check(cudaMemcpyAsync(d_box, box_init, sizeof(box_init), cudaMemcpyHostToDevice, s), "upload");
  if (n > 0) {
    k_reorder_f32<<<blocks_of(n, 256), 256, 0, s>>>(d_order, n, d_tris, d_n, d_uv, d_m, d_f, d_s, t_out, n_out,
                                                    uv_out, m_out, f_out, s_out);
    k_tangents<<<blocks_of(n, 256), 256, 0, s>>>(t_out, uv_out, n, tg_out, d_box);
  }
  check(cudaGetLastError(), "compile");
  double box[6];
  unsigned long long mc_bits = 0;
  check(cudaMemcpyAsync(box, d_box, sizeof(box), cudaMemcpyDeviceToHost, s), "download");
  check(cudaMemcpyAsync(&mc_bits, d_mc, sizeof(mc_bits), cudaMemcpyDeviceToHost, s), "download");
  int root[3] = {0, 0, 0};
  if (m > 0) check(cudaMemcpyAsync(root, d_nodes, sizeof(root), cudaMemcpyDeviceToHost, s), "download");
  check(cudaEventRecord(ev[3], s), "event");
  check(cudaStreamSynchronize(s), "compile");
  double max_coordinate;
  std::memcpy(&max_coordinate, &mc_bits, sizeof(double));
  const double diagonal = n > 0 ? js_hypot3(box[3] - box[0], box[4] - box[1], box[5] - box[2]) : 1.0;
  if (times_ms) {
    for (int i = 0; i < 3; i++) cudaEventElapsedTime(&times_ms[i], ev[i], ev[i + 1]);
  }
  for (auto& e : ev) cudaEventDestroy(e);
  DeviceGeometry g{};
  g.n = n;
  g.node_count = m;
  g.root_count = (m > 0 && root[1] > 0) ? root[1] : 0;
  g.epsilon = n > 0 ? std::max(diagonal * 1e-5, std::max(max_coordinate * 2e-6, 1e-7)) : std::max(1e-5, 1e-7);
  g.triangles = t_out;
  g.normals = n_out;
  g.uvs = uv_out;
  g.tangents = tg_out;
  g.materials = m_out;
  g.flags = f_out;
  g.sides = s_out;
  g.bounds = d_bounds;
  g.nodes = d_nodes;
  g.order = d_order;
  g.levels = last_levels_;
  *out = g;
}

size_t SceneBuilder::device_bytes() const {
  const BuildBuffers& B = *b_;
  size_t t = B.bmin.n * 16 * 3 + B.order_tmp.n * 4 + (B.slots[0].n + B.slots[1].n) * sizeof(Slot) +
             B.split.n * sizeof(Split) + (B.is_split.n + B.rank.n + B.nb.n + B.boff.n + B.wide.n + B.wid.n) * 4 +
             (B.blk_left.n + B.blk_pre.n) * 4 + B.acc.n * sizeof(WideAcc) + B.scan_sums.n * 4 + B.p.n * 8 + B.nrm.n * 8 +
             B.uv.n * 8 + B.colors.n * 8 + B.tris.n * 4 + B.tris_out.n * 4 + B.nrm_out.n * 4 + B.uv_out.n * 4 +
             B.col_out.n * 4 + B.tan_out.n * 4 + B.bounds.n * 4 + B.nodes.n * 4 + B.mats.n * 4 + B.mats_out.n * 4 +
             B.order.n * 4 + B.flags.n + B.sides.n + B.flags_out.n + B.sides_out.n + B.has_color.n +
             B.flat_nrm.n * 4 + B.flat_uv.n * 4 + B.inst.n * sizeof(DInstance);
  for (const auto& a : B.mesh_pos) t += a.n * 4;
  for (const auto& a : B.mesh_nrm) t += a.n * 4;
  for (const auto& a : B.mesh_uv) t += a.n * 4;
  for (const auto& a : B.mesh_idx) t += a.n * 4;
  return t;
}

int SceneBuilder::build_bvh_host(const float* tris, int n, float* bounds, int* nodes, uint32_t* order,
                                 cudaStream_t s) {
  if (n <= 0) return 0;
  BuildBuffers& B = *b_;
  const size_t cap = std::max(1, 2 * n - 1);
  float* d_tris = B.tris.ensure(9 * static_cast<size_t>(n));
  float* d_bounds = B.bounds.ensure(6 * cap);
  int* d_nodes = B.nodes.ensure(3 * cap);
  uint32_t* d_order = B.order.ensure(n);
  check(cudaMemcpyAsync(d_tris, tris, sizeof(float) * 9 * n, cudaMemcpyHostToDevice, s), "upload");
  const int m = build_device(d_tris, n, d_bounds, d_nodes, d_order, s);
  check(cudaMemcpyAsync(bounds, d_bounds, sizeof(float) * 6 * m, cudaMemcpyDeviceToHost, s), "download");
  check(cudaMemcpyAsync(nodes, d_nodes, sizeof(int) * 3 * m, cudaMemcpyDeviceToHost, s), "download");
  check(cudaMemcpyAsync(order, d_order, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s), "download");
  check(cudaStreamSynchronize(s), "download");
  return m;
}

void SceneBuilder::compile_host(int n, const double* p, const double* nrm, const double* uv, const double* colors,
                                const uint8_t* has_color, const uint32_t* materials, const uint8_t* flags,
                                const uint8_t* sides, float* triangles_out, float* normals_out, float* uvs_out,
                                float* tangents_out, float* colors_out, uint32_t* materials_out, uint8_t* flags_out,
                                uint8_t* sides_out, float* bounds_out, int* nodes_out, uint32_t* order_out,
                                int* node_count_out, double* epsilon_out, int* any_colors, cudaStream_t s) {
  int any = 0;
  for (int i = 0; i < n && has_color && colors; i++) any |= has_color[i] ? 1 : 0;
  *any_colors = any;
  if (n <= 0) {
    *node_count_out = 0;
    *epsilon_out = 1e-7;  // max(1 * 1e-5, 0, 1e-7) with diagonal 1: compile.ts:388, 401
    *epsilon_out = std::max(1e-5, 1e-7);
    return;
  }
  BuildBuffers& B = *b_;
  const size_t N = static_cast<size_t>(n);
  const size_t cap = std::max<size_t>(1, 2 * N - 1);
  auto up = [&](void* d, const void* h, size_t bytes) {
    check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s), "upload");
  };
  double* d_p = B.p.ensure(9 * N);
  up(d_p, p, sizeof(double) * 9 * N);
  float* d_tris = B.tris.ensure(9 * N);
  unsigned long long* d_mc = B.max_coord.ensure(1);
  check(cudaMemsetAsync(d_mc, 0, sizeof(unsigned long long), s), "memset");
  k_sink_triangles<<<blocks_of(n, 256), 256, 0, s>>>(d_p, n, d_tris, d_mc);
  float* d_bounds = B.bounds.ensure(6 * cap);
  int* d_nodes = B.nodes.ensure(3 * cap);
  uint32_t* d_order = B.order.ensure(N);
  const int m = build_device(d_tris, n, d_bounds, d_nodes, d_order, s);
  double* d_n = B.nrm.ensure(9 * N);
  up(d_n, nrm, sizeof(double) * 9 * N);
  double* d_uv = B.uv.ensure(6 * N);
  up(d_uv, uv, sizeof(double) * 6 * N);
  double* d_col = nullptr;
  uint8_t* d_hc = nullptr;
  if (any) {
    d_col = B.colors.ensure(12 * N);
    up(d_col, colors, sizeof(double) * 12 * N);
    d_hc = B.has_color.ensure(N);
    up(d_hc, has_color, N);
  }
  uint32_t* d_m = B.mats.ensure(N);
  up(d_m, materials, sizeof(uint32_t) * N);
  uint8_t* d_f = B.flags.ensure(N);
  up(d_f, flags, N);
  uint8_t* d_s = B.sides.ensure(N);
  up(d_s, sides, N);
  float* t_out = B.tris_out.ensure(9 * N);
  float* n_out = B.nrm_out.ensure(9 * N);
  float* uv_out = B.uv_out.ensure(6 * N);
  float* c_out = B.col_out.ensure(any ? 12 * N : 1);
  float* tg_out = B.tan_out.ensure(4 * N);
  uint32_t* m_out = B.mats_out.ensure(N);
  uint8_t* f_out = B.flags_out.ensure(N);
  uint8_t* s_out = B.sides_out.ensure(N);
  k_reorder<<<blocks_of(n, 256), 256, 0, s>>>(d_order, n, d_tris, d_n, d_uv, d_col, d_hc, any, d_m, d_f, d_s, t_out,
                                              n_out, uv_out, c_out, m_out, f_out, s_out);
  double box_init[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  double* d_box = B.box.ensure(6);
  up(d_box, box_init, sizeof(box_init));
  k_tangents<<<blocks_of(n, 256), 256, 0, s>>>(t_out, uv_out, n, tg_out, d_box);
  check(cudaGetLastError(), "compile");
  auto down = [&](void* h, const void* d, size_t bytes) {
    check(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s), "download");
  };
  down(triangles_out, t_out, sizeof(float) * 9 * N);
  down(normals_out, n_out, sizeof(float) * 9 * N);
  down(uvs_out, uv_out, sizeof(float) * 6 * N);
  down(tangents_out, tg_out, sizeof(float) * 4 * N);
  if (any && colors_out) down(colors_out, c_out, sizeof(float) * 12 * N);
  down(materials_out, m_out, sizeof(uint32_t) * N);
  down(flags_out, f_out, N);
  down(sides_out, s_out, N);
  down(bounds_out, d_bounds, sizeof(float) * 6 * m);
  down(nodes_out, d_nodes, sizeof(int) * 3 * m);
  down(order_out, d_order, sizeof(uint32_t) * N);
  double box[6];
  unsigned long long mc_bits = 0;
  down(box, d_box, sizeof(box));
  down(&mc_bits, d_mc, sizeof(mc_bits));
  check(cudaStreamSynchronize(s), "compile");
  double max_coordinate;
  std::memcpy(&max_coordinate, &mc_bits, sizeof(double));
  const double diagonal = js_hypot3(box[3] - box[0], box[4] - box[1], box[5] - box[2]);
  *node_count_out = m;
  *epsilon_out = std::max(diagonal * 1e-5, std::max(max_coordinate * 2e-6, 1e-7));
}

}  // namespace mcrt
