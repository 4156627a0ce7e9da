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

#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "scene_build.cuh"

namespace mcrt {

namespace {

constexpr int kBins = 16;      // bvh.ts:3
constexpr int kMaxLeaf = 4;    // bvh.ts:4
constexpr int kBuildDepth = 100;  // bvh.ts:5
constexpr int kBuildBlock = 256;

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

// mode: -1 leaf, 0 split at `bin` of `axis`, 1 split the run in half.
struct Split {
  int mode, axis, bin, nleft;
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

__device__ __forceinline__ int bin_of(float c, double lo, double scale) {
  return static_cast<int>(fmin(static_cast<double>(kBins - 1), floor((static_cast<double>(c) - lo) * scale)));
}

// Bounds, leaf test, binning and SAH choice of one node per block
// (bvh.ts:55-144).
__global__ void __launch_bounds__(kBuildBlock) k_split(const Slot* __restrict__ slots,
                                                       const uint32_t* __restrict__ order,
                                                       const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                                                       const float4* __restrict__ cent, float* __restrict__ bounds,
                                                       int* __restrict__ nodes, Split* __restrict__ split,
                                                       int* __restrict__ is_split) {
  const Slot s = slots[blockIdx.x];
  const int tid = threadIdx.x;
  __shared__ float red[kBuildBlock / 32][12];
  __shared__ float nb[12];  // node min xyz, -max xyz, centroid min xyz, -max xyz
  __shared__ int cnt[3][kBins];
  __shared__ float bbox[3][kBins][6];

  float m[12];
  for (int i = 0; i < 12; i++) m[i] = INFINITY;
  for (int k = s.first + tid; k < s.first + s.count; k += kBuildBlock) {
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
  for (int i = tid; i < 3 * kBins; i += kBuildBlock) {
    const int a = i / kBins, b = i % kBins;
    cnt[a][b] = 0;
    for (int j = 0; j < 3; j++) {
      bbox[a][b][j] = INFINITY;
      bbox[a][b][3 + j] = -INFINITY;
    }
  }
  __syncthreads();
  if (tid < 12) {
    float v = INFINITY;
    for (int w = 0; w < kBuildBlock / 32; w++) v = fminf(v, red[w][tid]);
    nb[tid] = v;
  }
  __syncthreads();
  const double nx0 = nb[0], ny0 = nb[1], nz0 = nb[2], nx1 = -nb[3], ny1 = -nb[4], nz1 = -nb[5];
  const double cmin[3] = {nb[6], nb[7], nb[8]};
  const double cmax[3] = {-nb[9], -nb[10], -nb[11]};
  if (tid == 0) {
    float* bo = bounds + 6 * static_cast<size_t>(s.node);
    bo[0] = nb[0]; bo[1] = nb[1]; bo[2] = nb[2];
    bo[3] = -nb[3]; bo[4] = -nb[4]; bo[5] = -nb[5];
  }
  if (s.count <= kMaxLeaf || s.depth >= kBuildDepth) {
    if (tid == 0) {
      int* nd = nodes + 3 * static_cast<size_t>(s.node);
      nd[0] = s.first; nd[1] = s.count; nd[2] = 0;
      split[blockIdx.x] = Split{-1, 0, 0, 0};
      is_split[blockIdx.x] = 0;
    }
    return;
  }
  // Bin the centroids along every axis with extent (bvh.ts:89-109).
  double lo[3], scale[3];
  bool live[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = cmin[a];
    const double extent = cmax[a] - lo[a];
    live[a] = extent > 0;
    scale[a] = live[a] ? kBins / extent : 0.0;
  }
  for (int k = s.first + tid; k < s.first + s.count; k += kBuildBlock) {
    const uint32_t t = order[k];
    const float4 a4 = bmin[t], b4 = bmax[t], c4 = cent[t];
    for (int a = 0; a < 3; a++) {
      if (!live[a]) continue;
      const int b = bin_of(comp4(c4, a), lo[a], scale[a]);
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
  if (tid == 0) {
    // SAH sweeps, bvh.ts:110-134, and the choice, bvh.ts:137-163.
    double best_cost = INFINITY;
    int best_axis = -1, best_split = -1;
    double right_area[kBins];
    int right_count[kBins];
    for (int a = 0; a < 3; a++) {
      if (!live[a]) continue;
      double rx0 = INFINITY, ry0 = INFINITY, rz0 = INFINITY, rx1 = -INFINITY, ry1 = -INFINITY, rz1 = -INFINITY;
      int rc = 0;
      for (int i = kBins - 1; i > 0; i--) {
        const float* o = bbox[a][i];
        rc += cnt[a][i];
        rx0 = fmin(rx0, static_cast<double>(o[0])); ry0 = fmin(ry0, static_cast<double>(o[1]));
        rz0 = fmin(rz0, static_cast<double>(o[2]));
        rx1 = fmax(rx1, static_cast<double>(o[3])); ry1 = fmax(ry1, static_cast<double>(o[4]));
        rz1 = fmax(rz1, static_cast<double>(o[5]));
        right_count[i] = rc;
        right_area[i] = rc > 0 ? area(rx0, ry0, rz0, rx1, ry1, rz1) : 0;
      }
      double lx0 = INFINITY, ly0 = INFINITY, lz0 = INFINITY, lx1 = -INFINITY, ly1 = -INFINITY, lz1 = -INFINITY;
      int lc = 0;
      for (int i = 0; i < kBins - 1; i++) {
        const float* o = bbox[a][i];
        lc += cnt[a][i];
        lx0 = fmin(lx0, static_cast<double>(o[0])); ly0 = fmin(ly0, static_cast<double>(o[1]));
        lz0 = fmin(lz0, static_cast<double>(o[2]));
        lx1 = fmax(lx1, static_cast<double>(o[3])); ly1 = fmax(ly1, static_cast<double>(o[4]));
        lz1 = fmax(lz1, static_cast<double>(o[5]));
        const int rc2 = right_count[i + 1];
        if (lc == 0 || rc2 == 0) continue;
        const double cost = lc * area(lx0, ly0, lz0, lx1, ly1, lz1) + rc2 * right_area[i + 1];
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_split = i;
        }
      }
    }
    Split d{1, 0, 0, s.count >> 1};
    bool leaf = false;
    if (best_axis >= 0) {
      const double parent_area = area(nx0, ny0, nz0, nx1, ny1, nz1);
      const double split_cost = 1 + (1 * best_cost) / fmax(parent_area, 1e-30);
      if (split_cost >= 1.0 * s.count && s.count <= 16) {
        leaf = true;
      } else {
        int nleft = 0;
        for (int i = 0; i <= best_split; i++) nleft += cnt[best_axis][i];
        d = Split{0, best_axis, best_split, nleft};
        if (nleft == 0 || nleft == s.count) d = Split{1, best_axis, 0, s.count >> 1};
      }
    }
    if (leaf) {
      int* nd = nodes + 3 * static_cast<size_t>(s.node);
      nd[0] = s.first; nd[1] = s.count; nd[2] = 0;
      split[blockIdx.x] = Split{-1, 0, 0, 0};
      is_split[blockIdx.x] = 0;
    } else {
      split[blockIdx.x] = d;
      is_split[blockIdx.x] = 1;
    }
  }
}

// Stable partition of each split node's run and its two children
// (bvh.ts:145-171); leaves copy their run unchanged.
__global__ void __launch_bounds__(kBuildBlock) k_scatter(const Slot* __restrict__ slots,
                                                         const Split* __restrict__ split,
                                                         const int* __restrict__ rank, int child_base,
                                                         const uint32_t* __restrict__ order,
                                                         uint32_t* __restrict__ order_out,
                                                         const float4* __restrict__ cent, int* __restrict__ nodes,
                                                         Slot* __restrict__ next) {
  using Scan = cub::BlockScan<int, kBuildBlock>;
  __shared__ typename Scan::TempStorage scan_tmp;
  const Slot s = slots[blockIdx.x];
  const Split d = split[blockIdx.x];
  const int tid = threadIdx.x;
  const int end = s.first + s.count;
  if (d.mode < 0) {
    for (int k = s.first + tid; k < end; k += kBuildBlock) order_out[k] = order[k];
    return;
  }
  double lo = 0, scale = 0;
  if (d.mode == 0) {
    // The same bins as k_split: recompute the centroid range along the axis.
    float mn = INFINITY, mx = -INFINITY;
    for (int k = s.first + tid; k < end; k += kBuildBlock) {
      const float c = comp4(cent[order[k]], d.axis);
      mn = fminf(mn, c);
      mx = fmaxf(mx, c);
    }
    __shared__ float rmn[kBuildBlock / 32], rmx[kBuildBlock / 32];
    __shared__ float fmn, fmx;
    for (int off = 16; off > 0; off >>= 1) {
      mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, off));
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    if ((tid & 31) == 0) {
      rmn[tid >> 5] = mn;
      rmx[tid >> 5] = mx;
    }
    __syncthreads();
    if (tid == 0) {
      float a = INFINITY, b = -INFINITY;
      for (int w = 0; w < kBuildBlock / 32; w++) {
        a = fminf(a, rmn[w]);
        b = fmaxf(b, rmx[w]);
      }
      fmn = a;
      fmx = b;
    }
    __syncthreads();
    lo = fmn;
    scale = kBins / (static_cast<double>(fmx) - lo);
  }
  int left_off = 0;
  for (int base = s.first; base < end; base += kBuildBlock) {
    const int k = base + tid;
    int f = 0;
    uint32_t t = 0;
    if (k < end) {
      t = order[k];
      f = d.mode == 0 ? (bin_of(comp4(cent[t], d.axis), lo, scale) <= d.bin ? 1 : 0) : (k - s.first < d.nleft ? 1 : 0);
    }
    int pre = 0, total = 0;
    Scan(scan_tmp).ExclusiveSum(f, pre, total);
    if (k < end) {
      const int right_before = (base - s.first) - left_off;
      const int dst = f ? s.first + left_off + pre : s.first + d.nleft + right_before + (tid - pre);
      order_out[dst] = t;
    }
    left_off += total;
    __syncthreads();
  }
  if (tid == 0) {
    const int left = child_base + 2 * rank[blockIdx.x];
    int* nd = nodes + 3 * static_cast<size_t>(s.node);
    nd[0] = left; nd[1] = 0; nd[2] = d.axis;
    next[2 * rank[blockIdx.x]] = Slot{left, s.first, d.nleft, s.depth + 1};
    next[2 * rank[blockIdx.x] + 1] = Slot{left + 1, s.first + d.nleft, s.count - d.nleft, s.depth + 1};
  }
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

}  // namespace

struct BuildBuffers {
  DevArray<float4> bmin, bmax, cent;
  DevArray<uint32_t> order_tmp;
  DevArray<Slot> slots[2];
  DevArray<Split> split;
  DevArray<int> is_split, rank;
  DevArray<uint8_t> scan_tmp;
  DevArray<int> host_pair;
  // compile
  DevArray<double> p, nrm, uv, colors, box;
  DevArray<uint8_t> has_color, flags, sides, flags_out, sides_out;
  DevArray<uint32_t> mats, mats_out, order;
  DevArray<float> tris, tris_out, nrm_out, uv_out, col_out, tan_out, bounds;
  DevArray<int> nodes;
  DevArray<unsigned long long> max_coord;
};

SceneBuilder::SceneBuilder() : b_(new BuildBuffers()) {}
SceneBuilder::~SceneBuilder() { delete b_; }

int SceneBuilder::build_device(const float* d_tris, int n, float* d_bounds, int* d_nodes, uint32_t* d_order,
                               cudaStream_t s) {
  last_levels_ = 0;
  if (n <= 0) return 0;
  BuildBuffers& B = *b_;
  float4* bmin = B.bmin.ensure(n);
  float4* bmax = B.bmax.ensure(n);
  float4* cent = B.cent.ensure(n);
  uint32_t* tmp = B.order_tmp.ensure(n);
  const int max_slots = std::max(1, n);
  Slot* slots[2] = {B.slots[0].ensure(max_slots), B.slots[1].ensure(max_slots)};
  Split* split = B.split.ensure(max_slots);
  int* is_split = B.is_split.ensure(max_slots);
  int* rank = B.rank.ensure(max_slots);
  k_prepare<<<blocks_of(n, 256), 256, 0, s>>>(d_tris, n, bmin, bmax, cent, d_order);
  Slot root{0, 0, n, 0};
  check(cudaMemcpyAsync(slots[0], &root, sizeof(Slot), cudaMemcpyHostToDevice, s), "upload");
  size_t scan_bytes = 0;
  check(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, is_split, rank, max_slots, s), "scan");
  uint8_t* scan_tmp = B.scan_tmp.ensure(scan_bytes);
  int active = 1, total = 1, cur = 0;
  uint32_t* order_a = d_order;
  uint32_t* order_b = tmp;
  int pair[2];
  while (active > 0) {
    k_split<<<active, kBuildBlock, 0, s>>>(slots[cur], order_a, bmin, bmax, cent, d_bounds, d_nodes, split, is_split);
    check(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, is_split, rank, active, s), "scan");
    check(cudaMemcpyAsync(&pair[0], rank + active - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
    check(cudaMemcpyAsync(&pair[1], is_split + active - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
    k_scatter<<<active, kBuildBlock, 0, s>>>(slots[cur], split, rank, total, order_a, order_b, cent, d_nodes,
                                             slots[cur ^ 1]);
    check(cudaStreamSynchronize(s), "BVH level");
    const int splits = pair[0] + pair[1];
    std::swap(order_a, order_b);
    total += 2 * splits;
    active = 2 * splits;
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
