// Device build of the compressed 8-wide BVH (wide_bvh.cuh) from the binary
// SAH tree, one level of wide nodes per launch and one thread per wide node.
//
// A wide node starts from one entry of the binary tree (an inner node, or a
// range of triangles) and repeatedly opens the child entry of largest surface
// area until it has eight children or nothing is left to open: an inner node
// opens into its two children, a range of more than three triangles (a
// binary leaf holds up to sixteen) into its two halves. Children that are
// still inner nodes or ranges of more than three triangles become the next
// level's wide nodes; the rest are leaves, whose triangles are copied into
// the wide-order triangle array. Boxes come from the binary tree's bounds
// (buildBvh's, src/bvh.ts:55-64, which contain the float vertices exactly)
// and, for the halves of a split range, from the triangles' vertices.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "wide_bvh.cuh"

namespace mcrt {
namespace {

struct WideItem {
  int node;   // binary node index, or -1 for a split range
  int first;  // range of triangles (binary order), when count > 0
  int count;  // 0: `node` is an inner binary node
  int wide;   // the wide node this item becomes
};

struct Entry {
  int node, first, count;
  float lo[3], hi[3];
};

MCRT_D void range_box(const float4* tris, int first, int count, float* lo, float* hi) {
  for (int a = 0; a < 3; a++) {
    lo[a] = FLT_MAX;
    hi[a] = -FLT_MAX;
  }
  for (int k = first; k < first + count; k++) {
    for (int v = 0; v < 3; v++) {
      const float4 p = tris[3 * static_cast<size_t>(k) + v];
      lo[0] = fminf(lo[0], p.x), hi[0] = fmaxf(hi[0], p.x);
      lo[1] = fminf(lo[1], p.y), hi[1] = fmaxf(hi[1], p.y);
      lo[2] = fminf(lo[2], p.z), hi[2] = fmaxf(hi[2], p.z);
    }
  }
}

MCRT_D Entry node_entry(const int* nodes, const float* bounds, int i) {
  Entry e;
  e.node = i;
  e.first = nodes[3 * i];
  e.count = nodes[3 * i + 1];
  for (int a = 0; a < 3; a++) {
    e.lo[a] = bounds[6 * static_cast<size_t>(i) + a];
    e.hi[a] = bounds[6 * static_cast<size_t>(i) + 3 + a];
  }
  return e;
}

MCRT_D Entry range_entry(const float4* tris, int first, int count) {
  Entry e;
  e.node = -1;
  e.first = first;
  e.count = count;
  range_box(tris, first, count, e.lo, e.hi);
  return e;
}

MCRT_D bool openable(const Entry& e) { return e.count == 0 || e.count > kWideLeafMax; }

MCRT_D float half_area(const Entry& e) {
  const float dx = fmaxf(e.hi[0] - e.lo[0], 0.0f), dy = fmaxf(e.hi[1] - e.lo[1], 0.0f),
              dz = fmaxf(e.hi[2] - e.lo[2], 0.0f);
  return dx * dy + dy * dz + dz * dx;
}

// Scale of the 8-bit grid over [lo, hi] on one axis: the smallest power of two
// s with lo + 255 s >= hi (exact in double), as its float exponent byte.
MCRT_D unsigned grid_exponent(float lo, float hi) {
  const double ext = static_cast<double>(hi) - static_cast<double>(lo);
  if (!(ext > 0.0)) return 27u;  // 2^-100: a flat extent, every coordinate 0
  int e = 0;
  const double m = frexp(ext / 255.0, &e);  // ext / 255 = m 2^e, m in [0.5, 1)
  if (m == 0.5) e -= 1;
  e = max(e, -100);
  while (static_cast<double>(lo) + 255.0 * ldexp(1.0, e) < static_cast<double>(hi)) e++;
  return static_cast<unsigned>(min(e, 100) + 127);
}

// counters: [0] wide nodes made, [1] triangles placed, [2] next level's
// items, [3] set when a tree reaches a node or triangle twice (then the
// buffers, sized for a tree, would overflow: nothing more is written).
__global__ void __launch_bounds__(128) k_wide_level(const int* __restrict__ nodes, const float* __restrict__ bounds,
                                                    const float4* __restrict__ tris, const WideItem* __restrict__ in,
                                                    int n_in, WideItem* __restrict__ out, uint4* __restrict__ wnodes,
                                                    float4* __restrict__ wtris, unsigned* __restrict__ counters,
                                                    unsigned capacity) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_in) return;
  const WideItem it = in[i];
  Entry e[8];
  int k = 1;
  e[0] = it.node >= 0 ? node_entry(nodes, bounds, it.node) : range_entry(tris, it.first, it.count);
  // Open the largest openable child until there are eight.
  while (k < 8) {
    int best = -1;
    float best_area = -1.0f;
    for (int j = 0; j < k; j++) {
      if (!openable(e[j])) continue;
      const float a = half_area(e[j]);
      if (a > best_area) {
        best_area = a;
        best = j;
      }
    }
    if (best < 0) break;
    const Entry p = e[best];
    if (p.count == 0) {
      e[best] = node_entry(nodes, bounds, p.first);
      e[k++] = node_entry(nodes, bounds, p.first + 1);
    } else {
      const int half = p.count / 2;
      e[best] = range_entry(tris, p.first, half);
      e[k++] = range_entry(tris, p.first + half, p.count - half);
    }
  }
  // The node's box and grid.
  float plo[3], phi[3];
  for (int a = 0; a < 3; a++) {
    plo[a] = e[0].lo[a];
    phi[a] = e[0].hi[a];
    for (int j = 1; j < k; j++) {
      plo[a] = fminf(plo[a], e[j].lo[a]);
      phi[a] = fmaxf(phi[a], e[j].hi[a]);
    }
  }
  unsigned ebyte[3];
  double scale[3];
  for (int a = 0; a < 3; a++) {
    ebyte[a] = grid_exponent(plo[a], phi[a]);
    scale[a] = ldexp(1.0, static_cast<int>(ebyte[a]) - 127);
  }
  // Slots by direction: slot bit a set for a child below the node's centre on
  // axis a. Greedy on the cost of each (child, slot) pair.
  int slot_child[8];
  for (int s = 0; s < 8; s++) slot_child[s] = -1;
  {
    float cost[8][8];
    for (int j = 0; j < k; j++) {
      for (int s = 0; s < 8; s++) {
        float c = 0.0f;
        for (int a = 0; a < 3; a++) {
          const float v = (e[j].lo[a] + e[j].hi[a]) - (plo[a] + phi[a]);
          c += (s >> a) & 1 ? v : -v;
        }
        cost[j][s] = c;
      }
    }
    unsigned child_done = 0;
    for (int round = 0; round < k; round++) {
      float best = FLT_MAX;
      int bj = -1, bs = -1;
      for (int j = 0; j < k; j++) {
        if ((child_done >> j) & 1) continue;
        for (int s = 0; s < 8; s++) {
          if (slot_child[s] >= 0) continue;
          if (bj < 0 || cost[j][s] < best) {
            best = cost[j][s];
            bj = j;
            bs = s;
          }
        }
      }
      slot_child[bs] = bj;
      child_done |= 1u << bj;
    }
  }
  int n_inner = 0, n_tris = 0;
  for (int j = 0; j < k; j++) {
    if (openable(e[j])) {
      n_inner++;
    } else {
      n_tris += e[j].count;
    }
  }
  const unsigned child_base = n_inner ? atomicAdd(&counters[0], static_cast<unsigned>(n_inner)) : 0u;
  const unsigned tri_base = n_tris ? atomicAdd(&counters[1], static_cast<unsigned>(n_tris)) : 0u;
  const unsigned out_base = n_inner ? atomicAdd(&counters[2], static_cast<unsigned>(n_inner)) : 0u;
  // A tree of n triangles has at most n wide nodes, n placed triangles and n
  // items on a level (every wide node but the root has two or more children).
  if (static_cast<unsigned long long>(child_base) + n_inner > capacity ||
      static_cast<unsigned long long>(tri_base) + n_tris > capacity ||
      static_cast<unsigned long long>(out_base) + n_inner > capacity || static_cast<unsigned>(it.wide) >= capacity) {
    atomicOr(&counters[3], 1u);
    return;
  }
  unsigned meta[2] = {0u, 0u}, qlo[3][2] = {{0u, 0u}, {0u, 0u}, {0u, 0u}}, qhi[3][2] = {{0u, 0u}, {0u, 0u}, {0u, 0u}};
  unsigned imask = 0;
  int rank = 0, offset = 0;
  for (int s = 0; s < 8; s++) {
    const int j = slot_child[s];
    if (j < 0) continue;
    const Entry& c = e[j];
    const int word = s >> 2, shift = 8 * (s & 3);
    for (int a = 0; a < 3; a++) {
      // Rounded outwards: the decoded box contains the child's in exact arithmetic.
      const double lo = floor((static_cast<double>(c.lo[a]) - plo[a]) / scale[a]);
      const double hi = ceil((static_cast<double>(c.hi[a]) - plo[a]) / scale[a]);
      const unsigned ql = static_cast<unsigned>(fmin(fmax(lo, 0.0), 255.0));
      const unsigned qh = static_cast<unsigned>(fmin(fmax(hi, 0.0), 255.0));
      qlo[a][word] |= ql << shift;
      qhi[a][word] |= qh << shift;
    }
    unsigned m;
    if (openable(c)) {
      m = 0x38u + static_cast<unsigned>(s);
      imask |= 1u << s;
      out[out_base + rank] = WideItem{c.node, c.first, c.count, static_cast<int>(child_base) + rank};
      rank++;
    } else {
      m = (((1u << c.count) - 1u) << 5) | static_cast<unsigned>(offset);
      for (int t = 0; t < c.count; t++) {
        const size_t src = 3 * static_cast<size_t>(c.first + t);
        const size_t dst = 3 * (static_cast<size_t>(tri_base) + offset + t);
        wtris[dst] = tris[src];
        wtris[dst + 1] = tris[src + 1];
        float4 v2 = tris[src + 2];
        v2.w = __int_as_float(c.first + t);  // the compiled geometry's index of the triangle
        wtris[dst + 2] = v2;
      }
      offset += c.count;
    }
    meta[word] |= m << shift;
  }
  uint4* node = wnodes + static_cast<size_t>(kWideNodeWords) * it.wide;
  node[0] = make_uint4(__float_as_uint(plo[0]), __float_as_uint(plo[1]), __float_as_uint(plo[2]),
                       ebyte[0] | (ebyte[1] << 8) | (ebyte[2] << 16) | (imask << 24));
  node[1] = make_uint4(child_base, tri_base, meta[0], meta[1]);
  node[2] = make_uint4(qlo[0][0], qlo[0][1], qlo[1][0], qlo[1][1]);
  node[3] = make_uint4(qlo[2][0], qlo[2][1], qhi[0][0], qhi[0][1]);
  node[4] = make_uint4(qhi[1][0], qhi[1][1], qhi[2][0], qhi[2][1]);
}

}  // namespace

size_t wide_bvh_item_bytes(int n) { return sizeof(WideItem) * 2 * static_cast<size_t>(std::max(n, 1)); }

cudaError_t build_wide_bvh(const int* nodes, const float* bounds, int root_count, const float4* tris, int n,
                           uint4* wnodes, float4* wtris, void* items, unsigned* counters, int* wide_nodes,
                           cudaStream_t s) {
  *wide_nodes = 0;
  if (n <= 0) return cudaSuccess;
  (void)root_count;  // node 0 is the root either way: an inner node, or a leaf of root_count triangles
  WideItem* a = static_cast<WideItem*>(items);
  WideItem* b = a + std::max(n, 1);
  const WideItem root{0, 0, 0, 0};
  const unsigned start[4] = {1u, 0u, 0u, 0u};
  cudaError_t e = cudaMemcpyAsync(a, &root, sizeof(root), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(counters, start, sizeof(start), cudaMemcpyHostToDevice, s);
  int n_in = 1;
  // Every level is at least one binary level deeper (or halves a range), so
  // the depth is bounded by the binary tree's plus four; the cap guards
  // against a malformed tree.
  for (int level = 0; e == cudaSuccess && n_in > 0; level++) {
    if (level > 4096) return cudaErrorInvalidValue;
    e = cudaMemsetAsync(counters + 2, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) break;
    k_wide_level<<<(n_in + 127) / 128, 128, 0, s>>>(nodes, bounds, tris, a, n_in, b, wnodes, wtris, counters,
                                                    static_cast<unsigned>(n));
    unsigned next[2] = {0u, 0u};
    e = cudaMemcpyAsync(next, counters + 2, sizeof(next), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && next[1]) return cudaErrorInvalidValue;  // not a tree
    n_in = static_cast<int>(next[0]);
    std::swap(a, b);
  }
  unsigned total = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, counters, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  *wide_nodes = static_cast<int>(total);
  return e;
}

}  // namespace mcrt
