// BVH traversal on the device.
//
// Triangles are tested with the watertight ray-triangle test of Woop,
// Benthin and Wald (JCGT 2013) in FP32: vertices are translated to the ray
// origin, permuted so the ray's dominant axis is z, and sheared so the ray
// runs along +z; the three 2D edge functions then decide the hit, with a
// double-precision recomputation of any edge function that comes out exactly
// zero. Edge functions are formed without fused multiply-adds so a shared
// edge evaluates to exact negatives in its two triangles. Hits follow the
// reference's rules (src/bvh.ts:226-253): edges inclusive, det == 0 misses,
// FrontSide culls det < 0 and BackSide det > 0, accept 0 < t < t_max.
//
// Boxes are tested with the slab test made conservative as in Ize, "Robust
// BVH Ray Traversal" (JCGT 2013): exit distances are scaled by 1 + 2*gamma(3)
// so rounding can't lose a box a ray grazes, which keeps flat boxes (planes)
// hit as the reference's boxEntry does (src/bvh.ts:340-356).
//
// The walk is the persistent "while-while" traversal of Aila and Laine
// ("Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009, and its
// Kepler/Fermi follow-up): each lane descends inner nodes (nearer child
// first, the other pushed) until every lane of the warp holds a leaf, then
// the warp tests leaves together, which keeps SIMD lanes busy; when enough
// lanes have finished their rays the warp refills them from a global counter
// (dynamic fetch), so a warp never idles waiting on its slowest ray. The
// stack keeps its top kShort entries in shared memory (one column per
// thread, bank-conflict free) and spills to local memory; the builder bounds
// depth at 100, and a deeper foreign tree sets a status bit instead of
// overflowing.
//
// Child references: >= 0 an inner node index; < 0 a leaf whose first triangle
// is ~ref. The last triangle of every leaf carries kLeafEnd in its flag word.
#pragma once

#include "device_scene.cuh"

namespace mcrt {

constexpr int kShort = 16;  // shared-memory stack entries per thread of the debugging kernels (k_trace_rays, k_count_hits)
constexpr int kSentinel = 0x7fffffff;  // empty stack / finished ray
constexpr int kLeafEnd = 1 << 16;      // in tris[3k].w: last triangle of its leaf
constexpr int kRefill = 16;            // refill a warp's finished lanes once this many are idle
// The same threshold for the render's own kernels, measured on the mid workload
// (closest hits: 12, shadow rays: 24, of thresholds between 4 and 32).
constexpr int kRefillClosest = 12;
constexpr int kRefillShadow = 24;

// Status bits a kernel reports back (never a trap).
constexpr unsigned kStatusStackOverflow = 1u;
constexpr unsigned kStatusShadowListOverflow = 2u;
constexpr unsigned kStatusStepLimit = 4u;  // a query hit the step budget and was ended
constexpr unsigned kStatusLeafRange = 8u;  // a leaf ran past the last triangle and was cut

// Node visits plus leaves one query may take: a walk of a well-formed BVH of
// N triangles enters each of its fewer than 2N nodes at most once, so past
// 2N + 64 steps something is wrong and the query ends (kStatusStepLimit)
// instead of looping. A positive sc.step_limit (a test hook) replaces it.
MCRT_D int max_steps(const DScene& sc) { return sc.step_limit > 0 ? sc.step_limit : 2 * sc.tri_count + 64; }

struct TravRay {
  V3 o, d, inv;
  int kx, ky, kz;
  float sx, sy, sz;
};

MCRT_D float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

MCRT_D TravRay make_trav_ray(V3 o, V3 d) {
  TravRay r;
  r.o = o;
  r.d = d;
  // safeInverse, src/bvh.ts:336-338: a large finite value for a zero component.
  r.inv = V3{d.x != 0.0f ? 1.0f / d.x : 1e30f, d.y != 0.0f ? 1.0f / d.y : 1e30f, d.z != 0.0f ? 1.0f / d.z : 1e30f};
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  float dz = comp(d, kz);
  if (dz < 0.0f) {
    int tmp = kx;
    kx = ky;
    ky = tmp;
  }
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.sx = comp(d, kx) / dz;
  r.sy = comp(d, ky) / dz;
  r.sz = 1.0f / dz;
  return r;
}

struct TriHit {
  float t, u, v;
  bool front;
};

// Watertight test against the triangle (a, b, c). cull_side: 0 culls back
// faces, 1 culls front faces, anything else culls nothing.
MCRT_D bool intersect_triangle(const TravRay& r, V3 a, V3 b, V3 c, float t_max, int cull_side, TriHit& out) {
  V3 A = a - r.o, B = b - r.o, C = c - r.o;
  const float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
  const float Ax = __fmaf_rn(-r.sx, Akz, comp(A, r.kx)), Ay = __fmaf_rn(-r.sy, Akz, comp(A, r.ky));
  const float Bx = __fmaf_rn(-r.sx, Bkz, comp(B, r.kx)), By = __fmaf_rn(-r.sy, Bkz, comp(B, r.ky));
  const float Cx = __fmaf_rn(-r.sx, Ckz, comp(C, r.kx)), Cy = __fmaf_rn(-r.sy, Ckz, comp(C, r.ky));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = static_cast<float>(static_cast<double>(Cx) * By - static_cast<double>(Cy) * Bx);
    V = static_cast<float>(static_cast<double>(Ax) * Cy - static_cast<double>(Ay) * Cx);
    W = static_cast<float>(static_cast<double>(Bx) * Ay - static_cast<double>(By) * Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = U + V + W;
  if (det == 0.0f) return false;
  if (cull_side == 0 && det < 0.0f) return false;
  if (cull_side == 1 && det > 0.0f) return false;
  const float Az = r.sz * Akz, Bz = r.sz * Bkz, Cz = r.sz * Ckz;
  const float T = U * Az + V * Bz + W * Cz;
  const float inv = 1.0f / det;
  const float t = T * inv;
  if (!(t > 0.0f && t < t_max)) return false;
  out.t = t;
  out.u = V * inv;
  out.v = W * inv;
  out.front = det > 0.0f;
  return true;
}

// Robust slab test of one box; returns the entry distance (>= 0), or -1 on a miss.
MCRT_D float box_entry(const TravRay& r, float x0, float x1, float y0, float y1, float z0, float z1,
                       float t_max) {
  const float g = 1.0000003576f;  // 1 + 2 * gamma(3) for float
  float tx0 = (x0 - r.o.x) * r.inv.x, tx1 = (x1 - r.o.x) * r.inv.x;
  float ty0 = (y0 - r.o.y) * r.inv.y, ty1 = (y1 - r.o.y) * r.inv.y;
  float tz0 = (z0 - r.o.z) * r.inv.z, tz1 = (z1 - r.o.z) * r.inv.z;
  float lo = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
  // Each exit scaled by g, then the least: rounding x * g is monotone in x, so
  // scaling the least exit once gives the same value.
  float hi = fminf(fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * g, t_max);
  return lo <= hi ? lo : -1.0f;
}

struct NodeRefs {
  float4 lxy, rxy, lrz;
  int left, right;
};

MCRT_D NodeRefs load_node(const DNode* nodes, int i) {
  const float4* p = reinterpret_cast<const float4*>(nodes + i);
  NodeRefs n;
  n.lxy = __ldg(p);
  n.rxy = __ldg(p + 1);
  n.lrz = __ldg(p + 2);
  const float4 k = __ldg(p + 3);
  n.left = __float_as_int(k.x);
  n.right = __float_as_int(k.y);
  return n;
}

// Two-level traversal stack: SHORT entries in shared memory, the rest local.
template <int SHORT>
struct TravStackT {
  static_assert(SHORT > 0 && SHORT < kStackMax, "short stack depth out of range");
  int* smem;  // this thread's column: entry i at smem[i * stride]
  int stride;
  int sp;
  int spill[kStackMax - SHORT];
  MCRT_D bool push(int v) {
    if (sp < SHORT) {
      smem[sp * stride] = v;
    } else if (sp < kStackMax) {
      spill[sp - SHORT] = v;
    } else {
      return false;
    }
    sp++;
    return true;
  }
  // The top entry, or kSentinel when empty.
  MCRT_D int pop() {
    if (sp == 0) return kSentinel;
    --sp;
    return sp < SHORT ? smem[sp * stride] : spill[sp - SHORT];
  }
};
using TravStack = TravStackT<kShort>;

MCRT_D void load_tri(const DScene& sc, int k, V3& a, V3& b, V3& c, float4& w0, float4& w1) {
  const float4* p = sc.tris + 3 * static_cast<size_t>(k);
  w0 = __ldg(p);
  w1 = __ldg(p + 1);
  float4 t2 = __ldg(p + 2);
  a = V3{w0.x, w0.y, w0.z};
  b = V3{w1.x, w1.y, w1.z};
  c = V3{t2.x, t2.y, t2.z};
}

MCRT_D bool leaf_end(float w) { return (__float_as_int(w) & kLeafEnd) != 0; }

MCRT_D unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Root reference of the scene: node 0, or the single leaf at triangle 0.
MCRT_D int root_ref(const DScene& sc) { return sc.root_count > 0 ? ~0 : 0; }

// Persistent while-while traversal of queries [0, n) for one warp, taking
// work from *counter. Q supplies, per lane:
//   void load(int index)      start query `index` (ray, limits, result state)
//   const TravRay& ray()
//   float t_max()             current upper limit (closest hit lowers it)
//   bool leaf(int first)      test the leaf starting at triangle `first`;
//                             false ends the query (any hit: blocked)
//   void finish()             write the query's result
// REFILL: a warp takes new queries once that many of its lanes are idle.
template <int REFILL = kRefill, class Q, class ST>
MCRT_D void traverse_persistent(const DScene& sc, Q& q, int n, unsigned* counter, ST& st,
                                unsigned& status) {
  const unsigned lane = threadIdx.x & 31;
  const bool empty = sc.tri_count == 0;
  const int step_limit = max_steps(sc);
  int node = kSentinel;  // next node to visit (kSentinel: none)
  int leaf = 0;          // postponed leaf (< 0), or 0
  int steps = 0;         // node visits and leaves of the current query
  bool has = false;      // this lane holds an unfinished query
  bool exhausted = false;
  for (;;) {
    // Refill finished lanes with one atomic per warp.
    const bool need = !has && !exhausted;
    const unsigned mneed = __ballot_sync(0xffffffffu, need);
    if (mneed) {
      const int leader = __ffs(mneed) - 1;
      unsigned base = 0;
      if (static_cast<int>(lane) == leader) base = atomicAdd(counter, __popc(mneed));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const unsigned idx = base + __popc(mneed & lanemask_lt());
        if (idx < static_cast<unsigned>(n)) {
          q.load(static_cast<int>(idx));
          has = true;
          st.sp = 0;
          leaf = 0;
          steps = 0;
          node = empty ? kSentinel : root_ref(sc);
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, !has)) return;  // every lane is exhausted
    do {
      // A lane may start at, or come back to, a leaf with none postponed.
      if (node < 0 && leaf == 0) {
        leaf = node;
        node = st.pop();
      }
      // Descend until every lane holds a leaf (or has finished).
      while (node >= 0 && node != kSentinel) {
        if (++steps > step_limit) {
          status |= kStatusStepLimit;
          node = kSentinel;
          leaf = 0;
          break;
        }
        const NodeRefs nd = load_node(sc.nodes, node);
        const float tm = q.t_max();
        const TravRay& r = q.ray();
        const float e0 = box_entry(r, nd.lxy.x, nd.lxy.y, nd.lxy.z, nd.lxy.w, nd.lrz.x, nd.lrz.y, tm);
        const float e1 = box_entry(r, nd.rxy.x, nd.rxy.y, nd.rxy.z, nd.rxy.w, nd.lrz.z, nd.lrz.w, tm);
        const bool h0 = e0 >= 0.0f, h1 = e1 >= 0.0f;
        if (!h0 && !h1) {
          node = st.pop();
        } else {
          // Nearer child next, the other pushed. The far reference is
          // derived from the near one by xor rather than by a second select
          // on the same condition: nvcc 12.9 at -O1 and above merged such a
          // select pair into one value, pushing the near child twice.
          const int near_ref = (h0 && (!h1 || e0 <= e1)) ? nd.left : nd.right;
          node = near_ref;
          if (h0 && h1 && !st.push(nd.left ^ nd.right ^ near_ref)) status |= kStatusStackOverflow;
        }
        if (node < 0 && leaf == 0) {  // postpone the leaf, keep descending
          leaf = node;
          node = st.pop();
        }
        if (!__any_sync(__activemask(), leaf == 0)) break;
      }
      // Test the postponed leaf, then any leaf reached right after it.
      while (leaf < 0) {
        if (++steps > step_limit) {
          status |= kStatusStepLimit;
          node = kSentinel;
          leaf = 0;
          break;
        }
        if (!q.leaf(~leaf)) {
          node = kSentinel;
          leaf = 0;
          st.sp = 0;
          break;
        }
        leaf = 0;
        if (node < 0) {
          leaf = node;
          node = st.pop();
        }
      }
      if (has && node == kSentinel && leaf == 0) {
        q.finish();
        has = false;
      }
    } while (__popc(__ballot_sync(0xffffffffu, !has)) < REFILL && __any_sync(0xffffffffu, has));
  }
}

// Warp-coherent traversal of queries [0, n): each warp takes 32 consecutive
// queries and walks the union of their paths through the tree together, one
// node at a time, every lane testing that node's child boxes against its own
// ray (the node is one broadcast load). A child is entered with the lanes
// whose ray enters its box, first the child most of those lanes reach first;
// the other is pushed with its lane mask on a warp stack in shared memory
// (`stack`, kStackMax entries, written by every lane with the same value).
// Each lane thus visits exactly the nodes its own box tests admit, with the
// same closest hit or blocking result as the per-lane walk; only the order
// among a lane's subtrees can differ, which matters for hits at exactly equal
// distance. With no divergence the warp runs at full width, which pays for
// rays that share most of their paths and all run to the end: camera rays,
// where a warp holds the passes of one or two pixels. Q is the same query
// interface as traverse_persistent's.
template <class Q>
MCRT_D void traverse_packet(const DScene& sc, Q& q, int n, unsigned* counter, int2* stack, unsigned& status) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned bit = 1u << lane;
  const int step_limit = max_steps(sc);
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= static_cast<unsigned>(n)) return;
    const bool has = base + lane < static_cast<unsigned>(n);
    if (has) q.load(static_cast<int>(base + lane));
    unsigned live = __ballot_sync(0xffffffffu, has);
    int node = sc.tri_count == 0 ? kSentinel : root_ref(sc);
    unsigned mask = live;
    int sp = 0;
    int steps = 0;
    while (node != kSentinel && live != 0) {
      mask &= live;
      if (mask != 0) {
        if (++steps > step_limit) {
          if (live & bit) status |= kStatusStepLimit;
          break;
        }
        if (node >= 0) {
          const NodeRefs nd = load_node(sc.nodes, node);
          float e0 = -1.0f, e1 = -1.0f;
          if (mask & bit) {
            const float tm = q.t_max();
            const TravRay& r = q.ray();
            e0 = box_entry(r, nd.lxy.x, nd.lxy.y, nd.lxy.z, nd.lxy.w, nd.lrz.x, nd.lrz.y, tm);
            e1 = box_entry(r, nd.rxy.x, nd.rxy.y, nd.rxy.z, nd.rxy.w, nd.lrz.z, nd.lrz.w, tm);
          }
          const bool h0 = e0 >= 0.0f, h1 = e1 >= 0.0f;
          const unsigned m0 = __ballot_sync(0xffffffffu, h0), m1 = __ballot_sync(0xffffffffu, h1);
          if (m0 != 0 && m1 != 0) {
            const unsigned first_left = __ballot_sync(0xffffffffu, h0 && (!h1 || e0 <= e1));
            const bool left = 2 * __popc(first_left) >= __popc(m0 | m1);
            if (sp < kStackMax) {
              stack[sp] = left ? make_int2(nd.right, static_cast<int>(m1)) : make_int2(nd.left, static_cast<int>(m0));
              sp++;
            } else if (live & bit) {
              status |= kStatusStackOverflow;
            }
            node = left ? nd.left : nd.right;
            mask = left ? m0 : m1;
            continue;
          }
          if (m0 != 0 || m1 != 0) {
            node = m0 != 0 ? nd.left : nd.right;
            mask = m0 | m1;
            continue;
          }
        } else {
          bool on = true;
          if (mask & bit) on = q.leaf(~node);
          live = __ballot_sync(0xffffffffu, (live & bit) != 0 && on);
        }
      }
      if (sp == 0) break;
      --sp;
      const int2 e = stack[sp];
      node = e.x;
      mask = static_cast<unsigned>(e.y);
    }
    if (has) q.finish();
  }
}

// Closest hit of one query: intersectClosest, src/bvh.ts:202-282.
struct ClosestHit {
  int tri;
  float t, u, v;
  bool front;
  int material;  // the hit triangle's material (its tris[3k + 1].w)
};

struct ClosestState {
  TravRay r;
  float tmax;
  bool cull;
  ClosestHit h;
  MCRT_D void start(V3 o, V3 d, bool c) {
    r = make_trav_ray(o, d);
    tmax = __int_as_float(0x7f800000);
    cull = c;
    tests = 0;
    h = ClosestHit{-1, 0.0f, 0.0f, 0.0f, true, 0};
  }
  int tests;
  MCRT_D bool leaf(const DScene& sc, int first) {
    for (int k = first; k < sc.tri_count; k++) {
      V3 a, b, c;
      float4 w0, w1;
      load_tri(sc, k, a, b, c, w0, w1);
      tests++;
      TriHit th;
      if (intersect_triangle(r, a, b, c, tmax, cull ? tri_side(w0.w) : 2, th)) {
        tmax = th.t;
        h = ClosestHit{k, th.t, th.u, th.v, th.front, __float_as_int(w1.w)};
      }
      if (leaf_end(w0.w)) break;
    }
    return true;
  }
};

}  // namespace mcrt
