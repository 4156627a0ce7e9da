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
// Traversal visits the nearer child first and pushes the other on a short
// stack whose top kShort entries live in shared memory (one column per
// thread, bank-conflict free) and whose rest spills to local memory; BVH depth
// is at most kMaxDepth, so the stack is bounded.
#pragma once

#include "device_scene.cuh"

namespace mcrt {

constexpr int kShort = 16;  // shared-memory stack entries per thread

// Status bits a kernel reports back (never a trap).
constexpr unsigned kStatusStackOverflow = 1u;
constexpr unsigned kStatusShadowListOverflow = 2u;

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
  float hi = fminf(fminf(fmaxf(tx0, tx1) * g, fmaxf(ty0, ty1) * g), fminf(fmaxf(tz0, tz1) * g, t_max));
  return lo <= hi ? lo : -1.0f;
}

MCRT_D DNode load_node(const DNode* nodes, int i) {
  const float4* p = reinterpret_cast<const float4*>(nodes + i);
  DNode n;
  n.lxy = __ldg(p);
  n.rxy = __ldg(p + 1);
  n.lrz = __ldg(p + 2);
  float4 k = __ldg(p + 3);
  n.kids = make_int4(__float_as_int(k.x), __float_as_int(k.y), __float_as_int(k.z), __float_as_int(k.w));
  return n;
}

// Two-level traversal stack: kShort entries in shared memory, the rest local.
struct TravStack {
  int* smem;  // this thread's column: entry i at smem[i * stride]
  int stride;
  int sp;
  int spill[kStackMax - kShort];
  MCRT_D bool push(int v) {
    if (sp < kShort) {
      smem[sp * stride] = v;
    } else if (sp < kStackMax) {
      spill[sp - kShort] = v;
    } else {
      return false;
    }
    sp++;
    return true;
  }
  MCRT_D int pop() {
    --sp;
    return sp < kShort ? smem[sp * stride] : spill[sp - kShort];
  }
};

// Walks the BVH, nearer child first, calling leaf(first, count, t_max) for
// every leaf whose box the ray enters before t_max. `leaf` may lower t_max
// (closest hit) and returns false to end the walk (any hit blocked).
template <class Leaf>
MCRT_D void traverse(const DScene& sc, const TravRay& r, float& t_max, TravStack& st, unsigned& status, Leaf&& leaf) {
  if (sc.tri_count == 0) return;
  if (sc.root_count > 0) {
    leaf(0, sc.root_count, t_max);
    return;
  }
  st.sp = 0;
  int node = 0;
  for (;;) {
    const DNode n = load_node(sc.nodes, node);
    float e0 = box_entry(r, n.lxy.x, n.lxy.y, n.lxy.z, n.lxy.w, n.lrz.x, n.lrz.y, t_max);
    float e1 = box_entry(r, n.rxy.x, n.rxy.y, n.rxy.z, n.rxy.w, n.lrz.z, n.lrz.w, t_max);
    int r0 = n.kids.x, c0 = n.kids.z, r1 = n.kids.y, c1 = n.kids.w;
    bool h0 = e0 >= 0.0f && c0 >= 0;
    bool h1 = e1 >= 0.0f && c1 >= 0;
    if (h1 && (!h0 || e1 < e0)) {  // visit the nearer child first
      int tr = r0; r0 = r1; r1 = tr;
      int tc = c0; c0 = c1; c1 = tc;
      float te = e0; e0 = e1; e1 = te;
      bool th = h0; h0 = h1; h1 = th;
    }
    int next = -1;
    if (h0) {
      if (c0 > 0) {
        if (!leaf(r0, c0, t_max)) return;
      } else {
        next = r0;
      }
    }
    if (h1 && e1 <= t_max) {
      if (c1 > 0) {
        if (!leaf(r1, c1, t_max)) return;
      } else if (next < 0) {
        next = r1;
      } else if (!st.push(r1)) {
        status |= kStatusStackOverflow;
      }
    }
    if (next >= 0) {
      node = next;
      continue;
    }
    if (st.sp == 0) return;
    node = st.pop();
  }
}

MCRT_D void load_tri(const DScene& sc, int k, V3& a, V3& b, V3& c, float4& w0, float4& w1) {
  const float4* p = sc.tris + 3 * static_cast<size_t>(k);
  w0 = __ldg(p);
  w1 = __ldg(p + 1);
  float4 t2 = __ldg(p + 2);
  a = V3{w0.x, w0.y, w0.z};
  b = V3{w1.x, w1.y, w1.z};
  c = V3{t2.x, t2.y, t2.z};
}

struct ClosestHit {
  int tri;
  float t, u, v;
  bool front;
};

// intersectClosest, src/bvh.ts:202-282: nearest hit with side culling.
MCRT_D ClosestHit trace_closest(const DScene& sc, const TravRay& r, bool cull, TravStack& st, unsigned& status) {
  ClosestHit h{-1, 0.0f, 0.0f, 0.0f, true};
  float t_max = __int_as_float(0x7f800000);
  traverse(sc, r, t_max, st, status, [&](int first, int count, float& tm) {
    for (int k = first; k < first + count; k++) {
      V3 a, b, c;
      float4 w0, w1;
      load_tri(sc, k, a, b, c, w0, w1);
      TriHit th;
      if (intersect_triangle(r, a, b, c, tm, cull ? tri_side(w0.w) : 2, th)) {
        tm = th.t;
        h.tri = k;
        h.t = th.t;
        h.u = th.u;
        h.v = th.v;
        h.front = th.front;
      }
    }
    return true;
  });
  return h;
}

}  // namespace mcrt
