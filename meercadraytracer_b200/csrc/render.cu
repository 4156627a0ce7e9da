// Wavefront path tracer: the reference's Tracer (src/tracer.ts) as a series
// of kernels over queues of paths.
//
//   raygen    one path per (pixel, pass): seed, jitter and camera ray in FP64
//             (Tracer.renderTile, tracer.ts:62-80; cameraRay, tracer.ts:705-727)
//   extend    closest hit of every queued ray (intersectClosest, bvh.ts:202-282)
//   shade     one iteration of samplePixel's loop (tracer.ts:113-470): surface,
//             materials, direct light split into shadow rays, continuation
//   shadow    any-hit transmittance of every shadow ray (visibleLight,
//             transmittance, attenuateShadow, tracer.ts:515-594)
//   resolve   adds each path's shadowed light, finishes ended paths (tone map
//             and fog, tracer.ts:472-477)
//   accumulate  Float32 running sum in pass order and the RGBA8 encode
//             (writeTile, progressive.ts:288-313)
//
// A path's random numbers are drawn in the reference's order because each
// path's stages run in sequence; shadow rays draw none. Shadowed light goes to
// a per-path, per-light slot and is summed in slot order, so results do not
// depend on queue order and renders are deterministic.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "render.cuh"
#include "traverse.cuh"

namespace cg = cooperative_groups;

namespace mcrt {

constexpr int kBlock = 128;
// De-duplicated see-through hits per shadow ray. The list is indexed at run
// time, so it lives in local memory and costs nothing until a ray uses it; a
// ray with more distinct see-through hits sets kStatusShadowListOverflow.
constexpr int kShadowSeen = 64;
constexpr int kSortMin = 1 << 16;  // shorter queues are shaded in the order they are in
constexpr int kMaxIterations = 1 << 16;  // bounce / pass-through iterations of one chunk

// Appends to a queue counter with one atomic per coalesced group of threads.
MCRT_D unsigned int queue_append(unsigned int* counter) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, g.size());
  base = g.shfl(base, 0);
  return base + g.thread_rank();
}

// ------------------------------------------------------------------- walks
// The traversal every query kernel runs (traverse_persistent): B threads per
// block, S shared-memory stack entries per thread, warps refilled once REFILL
// lanes are idle.
template <int REFILL, int B, int S, class Q>
MCRT_D void walk(const DScene& sc, Q& q, int n, unsigned* counter, unsigned& status) {
  __shared__ int stack[S * B];
  TravStackT<S> st;
  st.smem = stack + threadIdx.x;
  st.stride = B;
  st.sp = 0;
  traverse_persistent<REFILL>(sc, q, n, counter, st, status);
}

// ---------------------------------------------------------------- mapping
MCRT_D void path_pixel(const FrameParams& fp, int pid, int& px, int& py, int& pass) {
  const int k = pid - fp.path_base;
  int i, j;
  if (fp.npass > 0) {
    i = k / fp.npass;
    j = k - i * fp.npass;
  } else {
    j = k / fp.npix;
    i = k - j * fp.npix;
  }
  i += fp.pix0;
  pass = fp.pass0 + j;
  if (fp.mode == 1) {
    px = fp.list_x[i];
    py = fp.list_y[i];
  } else {
    int by = i / fp.nbx;
    int bx = i - by * fp.nbx;
    px = fp.tile_x + bx * fp.block;
    py = fp.tile_y + by * fp.block;
  }
}

// Seeds the path's generator and returns the screen position (tracer.ts:69-78).
MCRT_D void jitter(const FrameParams& fp, int px, int py, int pass, uint32_t& rng, double& sx, double& sy) {
  rng = rng_seed(static_cast<uint32_t>(px), static_cast<uint32_t>(py), static_cast<uint32_t>(pass), fp.seed);
  double jx = 0.5, jy = 0.5;
  if (fp.block > 1) {
    jx = min(fp.block, fp.width - px) * 0.5;
    jy = min(fp.block, fp.height - py) * 0.5;
  } else if (pass > 0) {
    jx = rng_next(rng);
    jy = rng_next(rng);
  }
  sx = (px + jx) / fp.width;
  sy = (py + jy) / fp.height;
}

// unproject, tracer.ts:715-727, in double.
MCRT_D void unproject(const FrameParams& fp, double x, double y, double z, double* out) {
  const double* p = fp.proj_inv;
  double w = p[3] * x + p[7] * y + p[11] * z + p[15];
  double vx = (p[0] * x + p[4] * y + p[8] * z + p[12]) / w;
  double vy = (p[1] * x + p[5] * y + p[9] * z + p[13]) / w;
  double vz = (p[2] * x + p[6] * y + p[10] * z + p[14]) / w;
  const double* m = fp.world;
  out[0] = m[0] * vx + m[4] * vy + m[8] * vz + m[12];
  out[1] = m[1] * vx + m[5] * vy + m[9] * vz + m[13];
  out[2] = m[2] * vx + m[6] * vy + m[10] * vz + m[14];
}

// ------------------------------------------------------------------ raygen
MCRT_D void raygen_path(const FrameParams& fp, const PathState& ps, int pid) {
  int px, py, pass;
  path_pixel(fp, pid, px, py, pass);
  uint32_t rng;
  double sx, sy;
  jitter(fp, px, py, pass, rng, sx, sy);
  double near_[3], far_[3];
  unproject(fp, sx * 2 - 1, 1 - sy * 2, -1.0, near_);
  unproject(fp, sx * 2 - 1, 1 - sy * 2, 1.0, far_);
  double dx = far_[0] - near_[0], dy = far_[1] - near_[1], dz = far_[2] - near_[2];
  double len = sqrt(dx * dx + dy * dy + dz * dz);
  if (!(len > 0)) len = 1;
  ps.ray_o[pid] = make_float4(static_cast<float>(near_[0]), static_cast<float>(near_[1]),
                              static_cast<float>(near_[2]), 0.0f);
  ps.ray_d[pid] = make_float4(static_cast<float>(dx / len), static_cast<float>(dy / len),
                              static_cast<float>(dz / len), 0.0f);
  // Throughput, radiance and medium are not written here: until its first
  // shaded hit (kFlagSeen) a path's are always (1, 1, 1, fog 0), (0, 0, 0,
  // env scale 1) and no medium, which shade_path uses without loading them.
  ps.rng[pid] = rng;
  ps.flags[pid] = kFlagToneMap | kFlagCull;
  ps.smask[pid] = 0ull;
  ps.queue[0][pid] = pid;
}

__global__ void __launch_bounds__(kBlock) k_raygen(FrameParams fp, PathState ps, int n) {
  const int pid = blockIdx.x * blockDim.x + threadIdx.x;
  if (pid < n) raygen_path(fp, ps, pid);
}

// Shading class of a hit on material m (the shading-order sort's key): 1 +
// 2 x the material model + 1 if transmissive; a miss is class 0.
MCRT_D int material_class(const DScene& sc, int m) {
  const DMaterial& mat = sc.materials[m];
  return 1 + 2 * min(max(mat.model, 0), 6) + (mat.transmission > 0.0f ? 1 : 0);
}

// ------------------------------------------------------------------ extend
// Closest hit of each queued path's ray (intersectClosest, bvh.ts:202-282),
// persistent: warps take rays from cnt->fetch until the queue is drained.
// With `hist` (shared memory, kShadeClasses counters) each finished query
// also stores its hit's shading class by queue position (ps.cls) and counts
// it, the first half of the shading-order sort.
struct ExtendQuery {
  const DScene& sc;
  const PathState& ps;
  const int* queue;
  int pid;
  ClosestState cs;
  unsigned int* hist;
  int qi;
  MCRT_D void load(int i) {
    qi = i;
    pid = queue[i];
    const float4 o = ps.ray_o[pid], d = ps.ray_d[pid];
    cs.start(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, (ps.flags[pid] & kFlagCull) != 0);
  }
  MCRT_D const TravRay& ray() const { return cs.r; }
  MCRT_D float t_max() const { return cs.tmax; }
  MCRT_D bool leaf(int first) { return cs.leaf(sc, first); }
  MCRT_D void finish() {
    const ClosestHit& h = cs.h;
    const unsigned word = h.tri >= 0 ? ((h.front ? 0x80000000u : 0u) | static_cast<unsigned>(h.tri + 1)) : 0u;
    ps.hit[pid] = make_float4(h.t, h.u, h.v, __uint_as_float(word));
    if (hist) {
      const int c = h.tri >= 0 ? material_class(sc, h.material) : 0;
      ps.cls[qi] = static_cast<uint8_t>(c);
      atomicAdd(hist + c, 1u);
    }
  }
};

// The shared histogram of a closest-hit kernel that counts shading classes
// (`bins` given): cleared before the walk, added to `bins` after it.
struct ClassHistogram {
  unsigned int* bins;
  unsigned int* hist;
  MCRT_D unsigned int* begin() {
    if (!bins) return nullptr;
    if (threadIdx.x < kShadeClasses) hist[threadIdx.x] = 0;
    __syncthreads();
    return hist;
  }
  MCRT_D void end() {
    if (!bins) return;
    __syncthreads();
    if (threadIdx.x < kShadeClasses && hist[threadIdx.x]) atomicAdd(bins + threadIdx.x, hist[threadIdx.x]);
  }
};

// B threads per block, S short-stack entries per thread (a traversal variant).
// 1280 / B blocks per SM: the register cap (48) costs a few bytes of spills
// and buys a ninth more resident warps than the unconstrained 56 registers.
template <int B, int S>
__global__ void __launch_bounds__(B, 1280 / B) k_extend(DScene sc, PathState ps, const int* __restrict__ queue, int n,
                                              Counters* cnt, unsigned int* bins) {
  __shared__ unsigned int hist[kShadeClasses];
  ClassHistogram ch{bins, hist};
  unsigned status = 0;
  ExtendQuery q{sc, ps, queue, 0, {}, ch.begin(), 0};
  walk<kRefillClosest, B, S>(sc, q, n, &cnt->fetch, status);
  if (status) atomicOr(&cnt->status, status);
  ch.end();
}

// The same over a queue of coherent rays (the camera rays), warp by warp
// (traverse_packet); B / 32 warp stacks of kStackMax entries in shared memory.
template <int B>
__global__ void __launch_bounds__(B) k_extend_packet(DScene sc, PathState ps, const int* __restrict__ queue, int n,
                                                     Counters* cnt, unsigned int* bins) {
  __shared__ int2 stack[(B / 32) * kStackMax];
  __shared__ unsigned int hist[kShadeClasses];
  ClassHistogram ch{bins, hist};
  unsigned status = 0;
  ExtendQuery q{sc, ps, queue, 0, {}, ch.begin(), 0};
  traverse_packet(sc, q, n, &cnt->fetch, stack + (threadIdx.x >> 5) * kStackMax, status);
  if (status) atomicOr(&cnt->status, status);
  ch.end();
}

// ------------------------------------------------------- shading order
// The shading step branches on what a path hit: nothing (background), or a
// material of one model, transmissive or not. Shading the queue in that
// class order gives each warp lanes that take the same branches (and run
// the same code) instead of a mix; results do not depend on queue order.

MCRT_D int shade_class(const DScene& sc, const PathState& ps, int pid) {
  const unsigned word = __float_as_uint(__ldg(reinterpret_cast<const float*>(ps.hit + pid) + 3));
  const int tri = static_cast<int>(word & 0x7fffffffu) - 1;
  if (tri < 0) return 0;
  return material_class(sc, __float_as_int(__ldg(&sc.tris[3 * static_cast<size_t>(tri) + 1].w)));
}

// Places the block's tile [first, first + blockDim.x) of the queue: ranks
// within each warp's class groups, then within the block (shared counters),
// then one global cursor increment per class and block.
MCRT_D void scatter_block(const int* __restrict__ queue, const uint8_t* __restrict__ cls, int n, int first,
                          const unsigned int* base, unsigned int* cursor, int* __restrict__ out) {
  __shared__ unsigned int blk_count[kShadeClasses], blk_base[kShadeClasses];
  if (threadIdx.x < kShadeClasses) blk_count[threadIdx.x] = 0;
  __syncthreads();
  const int i = first + threadIdx.x;
  int c = 0, pid = 0;
  unsigned int pos = 0;
  if (i < n) {
    pid = queue[i];
    c = cls[i];
    const unsigned int peers = __match_any_sync(__activemask(), c);
    const int leader = __ffs(peers) - 1;
    unsigned int w = 0;
    if (static_cast<int>(threadIdx.x & 31) == leader) w = atomicAdd(&blk_count[c], __popc(peers));
    pos = __shfl_sync(peers, w, leader) + __popc(peers & lanemask_lt());
  }
  __syncthreads();
  if (threadIdx.x < kShadeClasses && blk_count[threadIdx.x])
    blk_base[threadIdx.x] = atomicAdd(&cursor[threadIdx.x], blk_count[threadIdx.x]);
  __syncthreads();
  if (i < n) out[base[c] + blk_base[c] + pos] = pid;
}

__global__ void __launch_bounds__(256) k_class_scatter(DScene sc, PathState ps, const int* __restrict__ queue, int n,
                                                       unsigned int* __restrict__ bins, int* __restrict__ out) {
  __shared__ unsigned int base[kShadeClasses];
  if (threadIdx.x == 0) {
    unsigned int sum = 0;
    for (int b = 0; b < kShadeClasses; b++) {
      base[b] = sum;
      sum += bins[b];
    }
  }
  scatter_block(queue, ps.cls, n, blockIdx.x * blockDim.x, base, bins + kShadeClasses, out);
}

// ------------------------------------------------------------------- shade
// lightAt, tracer.ts:486-512: direction to a punctual light, its radiance and distance.
MCRT_D bool light_at(const DLight& L, V3 p, V3& l, V3& radiance, float& distance) {
  if (L.type == 2) {
    l = V3{L.direction[0], L.direction[1], L.direction[2]};
    radiance = V3{L.color[0], L.color[1], L.color[2]};
    distance = __int_as_float(0x7f800000);
    return true;
  }
  if (L.type == 3 || L.type == 4) {
    V3 v = V3{L.position[0], L.position[1], L.position[2]} - p;
    float dist = length3(v);
    if (dist == 0.0f) return false;
    l = v * (1.0f / dist);
    float scale = distance_attenuation(dist, L.distance, L.decay);
    if (L.type == 4) {
      float angle_cos = l.x * L.direction[0] + l.y * L.direction[1] + l.z * L.direction[2];
      scale *= smoothstep(L.cone_cos, L.penumbra_cos, angle_cos);
    }
    if (scale <= 0.0f) return false;
    radiance = V3{L.color[0] * scale, L.color[1] * scale, L.color[2] * scale};
    distance = dist;
    return true;
  }
  return false;
}

// Where a shade step puts its output: continuing paths and shadow rays.
struct StageQueues {
  int* next;
  unsigned int* next_count;
  float4* shadow;  // 3 float4 per shadow ray
  unsigned int* shadow_count;
};

struct ShadowEmitter {
  float4* queue;
  unsigned int* counter;
  int pid;
  unsigned long long mask;
  // Queues a shadow ray whose unshadowed contribution is `w`.
  MCRT_D void emit(V3 o, V3 d, float max_t, V3 w, int slot, bool cast_only) {
    unsigned idx = queue_append(counter);
    float4* e = queue + 3 * static_cast<size_t>(idx);
    e[0] = make_float4(o.x, o.y, o.z, max_t);
    e[1] = make_float4(d.x, d.y, d.z, __int_as_float(pid));
    e[2] = make_float4(w.x, w.y, w.z, __int_as_float(slot | (cast_only ? 0x10000 : 0)));
    mask |= 1ull << slot;
  }
};

// Direct light of one light: the unshadowed contribution goes straight into
// `out` when no shadow ray is needed (visibleLight, tracer.ts:515-526), or to
// a shadow ray weighted by throughput and the environment combine factor.
MCRT_D void direct_light(const FrameParams& fp, const DScene& sc, ShadowEmitter& em, const DLight& L, int li,
                         bool receive, V3 p, V3 g, V3 l, float light_distance, V3 c, V3& out, V3 weight) {
  if (fp.shadows == 2 || (fp.shadows == 1 && (!L.cast_shadow || !receive))) {
    out = out + c;
    return;
  }
  const float eps = sc.eps;
  const float side = dot(g, l) > 0.0f ? eps : -eps;
  const float inf = __int_as_float(0x7f800000);
  const float max_t = light_distance == inf ? inf : light_distance - 2.0f * eps;
  em.emit(p + g * side, l, max_t, c * weight, li, fp.shadows == 1);
}

// One iteration of samplePixel's loop for path `pid`.
MCRT_D void shade_path(const DScene& sc, const FrameParams& fp, const PathState& ps, int pid, const StageQueues& qs) {
  // The hit word and flags first: a miss (most camera rays of open scenes)
  // reads little more, so the rest of the path state is loaded after the test.
  const float4 h4 = ps.hit[pid];
  uint32_t fl = ps.flags[pid];
  const unsigned word = __float_as_uint(h4.w);
  const int tri = static_cast<int>(word & 0x7fffffffu) - 1;

  if (tri < 0) {
    if (!(fl & kFlagSeen)) {
      // background, tracer.ts:659-691.
      float4 out;
      const DBackground& bg = sc.background;
      if (bg.kind == 1) {
        out = make_float4(bg.color[0], bg.color[1], bg.color[2], 1.0f);
      } else if (bg.kind == 2 || bg.kind == 3) {
        float c[3];
        int srgb_tex;
        if (bg.kind == 2) {
          int px, py, pass;
          path_pixel(fp, pid, px, py, pass);
          uint32_t r2;
          double sx, sy;
          jitter(fp, px, py, pass, r2, sx, sy);
          float4 t = sample_texture(sc, bg.texture, static_cast<float>(sx), static_cast<float>(1.0 - sy));
          c[0] = t.x * bg.intensity;
          c[1] = t.y * bg.intensity;
          c[2] = t.z * bg.intensity;
          srgb_tex = sc.textures[bg.texture].srgb;
        } else {
          const float4 d4 = ps.ray_d[pid];
          V3 e = sample_environment(sc, bg.environment, V3{d4.x, d4.y, d4.z});
          c[0] = e.x;
          c[1] = e.y;
          c[2] = e.z;
          const DEnvironment& env = sc.envs[bg.environment];
          srgb_tex = sc.textures[env.kind == 0 ? env.faces[0] : env.texture].srgb;
        }
        if (!srgb_tex && fp.tone_mapping != 0) tone_map(c, fp.tone_mapping, fp.exposure);
        out = make_float4(c[0], c[1], c[2], 1.0f);
      } else {
        const float a = fp.clear_alpha;
        out = make_float4(fp.clear_color[0] * a, fp.clear_color[1] * a, fp.clear_color[2] * a, a);
      }
      ps.sample[pid] = out;
      ps.flags[pid] = fl | kFlagDone | kFlagDirect;  // the radiance is left as it is
      return;
    }
    const float4 L4 = ps.rad[pid];
    V3 Lr = V3{L4.x, L4.y, L4.z};
    const int le = flag_last_env(fl);
    if (le >= 0) {
      const float4 d4 = ps.ray_d[pid], T4 = ps.thr[pid];
      V3 e = sample_environment(sc, le, V3{d4.x, d4.y, d4.z});
      Lr = Lr + V3{T4.x, T4.y, T4.z} * e * L4.w;
    }
    ps.rad[pid] = make_float4(Lr.x, Lr.y, Lr.z, L4.w);
    ps.flags[pid] = fl | kFlagDone;
    return;
  }

  const float4 o4 = ps.ray_o[pid], d4 = ps.ray_d[pid];
  const bool seen = (fl & kFlagSeen) != 0;
  float4 T4 = make_float4(1.0f, 1.0f, 1.0f, 0.0f), L4 = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  float4 m4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (seen) {
    T4 = ps.thr[pid];
    L4 = ps.rad[pid];
    m4 = ps.med[pid];
  }
  uint32_t rng = ps.rng[pid];
  V3 d = V3{d4.x, d4.y, d4.z};
  V3 T = V3{T4.x, T4.y, T4.z};
  V3 Lr = V3{L4.x, L4.y, L4.z};
  float fog_factor = T4.w;
  float last_env_scale = L4.w;
  ShadowEmitter em{qs.shadow, qs.shadow_count, pid, 0ull};
  const bool front = (word & 0x80000000u) != 0;
  const float inf = __int_as_float(0x7f800000);

  const float t = h4.x;
  if (m4.x > 0.0f || m4.y > 0.0f || m4.z > 0.0f) {
    // Beer-Lambert absorption inside the volume, tracer.ts:128-131.
    T.x *= expf(-m4.x * t);
    T.y *= expf(-m4.y * t);
    T.z *= expf(-m4.z * t);
  }
  V3 va, vb, vc;
  float4 tw0, tw1;
  load_tri(sc, tri, va, vb, vc, tw0, tw1);
  const DMaterial& mat = sc.materials[__float_as_int(tw1.w)];
  const int tflags = tri_flags(tw0.w);
  const V3 o = V3{o4.x, o4.y, o4.z};
  const V3 p = o + d * t;
  const float w1 = h4.y, w2 = h4.z, w0 = 1.0f - w1 - w2;
  const float face = front ? 1.0f : -1.0f;
  V3 g = normalize_or_keep(cross(vb - va, vc - va)) * face;  // geometric normal, tracer.ts:140-145

  const float4* at = sc.attrs + 4 * static_cast<size_t>(tri);
  const float4 a0 = __ldg(at), a1 = __ldg(at + 1), a2 = __ldg(at + 2), a3 = __ldg(at + 3);
  const float u = a2.y * w0 + a2.w * w1 + a3.y * w2;
  const float v = a2.z * w0 + a3.x * w1 + a3.z * w2;

  // Base colour and coverage, tracer.ts:151-168.
  V3 c = V3{mat.color[0], mat.color[1], mat.color[2]};
  float alpha = mat.opacity;
  if (mat.map >= 0) {
    float4 tx = sample_texture(sc, mat.map, u, v);
    c = c * V3{tx.x, tx.y, tx.z};
    alpha *= tx.w;
  }
  if (mat.vertex_colors && sc.colors) {
    const float4* cp = sc.colors + 3 * static_cast<size_t>(tri);
    float4 k0 = __ldg(cp), k1 = __ldg(cp + 1), k2 = __ldg(cp + 2);
    c.x *= k0.x * w0 + k1.x * w1 + k2.x * w2;
    c.y *= k0.y * w0 + k1.y * w1 + k2.y * w2;
    c.z *= k0.z * w0 + k1.z * w1 + k2.z * w2;
    alpha *= k0.w * w0 + k1.w * w1 + k2.w * w2;
  }
  if (mat.alpha_map >= 0) alpha *= sample_texture(sc, mat.alpha_map, u, v).y;
  const bool cut_out = mat.alpha_test > 0.0f && alpha < mat.alpha_test;
  if (cut_out || (mat.transparent && rng_next(rng) >= static_cast<double>(alpha))) {
    // Pass straight through, tracer.ts:170-176.
    uint32_t passes = flag_passes(fl) + 1;
    fl = (fl & ~0xff00u) | (min(passes, 255u) << 8);
    if (passes > static_cast<uint32_t>(kMaxPassThrough)) {
      fl |= kFlagDone;
    } else {
      const float side = dot(g, d) > 0.0f ? sc.eps : -sc.eps;
      V3 no = p + g * side;
      ps.ray_o[pid] = make_float4(no.x, no.y, no.z, 0.0f);
      qs.next[queue_append(qs.next_count)] = pid;
    }
    ps.thr[pid] = make_float4(T.x, T.y, T.z, fog_factor);
    if (!seen) ps.rad[pid] = L4;  // read by resolve if the path ends here
    ps.rng[pid] = rng;
    ps.flags[pid] = fl;
    return;
  }
  if (!seen) {
    fl |= kFlagSeen;
    if (!mat.tone_mapped) fl &= ~kFlagToneMap;
    // fog, tracer.ts:649-656.
    if (sc.fog.kind != 0) {
      const float depth = (p.x - fp.cam_position[0]) * fp.cam_forward[0] +
                          (p.y - fp.cam_position[1]) * fp.cam_forward[1] +
                          (p.z - fp.cam_position[2]) * fp.cam_forward[2];
      fog_factor = sc.fog.kind == 1 ? smoothstep(sc.fog.near_, sc.fog.far_, depth)
                                    : 1.0f - expf(-sc.fog.density * sc.fog.density * depth * depth);
    }
  }

  // Shading normal, tracer.ts:184-209.
  V3 nrm = normalize_or_keep(V3{(a0.x * w0 + a0.w * w1 + a1.z * w2) * face, (a0.y * w0 + a1.x * w1 + a1.w * w2) * face,
                                (a0.z * w0 + a1.y * w1 + a2.x * w2) * face});
  if (mat.normal_map >= 0) {
    float4 tx = sample_texture(sc, mat.normal_map, u, v);
    const float mx = (tx.x * 2.0f - 1.0f) * mat.normal_scale[0];
    const float my = (tx.y * 2.0f - 1.0f) * mat.normal_scale[1];
    const float mz = tx.z * 2.0f - 1.0f;
    const float4 tg = __ldg(sc.tangents + tri);
    V3 ta = V3{tg.x, tg.y, tg.z};
    ta = ta - nrm * dot(ta, nrm);
    ta = normalize_or_keep(ta) * face;
    V3 bt = cross(nrm, ta) * tg.w;
    nrm = normalize_or_keep(ta * mx + bt * my + nrm * mz);
  }
  const V3 vv = V3{-d.x, -d.y, -d.z};
  const float dot_nv = clamp01(dot(nrm, vv));

  // Emission, tracer.ts:216-220.
  V3 e = V3{mat.emissive[0], mat.emissive[1], mat.emissive[2]};
  if (mat.emissive_map >= 0 && (e.x > 0.0f || e.y > 0.0f || e.z > 0.0f)) {
    float4 tx = sample_texture(sc, mat.emissive_map, u, v);
    e = e * V3{tx.x, tx.y, tx.z};
  }
  const bool receive = (tflags & 4) != 0;
  const uint32_t bounce = flag_bounce(fl);
  const bool can_continue = static_cast<int>(bounce) < fp.max_bounces;

  // Environment combine of Lambert, Phong and Basic materials (tracer.ts:393-406)
  // is affine in their colour: out' = alpha_c * out + beta_c. It is known before
  // the lights are, so shadowed light is weighted by alpha_c.
  V3 alpha_c = V3{1.0f, 1.0f, 1.0f}, beta_c = V3{0.0f, 0.0f, 0.0f};
  if (mat.model != 0 && mat.env_map >= 0) {
    const float dn = dot(d, nrm);
    V3 env = sample_environment(sc, mat.env_map, d - nrm * (2.0f * dn));
    const float s = mat.reflectivity;
    if (mat.combine == 0) {
      alpha_c = V3{1.0f - s + s * env.x, 1.0f - s + s * env.y, 1.0f - s + s * env.z};
    } else if (mat.combine == 1) {
      alpha_c = V3{1.0f - s, 1.0f - s, 1.0f - s};
      beta_c = env * s;
    } else if (mat.combine == 2) {
      beta_c = env * s;
    }
  }
  const V3 w_light = T * alpha_c;

  V3 spec = V3{0, 0, 0}, diff = V3{0, 0, 0}, trans = V3{0, 0, 0};
  float roughness = 1.0f;
  int environment = -1;
  float environment_scale = 1.0f;
  V3 out = V3{0, 0, 0};

  if (mat.model == 4) {
    out = c;
  } else {
    // Ambient and hemisphere irradiance, tracer.ts:237-247.
    V3 ir = V3{0, 0, 0};
    for (int li = 0; li < sc.light_count; li++) {
      const DLight& L = sc.lights[li];
      if (L.type == 0) {
        ir = ir + V3{L.color[0], L.color[1], L.color[2]};
      } else if (L.type == 1) {
        const float w = 0.5f * (nrm.x * L.direction[0] + nrm.y * L.direction[1] + nrm.z * L.direction[2]) + 0.5f;
        ir.x += L.ground[0] + (L.color[0] - L.ground[0]) * w;
        ir.y += L.ground[1] + (L.color[1] - L.ground[1]) * w;
        ir.z += L.ground[2] + (L.color[2] - L.ground[2]) * w;
      }
    }
    float ao = 1.0f;
    if (mat.ao_map >= 0) ao = (sample_texture(sc, mat.ao_map, u, v).x - 1.0f) * mat.ao_map_intensity + 1.0f;

    if (mat.model == 0) {
      // Physical, tracer.ts:254-354.
      float metalness = mat.metalness;
      roughness = mat.roughness;
      if (mat.roughness_map >= 0) roughness *= sample_texture(sc, mat.roughness_map, u, v).y;
      if (mat.metalness_map >= 0) metalness *= sample_texture(sc, mat.metalness_map, u, v).z;
      const float shade_roughness = fminf(fmaxf(roughness, 0.045f), 1.0f);
      V3 s0 = V3{0.04f, 0.04f, 0.04f};
      float f90 = 1.0f;
      if (mat.physical) {
        const float q = (mat.ior - 1.0f) / (mat.ior + 1.0f);
        const float f = q * q;
        s0.x = fminf(f * mat.specular_color[0], 1.0f) * mat.specular_intensity;
        s0.y = fminf(f * mat.specular_color[1], 1.0f) * mat.specular_intensity;
        s0.z = fminf(f * mat.specular_color[2], 1.0f) * mat.specular_intensity;
        f90 = mat.specular_intensity + (1.0f - mat.specular_intensity) * metalness;
      }
      const V3 base = s0 + (c - s0) * metalness;
      const V3 dcol = c * (1.0f - metalness);
      float fa, fb;
      dfg_lookup(sc, shade_roughness, dot_nv, fa, fb);
      const float ess_ms = fa + fb, ems = 1.0f - ess_ms;
      const V3 comp3 = V3{1.0f, 1.0f, 1.0f} + base * (1.0f / ess_ms - 1.0f);
      const float ggx_alpha = shade_roughness * shade_roughness;
      const float transmission = mat.transmission;
      const float keep_diffuse = 1.0f - transmission;

      for (int li = 0; li < sc.light_count; li++) {
        const DLight& L = sc.lights[li];
        V3 l, rad;
        float dist;
        if (!light_at(L, p, l, rad, dist)) continue;
        const float dot_nl = dot(nrm, l);
        if (dot_nl <= 0.0f) continue;
        const V3 h = normalize_or_keep(l + vv);
        const float dot_nh = clamp01(dot(nrm, h));
        const float dot_vh = clamp01(dot(vv, h));
        const float fw = fresnel_weight(dot_vh);
        const float vd = visibility_ggx(ggx_alpha, dot_nl, dot_nv) * distribution_ggx(ggx_alpha, dot_nh);
        V3 cc;
        cc.x = ((base.x * (1.0f - fw) + f90 * fw) * vd * comp3.x +
                dcol.x * kInvPi * (1.0f - (s0.x * (1.0f - fw) + f90 * fw)) * keep_diffuse) * dot_nl * rad.x;
        cc.y = ((base.y * (1.0f - fw) + f90 * fw) * vd * comp3.y +
                dcol.y * kInvPi * (1.0f - (s0.y * (1.0f - fw) + f90 * fw)) * keep_diffuse) * dot_nl * rad.y;
        cc.z = ((base.z * (1.0f - fw) + f90 * fw) * vd * comp3.z +
                dcol.z * kInvPi * (1.0f - (s0.z * (1.0f - fw) + f90 * fw)) * keep_diffuse) * dot_nl * rad.z;
        if (cc.x + cc.y + cc.z <= 0.0f) continue;
        direct_light(fp, sc, em, L, li, receive, p, g, l, dist, cc, out, w_light);
      }
      const V3 fss = s0 * fa + V3{f90 * fb, f90 * fb, f90 * fb};
      const V3 scatter = V3{fss.x + multi_scatter(fss.x, s0.x, ems), fss.y + multi_scatter(fss.y, s0.y, ems),
                            fss.z + multi_scatter(fss.z, s0.z, ems)};
      out.x += ir.x * kInvPi * dcol.x * (1.0f - scatter.x) * ao * keep_diffuse;
      out.y += ir.y * kInvPi * dcol.y * (1.0f - scatter.y) * ao * keep_diffuse;
      out.z += ir.z * kInvPi * dcol.z * (1.0f - scatter.z) * ao * keep_diffuse;
      const V3 mf = c * fa + V3{f90 * fb, f90 * fb, f90 * fb};
      spec = fss + (mf - fss) * metalness;
      diff = V3{dcol.x * (1.0f - scatter.x) * keep_diffuse, dcol.y * (1.0f - scatter.y) * keep_diffuse,
                dcol.z * (1.0f - scatter.z) * keep_diffuse};
      if (transmission > 0.0f) {
        trans = V3{transmission * (1.0f - fss.x) * c.x, transmission * (1.0f - fss.y) * c.y,
                   transmission * (1.0f - fss.z) * c.z};
      }
      if (mat.env_map >= 0) {
        environment = mat.env_map;
      } else if (sc.environment >= 0) {
        environment = sc.environment;
        environment_scale = mat.env_map_intensity;
      }
      if (environment >= 0 && !fp.gi) {
        // Environment light on the diffuse layer from one cosine-weighted
        // direction, tracer.ts:343-353: a shadow ray to infinity.
        const double r1 = rng_next(rng), r2 = rng_next(rng);
        const float phi = 2.0f * kPi * static_cast<float>(r1);
        const float radius = sqrtf(static_cast<float>(r2));
        float sphi, cphi;
        sincosf(phi, &sphi, &cphi);
        const V3 sd = to_world(nrm, radius * cphi, radius * sphi, sqrtf(fmaxf(0.0f, 1.0f - static_cast<float>(r2))));
        if (dot(sd, g) > 0.0f) {
          const V3 env = sample_environment(sc, environment, sd);
          em.emit(p + g * sc.eps, sd, inf, T * env * environment_scale * diff, sc.light_count, false);
        }
      }
      if (!fp.gi) diff = V3{0, 0, 0};
    } else {
      // Lambert, Phong and Toon, tracer.ts:355-389.
      for (int li = 0; li < sc.light_count; li++) {
        const DLight& L = sc.lights[li];
        V3 l, rad;
        float dist;
        if (!light_at(L, p, l, rad, dist)) continue;
        const float cosine = dot(nrm, l);
        float irradiance;
        if (mat.model == 3) {
          irradiance = cosine * 0.5f + 0.5f < 0.7f ? 0.7f : 1.0f;
        } else if (cosine <= 0.0f) {
          continue;
        } else {
          irradiance = cosine;
        }
        V3 cc = c * kInvPi;
        if (mat.model == 1 && cosine > 0.0f) {
          const V3 h = normalize_or_keep(l + vv);
          const float dot_nh = clamp01(dot(nrm, h));
          const float dot_vh = clamp01(dot(vv, h));
          const float fw = fresnel_weight(dot_vh);
          const float dd = blinn_phong(mat.shininess, dot_nh);
          cc.x += (mat.specular[0] * (1.0f - fw) + fw) * dd;
          cc.y += (mat.specular[1] * (1.0f - fw) + fw) * dd;
          cc.z += (mat.specular[2] * (1.0f - fw) + fw) * dd;
        }
        cc = cc * rad * irradiance;
        if (cc.x + cc.y + cc.z <= 0.0f) continue;
        direct_light(fp, sc, em, L, li, receive, p, g, l, dist, cc, out, w_light);
      }
      out = out + ir * c * (kInvPi * ao);
      if (fp.gi) diff = c;
    }
  }

  // Everything but the shadowed light, tracer.ts:408-410.
  Lr = Lr + T * (alpha_c * out + beta_c + e);

  bool done = !can_continue;
  if (!done) {
    // Continuation, tracer.ts:414-469.
    const float ws = luminance(spec.x, spec.y, spec.z);
    const float wt = luminance(trans.x, trans.y, trans.z);
    const float wd = luminance(diff.x, diff.y, diff.z);
    const float total = ws + wt + wd;
    if (total <= 1e-6f) {
      done = true;
    } else {
      const double pick = rng_next(rng) * static_cast<double>(total);
      V3 wv, sdir;
      float pr;
      bool cull = (fl & kFlagCull) != 0;
      V3 med = V3{m4.x, m4.y, m4.z};
      if (pick < static_cast<double>(ws)) {
        pr = ws / total;
        wv = spec;
        V3 hn = nrm;
        if (roughness > 0.02f) {
          // GGX-distributed microfacet normal, tracer.ts:608-621.
          const float a = roughness * roughness;
          const double r1 = rng_next(rng), r2 = rng_next(rng);
          const float phi = 2.0f * kPi * static_cast<float>(r1);
          const float r2f = static_cast<float>(r2);
          const float cos_t = sqrtf((1.0f - r2f) / (1.0f + (a * a - 1.0f) * r2f));
          const float sin_t = sqrtf(fmaxf(0.0f, 1.0f - cos_t * cos_t));
          float sphi, cphi;
          sincosf(phi, &sphi, &cphi);
          hn = to_world(nrm, sin_t * cphi, sin_t * sphi, cos_t);
        }
        sdir = d - hn * (2.0f * dot(d, hn));
        if (dot(sdir, g) <= 0.0f) done = true;
      } else if (pick < static_cast<double>(ws) + static_cast<double>(wt)) {
        pr = wt / total;
        wv = trans;
        if (mat.thickness > 0.0f) {
          // refract, tracer.ts:624-633, into or out of a solid.
          const float eta = front ? 1.0f / mat.ior : mat.ior;
          const float cosi = -dot(d, nrm);
          const float k = 1.0f - eta * eta * (1.0f - cosi * cosi);
          if (k >= 0.0f) {
            const float s = eta * cosi - sqrtf(k);
            sdir = normalize_or_keep(d * eta + nrm * s);
            cull = !front;
            med = front ? V3{mat.attenuation[0], mat.attenuation[1], mat.attenuation[2]} : V3{0, 0, 0};
          } else {
            sdir = d - nrm * (2.0f * dot(d, nrm));  // total internal reflection
          }
        } else {
          sdir = d;
        }
      } else {
        pr = wd / total;
        wv = diff;
        const double r1 = rng_next(rng), r2 = rng_next(rng);
        const float phi = 2.0f * kPi * static_cast<float>(r1);
        const float radius = sqrtf(static_cast<float>(r2));
        float sphi, cphi;
        sincosf(phi, &sphi, &cphi);
        sdir = to_world(nrm, radius * cphi, radius * sphi, sqrtf(fmaxf(0.0f, 1.0f - static_cast<float>(r2))));
        if (dot(sdir, g) <= 0.0f) done = true;
      }
      if (!done) {
        T = T * wv * (1.0f / pr);
        const float side = dot(sdir, g) > 0.0f ? sc.eps : -sc.eps;
        const V3 no = p + g * side;
        const uint32_t nb = bounce + 1;
        if (nb >= 3) {
          const float qq = fminf(0.95f, fmaxf(T.x, fmaxf(T.y, T.z)));
          if (rng_next(rng) >= static_cast<double>(qq)) {
            done = true;
          } else {
            T = T * (1.0f / qq);
          }
        }
        // Every continuation records the environment its ray may reach.
        fl = (fl & 0x00ffffffu) | (static_cast<uint32_t>(environment + 1) << 24);
        last_env_scale = environment_scale;
        fl = (fl & ~0xff0000u) | (min(nb, 255u) << 16);
        fl = cull ? (fl | kFlagCull) : (fl & ~kFlagCull);
        if (!done) {
          ps.ray_o[pid] = make_float4(no.x, no.y, no.z, 0.0f);
          ps.ray_d[pid] = make_float4(sdir.x, sdir.y, sdir.z, 0.0f);
          ps.med[pid] = make_float4(med.x, med.y, med.z, 0.0f);
          qs.next[queue_append(qs.next_count)] = pid;
        }
      }
    }
  }
  if (done) fl |= kFlagDone;
  ps.thr[pid] = make_float4(T.x, T.y, T.z, fog_factor);
  ps.rad[pid] = make_float4(Lr.x, Lr.y, Lr.z, last_env_scale);
  ps.rng[pid] = rng;
  ps.flags[pid] = fl;
  ps.smask[pid] = em.mask;
}

// Eight blocks of kBlock threads per SM (64 registers): the shading step then
// spills about 300 bytes per thread to L1, but the extra resident warps hide
// more of its memory latency. Measured on the mid workload: 10.9 ms of
// shading per frame at 5 blocks (95 registers, no spills), 10.5 at 6, 10.2 at
// 8, 10.6 at 10 and 11.4 at 12.
constexpr int kShadeBlocksPerSM = 8;
constexpr long long kShadeGridFactor = 16;  // batched shading grid, in resident grids

__global__ void __launch_bounds__(kBlock, kShadeBlocksPerSM) k_shade(DScene sc, FrameParams fp, PathState ps,
                                                  const int* __restrict__ qin, int n, int* __restrict__ qout,
                                                  Counters* cnt) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const StageQueues qs{qout, &cnt->next_count, ps.shadow_queue, &cnt->shadow_count};
  shade_path(sc, fp, ps, qin[q], qs);
}

// ------------------------------------------------------------------ shadow
// transmittance / attenuateShadow, tracer.ts:529-594, for one shadow ray: the
// any-hit walk stops at an opaque triangle or when almost no light is left.
struct ShadowQuery {
  const DScene& sc;
  const PathState& ps;
  int capacity;
  unsigned* status;
  int pid, slot;
  bool cast_only, blocked;
  float max_t;
  TravRay r;
  V3 w, shadow, depth;
  int nseen;
  float seen[kShadowSeen];
  MCRT_D void load(int i) {
    const float4* e = ps.shadow_queue + 3 * static_cast<size_t>(i);
    const float4 e0 = e[0], e1 = e[1], e2 = e[2];
    pid = __float_as_int(e1.w);
    const int tag = __float_as_int(e2.w);
    slot = tag & 0xffff;
    cast_only = (tag & 0x10000) != 0;
    max_t = e0.w;
    r = make_trav_ray(V3{e0.x, e0.y, e0.z}, V3{e1.x, e1.y, e1.z});
    w = V3{e2.x, e2.y, e2.z};
    shadow = V3{1.0f, 1.0f, 1.0f};
    depth = V3{0.0f, 0.0f, 0.0f};
    nseen = 0;
    blocked = false;
  }
  MCRT_D const TravRay& ray() const { return r; }
  MCRT_D float t_max() const { return max_t; }
  MCRT_D bool leaf(int first) {
    for (int k = first; k < sc.tri_count; k++) {
      V3 a, b, c;
      float4 w0, w1;
      load_tri(sc, k, a, b, c, w0, w1);
      const bool last = leaf_end(w0.w);
      TriHit th;
      if (intersect_triangle(r, a, b, c, max_t, 2, th) && visit(k, th, w0, w1)) return false;
      if (last) break;
    }
    return true;
  }
  // One hit of the visitor; true once the ray is blocked.
  MCRT_D bool visit(int k, const TriHit& th, float4 w0, float4 w1) {
    const int fl = tri_flags(w0.w);
    if (cast_only && (fl & 2) == 0) return false;
    if (fl & 1) {
      blocked = true;
      return true;
    }
    const DMaterial& mat = sc.materials[__float_as_int(w1.w)];
    float alpha = mat.opacity;
    V3 col = V3{mat.color[0], mat.color[1], mat.color[2]};
    if (mat.map >= 0 || mat.alpha_map >= 0) {
      const float4* at = sc.attrs + 4 * static_cast<size_t>(k);
      const float4 a2 = __ldg(at + 2), a3 = __ldg(at + 3);
      const float ww0 = 1.0f - th.u - th.v;
      const float tu = a2.y * ww0 + a2.w * th.u + a3.y * th.v;
      const float tv = a2.z * ww0 + a3.x * th.u + a3.z * th.v;
      if (mat.map >= 0) {
        const float4 tx = sample_texture(sc, mat.map, tu, tv);
        alpha *= tx.w;
        col = col * V3{tx.x, tx.y, tx.z};
      }
      if (mat.alpha_map >= 0) alpha *= sample_texture(sc, mat.alpha_map, tu, tv).y;
    }
    if (mat.alpha_test > 0.0f && alpha < mat.alpha_test) return false;
    if (!mat.transparent) alpha = 1.0f;
    bool dup = false;
    for (int i = 0; i < nseen; i++) dup |= fabsf(seen[i] - th.t) <= sc.eps;
    if (dup) return false;
    if (nseen < kShadowSeen) {
      seen[nseen++] = th.t;
    } else {
      *status |= kStatusShadowListOverflow;
    }
    if (mat.thickness > 0.0f) {
      const float sgn = th.front ? -th.t : th.t;
      depth = depth + V3{mat.attenuation[0], mat.attenuation[1], mat.attenuation[2]} * sgn;
    }
    const float open = 1.0f - alpha;
    const float through = mat.transmission;
    shadow = shadow * (V3{open, open, open} + col * (alpha * through));
    if (shadow.x + shadow.y + shadow.z < 1e-4f) {
      blocked = true;
      return true;
    }
    return false;
  }
  MCRT_D void finish() {
    V3 result = V3{0.0f, 0.0f, 0.0f};
    if (!blocked) {
      V3 s = shadow;
      if (depth.x > 0.0f) s.x *= expf(-depth.x);
      if (depth.y > 0.0f) s.y *= expf(-depth.y);
      if (depth.z > 0.0f) s.z *= expf(-depth.z);
      if (s.x + s.y + s.z > 0.0f) result = w * s;
    }
    ps.slots[static_cast<size_t>(slot) * capacity + pid] = make_float4(result.x, result.y, result.z, 0.0f);
  }
};

// 1152 / B blocks per SM: at 128 threads a cap of 56 registers (about 30 bytes
// of spills) keeps nine blocks resident instead of eight, 0.7 % faster; a cap
// of 48 spills in the walk itself and measured 40 % slower.
template <int B, int S>
__global__ void __launch_bounds__(B, 1152 / B) k_shadow(DScene sc, PathState ps, int n, int capacity, Counters* cnt) {
  unsigned status = 0;
  ShadowQuery q{sc, ps, capacity, &status};
  walk<kRefillShadow, B, S>(sc, q, n, &cnt->fetch_shadow, status);
  if (status) atomicOr(&cnt->status, status);
}

// ----------------------------------------------------------------- resolve
// Adds the path's shadowed light; tone maps and fogs a finished path.
MCRT_D void resolve_path(const DScene& sc, const FrameParams& fp, const PathState& ps, int pid, int capacity) {
  const uint32_t fl = ps.flags[pid];
  if (fl & kFlagDirect) return;  // a background sample, written by shading; no shadow rays
  unsigned long long mask = ps.smask[pid];
  if (mask == 0ull && !(fl & kFlagDone)) return;
  float4 L4 = ps.rad[pid];
  while (mask) {
    const int slot = __ffsll(static_cast<long long>(mask)) - 1;
    mask &= mask - 1;
    const float4 c = ps.slots[static_cast<size_t>(slot) * capacity + pid];
    L4.x += c.x;
    L4.y += c.y;
    L4.z += c.z;
  }
  ps.smask[pid] = 0ull;
  if (!(fl & kFlagDone)) {
    ps.rad[pid] = L4;
    return;
  }
  // Tone map and fog the finished path, tracer.ts:472-477.
  float c[3] = {L4.x, L4.y, L4.z};
  if ((fl & kFlagToneMap) && fp.tone_mapping != 0) tone_map(c, fp.tone_mapping, fp.exposure);
  const float fog_factor = ps.thr[pid].w;
  if (fog_factor > 0.0f && sc.fog.kind != 0) {
    for (int i = 0; i < 3; i++) c[i] = c[i] + (sc.fog.color[i] - c[i]) * fog_factor;
  }
  ps.sample[pid] = make_float4(c[0], c[1], c[2], 1.0f);
}

__global__ void __launch_bounds__(kBlock) k_resolve(DScene sc, FrameParams fp, PathState ps,
                                                    const int* __restrict__ queue, int n, int capacity) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) resolve_path(sc, fp, ps, queue[q], capacity);
}

// -------------------------------------------------------------- accumulate
// writeTile's encode, progressive.ts:299-310: average, un-premultiply, sRGB,
// then the Uint8ClampedArray store.
MCRT_D uchar4 encode_rgba(double r, double g, double b, double a, double scale, int srgb) {
  r *= scale;
  g *= scale;
  b *= scale;
  a *= scale;
  if (a > 0) {
    r /= a;
    g /= a;
    b /= a;
  }
  if (srgb) {
    r = linear_to_srgb_f64(fmax(0.0, r));
    g = linear_to_srgb_f64(fmax(0.0, g));
    b = linear_to_srgb_f64(fmax(0.0, b));
  }
  uchar4 o;
  o.x = encode_byte(r);
  o.y = encode_byte(g);
  o.z = encode_byte(b);
  o.w = encode_byte(a);
  return o;
}

// writeTile, progressive.ts:295-310, over the passes of one chunk in order
// (the plain wavefront runs a chunk's paths pixel-major, so pixel i's samples
// are the `passes` consecutive ones from i * passes). The running sum is Float32; the encode reads the last pass's sum unrounded,
// as `r = sum[d] = sum[d] + r` does, in double.
__global__ void __launch_bounds__(256) k_accumulate(const float4* __restrict__ samples, int npix, int passes,
                                                    float4* __restrict__ sum, int total_passes, int last_chunk,
                                                    uint8_t* __restrict__ image, FrameParams fp, int srgb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const int gi = fp.pix0 + i;  // pixel index in the tile or list
  float4 s = sum[gi];
  double r = 0, g = 0, b = 0, a = 0;
  for (int j = 0; j < passes; j++) {
    const float4 x = samples[static_cast<size_t>(i) * passes + j];
    r = static_cast<double>(s.x) + x.x;
    g = static_cast<double>(s.y) + x.y;
    b = static_cast<double>(s.z) + x.z;
    a = static_cast<double>(s.w) + x.w;
    s = make_float4(static_cast<float>(r), static_cast<float>(g), static_cast<float>(b), static_cast<float>(a));
  }
  sum[gi] = s;
  if (!last_chunk || !image) return;
  const uchar4 o = encode_rgba(r, g, b, a, 1.0 / total_passes, srgb);
  if (fp.mode == 1) {
    reinterpret_cast<uchar4*>(image)[gi] = o;
  } else {
    const int px = fp.tile_x + gi % fp.tile_w, py = fp.tile_y + gi / fp.tile_w;
    reinterpret_cast<uchar4*>(image)[static_cast<size_t>(py) * fp.width + px] = o;
  }
}

// Tile output of renderTile (tracer.ts:62-89): each pixel takes the sample of
// its block; this launch series holds blocks [pix0, pix0 + npix).
__global__ void k_tile_output(const float4* __restrict__ samples, FrameParams fp, float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = fp.tile_w * fp.tile_h;
  if (i >= n) return;
  const int x = i % fp.tile_w, y = i / fp.tile_w;
  const int b = (y / fp.block) * fp.nbx + (x / fp.block) - fp.pix0;
  if (b < 0 || b >= fp.npix) return;
  out[i] = samples[b];
}

// Closest hits of arbitrary rays (origin, -, direction, -): debugging and parity.
struct RayQuery {
  const DScene& sc;
  const float4* rays;
  int cull;
  int4* hits;
  int i;
  ClosestState cs;
  MCRT_D void load(int k) {
    i = k;
    const float4 o = rays[2 * k], d = rays[2 * k + 1];
    cs.start(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z}, cull != 0);
  }
  MCRT_D const TravRay& ray() const { return cs.r; }
  MCRT_D float t_max() const { return cs.tmax; }
  MCRT_D bool leaf(int first) { return cs.leaf(sc, first); }
  MCRT_D void finish() {
    hits[i] = make_int4(cs.h.tri, __float_as_int(cs.h.t), __float_as_int(cs.h.u),
                        (cs.h.front ? 1 : 0) | (min(cs.tests, 0xffffff) << 8));
  }
};

__global__ void __launch_bounds__(kBlock) k_trace_rays(DScene sc, const float4* __restrict__ rays, int n, int cull,
                                                       int4* __restrict__ hits, unsigned* fetch) {
  unsigned status = 0;
  RayQuery q{sc, rays, cull, hits, 0, {}};
  walk<kRefill, kBlock, kShort>(sc, q, n, fetch, status);
  if (status) atomicOr(fetch + 1, status);
}

// Number of hits along each ray (intersectAny with a counting visitor).
struct CountQuery {
  const DScene& sc;
  const float4* rays;
  int* counts;
  int i, hits;
  float limit;
  TravRay r;
  MCRT_D void load(int k) {
    i = k;
    hits = 0;
    const float4 o = rays[2 * k], d = rays[2 * k + 1];
    limit = o.w > 0.0f ? o.w : __int_as_float(0x7f800000);
    r = make_trav_ray(V3{o.x, o.y, o.z}, V3{d.x, d.y, d.z});
  }
  MCRT_D const TravRay& ray() const { return r; }
  MCRT_D float t_max() const { return limit; }
  MCRT_D bool leaf(int first) {
    for (int k = first; k < sc.tri_count; k++) {
      V3 a, b, c;
      float4 w0, w1;
      load_tri(sc, k, a, b, c, w0, w1);
      TriHit th;
      if (intersect_triangle(r, a, b, c, limit, 2, th)) hits++;
      if (leaf_end(w0.w)) break;
    }
    return true;
  }
  MCRT_D void finish() { counts[i] = hits; }
};

__global__ void __launch_bounds__(kBlock) k_count_hits(DScene sc, const float4* __restrict__ rays, int n,
                                                       int* __restrict__ counts, unsigned* fetch) {
  unsigned status = 0;
  CountQuery q{sc, rays, counts, 0, 0, 0.0f, {}};
  walk<kRefill, kBlock, kShort>(sc, q, n, fetch, status);
  if (status) atomicOr(fetch + 1, status);
}

// ------------------------------------------------------------------- host
PathBuffers::~PathBuffers() {
  release();
  if (fork_) cudaEventDestroy(fork_);
  if (join_) cudaEventDestroy(join_);
  if (side_) cudaStreamDestroy(side_);
}

cudaError_t PathBuffers::side_stream(cudaStream_t* side, cudaEvent_t* fork, cudaEvent_t* join) {
  cudaError_t e = cudaSuccess;
  if (!side_) e = cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking);
  if (e == cudaSuccess && !fork_) e = cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming);
  if (e == cudaSuccess && !join_) e = cudaEventCreateWithFlags(&join_, cudaEventDisableTiming);
  *side = side_;
  *fork = fork_;
  *join = join_;
  return e;
}

void PathBuffers::release() {
  for (void* p : allocations_) cudaFree(p);
  allocations_.clear();
  if (counters_) cudaFree(counters_);
  if (host_counters_) cudaFreeHost(host_counters_);
  counters_ = nullptr;
  host_counters_ = nullptr;
  st_ = PathState{};
  capacity_ = slots_ = 0;
  bytes_ = 0;
}

cudaError_t PathBuffers::reserve(int capacity, int slots) {
  if (capacity <= capacity_ && slots <= slots_ && counters_) return cudaSuccess;
  release();
  capacity = std::max(capacity, 1);
  slots = std::max(slots, 1);
  const size_t n = static_cast<size_t>(capacity);
  auto alloc = [&](size_t bytes, void** out) -> cudaError_t {
    cudaError_t e = cudaMalloc(out, bytes);
    if (e == cudaSuccess) {
      allocations_.push_back(*out);
      bytes_ += bytes;
    }
    return e;
  };
  cudaError_t e = cudaSuccess;
#define MCRT_ALLOC(field, count)                                                   \
  if (e == cudaSuccess) {                                                          \
    void* p = nullptr;                                                             \
    e = alloc(sizeof(*st_.field) * (count), &p);                                  \
    st_.field = static_cast<decltype(st_.field)>(p);                              \
  }
  MCRT_ALLOC(ray_o, n)
  MCRT_ALLOC(ray_d, n)
  MCRT_ALLOC(hit, n)
  MCRT_ALLOC(thr, n)
  MCRT_ALLOC(rad, n)
  MCRT_ALLOC(med, n)
  MCRT_ALLOC(rng, n)
  MCRT_ALLOC(flags, n)
  MCRT_ALLOC(smask, n)
  MCRT_ALLOC(sample, n)
  MCRT_ALLOC(seg, n)
  MCRT_ALLOC(slots, n * slots)
  MCRT_ALLOC(shadow_queue, n * slots * 3)
#undef MCRT_ALLOC
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    void* p = nullptr;
    e = alloc(sizeof(int) * n, &p);
    st_.queue[i] = static_cast<int*>(p);
  }
  if (e == cudaSuccess) {
    void* p = nullptr;
    e = alloc(sizeof(int) * n, &p);
    st_.binned = static_cast<int*>(p);
  }
  if (e == cudaSuccess) {
    void* p = nullptr;
    e = alloc(n, &p);
    st_.cls = static_cast<uint8_t*>(p);
  }
  if (e == cudaSuccess) {
    void* p = nullptr;
    e = alloc(sizeof(unsigned int) * 2 * kShadeClasses * kMaxBatchScenes, &p);
    st_.bins = static_cast<unsigned int*>(p);
    if (e == cudaSuccess) e = cudaMemset(p, 0, sizeof(unsigned int) * 2 * kShadeClasses * kMaxBatchScenes);
  }
  if (e == cudaSuccess) e = cudaMalloc(&counters_, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMallocHost(&host_counters_, sizeof(Counters));
  if (e != cudaSuccess) {
    release();
    return e;
  }
  capacity_ = capacity;
  slots_ = slots;
  return cudaSuccess;
}

namespace {

struct Timer {
  bool on;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  Timer(bool enabled, cudaStream_t stream) : on(enabled), s(stream) {
    if (on) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
    }
  }
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  void start() {
    if (on) cudaEventRecord(a, s);
  }
  void stop(double& total, unsigned long long& count) {
    if (!on) return;
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    total += ms;
    count++;
  }
};

inline int blocks_for(long long n, int block) { return static_cast<int>((n + block - 1) / block); }

// Blocks of a persistent launch of `kernel` with `block` threads: enough to
// fill every SM at the kernel's occupancy (cached per device and kernel),
// fewer when there is less work.
int resident_limit(const void* kernel, int block) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({kernel, dev});
  if (it != cache.end()) return it->second;
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
  const int r = std::max(1, sms) * std::max(1, per_sm);
  cache[{kernel, dev}] = r;
  return r;
}

template <class K>
int persistent_blocks(K kernel, long long n, int block = kBlock) {
  const int limit = resident_limit(reinterpret_cast<const void*>(kernel), block);
  return static_cast<int>(std::min<long long>(blocks_for(n, block), limit));
}

// The traversal kernels compiled for each variant (block size, short-stack
// depth); the autotuner picks one per scene and workload.
using ExtendFn = void (*)(DScene, PathState, const int*, int, Counters*, unsigned int*);
using ShadowFn = void (*)(DScene, PathState, int, int, Counters*);

struct PlainVariant {
  int block, stack;
  ExtendFn extend;
  ShadowFn shadow;
};

#define MCRT_PLAIN_VARIANT(B, S) PlainVariant{B, S, k_extend<B, S>, k_shadow<B, S>}
const PlainVariant kPlainVariants[] = {
    MCRT_PLAIN_VARIANT(128, 4), MCRT_PLAIN_VARIANT(128, 8), MCRT_PLAIN_VARIANT(64, 16),
    MCRT_PLAIN_VARIANT(128, 16), MCRT_PLAIN_VARIANT(256, 8), MCRT_PLAIN_VARIANT(256, 16),
};
#undef MCRT_PLAIN_VARIANT
constexpr int kVariantCount = static_cast<int>(sizeof(kPlainVariants) / sizeof(kPlainVariants[0]));

const PlainVariant& plain_variant(int v) { return kPlainVariants[(v >= 0 && v < kVariantCount) ? v : 0]; }

}  // namespace

int traversal_variant_count() { return kVariantCount; }

void traversal_variant_info(int v, int* block, int* stack) {
  const PlainVariant& p = plain_variant(v);
  if (block) *block = p.block;
  if (stack) *stack = p.stack;
}

int find_traversal_variant(int block, int stack) {
  for (int i = 0; i < kVariantCount; i++)
    if (kPlainVariants[i].block == block && kPlainVariants[i].stack == stack) return i;
  return -1;
}

cudaError_t Wavefront::run(const DScene& scene, FrameParams fp, int passes, PathBuffers& buffers,
                           cudaStream_t stream, RenderStats* stats, bool timed,
                           cudaError_t (*on_chunk)(void*, int, int), void* ctx) {
  const int npix = fp.npix;
  if (npix <= 0 || passes <= 0) return cudaSuccess;
  const int cap = buffers.capacity();
  const int chunk_passes = std::max(1, std::min(passes, cap / npix));
  if (static_cast<long long>(chunk_passes) * npix > cap) return cudaErrorInvalidValue;
  PathState ps = buffers.state();
  Counters* cnt = buffers.counters();
  Counters* host = buffers.host_counters();
  fp.capacity = cap;
  fp.slot_count = buffers.slots();
  Timer tm(timed, stream);
  const PlainVariant& tv = plain_variant(variant);
  RenderStats local;
  RenderStats& st = stats ? *stats : local;
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(Counters), stream);
  // Untimed renders trace bounce k's shadow rays and resolve its paths on a
  // side stream while bounce k + 1's closest hits (and shading sort) run on
  // the main one: neither touches what the other reads or writes, and each
  // fills the other's tail of idle SMs. Shading k + 1 waits for the side
  // stream (it rewrites the shadow queue, the slots and the path queue that
  // resolve reads). Timed renders keep one stream, so every kernel's events
  // bracket it alone.
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  bool overlap = !timed;
  if (overlap && e == cudaSuccess) {
    e = buffers.side_stream(&side, &fork, &join);
    overlap = e == cudaSuccess;
  }
  bool side_busy = false;  // side work queued since the main stream last joined it
  auto join_side = [&]() {
    if (side_busy) {
      cudaStreamWaitEvent(stream, join, 0);
      side_busy = false;
    }
  };
  for (int first = 0; first < passes && e == cudaSuccess; first += chunk_passes) {
    const int np = std::min(chunk_passes, passes - first);
    int n = np * npix;
    FrameParams f = fp;
    f.pass0 = fp.pass0 + first;
    f.npass = np;
    tm.start();
    k_raygen<<<blocks_for(n, kBlock), kBlock, 0, stream>>>(f, ps, n);
    tm.stop(st.ms_raygen, st.n_raygen);
    st.launches++;
    st.samples += n;
    int cur = 0;
    int iterations = 0;
    while (n > 0) {
      // Paths end by bounce count, pass-through count or Russian roulette; a
      // loop this long means corrupt state, reported rather than spun on.
      if (++iterations > kMaxIterations) {
        e = cudaErrorLaunchTimeout;
        break;
      }
      // The camera rays walk warp-coherent where a warp's 32 rays (passes of
      // 32 / npass pixels of a row) span at most 1/360 of the image height:
      // measured on the mid scene at 64 passes, the coherent walk was 1-3 %
      // faster per frame from 640x360 to 2560x1440 and a third slower per
      // launch at 320x180. (Their shadow rays lose with it at every size: lanes
      // blocked early idle until the warp's last ray ends, where the per-lane
      // walk refills them.)
      const int warp_pixels = 32 / std::max(1, std::min(f.npass, 32));
      const bool coherent = packet_first && iterations == 1 && warp_pixels * 360 <= f.height;
      // A queue long enough to shade in hit-class order has its classes
      // counted by the closest-hit kernel itself (ExtendQuery with a
      // histogram); the scatter then puts the queue in that order.
      const bool sort = sort_shading && n >= kSortMin;
      unsigned int* class_bins = sort ? ps.bins : nullptr;
      if (sort) cudaMemsetAsync(ps.bins, 0, 2 * kShadeClasses * sizeof(unsigned int), stream);
      cudaMemsetAsync(&cnt->fetch, 0, sizeof(unsigned int), stream);
      tm.start();
      if (coherent) {
        k_extend_packet<kBlock><<<persistent_blocks(k_extend_packet<kBlock>, n), kBlock, 0, stream>>>(
            scene, ps, ps.queue[cur], n, cnt, class_bins);
      } else {
        tv.extend<<<persistent_blocks(tv.extend, n, tv.block), tv.block, 0, stream>>>(scene, ps, ps.queue[cur], n,
                                                                                      cnt, class_bins);
      }
      tm.stop(st.ms_extend, st.n_extend);
      st.closest_rays += n;
      const int* shade_queue = ps.queue[cur];
      if (sort) {
        k_class_scatter<<<blocks_for(n, 256), 256, 0, stream>>>(scene, ps, ps.queue[cur], n, ps.bins, ps.binned);
        shade_queue = ps.binned;
        st.launches += 1;
      }
      join_side();
      cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned int), stream);
      tm.start();
      k_shade<<<blocks_for(n, kBlock), kBlock, 0, stream>>>(scene, f, ps, shade_queue, n, ps.queue[cur ^ 1], cnt);
      tm.stop(st.ms_shade, st.n_shade);
      cudaMemcpyAsync(host, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, stream);
      e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) break;
      const int n_next = static_cast<int>(host->next_count);
      const int n_shadow = static_cast<int>(host->shadow_count);
      st.status |= host->status;
      cudaStream_t sh = stream;
      if (overlap) {
        cudaEventRecord(fork, stream);
        cudaStreamWaitEvent(side, fork, 0);
        sh = side;
      }
      if (n_shadow > 0) {
        cudaMemsetAsync(&cnt->fetch_shadow, 0, sizeof(unsigned int), sh);
        tm.start();
        tv.shadow<<<persistent_blocks(tv.shadow, n_shadow, tv.block), tv.block, 0, sh>>>(scene, ps, n_shadow, cap,
                                                                                         cnt);
        tm.stop(st.ms_shadow, st.n_shadow);
        st.any_rays += n_shadow;
        st.launches++;
      }
      tm.start();
      k_resolve<<<blocks_for(n, kBlock), kBlock, 0, sh>>>(scene, f, ps, ps.queue[cur], n, cap);
      tm.stop(st.ms_resolve, st.n_resolve);
      if (overlap) {
        cudaEventRecord(join, side);
        side_busy = true;
      }
      st.launches += 3;
      n = n_next;
      cur ^= 1;
    }
    join_side();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess && on_chunk) {
      tm.start();
      e = on_chunk(ctx, first, np);
      tm.stop(st.ms_accumulate, st.n_accumulate);
    }
  }
  join_side();
  if (side) {
    const cudaError_t es = cudaStreamSynchronize(side);
    if (e == cudaSuccess) e = es;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(host, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) st.status |= host->status;
  }
  return e;
}

cudaError_t primary_hits(const DScene& scene, FrameParams fp, PathBuffers& buffers, cudaStream_t stream) {
  const int n = fp.npix;
  if (n <= 0) return cudaSuccess;
  if (n > buffers.capacity()) return cudaErrorInvalidValue;
  PathState ps = buffers.state();
  fp.capacity = buffers.capacity();
  fp.slot_count = buffers.slots();
  k_raygen<<<blocks_for(n, kBlock), kBlock, 0, stream>>>(fp, ps, n);
  cudaMemsetAsync(&buffers.counters()->fetch, 0, sizeof(unsigned int), stream);
  const PlainVariant& tv = plain_variant(0);
  tv.extend<<<persistent_blocks(tv.extend, n, tv.block), tv.block, 0, stream>>>(scene, ps, ps.queue[0], n,
                                                                                  buffers.counters(), nullptr);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const float4* samples, int npix, int passes_in_chunk, float4* sum, int total_passes,
                              int last_chunk, uint8_t* image, const FrameParams& fp, int srgb, cudaStream_t s) {
  k_accumulate<<<blocks_for(npix, 256), 256, 0, s>>>(samples, npix, passes_in_chunk, sum, total_passes, last_chunk,
                                                     image, fp, srgb);
  return cudaGetLastError();
}

cudaError_t launch_tile_output(const float4* samples, const FrameParams& fp, float* out, cudaStream_t s) {
  const int n = fp.tile_w * fp.tile_h;
  k_tile_output<<<blocks_for(n, 256), 256, 0, s>>>(samples, fp, reinterpret_cast<float4*>(out));
  return cudaGetLastError();
}

cudaError_t launch_trace_rays(const DScene& scene, const float4* rays, int count, int cull, int4* hits,
                              unsigned* fetch, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  cudaMemsetAsync(fetch, 0, sizeof(unsigned), s);
  k_trace_rays<<<persistent_blocks(k_trace_rays, count), kBlock, 0, s>>>(scene, rays, count, cull, hits, fetch);
  return cudaGetLastError();
}

cudaError_t launch_count_hits(const DScene& scene, const float4* rays, int count, int* counts, unsigned* fetch,
                              cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  cudaMemsetAsync(fetch, 0, sizeof(unsigned), s);
  k_count_hits<<<persistent_blocks(k_count_hits, count), kBlock, 0, s>>>(scene, rays, count, counts, fetch);
  return cudaGetLastError();
}

// ------------------------------------------------------------ batched renders
namespace {

// The segment holding item `k`: the last j < n with base[j] <= k.
MCRT_D int find_segment(const int* base, int n, int k) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= k) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

__global__ void __launch_bounds__(kBlock) k_batch_raygen(const BatchTables* __restrict__ t, PathState ps) {
  __shared__ int base[kMaxSegments + 1];
  const int nseg = t->segments;
  for (int i = threadIdx.x; i <= nseg; i += blockDim.x) base[i] = t->seg_base[i];
  __syncthreads();
  const int n = t->paths;
  for (int pid = blockIdx.x * blockDim.x + threadIdx.x; pid < n; pid += gridDim.x * blockDim.x) {
    const int j = find_segment(base, nseg, pid);
    ps.seg[pid] = j;
    raygen_path(t->fp[j], ps, pid);
  }
}

template <int B, int S>
__global__ void __launch_bounds__(B, 1280 / B) k_batch_extend(DScene sc, int s, BatchTables* t, PathState ps,
                                                    BatchCounters* bc) {
  SceneQueues* sq = &t->scenes[s];
  const int n = static_cast<int>(sq->count);
  if (n == 0) return;
  unsigned status = 0;
  ExtendQuery q{sc, ps, ps.queue[t->iteration & 1] + sq->base, 0, {}, nullptr, 0};
  walk<kRefillClosest, B, S>(sc, q, n, &sq->fetch, status);
  if (status) atomicOr(&bc->status, status);
}

__global__ void __launch_bounds__(kBlock, kShadeBlocksPerSM) k_batch_shade(DScene sc, int s, BatchTables* t, PathState ps, int slots) {
  SceneQueues* sq = &t->scenes[s];
  const int n = static_cast<int>(sq->count);
  const int cur = t->iteration & 1;
  // In shading order once the queue is long enough to be sorted (k_batch_class_*).
  const int* qin = (n >= kSortMin ? ps.binned : ps.queue[cur]) + sq->base;
  const StageQueues qs{ps.queue[cur ^ 1] + sq->base, &sq->next_count,
                       ps.shadow_queue + 3ull * sq->base * static_cast<unsigned>(slots), &sq->shadow_count};
  // Every lane of a warp runs the same number of iterations and the warp
  // reconverges after each path: shading diverges by material, and a warp
  // whose lanes drifted apart across iterations ran each path's code once per
  // lane group (a third of the lanes active, instruction-cache misses).
  const FrameParams* __restrict__ params = t->fp;
  const int stride = gridDim.x * blockDim.x;
#pragma unroll 1
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int q = base + threadIdx.x;
    if (q < n) {
      const int pid = qin[q];
      // The segment's parameters through a read-only, non-aliasing view of
      // the table: through `t` itself every field would be reloaded after
      // each store of the shading step, one dependent L1 round trip each.
      shade_path(sc, params[ps.seg[pid]], ps, pid, qs);
    }
    __syncwarp();
  }
}

template <int B, int S>
__global__ void __launch_bounds__(B, 1152 / B) k_batch_shadow(DScene sc, int s, BatchTables* t, PathState ps, int capacity,
                                                    int slots, BatchCounters* bc) {
  SceneQueues* sq = &t->scenes[s];
  const int n = static_cast<int>(sq->shadow_count);
  if (n == 0) return;
  unsigned status = 0;
  PathState pq = ps;
  pq.shadow_queue += 3ull * sq->base * static_cast<unsigned>(slots);
  ShadowQuery q{sc, pq, capacity, &status};
  walk<kRefillShadow, B, S>(sc, q, n, &sq->fetch_shadow, status);
  if (status) atomicOr(&bc->status, status);
}

__global__ void __launch_bounds__(kBlock) k_batch_resolve(DScene sc, int s, BatchTables* t, PathState ps,
                                                          int capacity) {
  SceneQueues* sq = &t->scenes[s];
  const int n = static_cast<int>(sq->count);
  const int* qin = ps.queue[t->iteration & 1] + sq->base;
  const FrameParams* __restrict__ params = t->fp;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int q = base + threadIdx.x;
    if (q < n) {
      const int pid = qin[q];
      resolve_path(sc, params[ps.seg[pid]], ps, pid, capacity);
    }
    __syncwarp();
  }
}

// Shading order of one scene's queue range (the class count, then
// k_class_scatter's scatter, over a resident grid): bins of scene s are
// bins[32 s, 32 s + 32).
__global__ void __launch_bounds__(256) k_batch_class_count(DScene sc, int s, BatchTables* t, PathState ps) {
  SceneQueues* sq = &t->scenes[s];
  const int n = static_cast<int>(sq->count);
  if (n < kSortMin) return;
  const int* qin = ps.queue[t->iteration & 1] + sq->base;
  unsigned int* bins = ps.bins + 2 * kShadeClasses * s;
  __shared__ unsigned int h[kShadeClasses];
  if (threadIdx.x < kShadeClasses) h[threadIdx.x] = 0;
  __syncthreads();
  uint8_t* cls = ps.cls + sq->base;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = shade_class(sc, ps, qin[i]);
    cls[i] = static_cast<uint8_t>(c);
    atomicAdd(&h[c], 1u);
  }
  __syncthreads();
  if (threadIdx.x < kShadeClasses && h[threadIdx.x]) atomicAdd(&bins[threadIdx.x], h[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_batch_class_scatter(DScene sc, int s, BatchTables* t, PathState ps) {
  SceneQueues* sq = &t->scenes[s];
  const int n = static_cast<int>(sq->count);
  if (n < kSortMin) return;
  const int* qin = ps.queue[t->iteration & 1] + sq->base;
  unsigned int* bins = ps.bins + 2 * kShadeClasses * s;
  int* out = ps.binned + sq->base;
  __shared__ unsigned int base[kShadeClasses];
  if (threadIdx.x == 0) {
    unsigned int sum = 0;
    for (int b = 0; b < kShadeClasses; b++) {
      base[b] = sum;
      sum += bins[b];
    }
  }
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  for (int first = blockIdx.x * blockDim.x; first < n; first += stride) {
    scatter_block(qin, ps.cls + sq->base, n, first, base, bins + kShadeClasses, out);
    __syncthreads();  // the block's shared counters are reused by the next tile
  }
}

// Queue swap after an iteration, on one thread: counts the queries traced,
// makes the continued paths the next iteration's queue and says whether
// another iteration is needed.
__global__ void k_batch_advance(BatchTables* t, int nscenes, BatchCounters* bc, unsigned int* bins, int graph,
                                cudaGraphConditionalHandle handle) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  bool more = false;
  unsigned long long closest = 0, any = 0;
  for (int s = 0; s < nscenes; s++) {
    SceneQueues& q = t->scenes[s];
    closest += q.count;
    any += q.shadow_count;
    q.count = q.next_count;
    q.next_count = 0;
    q.shadow_count = 0;
    q.fetch = 0;
    q.fetch_shadow = 0;
    more = more || q.count > 0;
  }
  bc->closest += closest;
  bc->any += any;
  for (int i = 0; i < 2 * kShadeClasses * nscenes; i++) bins[i] = 0;  // the next iteration's shading order
  const int it = t->iteration + 1;
  t->iteration = it;
  if (more && it >= t->max_iterations) {
    bc->status |= kStatusIterationLimit;
    more = false;
  }
  bc->more = more ? 1u : 0u;
  if (graph) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// writeTile for one segment item: a preview block written straight into the
// image (no running sum, count 1), or one pixel's passes (consecutive paths:
// segments run pixel-major) added in order to the Float32 sum and the average
// encoded.
__global__ void __launch_bounds__(256) k_batch_accumulate(const BatchTables* __restrict__ t, PathState ps) {
  __shared__ int base[kMaxSegments + 1];
  const int nseg = t->segments;
  for (int i = threadIdx.x; i <= nseg; i += blockDim.x) base[i] = t->pix_base[i];
  __syncthreads();
  const int total = base[nseg];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    const int j = find_segment(base, nseg, k);
    const int i = k - base[j];
    const FrameParams& fp = t->fp[j];
    const SegmentOut& o = t->out[j];
    const float4* samples = ps.sample + t->seg_base[j];
    uchar4* image = reinterpret_cast<uchar4*>(o.image);
    if (o.preview) {
      const float4 x = samples[i];
      const uchar4 c = encode_rgba(x.x, x.y, x.z, x.w, 1.0, o.srgb);
      const int bi = fp.pix0 + i;
      const int by = bi / fp.nbx, bx = bi - by * fp.nbx;
      const int x0 = fp.tile_x + bx * fp.block, y0 = fp.tile_y + by * fp.block;
      const int x1 = min(x0 + fp.block, fp.tile_x + fp.tile_w), y1 = min(y0 + fp.block, fp.tile_y + fp.tile_h);
      for (int y = y0; y < y1; y++)
        for (int xx = x0; xx < x1; xx++) image[static_cast<size_t>(y) * fp.width + xx] = c;
      continue;
    }
    const int gi = fp.pix0 + i;
    // A segment starting at pass 0 starts the pixel's running sum (request
    // buffers are not cleared when they are taken from the arena).
    float4 sm = fp.pass0 == 0 ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : o.sum[gi];
    double r = 0, g = 0, b = 0, a = 0;
    for (int jj = 0; jj < o.passes; jj++) {
      const float4 x = samples[static_cast<size_t>(i) * o.passes + jj];
      r = static_cast<double>(sm.x) + x.x;
      g = static_cast<double>(sm.y) + x.y;
      b = static_cast<double>(sm.z) + x.z;
      a = static_cast<double>(sm.w) + x.w;
      sm = make_float4(static_cast<float>(r), static_cast<float>(g), static_cast<float>(b), static_cast<float>(a));
    }
    o.sum[gi] = sm;
    const int px = fp.tile_x + gi % fp.tile_w, py = fp.tile_y + gi / fp.tile_w;
    image[static_cast<size_t>(py) * fp.width + px] = encode_rgba(r, g, b, a, 1.0 / o.done_after, o.srgb);
  }
}

int resident_blocks(const void* kernel, int block) { return resident_limit(kernel, block); }

using BatchExtendFn = void (*)(DScene, int, BatchTables*, PathState, BatchCounters*);
using BatchShadowFn = void (*)(DScene, int, BatchTables*, PathState, int, int, BatchCounters*);

struct BatchVariant {
  int block, stack;
  BatchExtendFn extend;
  BatchShadowFn shadow;
};

// The same variants, in the same order, as kPlainVariants.
#define MCRT_BATCH_VARIANT(B, S) BatchVariant{B, S, k_batch_extend<B, S>, k_batch_shadow<B, S>}
const BatchVariant kBatchVariants[] = {
    MCRT_BATCH_VARIANT(128, 4), MCRT_BATCH_VARIANT(128, 8), MCRT_BATCH_VARIANT(64, 16),
    MCRT_BATCH_VARIANT(128, 16), MCRT_BATCH_VARIANT(256, 8), MCRT_BATCH_VARIANT(256, 16),
};
#undef MCRT_BATCH_VARIANT
static_assert(sizeof(kBatchVariants) / sizeof(kBatchVariants[0]) == kVariantCount, "variant tables differ");

const BatchVariant& batch_variant(int v) { return kBatchVariants[(v >= 0 && v < kVariantCount) ? v : 0]; }

}  // namespace

cudaError_t batch_grids(BatchGrids* g, int variant, int capacity) {
  const BatchVariant& bv = batch_variant(variant);
  g->variant = (variant >= 0 && variant < kVariantCount) ? variant : 0;
  g->block = bv.block;
  g->raygen = resident_blocks(reinterpret_cast<const void*>(k_batch_raygen), kBlock);
  g->extend = resident_blocks(reinterpret_cast<const void*>(bv.extend), bv.block);
  // Shading launches many more blocks than fit at once (each taking a few
  // 128-path tiles): blocks that finish make room for fresh ones, as in the
  // one-path-per-thread launch of the plain path, instead of a resident grid
  // whose warps stay in the shading code for every tile.
  {
    const int resident = resident_blocks(reinterpret_cast<const void*>(k_batch_shade), kBlock);
    const long long tiles = (static_cast<long long>(std::max(capacity, 1)) + kBlock - 1) / kBlock;
    g->shade = static_cast<int>(std::max<long long>(resident, std::min<long long>(tiles, kShadeGridFactor * resident)));
  }
  g->shadow = resident_blocks(reinterpret_cast<const void*>(bv.shadow), bv.block);
  g->resolve = resident_blocks(reinterpret_cast<const void*>(k_batch_resolve), kBlock);
  g->accumulate = resident_blocks(reinterpret_cast<const void*>(k_batch_accumulate), 256);
  g->sort = resident_blocks(reinterpret_cast<const void*>(k_batch_class_scatter), 256);
  return cudaGetLastError();
}

cudaError_t launch_batch_raygen(const BatchTables* t, const PathState& ps, const BatchGrids& g, cudaStream_t s) {
  k_batch_raygen<<<g.raygen, kBlock, 0, s>>>(t, ps);
  return cudaGetLastError();
}

cudaError_t launch_batch_iteration(const DScene* scenes, int nscenes, BatchTables* t, const PathState& ps,
                                   int capacity, int slots, BatchCounters* counters, const BatchGrids& g, bool graph,
                                   cudaGraphConditionalHandle handle, cudaStream_t s, const SceneLanes* lanes) {
  const BatchVariant& bv = batch_variant(g.variant);
  // One scene's stages, in order: closest hits, shading order, shading, shadow
  // rays, resolve. Scenes touch disjoint queue ranges, bins and slots.
  auto chain = [&](int i, cudaStream_t q) {
    bv.extend<<<g.extend, bv.block, 0, q>>>(scenes[i], i, t, ps, counters);
    k_batch_class_count<<<g.sort, 256, 0, q>>>(scenes[i], i, t, ps);
    k_batch_class_scatter<<<g.sort, 256, 0, q>>>(scenes[i], i, t, ps);
    k_batch_shade<<<g.shade, kBlock, 0, q>>>(scenes[i], i, t, ps, slots);
    bv.shadow<<<g.shadow, bv.block, 0, q>>>(scenes[i], i, t, ps, capacity, slots, counters);
    k_batch_resolve<<<g.resolve, kBlock, 0, q>>>(scenes[i], i, t, ps, capacity);
  };
  cudaError_t e = cudaSuccess;
  if (lanes && nscenes > 1) {
    // The scenes' chains as parallel branches: one scene's kernels fill the
    // tails of another's instead of waiting for them.
    e = cudaEventRecord(lanes->fork, s);
    for (int i = 0; i < nscenes && e == cudaSuccess; i++) {
      e = cudaStreamWaitEvent(lanes->stream[i], lanes->fork, 0);
      if (e != cudaSuccess) break;
      chain(i, lanes->stream[i]);
      e = cudaEventRecord(lanes->join[i], lanes->stream[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, lanes->join[i], 0);
    }
  } else {
    for (int i = 0; i < nscenes; i++) chain(i, s);
  }
  if (e != cudaSuccess) return e;
  k_batch_advance<<<1, 32, 0, s>>>(t, nscenes, counters, ps.bins, graph ? 1 : 0, handle);
  return cudaGetLastError();
}

cudaError_t launch_batch_accumulate(const BatchTables* t, const PathState& ps, const BatchGrids& g, cudaStream_t s) {
  k_batch_accumulate<<<g.accumulate, 256, 0, s>>>(t, ps);
  return cudaGetLastError();
}

// The used part of the plan's current table (its fixed fields and the
// segments' frame parameters), copied word by word into the chunk's table.
__global__ void k_batch_load_chunk(const BatchPlan* plan, BatchTables* dst, cudaGraphConditionalHandle inner) {
  const int c = min(plan->index, plan->count - 1);
  const BatchTables* src = plan->tables + c;
  const size_t bytes = offsetof(BatchTables, fp) + sizeof(FrameParams) * static_cast<size_t>(src->segments);
  const int words = static_cast<int>(bytes / sizeof(int));
  const int* from = reinterpret_cast<const int*>(src);
  int* to = reinterpret_cast<int*>(dst);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) to[i] = from[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(inner, 1u);
}

__global__ void k_batch_next_chunk(BatchPlan* plan, cudaGraphConditionalHandle outer) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int next = plan->index + 1;
  plan->index = next;
  cudaGraphSetConditional(outer, next < plan->count ? 1u : 0u);
}

cudaError_t launch_batch_load_chunk(const BatchPlan* plan, BatchTables* dst, cudaGraphConditionalHandle inner,
                                    cudaStream_t s) {
  static_assert(offsetof(BatchTables, fp) % sizeof(int) == 0 && sizeof(FrameParams) % sizeof(int) == 0,
                "tables are copied in 4-byte words");
  k_batch_load_chunk<<<8, 256, 0, s>>>(plan, dst, inner);
  return cudaGetLastError();
}

cudaError_t launch_batch_next_chunk(BatchPlan* plan, cudaGraphConditionalHandle outer, cudaStream_t s) {
  k_batch_next_chunk<<<1, 32, 0, s>>>(plan, outer);
  return cudaGetLastError();
}

}  // namespace mcrt
