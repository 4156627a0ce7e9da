// Device-resident scene: the layout of a compiled scene in HBM.
//
//  nodes   64 B per inner BVH node: both children's boxes and references, so
//          one inner-node visit is one aligned 64 B fetch (4 x 128-bit loads).
//  tris    48 B per triangle: the three vertices (for the watertight test)
//          plus flags / culled side and the material index in the w lanes.
//  attrs   64 B per triangle: vertex normals and uvs, read once per hit.
//  tangents, colors: per triangle, only where a normal map / vertex colours
//          are used.
// Materials, lights, environments and texture descriptors are small arrays
// read through the read-only data cache; each texture's texels live in their
// own buffer. The DFG table is a CUDA texture object.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mcrt_math.cuh"

namespace mcrt {

constexpr int kMaxDepth = 100;       // bvh.ts:5: no leaf deeper than this
constexpr int kStackMax = kMaxDepth + 4;
constexpr int kMaxPassThrough = 64;  // tracer.ts:30
constexpr int kMaxLights = 63;       // shadow slots: one per light plus the environment estimate

// Child reference of an inner node: count == 0 -> inner node index in `ref`;
// count > 0 -> leaf covering triangles [ref, ref + count); count < 0 -> absent.
struct alignas(16) DNode {
  float4 lxy;   // left  min.x, max.x, min.y, max.y
  float4 rxy;   // right min.x, max.x, min.y, max.y
  float4 lrz;   // left  min.z, max.z, right min.z, max.z
  int4 kids;    // left ref, right ref, left count, right count
};

struct alignas(16) DMaterial {
  int model, side, transparent, vertex_colors;
  int flat_shading, tone_mapped, physical, combine;
  int map, alpha_map, emissive_map, normal_map;
  int ao_map, roughness_map, metalness_map, env_map;
  float color[3], opacity;
  float emissive[3], alpha_test;
  float normal_scale[2], ao_map_intensity, roughness;
  float metalness, ior, specular_intensity, transmission;
  float specular_color[3], thickness;
  float attenuation[3], shininess;
  float specular[3], env_map_intensity;
  float reflectivity, pad_[3];
};

struct alignas(16) DLight {
  int type, cast_shadow, pad_[2];
  float color[3], distance;
  float ground[3], decay;
  float direction[3], cone_cos;
  float position[3], penumbra_cos;
};

struct alignas(16) DTexture {
  const uint8_t* data;  // RGBA texels, first row first (uint8 or float32)
  int width, height, format, srgb;
  int flip_y, wrap_s, wrap_t, pad_;
  float matrix[9], pad2_[3];
};

struct alignas(16) DEnvironment {
  int kind, texture, flip_x, pad_;
  int faces[6], pad2_[2];
  float rotation[9], intensity;
};

struct DBackground {
  int kind, texture, environment, pad_;
  float color[3], intensity;
};

struct DFog {
  int kind, pad_[3];
  float color[3], near_;
  float far_, density, pad2_[2];
};

struct DScene {
  const DNode* nodes;
  const float4* tris;
  const float4* attrs;
  const float4* tangents;
  const float4* colors;  // 3 per triangle, or null
  int tri_count;
  int root_count;        // > 0: the root is a leaf of this many triangles (from 0); 0: node 0 is inner
  float eps;             // CompiledGeometry.epsilon
  int node_count;
  const DMaterial* materials;
  const DLight* lights;
  const DEnvironment* envs;
  const DTexture* textures;
  const float* srgb_lut;     // SRGB_TO_LINEAR_8BIT, 256 floats
  cudaTextureObject_t dfg;   // 512 floats: (scale, bias) per texel
  int light_count;
  int environment;           // scene.environment, or -1
  int step_limit;            // > 0: node visits plus leaves one query may take (a test hook)
  DBackground background;
  DFog fog;
};

// Per-triangle packed word in tris[3k].w: flags (bits 0-7), culled side (bits 8-15).
MCRT_D int tri_flags(float w) { return __float_as_int(w) & 0xff; }
MCRT_D int tri_side(float w) { return (__float_as_int(w) >> 8) & 0xff; }

// ----------------------------------------------------------------- textures
// wrap, src/textures.ts:229-236.
MCRT_D float wrap_coord(float c, int mode) {
  if (mode == 1001) return c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
  if (mode == 1002) {
    float period = c - 2.0f * floorf(c / 2.0f);
    return period > 1.0f ? 2.0f - period : period;
  }
  return c - floorf(c);
}

// texelIndex, src/textures.ts:238-241.
MCRT_D int texel_index(int i, int size, int mode) {
  if (mode == 1001 || mode == 1002) return i < 0 ? 0 : (i >= size ? size - 1 : i);
  int r = i % size;
  return r < 0 ? r + size : r;
}

// sampleTexel, src/textures.ts:255-281: bilinear at s * w - 0.5, 8-bit sRGB
// decoded per texel before blending.
MCRT_D float4 sample_texel(const DScene& sc, const DTexture& t, float s, float tt) {
  const int w = t.width, h = t.height;
  float row = t.flip_y ? 1.0f - tt : tt;
  float x = s * w - 0.5f, y = row * h - 0.5f;
  float x0 = floorf(x), y0 = floorf(y);
  float fx = x - x0, fy = y - y0;
  int ix = static_cast<int>(x0), iy = static_cast<int>(y0);
  int xa = texel_index(ix, w, t.wrap_s), xb = texel_index(ix + 1, w, t.wrap_s);
  int ya = texel_index(iy, h, t.wrap_t), yb = texel_index(iy + 1, h, t.wrap_t);
  float w00 = (1.0f - fx) * (1.0f - fy), w10 = fx * (1.0f - fy), w01 = (1.0f - fx) * fy, w11 = fx * fy;
  size_t i00 = static_cast<size_t>(ya) * w + xa, i10 = static_cast<size_t>(ya) * w + xb;
  size_t i01 = static_cast<size_t>(yb) * w + xa, i11 = static_cast<size_t>(yb) * w + xb;
  if (t.format == 1) {
    const float4* d = reinterpret_cast<const float4*>(t.data);
    float4 a = __ldg(d + i00), b = __ldg(d + i10), c = __ldg(d + i01), e = __ldg(d + i11);
    return make_float4(a.x * w00 + b.x * w10 + c.x * w01 + e.x * w11, a.y * w00 + b.y * w10 + c.y * w01 + e.y * w11,
                       a.z * w00 + b.z * w10 + c.z * w01 + e.z * w11, a.w * w00 + b.w * w10 + c.w * w01 + e.w * w11);
  }
  const uchar4* d = reinterpret_cast<const uchar4*>(t.data);
  uchar4 a = __ldg(d + i00), b = __ldg(d + i10), c = __ldg(d + i01), e = __ldg(d + i11);
  float4 out;
  if (t.srgb) {
    const float* lut = sc.srgb_lut;
    out.x = __ldg(lut + a.x) * w00 + __ldg(lut + b.x) * w10 + __ldg(lut + c.x) * w01 + __ldg(lut + e.x) * w11;
    out.y = __ldg(lut + a.y) * w00 + __ldg(lut + b.y) * w10 + __ldg(lut + c.y) * w01 + __ldg(lut + e.y) * w11;
    out.z = __ldg(lut + a.z) * w00 + __ldg(lut + b.z) * w10 + __ldg(lut + c.z) * w01 + __ldg(lut + e.z) * w11;
  } else {
    out.x = (a.x * w00 + b.x * w10 + c.x * w01 + e.x * w11) / 255.0f;
    out.y = (a.y * w00 + b.y * w10 + c.y * w01 + e.y * w11) / 255.0f;
    out.z = (a.z * w00 + b.z * w10 + c.z * w01 + e.z * w11) / 255.0f;
  }
  out.w = (a.w * w00 + b.w * w10 + c.w * w01 + e.w * w11) / 255.0f;
  return out;
}

// sampleTexture, src/textures.ts:247-252: uv transform, wrap, sample.
MCRT_D float4 sample_texture(const DScene& sc, int index, float u, float v) {
  const DTexture& t = sc.textures[index];
  float tu = t.matrix[0] * u + t.matrix[3] * v + t.matrix[6];
  float tv = t.matrix[1] * u + t.matrix[4] * v + t.matrix[7];
  return sample_texel(sc, t, wrap_coord(tu, t.wrap_s), wrap_coord(tv, t.wrap_t));
}

// sampleEnvironment, src/textures.ts:287-317: equirectangular or cube lookup.
MCRT_D V3 sample_environment(const DScene& sc, int index, V3 d) {
  const DEnvironment& e = sc.envs[index];
  const float* r = e.rotation;
  float x = r[0] * d.x + r[3] * d.y + r[6] * d.z;
  float y = r[1] * d.x + r[4] * d.y + r[7] * d.z;
  float z = r[2] * d.x + r[5] * d.y + r[8] * d.z;
  float4 t;
  if (e.kind == 1) {
    float l = sqrtf(x * x + y * y + z * z);
    if (!(l > 0.0f)) l = 1.0f;
    float u = atan2f(z, x) / (2.0f * kPi) + 0.5f;
    float v = asinf(fmaxf(-1.0f, fminf(1.0f, y / l))) / kPi + 0.5f;
    const DTexture& tex = sc.textures[e.texture];
    t = sample_texel(sc, tex, wrap_coord(u, tex.wrap_s), fmaxf(0.0f, fminf(1.0f, v)));
  } else {
    if (e.flip_x) x = -x;
    float ax = fabsf(x), ay = fabsf(y), az = fabsf(z);
    int face;
    float sc_, tc, ma;
    if (ax >= ay && ax >= az) {
      face = x > 0.0f ? 0 : 1; ma = ax; sc_ = x > 0.0f ? -z : z; tc = -y;
    } else if (ay >= az) {
      face = y > 0.0f ? 2 : 3; ma = ay; sc_ = x; tc = y > 0.0f ? z : -z;
    } else {
      face = z > 0.0f ? 4 : 5; ma = az; sc_ = z > 0.0f ? x : -x; tc = -y;
    }
    float s = (sc_ / ma + 1.0f) * 0.5f, tt = (tc / ma + 1.0f) * 0.5f;
    t = sample_texel(sc, sc.textures[e.faces[face]], fmaxf(0.0f, fminf(1.0f, s)), fmaxf(0.0f, fminf(1.0f, tt)));
  }
  return V3{t.x * e.intensity, t.y * e.intensity, t.z * e.intensity};
}

// dfg, src/brdf.ts:18-30: bilinear lookup of three.js's DFG table, by hand
// (hardware filtering has 8-bit weights) from the texture object.
MCRT_D void dfg_lookup(const DScene& sc, float roughness, float dot_nv, float& fa, float& fb) {
  const int n = 16;
  float x = fminf(fmaxf(roughness * n - 0.5f, 0.0f), static_cast<float>(n - 1));
  float y = fminf(fmaxf(dot_nv * n - 0.5f, 0.0f), static_cast<float>(n - 1));
  float x0f = floorf(x), y0f = floorf(y);
  int x0 = static_cast<int>(x0f), y0 = static_cast<int>(y0f);
  int x1 = min(x0 + 1, n - 1), y1 = min(y0 + 1, n - 1);
  float fx = x - x0f, fy = y - y0f;
  float r[2];
  for (int c = 0; c < 2; c++) {
    float a = tex1Dfetch<float>(sc.dfg, (y0 * n + x0) * 2 + c), b = tex1Dfetch<float>(sc.dfg, (y0 * n + x1) * 2 + c);
    float d = tex1Dfetch<float>(sc.dfg, (y1 * n + x0) * 2 + c), e = tex1Dfetch<float>(sc.dfg, (y1 * n + x1) * 2 + c);
    r[c] = (a * (1.0f - fx) + b * fx) * (1.0f - fy) + (d * (1.0f - fx) + e * fx) * fy;
  }
  fa = r[0];
  fb = r[1];
}

}  // namespace mcrt
