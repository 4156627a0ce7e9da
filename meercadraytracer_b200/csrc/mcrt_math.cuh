// Device math shared by the kernels: vectors, the reference's random number
// generator (bit-exact, integer), colour transforms, tone mapping and BRDF
// terms. Shading arithmetic is FP32; ray generation and the final 8-bit
// encode are FP64 so that they reproduce the reference's double-precision
// results exactly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define MCRT_HD __host__ __device__ __forceinline__
#define MCRT_D __device__ __forceinline__

namespace mcrt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;  // brdf.ts:6

// ------------------------------------------------------------------ vectors
struct V3 {
  float x, y, z;
};
MCRT_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
MCRT_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
MCRT_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
MCRT_HD V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
MCRT_HD V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
MCRT_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MCRT_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
MCRT_HD float length3(V3 a) { return sqrtf(dot(a, a)); }
// `v / (Math.hypot(v) || 1)`.
MCRT_HD V3 normalize_or_keep(V3 a) {
  float l = length3(a);
  if (!(l > 0.0f)) l = 1.0f;
  return a * (1.0f / l);
}
MCRT_HD float clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
MCRT_HD float luminance(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

// ------------------------------------------------------------------- random
// lowbias32 hash, src/random.ts:24-31.
MCRT_HD uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// Random.seed, src/random.ts:6-10.
MCRT_HD uint32_t rng_seed(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  uint32_t h = hash32(a ^ hash32(b ^ hash32(c ^ hash32(d))));
  return h == 0 ? 0x9e3779b9u : h;
}
// Random.next, src/random.ts:13-20: xorshift32, value state / 2^32 (exact in double).
MCRT_HD double rng_next(uint32_t& s) {
  uint32_t x = s;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  s = x;
  return static_cast<double>(x) * 2.3283064365386963e-10;
}

// ------------------------------------------------------------------- colour
// srgbToLinear / linearToSrgb, src/color.ts:11-18.
MCRT_HD float srgb_to_linear(float c) {
  return c < 0.04045f ? c * 0.0773993808f : powf(c * 0.9478672986f + 0.0521327014f, 2.4f);
}
MCRT_HD double linear_to_srgb_f64(double c) {
  return c < 0.0031308 ? c * 12.92 : 1.055 * pow(c, 0.41666) - 0.055;
}
MCRT_HD float saturate(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

// Column-major 3x3 times a vector, src/color.ts:54-59.
MCRT_HD void mul3(const float* m, float* c) {
  float x = c[0], y = c[1], z = c[2];
  c[0] = m[0] * x + m[3] * y + m[6] * z;
  c[1] = m[1] * x + m[4] * y + m[7] * z;
  c[2] = m[2] * x + m[5] * y + m[8] * z;
}

// toneMap, src/color.ts:81-136: three.js's tonemapping_pars_fragment operators.
// The matrices are three.js's GLSL mat3 constants (columns listed in order).
MCRT_HD void tone_map(float* c, int mapping, float exposure) {
  switch (mapping) {
    case 1:  // Linear
      for (int i = 0; i < 3; i++) c[i] = saturate(exposure * c[i]);
      return;
    case 2:  // Reinhard
      for (int i = 0; i < 3; i++) {
        float v = exposure * c[i];
        c[i] = saturate(v / (1.0f + v));
      }
      return;
    case 3:  // Cineon
      for (int i = 0; i < 3; i++) {
        float v = fmaxf(0.0f, exposure * c[i] - 0.004f);
        c[i] = powf((v * (6.2f * v + 0.5f)) / (v * (6.2f * v + 1.7f) + 0.06f), 2.2f);
      }
      return;
    case 4: {  // ACES filmic
      const float in_m[9] = {0.59719f, 0.076f, 0.0284f, 0.35458f, 0.90834f, 0.13383f, 0.04823f, 0.01566f, 0.83777f};
      const float out_m[9] = {1.60475f, -0.10208f, -0.00327f, -0.53108f, 1.10813f,
                              -0.07276f, -0.07367f, -0.00605f, 1.07602f};
      for (int i = 0; i < 3; i++) c[i] = (c[i] * exposure) / 0.6f;
      mul3(in_m, c);
      for (int i = 0; i < 3; i++) {
        float v = c[i];
        float a = v * (v + 0.0245786f) - 0.000090537f;
        float b = v * (0.983729f * v + 0.432951f) + 0.238081f;
        c[i] = a / b;
      }
      mul3(out_m, c);
      for (int i = 0; i < 3; i++) c[i] = saturate(c[i]);
      return;
    }
    case 6: {  // AgX
      const float to2020[9] = {0.6274f, 0.0691f, 0.0164f, 0.3293f, 0.9195f, 0.088f, 0.0433f, 0.0113f, 0.8956f};
      const float from2020[9] = {1.6605f, -0.1246f, -0.0182f, -0.5876f, 1.1329f, -0.1006f, -0.0728f, -0.0083f, 1.1187f};
      const float inset[9] = {0.856627153315983f, 0.137318972929847f, 0.11189821299995f,
                              0.0951212405381588f, 0.761241990602591f, 0.0767994186031903f,
                              0.0482516061458583f, 0.101439036467562f, 0.811302368396859f};
      const float outset[9] = {1.1271005818144368f, -0.1413297634984383f, -0.14132976349843826f,
                               -0.11060664309660323f, 1.157823702216272f, -0.11060664309660294f,
                               -0.016493938717834573f, -0.016493938717834257f, 1.2519364065950405f};
      const float min_ev = -12.47393f, max_ev = 4.026069f;
      for (int i = 0; i < 3; i++) c[i] = c[i] * exposure;
      mul3(to2020, c);
      mul3(inset, c);
      for (int i = 0; i < 3; i++) {
        float v = saturate((log2f(fmaxf(c[i], 1e-10f)) - min_ev) / (max_ev - min_ev));
        float x2 = v * v, x4 = x2 * x2;
        c[i] = 15.5f * x4 * x2 - 40.14f * x4 * v + 31.96f * x4 - 6.868f * x2 * v + 0.4298f * x2 + 0.1191f * v -
               0.00232f;
      }
      mul3(outset, c);
      for (int i = 0; i < 3; i++) c[i] = powf(fmaxf(0.0f, c[i]), 2.2f);
      mul3(from2020, c);
      for (int i = 0; i < 3; i++) c[i] = saturate(c[i]);
      return;
    }
    case 7: {  // Neutral
      const float start = 0.8f - 0.04f, desaturation = 0.15f;
      for (int i = 0; i < 3; i++) c[i] = c[i] * exposure;
      float x = fminf(c[0], fminf(c[1], c[2]));
      float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
      for (int i = 0; i < 3; i++) c[i] = c[i] - offset;
      float peak = fmaxf(c[0], fmaxf(c[1], c[2]));
      if (peak < start) return;
      float d = 1.0f - start;
      float new_peak = 1.0f - (d * d) / (peak + d - start);
      float g = 1.0f - 1.0f / (desaturation * (peak - new_peak) + 1.0f);
      for (int i = 0; i < 3; i++) c[i] = (c[i] * new_peak) / peak * (1.0f - g) + new_peak * g;
      return;
    }
    default:
      return;
  }
}

// ToUint8Clamp of `v * 255 + 0.5` computed as JavaScript does, in double and
// without a fused multiply-add: clamp to 0..255, NaN to 0, round half to even.
MCRT_HD uint8_t encode_byte(double v) {
#ifdef __CUDA_ARCH__
  double x = __dadd_rn(__dmul_rn(v, 255.0), 0.5);
#else
  volatile double prod = v * 255.0;
  double x = prod + 0.5;
#endif
  if (!(x > 0.0)) return 0;
  if (x >= 255.0) return 255;
  double f = floor(x);
  if (f + 0.5 < x) return static_cast<uint8_t>(f + 1.0);
  if (x < f + 0.5) return static_cast<uint8_t>(f);
  int fi = static_cast<int>(f);
  return static_cast<uint8_t>((fi & 1) ? fi + 1 : fi);
}

// -------------------------------------------------------------------- BRDF
// fresnelWeight, visibilityGgx, distributionGgx, blinnPhong, smoothstep and
// distanceAttenuation, src/brdf.ts:33-72 (three.js's shader chunk formulas).
MCRT_HD float fresnel_weight(float vh) { return exp2f((-5.55473f * vh - 6.98316f) * vh); }
MCRT_HD float visibility_ggx(float alpha, float nl, float nv) {
  float a2 = alpha * alpha;
  float gv = nl * sqrtf(a2 + (1.0f - a2) * nv * nv);
  float gl = nv * sqrtf(a2 + (1.0f - a2) * nl * nl);
  return 0.5f / fmaxf(gv + gl, 1e-6f);
}
MCRT_HD float distribution_ggx(float alpha, float nh) {
  float a2 = alpha * alpha;
  float denom = nh * nh * (a2 - 1.0f) + 1.0f;
  return (kInvPi * a2) / (denom * denom);
}
MCRT_HD float blinn_phong(float shininess, float nh) {
  return 0.25f * kInvPi * (shininess * 0.5f + 1.0f) * powf(nh, shininess);
}
MCRT_HD float smoothstep(float e0, float e1, float x) {
  if (e0 == e1) return x < e0 ? 0.0f : 1.0f;
  float t = fminf(fmaxf((x - e0) / (e1 - e0), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
MCRT_HD float distance_attenuation(float distance, float cutoff, float decay) {
  float falloff = 1.0f / fmaxf(powf(distance, decay), 0.01f);
  if (cutoff > 0.0f) {
    float r = fminf(fmaxf(1.0f - powf(distance / cutoff, 4.0f), 0.0f), 1.0f);
    falloff *= r * r;
  }
  return falloff;
}
// Multiple-scattering energy, tracer.ts:699-702.
MCRT_HD float multi_scatter(float fss_ess, float f0, float ems) {
  float f_avg = f0 + (1.0f - f0) * 0.047619f;
  return ((fss_ess * f_avg) / (1.0f - ems * f_avg)) * ems;
}

// Orthonormal basis about a normal (Duff et al. 2017), tracer.ts:636-646.
MCRT_HD V3 to_world(V3 n, float a, float b, float c) {
  float sign = n.z >= 0.0f ? 1.0f : -1.0f;
  float e = -1.0f / (sign + n.z);
  float f = n.x * n.y * e;
  V3 t = {1.0f + sign * n.x * n.x * e, sign * f, -sign * n.x};
  V3 bt = {f, sign + n.y * n.y * e, -n.y};
  return {t.x * a + bt.x * b + n.x * c, t.y * a + bt.y * b + n.y * c, t.z * a + bt.z * b + n.z * c};
}

}  // namespace mcrt
