// CPU oracle for the ray tracer's hot path. TEST INFRASTRUCTURE ONLY: the
// product never links or calls this file; tests, the smoke check and the
// benchmark's CPU-baseline leg use it as the checker.
//
// A restatement, in C++ with JavaScript numeric semantics, of the reference
// (VJigouline/MeerCADRaytracer): doubles everywhere, float rounding exactly
// where the reference stores into a Float32Array, uint32 hashing, and
// Uint8ClampedArray conversion. Each function names the reference lines it
// follows. Build with -ffp-contract=off so that no multiply-add is fused,
// as JavaScript never fuses them.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../meercadraytracer_b200/csrc/dfg_lut.h"

namespace {

const double kInf = std::numeric_limits<double>::infinity();
const double kPi = 3.141592653589793;
const double kInvPi = 1.0 / kPi;  // brdf.ts:6

inline float fround(double x) { return static_cast<float>(x); }

// Math.hypot as V8 computes it: scaled by the largest magnitude and summed
// with Kahan compensation.
double js_hypot(double a, double b, double c) {
  double x[3] = {std::fabs(a), std::fabs(b), std::fabs(c)};
  double mx = 0;
  for (double v : x) {
    if (std::isinf(v)) return kInf;
  }
  for (double v : x) {
    if (std::isnan(v)) return std::numeric_limits<double>::quiet_NaN();
    if (v > mx) mx = v;
  }
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (double v : x) {
    double n = v / mx;
    double summand = n * n - comp;
    double prelim = sum + summand;
    comp = (prelim - sum) - summand;
    sum = prelim;
  }
  return std::sqrt(sum) * mx;
}

// `Math.hypot(...) || 1`.
inline double hypot_or_one(double a, double b, double c) {
  double h = js_hypot(a, b, c);
  return (h == 0 || std::isnan(h)) ? 1.0 : h;
}

inline double clamp01(double x) { return std::min(std::max(x, 0.0), 1.0); }

// ---------------------------------------------------------------- random.ts

// hash, src/random.ts:24-31 (lowbias32).
uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

struct Random {
  uint32_t state = 1;
  // Random.seed, src/random.ts:6-10.
  void seed(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    uint32_t h = hash32(a ^ hash32(b ^ hash32(c ^ hash32(d))));
    if (h == 0) h = 0x9e3779b9u;
    state = h;
  }
  // Random.next, src/random.ts:13-20 (xorshift32).
  double next() {
    uint32_t x = state;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    state = x;
    return static_cast<double>(state) / 4294967296.0;
  }
};

// A mistake planted in the path loop's use of random numbers, for tests that
// show a comparison would catch a reordered, extra or missing draw. 0 (the
// default) is the reference's order. Set only by oracle_plant_draw_mistake.
//   1  the transparency test (tracer.ts:170) draws twice
//   2  the GI-off environment estimate's cosine draws (tracer.ts:343-344,
//      601) are taken in swapped order
//   3  the continuation pick (tracer.ts:420) draws twice
//   4  the diffuse continuation's cosine draws (tracer.ts:455, 601) swapped
//   5  the GGX half-vector draws (tracer.ts:610-612) swapped
//   6  Russian roulette (tracer.ts:465-467) draws from bounce 2 on, not 3
int g_planted_draw_mistake = 0;

// ----------------------------------------------------------------- color.ts

double srgb_to_linear(double c) {  // color.ts:11-13
  return c < 0.04045 ? c * 0.0773993808 : std::pow(c * 0.9478672986 + 0.0521327014, 2.4);
}

double linear_to_srgb(double c) {  // color.ts:16-18
  return c < 0.0031308 ? c * 12.92 : 1.055 * std::pow(c, 0.41666) - 0.055;
}

double half_to_float(uint32_t h) {  // color.ts:28-35
  double sign = (h & 0x8000) ? -1.0 : 1.0;
  int exponent = (h >> 10) & 0x1f;
  int fraction = h & 0x3ff;
  if (exponent == 0) return sign * std::pow(2.0, -14) * (fraction / 1024.0);
  if (exponent == 31) return fraction ? std::numeric_limits<double>::quiet_NaN() : sign * kInf;
  return sign * std::pow(2.0, exponent - 15) * (1 + fraction / 1024.0);
}

// SRGB_TO_LINEAR_8BIT, color.ts:21-25: a Float32Array of the 256 levels.
struct SrgbTable {
  float v[256];
  SrgbTable() {
    for (int i = 0; i < 256; i++) v[i] = fround(srgb_to_linear(i / 255.0));
  }
};
const SrgbTable kSrgb;

double saturate(double x) { return x < 0 ? 0 : x > 1 ? 1 : x; }  // color.ts:37-39

double rrt_and_odt_fit(double v) {  // color.ts:41-45
  double a = v * (v + 0.0245786) - 0.000090537;
  double b = v * (0.983729 * v + 0.432951) + 0.238081;
  return a / b;
}

double agx_contrast(double x) {  // color.ts:47-51
  double x2 = x * x;
  double x4 = x2 * x2;
  return 15.5 * x4 * x2 - 40.14 * x4 * x + 31.96 * x4 - 6.868 * x2 * x + 0.4298 * x2 + 0.1191 * x -
         0.00232;
}

void mul3(const double* m, double* c) {  // color.ts:54-59, column-major
  double x = c[0], y = c[1], z = c[2];
  c[0] = m[0] * x + m[3] * y + m[6] * z;
  c[1] = m[1] * x + m[4] * y + m[7] * z;
  c[2] = m[2] * x + m[5] * y + m[8] * z;
}

// three.js tone mapping matrices (GLSL mat3 columns), color.ts:62-75.
const double kAcesIn[9] = {0.59719, 0.076, 0.0284, 0.35458, 0.90834, 0.13383, 0.04823, 0.01566, 0.83777};
const double kAcesOut[9] = {1.60475, -0.10208, -0.00327, -0.53108, 1.10813, -0.07276, -0.07367, -0.00605, 1.07602};
const double kSrgbToRec2020[9] = {0.6274, 0.0691, 0.0164, 0.3293, 0.9195, 0.088, 0.0433, 0.0113, 0.8956};
const double kRec2020ToSrgb[9] = {1.6605, -0.1246, -0.0182, -0.5876, 1.1329, -0.1006, -0.0728, -0.0083, 1.1187};
const double kAgxInset[9] = {0.856627153315983, 0.137318972929847, 0.11189821299995,
                             0.0951212405381588, 0.761241990602591, 0.0767994186031903,
                             0.0482516061458583, 0.101439036467562, 0.811302368396859};
const double kAgxOutset[9] = {1.1271005818144368, -0.1413297634984383, -0.14132976349843826,
                              -0.11060664309660323, 1.157823702216272, -0.11060664309660294,
                              -0.016493938717834573, -0.016493938717834257, 1.2519364065950405};
const double kAgxMinEv = -12.47393;
const double kAgxMaxEv = 4.026069;

// toneMap, color.ts:81-136.
void tone_map(double* c, int mapping, double exposure) {
  switch (mapping) {
    case MCRT_LINEAR_TONE_MAPPING:
      for (int i = 0; i < 3; i++) c[i] = saturate(exposure * c[i]);
      return;
    case MCRT_REINHARD_TONE_MAPPING:
      for (int i = 0; i < 3; i++) {
        double v = exposure * c[i];
        c[i] = saturate(v / (1 + v));
      }
      return;
    case MCRT_CINEON_TONE_MAPPING:
      for (int i = 0; i < 3; i++) {
        double v = std::max(0.0, exposure * c[i] - 0.004);
        c[i] = std::pow((v * (6.2 * v + 0.5)) / (v * (6.2 * v + 1.7) + 0.06), 2.2);
      }
      return;
    case MCRT_ACES_FILMIC_TONE_MAPPING:
      for (int i = 0; i < 3; i++) c[i] = (c[i] * exposure) / 0.6;
      mul3(kAcesIn, c);
      for (int i = 0; i < 3; i++) c[i] = rrt_and_odt_fit(c[i]);
      mul3(kAcesOut, c);
      for (int i = 0; i < 3; i++) c[i] = saturate(c[i]);
      return;
    case MCRT_AGX_TONE_MAPPING:
      for (int i = 0; i < 3; i++) c[i] = c[i] * exposure;
      mul3(kSrgbToRec2020, c);
      mul3(kAgxInset, c);
      for (int i = 0; i < 3; i++) {
        double v = (std::log2(std::max(c[i], 1e-10)) - kAgxMinEv) / (kAgxMaxEv - kAgxMinEv);
        c[i] = agx_contrast(saturate(v));
      }
      mul3(kAgxOutset, c);
      for (int i = 0; i < 3; i++) c[i] = std::pow(std::max(0.0, c[i]), 2.2);
      mul3(kRec2020ToSrgb, c);
      for (int i = 0; i < 3; i++) c[i] = saturate(c[i]);
      return;
    case MCRT_NEUTRAL_TONE_MAPPING: {
      const double start = 0.8 - 0.04;
      const double desaturation = 0.15;
      for (int i = 0; i < 3; i++) c[i] = c[i] * exposure;
      double x = std::min(c[0], std::min(c[1], c[2]));
      double offset = x < 0.08 ? x - 6.25 * x * x : 0.04;
      for (int i = 0; i < 3; i++) c[i] = c[i] - offset;
      double peak = std::max(c[0], std::max(c[1], c[2]));
      if (peak < start) return;
      double d = 1 - start;
      double new_peak = 1 - (d * d) / (peak + d - start);
      double g = 1 - 1 / (desaturation * (peak - new_peak) + 1);
      for (int i = 0; i < 3; i++) c[i] = (c[i] * new_peak) / peak * (1 - g) + new_peak * g;
      return;
    }
    default:
      return;
  }
}

// ToUint8Clamp, the conversion a store into a Uint8ClampedArray makes:
// NaN to 0, clamp to 0..255, round half to even.
uint8_t uint8_clamp(double v) {
  if (!(v > 0)) return 0;
  if (v >= 255) return 255;
  double f = std::floor(v);
  if (f + 0.5 < v) return static_cast<uint8_t>(f + 1);
  if (v < f + 0.5) return static_cast<uint8_t>(f);
  int fi = static_cast<int>(f);
  return static_cast<uint8_t>((fi & 1) ? fi + 1 : fi);
}

// ------------------------------------------------------------------ brdf.ts

// DFG table decoded into a Float32Array, brdf.ts:8-12.
struct DfgTable {
  float v[512];
  DfgTable() {
    for (int i = 0; i < 512; i++) v[i] = fround(half_to_float(MCRT_DFG_LUT_HALF[i]));
  }
};
const DfgTable kDfg;

void dfg(double roughness, double dot_nv, double* out) {  // brdf.ts:18-30
  const int n = MCRT_DFG_LUT_SIZE;
  double x = std::min(std::max(roughness * n - 0.5, 0.0), static_cast<double>(n - 1));
  double y = std::min(std::max(dot_nv * n - 0.5, 0.0), static_cast<double>(n - 1));
  int x0 = static_cast<int>(std::floor(x)), y0 = static_cast<int>(std::floor(y));
  int x1 = std::min(x0 + 1, n - 1), y1 = std::min(y0 + 1, n - 1);
  double fx = x - x0, fy = y - y0;
  for (int c = 0; c < 2; c++) {
    double a = kDfg.v[(y0 * n + x0) * 2 + c], b = kDfg.v[(y0 * n + x1) * 2 + c];
    double d = kDfg.v[(y1 * n + x0) * 2 + c], e = kDfg.v[(y1 * n + x1) * 2 + c];
    out[c] = (a * (1 - fx) + b * fx) * (1 - fy) + (d * (1 - fx) + e * fx) * fy;
  }
}

double fresnel_weight(double dot_vh) {  // brdf.ts:33-35
  return std::pow(2.0, (-5.55473 * dot_vh - 6.98316) * dot_vh);
}

double visibility_ggx(double alpha, double dot_nl, double dot_nv) {  // brdf.ts:38-43
  double a2 = alpha * alpha;
  double gv = dot_nl * std::sqrt(a2 + (1 - a2) * dot_nv * dot_nv);
  double gl = dot_nv * std::sqrt(a2 + (1 - a2) * dot_nl * dot_nl);
  return 0.5 / std::max(gv + gl, 1e-6);
}

double distribution_ggx(double alpha, double dot_nh) {  // brdf.ts:46-50
  double a2 = alpha * alpha;
  double denom = dot_nh * dot_nh * (a2 - 1) + 1;
  return (kInvPi * a2) / (denom * denom);
}

double blinn_phong(double shininess, double dot_nh) {  // brdf.ts:53-55
  return 0.25 * kInvPi * (shininess * 0.5 + 1) * std::pow(dot_nh, shininess);
}

double smoothstep(double e0, double e1, double x) {  // brdf.ts:58-62
  if (e0 == e1) return x < e0 ? 0 : 1;
  double t = std::min(std::max((x - e0) / (e1 - e0), 0.0), 1.0);
  return t * t * (3 - 2 * t);
}

double distance_attenuation(double distance, double cutoff, double decay) {  // brdf.ts:65-72
  double falloff = 1 / std::max(std::pow(distance, decay), 0.01);
  if (cutoff > 0) {
    double r = std::min(std::max(1 - std::pow(distance / cutoff, 4.0), 0.0), 1.0);
    falloff *= r * r;
  }
  return falloff;
}

// -------------------------------------------------------------- textures.ts

double wrap(double coordinate, int mode) {  // textures.ts:229-236
  if (mode == MCRT_CLAMP_TO_EDGE_WRAPPING) return coordinate < 0 ? 0 : coordinate > 1 ? 1 : coordinate;
  if (mode == MCRT_MIRRORED_REPEAT_WRAPPING) {
    double period = coordinate - 2 * std::floor(coordinate / 2);
    return period > 1 ? 2 - period : period;
  }
  return coordinate - std::floor(coordinate);
}

// texelIndex, textures.ts:238-241. `i` is an integer-valued double.
int64_t texel_index(double i, int size, int mode) {
  if (mode == MCRT_CLAMP_TO_EDGE_WRAPPING || mode == MCRT_MIRRORED_REPEAT_WRAPPING) {
    return i < 0 ? 0 : i >= size ? size - 1 : static_cast<int64_t>(i);
  }
  // ((i % size) + size) % size with JavaScript's sign-of-dividend remainder.
  double r = std::fmod(i, static_cast<double>(size));
  r = std::fmod(r + size, static_cast<double>(size));
  return static_cast<int64_t>(r);
}

// sampleTexel, textures.ts:255-281.
void sample_texel(const mcrt_texture& tex, double s, double t, double* out) {
  int w = tex.width, h = tex.height;
  double row = tex.flip_y ? 1 - t : t;
  double x = s * w - 0.5, y = row * h - 0.5;
  double x0 = std::floor(x), y0 = std::floor(y);
  double fx = x - x0, fy = y - y0;
  int64_t xa = texel_index(x0, w, tex.wrap_s), xb = texel_index(x0 + 1, w, tex.wrap_s);
  int64_t ya = texel_index(y0, h, tex.wrap_t), yb = texel_index(y0 + 1, h, tex.wrap_t);
  int64_t i00 = (ya * w + xa) * 4, i10 = (ya * w + xb) * 4, i01 = (yb * w + xa) * 4, i11 = (yb * w + xb) * 4;
  double w00 = (1 - fx) * (1 - fy), w10 = fx * (1 - fy), w01 = (1 - fx) * fy, w11 = fx * fy;
  if (tex.format == MCRT_TEXEL_RGBA32F) {
    const float* d = static_cast<const float*>(tex.data);
    for (int c = 0; c < 4; c++) {
      out[c] = d[i00 + c] * w00 + d[i10 + c] * w10 + d[i01 + c] * w01 + d[i11 + c] * w11;
    }
    return;
  }
  const uint8_t* d = static_cast<const uint8_t*>(tex.data);
  for (int c = 0; c < 4; c++) {
    if (tex.srgb && c < 3) {
      out[c] = static_cast<double>(kSrgb.v[d[i00 + c]]) * w00 + static_cast<double>(kSrgb.v[d[i10 + c]]) * w10 +
               static_cast<double>(kSrgb.v[d[i01 + c]]) * w01 + static_cast<double>(kSrgb.v[d[i11 + c]]) * w11;
    } else {
      out[c] = (d[i00 + c] * w00 + d[i10 + c] * w10 + d[i01 + c] * w01 + d[i11 + c] * w11) / 255;
    }
  }
}

// sampleTexture, textures.ts:247-252.
void sample_texture(const mcrt_texture& tex, double u, double v, double* out) {
  const double* m = tex.matrix;
  double tu = m[0] * u + m[3] * v + m[6];
  double tv = m[1] * u + m[4] * v + m[7];
  sample_texel(tex, wrap(tu, tex.wrap_s), wrap(tv, tex.wrap_t), out);
}

// sampleEnvironment, textures.ts:287-317.
void sample_environment(const mcrt_environment& env, const mcrt_texture* textures, double dx,
                        double dy, double dz, double* out) {
  const double* r = env.rotation;
  double x = r[0] * dx + r[3] * dy + r[6] * dz;
  double y = r[1] * dx + r[4] * dy + r[7] * dz;
  double z = r[2] * dx + r[5] * dy + r[8] * dz;
  double texel[4];
  if (env.kind == MCRT_ENV_EQUIRECT) {
    double length = hypot_or_one(x, y, z);
    double u = std::atan2(z, x) / (2 * kPi) + 0.5;
    double v = std::asin(std::max(-1.0, std::min(1.0, y / length))) / kPi + 0.5;
    const mcrt_texture& tex = textures[env.texture];
    sample_texel(tex, wrap(u, tex.wrap_s), std::max(0.0, std::min(1.0, v)), texel);
  } else {
    if (env.flip_x) x = -x;
    double ax = std::fabs(x), ay = std::fabs(y), az = std::fabs(z);
    int face;
    double sc, tc, ma;
    if (ax >= ay && ax >= az) {
      face = x > 0 ? 0 : 1;
      ma = ax;
      sc = x > 0 ? -z : z;
      tc = -y;
    } else if (ay >= az) {
      face = y > 0 ? 2 : 3;
      ma = ay;
      sc = x;
      tc = y > 0 ? z : -z;
    } else {
      face = z > 0 ? 4 : 5;
      ma = az;
      sc = z > 0 ? x : -x;
      tc = -y;
    }
    double s = (sc / ma + 1) * 0.5, t = (tc / ma + 1) * 0.5;
    sample_texel(textures[env.faces[face]], std::max(0.0, std::min(1.0, s)), std::max(0.0, std::min(1.0, t)),
                 texel);
  }
  out[0] = texel[0] * env.intensity;
  out[1] = texel[1] * env.intensity;
  out[2] = texel[2] * env.intensity;
}

// ------------------------------------------------------------------- bvh.ts

const int kBins = 16;      // bvh.ts:3 (BINS); build_bvh takes the count as a parameter
const int kMaxBins = 64;
const int kMaxLeaf = 4;    // bvh.ts:4
const int kMaxDepth = 100; // bvh.ts:5

double area(double x0, double y0, double z0, double x1, double y1, double z1) {  // bvh.ts:180-183
  double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
  return dx * dy + dy * dz + dz * dx;
}

// buildBvh, bvh.ts:16-178, with BINS (bvh.ts:3) as the parameter `bins`: the
// reference's builder is written in terms of that one constant, so a build
// with another bin count is the same algorithm. Returns nodeCount.
int32_t build_bvh(const float* tris, int32_t count, float* bounds, int32_t* nodes, uint32_t* order,
                  int bins = kBins) {
  if (count == 0) return 0;
  if (bins < 2) bins = 2;
  if (bins > kMaxBins) bins = kMaxBins;
  std::vector<float> cent[3];
  for (auto& c : cent) c.resize(count);
  std::vector<float> bmin(static_cast<size_t>(count) * 3), bmax(static_cast<size_t>(count) * 3);
  for (int32_t i = 0; i < count; i++) {
    order[i] = i;
    const float* o = tris + static_cast<size_t>(i) * 9;
    double x0 = o[0], y0 = o[1], z0 = o[2];
    double x1 = x0 + o[3], y1 = y0 + o[4], z1 = z0 + o[5];
    double x2 = x0 + o[6], y2 = y0 + o[7], z2 = z0 + o[8];
    double ax = std::min(x0, std::min(x1, x2)), ay = std::min(y0, std::min(y1, y2)), az = std::min(z0, std::min(z1, z2));
    double bx = std::max(x0, std::max(x1, x2)), by = std::max(y0, std::max(y1, y2)), bz = std::max(z0, std::max(z1, z2));
    bmin[i * 3] = fround(ax); bmin[i * 3 + 1] = fround(ay); bmin[i * 3 + 2] = fround(az);
    bmax[i * 3] = fround(bx); bmax[i * 3 + 1] = fround(by); bmax[i * 3 + 2] = fround(bz);
    cent[0][i] = fround((ax + bx) * 0.5);
    cent[1][i] = fround((ay + by) * 0.5);
    cent[2][i] = fround((az + bz) * 0.5);
  }
  int32_t node_count = 1;
  struct Item { int32_t node, first, n, depth; };
  std::vector<Item> stack;
  stack.push_back({0, 0, count, 0});
  int32_t bin_count[kMaxBins];
  float bin_bounds[kMaxBins * 6];
  double right_area[kMaxBins];
  int32_t right_count[kMaxBins];
  while (!stack.empty()) {
    Item it = stack.back();
    stack.pop_back();
    const int32_t node = it.node, first = it.first, n = it.n, depth = it.depth;
    double nx0 = kInf, ny0 = kInf, nz0 = kInf, nx1 = -kInf, ny1 = -kInf, nz1 = -kInf;
    double cmin[3] = {kInf, kInf, kInf}, cmax[3] = {-kInf, -kInf, -kInf};
    for (int32_t k = first; k < first + n; k++) {
      uint32_t t = order[k];
      nx0 = std::min(nx0, static_cast<double>(bmin[t * 3]));
      ny0 = std::min(ny0, static_cast<double>(bmin[t * 3 + 1]));
      nz0 = std::min(nz0, static_cast<double>(bmin[t * 3 + 2]));
      nx1 = std::max(nx1, static_cast<double>(bmax[t * 3]));
      ny1 = std::max(ny1, static_cast<double>(bmax[t * 3 + 1]));
      nz1 = std::max(nz1, static_cast<double>(bmax[t * 3 + 2]));
      for (int a = 0; a < 3; a++) {
        double c = cent[a][t];
        if (c < cmin[a]) cmin[a] = c;
        if (c > cmax[a]) cmax[a] = c;
      }
    }
    float* b = bounds + static_cast<size_t>(node) * 6;
    if (n == 0) {
      b[0] = b[1] = b[2] = 0;
      b[3] = b[4] = b[5] = -1;
    } else {
      b[0] = fround(nx0); b[1] = fround(ny0); b[2] = fround(nz0);
      b[3] = fround(nx1); b[4] = fround(ny1); b[5] = fround(nz1);
    }
    int32_t* nd = nodes + static_cast<size_t>(node) * 3;
    if (n <= kMaxLeaf || depth >= kMaxDepth) {
      nd[0] = first; nd[1] = n; nd[2] = 0;
      continue;
    }
    double best_cost = kInf;
    int best_axis = -1, best_split = -1;
    for (int axis = 0; axis < 3; axis++) {
      double lo = cmin[axis], extent = cmax[axis] - lo;
      if (!(extent > 0)) continue;
      double scale = bins / extent;
      const std::vector<float>& c = cent[axis];
      std::fill(bin_count, bin_count + bins, 0);
      for (int i = 0; i < bins; i++) {
        float* o = bin_bounds + i * 6;
        o[0] = o[1] = o[2] = std::numeric_limits<float>::infinity();
        o[3] = o[4] = o[5] = -std::numeric_limits<float>::infinity();
      }
      for (int32_t k = first; k < first + n; k++) {
        uint32_t t = order[k];
        int bin = static_cast<int>(std::min(static_cast<double>(bins - 1), std::floor((c[t] - lo) * scale)));
        bin_count[bin]++;
        float* o = bin_bounds + bin * 6;
        for (int a = 0; a < 3; a++) {
          if (bmin[t * 3 + a] < o[a]) o[a] = bmin[t * 3 + a];
          if (bmax[t * 3 + a] > o[3 + a]) o[3 + a] = bmax[t * 3 + a];
        }
      }
      double rx0 = kInf, ry0 = kInf, rz0 = kInf, rx1 = -kInf, ry1 = -kInf, rz1 = -kInf;
      int32_t rc = 0;
      for (int i = bins - 1; i > 0; i--) {
        const float* o = bin_bounds + i * 6;
        rc += bin_count[i];
        rx0 = std::min(rx0, static_cast<double>(o[0])); ry0 = std::min(ry0, static_cast<double>(o[1]));
        rz0 = std::min(rz0, static_cast<double>(o[2]));
        rx1 = std::max(rx1, static_cast<double>(o[3])); ry1 = std::max(ry1, static_cast<double>(o[4]));
        rz1 = std::max(rz1, static_cast<double>(o[5]));
        right_count[i] = rc;
        right_area[i] = rc > 0 ? area(rx0, ry0, rz0, rx1, ry1, rz1) : 0;
      }
      double lx0 = kInf, ly0 = kInf, lz0 = kInf, lx1 = -kInf, ly1 = -kInf, lz1 = -kInf;
      int32_t lc = 0;
      for (int i = 0; i < bins - 1; i++) {
        const float* o = bin_bounds + i * 6;
        lc += bin_count[i];
        lx0 = std::min(lx0, static_cast<double>(o[0])); ly0 = std::min(ly0, static_cast<double>(o[1]));
        lz0 = std::min(lz0, static_cast<double>(o[2]));
        lx1 = std::max(lx1, static_cast<double>(o[3])); ly1 = std::max(ly1, static_cast<double>(o[4]));
        lz1 = std::max(lz1, static_cast<double>(o[5]));
        int32_t rc2 = right_count[i + 1];
        if (lc == 0 || rc2 == 0) continue;
        double cost = lc * area(lx0, ly0, lz0, lx1, ly1, lz1) + rc2 * right_area[i + 1];
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_split = i;
        }
      }
    }
    int32_t mid;
    if (best_axis >= 0) {
      double parent_area = area(nx0, ny0, nz0, nx1, ny1, nz1);
      double split_cost = 1 + (1 * best_cost) / std::max(parent_area, 1e-30);
      if (split_cost >= 1.0 * n && n <= 16) {
        nd[0] = first; nd[1] = n; nd[2] = 0;
        continue;
      }
      double lo = cmin[best_axis], scale = bins / (cmax[best_axis] - lo);
      const std::vector<float>& c = cent[best_axis];
      int32_t i = first, j = first + n - 1;
      while (i <= j) {
        int bin = static_cast<int>(std::min(static_cast<double>(bins - 1), std::floor((c[order[i]] - lo) * scale)));
        if (bin <= best_split) {
          i++;
        } else {
          std::swap(order[i], order[j]);
          j--;
        }
      }
      mid = i;
    } else {
      best_axis = 0;
      mid = first + (n >> 1);
    }
    if (mid == first || mid == first + n) mid = first + (n >> 1);
    int32_t left = node_count;
    node_count += 2;
    nd[0] = left; nd[1] = 0; nd[2] = best_axis;
    stack.push_back({left, first, mid - first, depth + 1});
    stack.push_back({left + 1, mid, first + n - mid, depth + 1});
  }
  return node_count;
}

inline double safe_inverse(double d) { return d != 0 ? 1 / d : 1e30; }  // bvh.ts:336-338

// boxEntry, bvh.ts:340-356.
inline double box_entry(const float* bounds, int32_t node, double ox, double oy, double oz, double ix,
                        double iy, double iz, double t_min, double t_max) {
  const float* b = bounds + static_cast<size_t>(node) * 6;
  double t0 = (b[0] - ox) * ix, t1 = (b[3] - ox) * ix;
  double lo = std::min(t0, t1), hi = std::max(t0, t1);
  t0 = (b[1] - oy) * iy; t1 = (b[4] - oy) * iy;
  lo = std::max(lo, std::min(t0, t1)); hi = std::min(hi, std::max(t0, t1));
  t0 = (b[2] - oz) * iz; t1 = (b[5] - oz) * iz;
  lo = std::max(lo, std::min(t0, t1)); hi = std::min(hi, std::max(t0, t1));
  if (hi >= lo && hi >= t_min && lo <= t_max) return std::max(lo, t_min);
  return kInf;
}

struct Bvh {
  const float* tris;
  const uint8_t* sides;
  const float* bounds;
  const int32_t* nodes;
  int32_t node_count;
};

struct Hit {
  int32_t triangle = -1;
  double t = kInf;
  double u = 0, v = 0;
  bool front = true;
};

// Moller-Trumbore on a (v0, e1, e2) record, as both traversals inline it
// (bvh.ts:226-253 and 315-329). Returns false on a miss.
inline bool intersect_triangle(const float* o9, double ox, double oy, double oz, double dx, double dy,
                               double dz, double* det_out, double* t, double* u, double* v,
                               int cull_side) {
  double e1x = o9[3], e1y = o9[4], e1z = o9[5];
  double e2x = o9[6], e2y = o9[7], e2z = o9[8];
  double px = dy * e2z - dz * e2y, py = dz * e2x - dx * e2z, pz = dx * e2y - dy * e2x;
  double det = e1x * px + e1y * py + e1z * pz;
  if (det == 0) return false;
  if (cull_side == 0 && det < 0) return false;
  if (cull_side == 1 && det > 0) return false;
  double inv = 1 / det;
  double sx = ox - o9[0], sy = oy - o9[1], sz = oz - o9[2];
  double uu = (sx * px + sy * py + sz * pz) * inv;
  if (uu < 0 || uu > 1) return false;
  double qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
  double vv = (dx * qx + dy * qy + dz * qz) * inv;
  if (vv < 0 || uu + vv > 1) return false;
  *t = (e2x * qx + e2y * qy + e2z * qz) * inv;
  *u = uu;
  *v = vv;
  *det_out = det;
  return true;
}

// intersectClosest, bvh.ts:202-282.
bool intersect_closest(const Bvh& bvh, double ox, double oy, double oz, double dx, double dy, double dz,
                       double t_min, double t_max, bool cull, Hit& hit, int32_t* stack, oracle_counters* cnt) {
  hit.triangle = -1;
  hit.t = t_max;
  if (cnt) cnt->closest_queries++;
  if (bvh.node_count == 0) return false;
  double ix = safe_inverse(dx), iy = safe_inverse(dy), iz = safe_inverse(dz);
  bool neg[3] = {ix < 0, iy < 0, iz < 0};
  int sp = 0;
  int32_t node = 0;
  for (;;) {
    const int32_t* nd = bvh.nodes + static_cast<size_t>(node) * 3;
    int32_t count = nd[1];
    if (count > 0) {
      int32_t first = nd[0];
      for (int32_t k = first; k < first + count; k++) {
        if (cnt) cnt->closest_tris++;
        double det, t, u, v;
        int side = cull ? bvh.sides[k] : 2;
        if (!intersect_triangle(bvh.tris + static_cast<size_t>(k) * 9, ox, oy, oz, dx, dy, dz, &det, &t, &u,
                                &v, side))
          continue;
        if (t > t_min && t < hit.t) {
          hit.t = t;
          hit.u = u;
          hit.v = v;
          hit.triangle = k;
          hit.front = det > 0;
        }
      }
    } else {
      int32_t left = nd[0];
      int32_t near_ = neg[nd[2]] ? left + 1 : left;
      int32_t far_ = near_ == left ? left + 1 : left;
      if (cnt) cnt->closest_boxes += 2;
      double tn = box_entry(bvh.bounds, near_, ox, oy, oz, ix, iy, iz, t_min, hit.t);
      double tf = box_entry(bvh.bounds, far_, ox, oy, oz, ix, iy, iz, t_min, hit.t);
      if (tn < kInf) {
        if (tf < kInf) {
          if (tf < tn) {
            stack[sp++] = near_;
            node = far_;
          } else {
            stack[sp++] = far_;
            node = near_;
          }
        } else {
          node = near_;
        }
        continue;
      }
      if (tf < kInf) {
        node = far_;
        continue;
      }
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
  return hit.triangle >= 0;
}

// intersectAny, bvh.ts:289-332, with the visitor as a functor.
template <class Visit>
void intersect_any(const Bvh& bvh, double ox, double oy, double oz, double dx, double dy, double dz,
                   double t_min, double t_max, int32_t* stack, oracle_counters* cnt, Visit&& visit) {
  if (cnt) cnt->any_queries++;
  if (bvh.node_count == 0) return;
  double ix = safe_inverse(dx), iy = safe_inverse(dy), iz = safe_inverse(dz);
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    int32_t node = stack[--sp];
    if (cnt) cnt->any_boxes++;
    if (box_entry(bvh.bounds, node, ox, oy, oz, ix, iy, iz, t_min, t_max) == kInf) continue;
    const int32_t* nd = bvh.nodes + static_cast<size_t>(node) * 3;
    int32_t count = nd[1];
    if (count == 0) {
      stack[sp++] = nd[0];
      stack[sp++] = nd[0] + 1;
      continue;
    }
    int32_t first = nd[0];
    for (int32_t k = first; k < first + count; k++) {
      if (cnt) cnt->any_tris++;
      double det, t, u, v;
      if (!intersect_triangle(bvh.tris + static_cast<size_t>(k) * 9, ox, oy, oz, dx, dy, dz, &det, &t, &u, &v,
                              2))
        continue;
      if (t > t_min && t < t_max && !visit(k, t, u, v, det > 0)) return;
    }
  }
}

// ---------------------------------------------------------------- tracer.ts

const int kMaxPassThrough = 64;  // tracer.ts:30

// cameraRay / unproject, tracer.ts:705-727.
void unproject(const mcrt_camera& cam, double x, double y, double z, double* out) {
  const double* p = cam.projection_inverse;
  double w = p[3] * x + p[7] * y + p[11] * z + p[15];
  double vx = (p[0] * x + p[4] * y + p[8] * z + p[12]) / w;
  double vy = (p[1] * x + p[5] * y + p[9] * z + p[13]) / w;
  double vz = (p[2] * x + p[6] * y + p[10] * z + p[14]) / w;
  const double* m = cam.world;
  out[0] = m[0] * vx + m[4] * vy + m[8] * vz + m[12];
  out[1] = m[1] * vx + m[5] * vy + m[9] * vz + m[13];
  out[2] = m[2] * vx + m[6] * vy + m[10] * vz + m[14];
}

void camera_ray(const mcrt_camera& cam, double x, double y, double* out) {
  double near_[3], far_[3];
  unproject(cam, x, y, -1, near_);
  unproject(cam, x, y, 1, far_);
  double dx = far_[0] - near_[0], dy = far_[1] - near_[1], dz = far_[2] - near_[2];
  double length = hypot_or_one(dx, dy, dz);
  dx /= length; dy /= length; dz /= length;
  out[0] = near_[0]; out[1] = near_[1]; out[2] = near_[2];
  out[3] = dx; out[4] = dy; out[5] = dz;
}

inline double luminance(double r, double g, double b) { return 0.2126 * r + 0.7152 * g + 0.0722 * b; }

inline double multi_scatter(double fss_ess, double f0, double ems) {  // tracer.ts:699-702
  double f_avg = f0 + (1 - f0) * 0.047619;
  return ((fss_ess * f_avg) / (1 - ems * f_avg)) * ems;
}

// Tracer, tracer.ts:36-692. One per thread: it holds scratch state.
struct Tracer {
  const mcrt_geometry& geo;
  const mcrt_shading& sh;
  const mcrt_settings& settings;
  Bvh bvh;
  oracle_counters* cnt;
  Hit hit;
  int32_t stack[256];
  Random random;
  double texel[4];
  double env[3];
  double color[3];
  double shadow_color[3];
  bool shadow_cast_only = false;
  std::vector<double> shadow_hits;
  double shadow_depth[3];
  double lx = 0, ly = 0, lz = 0, lr = 0, lg = 0, lb = 0, light_distance = kInf;
  double sx = 0, sy = 0, sz = 0;

  Tracer(const mcrt_geometry& g, const mcrt_shading& s, const mcrt_settings& st, oracle_counters* c)
      : geo(g), sh(s), settings(st), cnt(c) {
    bvh = {g.triangles, g.sides, g.bvh_bounds, g.bvh_nodes, g.node_count};
  }

  // renderTile, tracer.ts:62-89.
  void render_tile(const mcrt_camera& cam, const mcrt_tile& tile, int width, int height, int pass, int block,
                   float* out) {
    double sample[4];
    double ray[6];
    for (int y = 0; y < tile.height; y += block) {
      for (int x = 0; x < tile.width; x += block) {
        int px = tile.x + x, py = tile.y + y;
        sample_one(cam, px, py, width, height, pass, block, sample, ray);
        for (int by = y; by < std::min(y + block, tile.height); by++) {
          for (int bx = x; bx < std::min(x + block, tile.width); bx++) {
            float* o = out + (static_cast<size_t>(by) * tile.width + bx) * 4;
            for (int c = 0; c < 4; c++) o[c] = fround(sample[c]);
          }
        }
      }
    }
  }

  // The body of renderTile's pixel loop, tracer.ts:68-80.
  void sample_one(const mcrt_camera& cam, int px, int py, int width, int height, int pass, int block,
                  double* sample, double* ray) {
    random.seed(static_cast<uint32_t>(px), static_cast<uint32_t>(py), static_cast<uint32_t>(pass), settings.seed);
    double jx = 0.5, jy = 0.5;
    if (block > 1) {
      jx = std::min(block, width - px) * 0.5;
      jy = std::min(block, height - py) * 0.5;
    } else if (pass > 0) {
      jx = random.next();
      jy = random.next();
    }
    double sxp = (px + jx) / width, syp = (py + jy) / height;
    camera_ray(cam, sxp * 2 - 1, 1 - syp * 2, ray);
    sample_pixel(cam, ray, sxp, syp, sample);
    if (cnt) cnt->samples++;
  }

  // samplePixel, tracer.ts:92-478.
  void sample_pixel(const mcrt_camera& cam, const double* ray, double sxp, double syp, double* out) {
    const double eps = geo.epsilon;
    double ox = ray[0], oy = ray[1], oz = ray[2], dx = ray[3], dy = ray[4], dz = ray[5];
    double tr = 1, tg = 1, tb = 1;
    double Lr = 0, Lg = 0, Lb = 0;
    bool surface_seen = false;
    bool tone_mapped = true;
    double fog_factor = 0;
    const mcrt_environment* last_env = nullptr;
    double last_env_scale = 1;
    int bounce = 0;
    int passes = 0;
    bool cull = true;
    double mr = 0, mg = 0, mb = 0;

    for (;;) {
      if (!intersect_closest(bvh, ox, oy, oz, dx, dy, dz, 0, kInf, cull, hit, stack, cnt)) {
        if (!surface_seen) {
          background(dx, dy, dz, sxp, syp, out);
          return;
        }
        if (last_env) {
          sample_environment(*last_env, sh.textures, dx, dy, dz, env);
          Lr += tr * env[0] * last_env_scale;
          Lg += tg * env[1] * last_env_scale;
          Lb += tb * env[2] * last_env_scale;
        }
        break;
      }
      if (mr > 0 || mg > 0 || mb > 0) {
        tr *= std::exp(-mr * hit.t);
        tg *= std::exp(-mg * hit.t);
        tb *= std::exp(-mb * hit.t);
      }
      const int32_t k = hit.triangle;
      const mcrt_material& mat = sh.materials[geo.materials[k]];
      const double t = hit.t;
      const double px = ox + dx * t, py = oy + dy * t, pz = oz + dz * t;
      const double w1 = hit.u, w2 = hit.v, w0 = 1 - w1 - w2;
      const float* tri = geo.triangles + static_cast<size_t>(k) * 9;
      double gx = static_cast<double>(tri[4]) * tri[8] - static_cast<double>(tri[5]) * tri[7];
      double gy = static_cast<double>(tri[5]) * tri[6] - static_cast<double>(tri[3]) * tri[8];
      double gz = static_cast<double>(tri[3]) * tri[7] - static_cast<double>(tri[4]) * tri[6];
      double gl = hypot_or_one(gx, gy, gz);
      double face = hit.front ? 1 : -1;
      gx = (gx / gl) * face; gy = (gy / gl) * face; gz = (gz / gl) * face;

      const float* uv = geo.uvs + static_cast<size_t>(k) * 6;
      double u = uv[0] * w0 + uv[2] * w1 + uv[4] * w2;
      double v = uv[1] * w0 + uv[3] * w1 + uv[5] * w2;

      double cr = mat.color[0], cg = mat.color[1], cb = mat.color[2];
      double alpha = mat.opacity;
      if (mat.map >= 0) {
        sample_texture(sh.textures[mat.map], u, v, texel);
        cr *= texel[0]; cg *= texel[1]; cb *= texel[2]; alpha *= texel[3];
      }
      if (mat.vertex_colors && geo.colors) {
        const float* c = geo.colors + static_cast<size_t>(k) * 12;
        cr *= c[0] * w0 + c[4] * w1 + c[8] * w2;
        cg *= c[1] * w0 + c[5] * w1 + c[9] * w2;
        cb *= c[2] * w0 + c[6] * w1 + c[10] * w2;
        alpha *= c[3] * w0 + c[7] * w1 + c[11] * w2;
      }
      if (mat.alpha_map >= 0) {
        sample_texture(sh.textures[mat.alpha_map], u, v, texel);
        alpha *= texel[1];
      }
      bool cut_out = mat.alpha_test > 0 && alpha < mat.alpha_test;
      if (cut_out || (mat.transparent && (g_planted_draw_mistake == 1 ? (random.next(), random.next())
                                                                       : random.next()) >= alpha)) {
        if (++passes > kMaxPassThrough) break;
        double side = gx * dx + gy * dy + gz * dz > 0 ? eps : -eps;
        ox = px + gx * side; oy = py + gy * side; oz = pz + gz * side;
        continue;
      }
      if (!surface_seen) {
        surface_seen = true;
        tone_mapped = mat.tone_mapped != 0;
        fog_factor = fog(cam, px, py, pz);
      }

      const float* nrm = geo.normals + static_cast<size_t>(k) * 9;
      double nx = (nrm[0] * w0 + nrm[3] * w1 + nrm[6] * w2) * face;
      double ny = (nrm[1] * w0 + nrm[4] * w1 + nrm[7] * w2) * face;
      double nz = (nrm[2] * w0 + nrm[5] * w1 + nrm[8] * w2) * face;
      double nl = hypot_or_one(nx, ny, nz);
      nx /= nl; ny /= nl; nz /= nl;
      if (mat.normal_map >= 0) {
        sample_texture(sh.textures[mat.normal_map], u, v, texel);
        double mx = (texel[0] * 2 - 1) * mat.normal_scale[0];
        double my = (texel[1] * 2 - 1) * mat.normal_scale[1];
        double mz = texel[2] * 2 - 1;
        const float* tg4 = geo.tangents + static_cast<size_t>(k) * 4;
        double ax = tg4[0], ay = tg4[1], az = tg4[2];
        double along = ax * nx + ay * ny + az * nz;
        ax -= nx * along; ay -= ny * along; az -= nz * along;
        double al = hypot_or_one(ax, ay, az);
        ax = (ax / al) * face; ay = (ay / al) * face; az = (az / al) * face;
        double sign = tg4[3];
        double bx = (ny * az - nz * ay) * sign, by = (nz * ax - nx * az) * sign, bz = (nx * ay - ny * ax) * sign;
        nx = ax * mx + bx * my + nx * mz;
        ny = ay * mx + by * my + ny * mz;
        nz = az * mx + bz * my + nz * mz;
        nl = hypot_or_one(nx, ny, nz);
        nx /= nl; ny /= nl; nz /= nl;
      }

      const double vx = -dx, vy = -dy, vz = -dz;
      const double dot_nv = std::min(std::max(nx * vx + ny * vy + nz * vz, 0.0), 1.0);
      double out_r = 0, out_g = 0, out_b = 0;

      double er = mat.emissive[0], eg = mat.emissive[1], eb = mat.emissive[2];
      if (mat.emissive_map >= 0 && (er > 0 || eg > 0 || eb > 0)) {
        sample_texture(sh.textures[mat.emissive_map], u, v, texel);
        er *= texel[0]; eg *= texel[1]; eb *= texel[2];
      }

      const bool receive = (geo.flags[k] & MCRT_TRI_RECEIVE_SHADOW) != 0;
      const bool can_continue = bounce < settings.max_bounces;

      double spec_r = 0, spec_g = 0, spec_b = 0;
      double diff_r = 0, diff_g = 0, diff_b = 0;
      double trans_r = 0, trans_g = 0, trans_b = 0;
      double roughness = 1;
      const mcrt_environment* environment = nullptr;
      double environment_scale = 1;

      if (mat.model == MCRT_MODEL_BASIC) {
        out_r = cr; out_g = cg; out_b = cb;
      } else {
        double ir = 0, ig = 0, ib = 0;
        for (int li = 0; li < sh.light_count; li++) {
          const mcrt_light& light = sh.lights[li];
          if (light.type == MCRT_LIGHT_AMBIENT) {
            ir += light.color[0]; ig += light.color[1]; ib += light.color[2];
          } else if (light.type == MCRT_LIGHT_HEMISPHERE) {
            double w = 0.5 * (nx * light.direction[0] + ny * light.direction[1] + nz * light.direction[2]) + 0.5;
            ir += light.ground_color[0] + (light.color[0] - light.ground_color[0]) * w;
            ig += light.ground_color[1] + (light.color[1] - light.ground_color[1]) * w;
            ib += light.ground_color[2] + (light.color[2] - light.ground_color[2]) * w;
          }
        }
        double ao = 1;
        if (mat.ao_map >= 0) {
          sample_texture(sh.textures[mat.ao_map], u, v, texel);
          ao = (texel[0] - 1) * mat.ao_map_intensity + 1;
        }

        if (mat.model == MCRT_MODEL_PHYSICAL) {
          double metalness = mat.metalness;
          roughness = mat.roughness;
          if (mat.roughness_map >= 0) {
            sample_texture(sh.textures[mat.roughness_map], u, v, texel);
            roughness *= texel[1];
          }
          if (mat.metalness_map >= 0) {
            sample_texture(sh.textures[mat.metalness_map], u, v, texel);
            metalness *= texel[2];
          }
          const double shade_roughness = std::min(std::max(roughness, 0.045), 1.0);
          double sr = 0.04, sg = 0.04, sb = 0.04, f90 = 1;
          if (mat.physical) {
            double f = std::pow((mat.ior - 1) / (mat.ior + 1), 2.0);
            sr = std::min(f * mat.specular_color[0], 1.0) * mat.specular_intensity;
            sg = std::min(f * mat.specular_color[1], 1.0) * mat.specular_intensity;
            sb = std::min(f * mat.specular_color[2], 1.0) * mat.specular_intensity;
            f90 = mat.specular_intensity + (1 - mat.specular_intensity) * metalness;
          }
          const double br = sr + (cr - sr) * metalness, bg = sg + (cg - sg) * metalness,
                       bbl = sb + (cb - sb) * metalness;
          const double dr = cr * (1 - metalness), dg = cg * (1 - metalness), db = cb * (1 - metalness);
          double dfg_out[2];
          dfg(shade_roughness, dot_nv, dfg_out);
          const double fa = dfg_out[0], fb = dfg_out[1];
          const double ess_ms = fa + fb, ems = 1 - ess_ms;
          const double comp_r = 1 + br * (1 / ess_ms - 1), comp_g = 1 + bg * (1 / ess_ms - 1),
                       comp_b = 1 + bbl * (1 / ess_ms - 1);
          const double ggx_alpha = shade_roughness * shade_roughness;
          const double transmission = mat.transmission;
          const double keep_diffuse = 1 - transmission;

          for (int li = 0; li < sh.light_count; li++) {
            const mcrt_light& light = sh.lights[li];
            if (!light_at(light, px, py, pz)) continue;
            const double dot_nl = nx * lx + ny * ly + nz * lz;
            if (dot_nl <= 0) continue;
            double hx = lx + vx, hy = ly + vy, hz = lz + vz;
            double hl = hypot_or_one(hx, hy, hz);
            hx /= hl; hy /= hl; hz /= hl;
            const double dot_nh = std::min(std::max(nx * hx + ny * hy + nz * hz, 0.0), 1.0);
            const double dot_vh = std::min(std::max(vx * hx + vy * hy + vz * hz, 0.0), 1.0);
            const double fw = fresnel_weight(dot_vh);
            const double vd = visibility_ggx(ggx_alpha, dot_nl, dot_nv) * distribution_ggx(ggx_alpha, dot_nh);
            const double specular_r = (br * (1 - fw) + f90 * fw) * vd * comp_r;
            const double specular_g = (bg * (1 - fw) + f90 * fw) * vd * comp_g;
            const double specular_b = (bbl * (1 - fw) + f90 * fw) * vd * comp_b;
            const double diffuse_r = dr * kInvPi * (1 - (sr * (1 - fw) + f90 * fw)) * keep_diffuse;
            const double diffuse_g = dg * kInvPi * (1 - (sg * (1 - fw) + f90 * fw)) * keep_diffuse;
            const double diffuse_b = db * kInvPi * (1 - (sb * (1 - fw) + f90 * fw)) * keep_diffuse;
            const double scale = dot_nl;
            double r = (specular_r + diffuse_r) * scale * lr;
            double g = (specular_g + diffuse_g) * scale * lg;
            double b = (specular_b + diffuse_b) * scale * lb;
            if (r + g + b <= 0) continue;
            if (!visible_light(light, receive, px, py, pz, gx, gy, gz)) continue;
            r *= shadow_color[0]; g *= shadow_color[1]; b *= shadow_color[2];
            out_r += r; out_g += g; out_b += b;
          }

          const double fss_r = sr * fa + f90 * fb, fss_g = sg * fa + f90 * fb, fss_b = sb * fa + f90 * fb;
          const double scatter_r = fss_r + multi_scatter(fss_r, sr, ems);
          const double scatter_g = fss_g + multi_scatter(fss_g, sg, ems);
          const double scatter_b = fss_b + multi_scatter(fss_b, sb, ems);
          out_r += ir * kInvPi * dr * (1 - scatter_r) * ao * keep_diffuse;
          out_g += ig * kInvPi * dg * (1 - scatter_g) * ao * keep_diffuse;
          out_b += ib * kInvPi * db * (1 - scatter_b) * ao * keep_diffuse;

          const double mf_r = cr * fa + f90 * fb, mf_g = cg * fa + f90 * fb, mf_b = cb * fa + f90 * fb;
          spec_r = fss_r + (mf_r - fss_r) * metalness;
          spec_g = fss_g + (mf_g - fss_g) * metalness;
          spec_b = fss_b + (mf_b - fss_b) * metalness;
          diff_r = dr * (1 - scatter_r) * keep_diffuse;
          diff_g = dg * (1 - scatter_g) * keep_diffuse;
          diff_b = db * (1 - scatter_b) * keep_diffuse;
          if (transmission > 0) {
            const double fr = sr * fa + f90 * fb, fg = sg * fa + f90 * fb, fbl = sb * fa + f90 * fb;
            trans_r = transmission * (1 - fr) * cr;
            trans_g = transmission * (1 - fg) * cg;
            trans_b = transmission * (1 - fbl) * cb;
          }
          if (mat.env_map >= 0) {
            environment = &sh.environments[mat.env_map];
          } else if (sh.environment >= 0) {
            environment = &sh.environments[sh.environment];
            environment_scale = mat.env_map_intensity;
          }
          if (environment && !settings.global_illumination) {
            cosine_direction(nx, ny, nz, g_planted_draw_mistake == 2);
            const double sx2 = sx, sy2 = sy, sz2 = sz;
            if (sx2 * gx + sy2 * gy + sz2 * gz > 0 &&
                transmittance(px + gx * eps, py + gy * eps, pz + gz * eps, sx2, sy2, sz2, kInf, false)) {
              sample_environment(*environment, sh.textures, sx2, sy2, sz2, env);
              out_r += env[0] * environment_scale * diff_r * shadow_color[0];
              out_g += env[1] * environment_scale * diff_g * shadow_color[1];
              out_b += env[2] * environment_scale * diff_b * shadow_color[2];
            }
          }
          if (!settings.global_illumination) diff_r = diff_g = diff_b = 0;
        } else {
          for (int li = 0; li < sh.light_count; li++) {
            const mcrt_light& light = sh.lights[li];
            if (!light_at(light, px, py, pz)) continue;
            const double cosine = nx * lx + ny * ly + nz * lz;
            double irradiance;
            if (mat.model == MCRT_MODEL_TOON) {
              irradiance = cosine * 0.5 + 0.5 < 0.7 ? 0.7 : 1;
            } else if (cosine <= 0) {
              continue;
            } else {
              irradiance = cosine;
            }
            double r = cr * kInvPi, g = cg * kInvPi, b = cb * kInvPi;
            if (mat.model == MCRT_MODEL_PHONG && cosine > 0) {
              double hx = lx + vx, hy = ly + vy, hz = lz + vz;
              double hl = hypot_or_one(hx, hy, hz);
              hx /= hl; hy /= hl; hz /= hl;
              const double dot_nh = std::min(std::max(nx * hx + ny * hy + nz * hz, 0.0), 1.0);
              const double dot_vh = std::min(std::max(vx * hx + vy * hy + vz * hz, 0.0), 1.0);
              const double fw = fresnel_weight(dot_vh);
              const double d = blinn_phong(mat.shininess, dot_nh);
              r += (mat.specular[0] * (1 - fw) + fw) * d;
              g += (mat.specular[1] * (1 - fw) + fw) * d;
              b += (mat.specular[2] * (1 - fw) + fw) * d;
            }
            r *= irradiance * lr; g *= irradiance * lg; b *= irradiance * lb;
            if (r + g + b <= 0) continue;
            if (!visible_light(light, receive, px, py, pz, gx, gy, gz)) continue;
            out_r += r * shadow_color[0]; out_g += g * shadow_color[1]; out_b += b * shadow_color[2];
          }
          out_r += ir * kInvPi * cr * ao;
          out_g += ig * kInvPi * cg * ao;
          out_b += ib * kInvPi * cb * ao;
          if (settings.global_illumination) {
            diff_r = cr; diff_g = cg; diff_b = cb;
          }
        }
      }

      if (mat.model != MCRT_MODEL_PHYSICAL && mat.env_map >= 0) {
        const mcrt_environment& e = sh.environments[mat.env_map];
        const double dn = dx * nx + dy * ny + dz * nz;
        sample_environment(e, sh.textures, dx - 2 * dn * nx, dy - 2 * dn * ny, dz - 2 * dn * nz, env);
        const double s = mat.reflectivity;
        const double er2 = env[0], eg2 = env[1], eb2 = env[2];
        if (mat.combine == MCRT_MULTIPLY_OPERATION) {
          out_r *= 1 - s + s * er2; out_g *= 1 - s + s * eg2; out_b *= 1 - s + s * eb2;
        } else if (mat.combine == MCRT_MIX_OPERATION) {
          out_r += (er2 - out_r) * s; out_g += (eg2 - out_g) * s; out_b += (eb2 - out_b) * s;
        } else if (mat.combine == MCRT_ADD_OPERATION) {
          out_r += er2 * s; out_g += eg2 * s; out_b += eb2 * s;
        }
      }

      Lr += tr * (out_r + er);
      Lg += tg * (out_g + eg);
      Lb += tb * (out_b + eb);

      if (!can_continue) break;

      const double ws = luminance(spec_r, spec_g, spec_b);
      const double wt = luminance(trans_r, trans_g, trans_b);
      const double wd = luminance(diff_r, diff_g, diff_b);
      const double total = ws + wt + wd;
      if (total <= 1e-6) break;
      if (g_planted_draw_mistake == 3) random.next();
      const double pick = random.next() * total;
      double wr, wg, wb, p;
      if (pick < ws) {
        p = ws / total;
        wr = spec_r; wg = spec_g; wb = spec_b;
        reflection(dx, dy, dz, nx, ny, nz, roughness);
        if (sx * gx + sy * gy + sz * gz <= 0) break;
        last_env = environment;
        last_env_scale = environment_scale;
      } else if (pick < ws + wt) {
        p = wt / total;
        wr = trans_r; wg = trans_g; wb = trans_b;
        if (mat.thickness > 0) {
          const double eta = hit.front ? 1 / mat.ior : mat.ior;
          if (refract(dx, dy, dz, nx, ny, nz, eta)) {
            cull = !hit.front;
            if (hit.front) {
              mr = mat.attenuation[0]; mg = mat.attenuation[1]; mb = mat.attenuation[2];
            } else {
              mr = mg = mb = 0;
            }
          } else {
            reflection(dx, dy, dz, nx, ny, nz, 0);
          }
        } else {
          sx = dx; sy = dy; sz = dz;
        }
        last_env = environment;
        last_env_scale = environment_scale;
      } else {
        p = wd / total;
        wr = diff_r; wg = diff_g; wb = diff_b;
        cosine_direction(nx, ny, nz, g_planted_draw_mistake == 4);
        if (sx * gx + sy * gy + sz * gz <= 0) break;
        last_env = environment;
        last_env_scale = environment_scale;
      }
      tr *= wr / p; tg *= wg / p; tb *= wb / p;
      const double side = sx * gx + sy * gy + sz * gz > 0 ? eps : -eps;
      ox = px + gx * side; oy = py + gy * side; oz = pz + gz * side;
      dx = sx; dy = sy; dz = sz;
      bounce++;
      if (bounce >= (g_planted_draw_mistake == 6 ? 2 : 3)) {
        const double q = std::min(0.95, std::max(tr, std::max(tg, tb)));
        if (random.next() >= q) break;
        tr /= q; tg /= q; tb /= q;
      }
    }

    color[0] = Lr; color[1] = Lg; color[2] = Lb;
    if (tone_mapped && settings.tone_mapping != MCRT_NO_TONE_MAPPING)
      tone_map(color, settings.tone_mapping, settings.tone_mapping_exposure);
    if (fog_factor > 0 && sh.fog.kind != MCRT_FOG_NONE) {
      for (int c = 0; c < 3; c++) color[c] = color[c] + (sh.fog.color[c] - color[c]) * fog_factor;
    }
    out[0] = color[0]; out[1] = color[1]; out[2] = color[2]; out[3] = 1;
  }

  // lightAt, tracer.ts:486-512.
  bool light_at(const mcrt_light& light, double px, double py, double pz) {
    switch (light.type) {
      case MCRT_LIGHT_DIRECTIONAL:
        lx = light.direction[0]; ly = light.direction[1]; lz = light.direction[2];
        lr = light.color[0]; lg = light.color[1]; lb = light.color[2];
        light_distance = kInf;
        return true;
      case MCRT_LIGHT_POINT:
      case MCRT_LIGHT_SPOT: {
        double x = light.position[0] - px, y = light.position[1] - py, z = light.position[2] - pz;
        double distance = js_hypot(x, y, z);
        if (distance == 0) return false;
        lx = x / distance; ly = y / distance; lz = z / distance;
        double scale = distance_attenuation(distance, light.distance, light.decay);
        if (light.type == MCRT_LIGHT_SPOT) {
          double angle_cos = lx * light.direction[0] + ly * light.direction[1] + lz * light.direction[2];
          scale *= smoothstep(light.cone_cos, light.penumbra_cos, angle_cos);
        }
        if (scale <= 0) return false;
        lr = light.color[0] * scale; lg = light.color[1] * scale; lb = light.color[2] * scale;
        light_distance = distance;
        return true;
      }
      default:
        return false;
    }
  }

  // visibleLight, tracer.ts:515-526.
  bool visible_light(const mcrt_light& light, bool receive, double px, double py, double pz, double gx, double gy,
                     double gz) {
    shadow_color[0] = shadow_color[1] = shadow_color[2] = 1;
    const int mode = settings.shadows;
    if (mode == MCRT_SHADOWS_NONE) return true;
    const bool cast_only = mode == MCRT_SHADOWS_CAST_SHADOW;
    // Only directional, point and spot lights carry castShadow; lightAt
    // returns false for the others, so `'castShadow' in light` always holds here.
    if (cast_only && (!light.cast_shadow || !receive)) return true;
    const double eps = geo.epsilon;
    const double side = gx * lx + gy * ly + gz * lz > 0 ? eps : -eps;
    const double max_t = light_distance == kInf ? kInf : light_distance - 2 * eps;
    return transmittance(px + gx * side, py + gy * side, pz + gz * side, lx, ly, lz, max_t, cast_only);
  }

  // transmittance, tracer.ts:529-542.
  bool transmittance(double ox, double oy, double oz, double dx, double dy, double dz, double max_t,
                     bool cast_only) {
    shadow_color[0] = shadow_color[1] = shadow_color[2] = 1;
    shadow_cast_only = cast_only;
    shadow_hits.clear();
    shadow_depth[0] = shadow_depth[1] = shadow_depth[2] = 0;
    intersect_any(bvh, ox, oy, oz, dx, dy, dz, 0, max_t, stack, cnt,
                  [this](int32_t tri, double t, double u, double v, bool front) {
                    return attenuate_shadow(tri, t, u, v, front);
                  });
    for (int c = 0; c < 3; c++) {
      double depth = shadow_depth[c];
      if (depth > 0) shadow_color[c] = shadow_color[c] * std::exp(-depth);
    }
    return shadow_color[0] + shadow_color[1] + shadow_color[2] > 0;
  }

  // attenuateShadow, tracer.ts:544-594.
  bool attenuate_shadow(int32_t triangle, double t, double u, double v, bool front) {
    const uint8_t flags = geo.flags[triangle];
    if (shadow_cast_only && (flags & MCRT_TRI_CAST_SHADOW) == 0) return true;
    if (flags & MCRT_TRI_OPAQUE) {
      shadow_color[0] = shadow_color[1] = shadow_color[2] = 0;
      return false;
    }
    const mcrt_material& mat = sh.materials[geo.materials[triangle]];
    double alpha = mat.opacity;
    double cr = mat.color[0], cg = mat.color[1], cb = mat.color[2];
    if (mat.map >= 0 || mat.alpha_map >= 0) {
      const float* uv = geo.uvs + static_cast<size_t>(triangle) * 6;
      const double w0 = 1 - u - v;
      const double tu = uv[0] * w0 + uv[2] * u + uv[4] * v;
      const double tv = uv[1] * w0 + uv[3] * u + uv[5] * v;
      if (mat.map >= 0) {
        sample_texture(sh.textures[mat.map], tu, tv, texel);
        alpha *= texel[3];
        cr *= texel[0]; cg *= texel[1]; cb *= texel[2];
      }
      if (mat.alpha_map >= 0) {
        sample_texture(sh.textures[mat.alpha_map], tu, tv, texel);
        alpha *= texel[1];
      }
    }
    if (mat.alpha_test > 0 && alpha < mat.alpha_test) return true;
    if (!mat.transparent) alpha = 1;
    const double eps = geo.epsilon;
    for (double seen : shadow_hits)
      if (std::fabs(seen - t) <= eps) return true;
    shadow_hits.push_back(t);
    if (mat.thickness > 0) {
      const double signed_t = front ? -t : t;
      shadow_depth[0] = shadow_depth[0] + mat.attenuation[0] * signed_t;
      shadow_depth[1] = shadow_depth[1] + mat.attenuation[1] * signed_t;
      shadow_depth[2] = shadow_depth[2] + mat.attenuation[2] * signed_t;
    }
    const double open = 1 - alpha;
    const double through = mat.transmission;
    shadow_color[0] = shadow_color[0] * (open + alpha * through * cr);
    shadow_color[1] = shadow_color[1] * (open + alpha * through * cg);
    shadow_color[2] = shadow_color[2] * (open + alpha * through * cb);
    if (shadow_color[0] + shadow_color[1] + shadow_color[2] < 1e-4) {
      shadow_color[0] = shadow_color[1] = shadow_color[2] = 0;
      return false;
    }
    return true;
  }

  // cosineDirection, tracer.ts:600-605.
  void cosine_direction(double nx, double ny, double nz, bool swapped = false) {
    double r1 = random.next(), r2 = random.next();
    if (swapped) std::swap(r1, r2);
    const double phi = 2 * kPi * r1;
    const double radius = std::sqrt(r2);
    to_world(nx, ny, nz, radius * std::cos(phi), radius * std::sin(phi), std::sqrt(std::max(0.0, 1 - r2)));
  }

  // reflection, tracer.ts:608-621.
  void reflection(double dx, double dy, double dz, double nx, double ny, double nz, double roughness) {
    double hx = nx, hy = ny, hz = nz;
    if (roughness > 0.02) {
      const double a = roughness * roughness;
      double r1 = random.next(), r2 = random.next();
      if (g_planted_draw_mistake == 5) std::swap(r1, r2);
      const double phi = 2 * kPi * r1;
      const double cos_theta = std::sqrt((1 - r2) / (1 + (a * a - 1) * r2));
      const double sin_theta = std::sqrt(std::max(0.0, 1 - cos_theta * cos_theta));
      to_world(nx, ny, nz, sin_theta * std::cos(phi), sin_theta * std::sin(phi), cos_theta);
      hx = sx; hy = sy; hz = sz;
    }
    const double dn = dx * hx + dy * hy + dz * hz;
    sx = dx - 2 * dn * hx; sy = dy - 2 * dn * hy; sz = dz - 2 * dn * hz;
  }

  // refract, tracer.ts:624-633.
  bool refract(double dx, double dy, double dz, double nx, double ny, double nz, double eta) {
    const double cosi = -(dx * nx + dy * ny + dz * nz);
    const double k = 1 - eta * eta * (1 - cosi * cosi);
    if (k < 0) return false;
    const double s = eta * cosi - std::sqrt(k);
    sx = eta * dx + s * nx; sy = eta * dy + s * ny; sz = eta * dz + s * nz;
    const double length = hypot_or_one(sx, sy, sz);
    sx /= length; sy /= length; sz /= length;
    return true;
  }

  // toWorld, tracer.ts:636-646 (Duff et al. 2017 orthonormal basis).
  void to_world(double nx, double ny, double nz, double a, double b, double c) {
    const double sign = nz >= 0 ? 1 : -1;
    const double e = -1 / (sign + nz);
    const double f = nx * ny * e;
    const double tx = 1 + sign * nx * nx * e, ty = sign * f, tz = -sign * nx;
    const double bx = f, by = sign + ny * ny * e, bz = -ny;
    sx = tx * a + bx * b + nx * c;
    sy = ty * a + by * b + ny * c;
    sz = tz * a + bz * b + nz * c;
  }

  // fog, tracer.ts:649-656.
  double fog(const mcrt_camera& cam, double px, double py, double pz) {
    if (sh.fog.kind == MCRT_FOG_NONE) return 0;
    const double* f = cam.forward;
    const double* c = cam.position;
    const double depth = (px - c[0]) * f[0] + (py - c[1]) * f[1] + (pz - c[2]) * f[2];
    if (sh.fog.kind == MCRT_FOG_LINEAR) return smoothstep(sh.fog.near_, sh.fog.far_, depth);
    return 1 - std::exp(-sh.fog.density * sh.fog.density * depth * depth);
  }

  // background, tracer.ts:659-691.
  void background(double dx, double dy, double dz, double sxp, double syp, double* out) {
    const mcrt_background& bg = sh.background;
    switch (bg.kind) {
      case MCRT_BACKGROUND_COLOR:
        out[0] = bg.color[0]; out[1] = bg.color[1]; out[2] = bg.color[2]; out[3] = 1;
        return;
      case MCRT_BACKGROUND_SCREEN: {
        const mcrt_texture& tex = sh.textures[bg.texture];
        sample_texture(tex, sxp, 1 - syp, texel);
        color[0] = texel[0] * bg.intensity;
        color[1] = texel[1] * bg.intensity;
        color[2] = texel[2] * bg.intensity;
        if (!tex.srgb && settings.tone_mapping != MCRT_NO_TONE_MAPPING)
          tone_map(color, settings.tone_mapping, settings.tone_mapping_exposure);
        out[0] = color[0]; out[1] = color[1]; out[2] = color[2]; out[3] = 1;
        return;
      }
      case MCRT_BACKGROUND_ENVIRONMENT: {
        const mcrt_environment& e = sh.environments[bg.environment];
        sample_environment(e, sh.textures, dx, dy, dz, color);
        const int tex_index = e.kind == MCRT_ENV_CUBE ? e.faces[0] : e.texture;
        if (!sh.textures[tex_index].srgb && settings.tone_mapping != MCRT_NO_TONE_MAPPING)
          tone_map(color, settings.tone_mapping, settings.tone_mapping_exposure);
        out[0] = color[0]; out[1] = color[1]; out[2] = color[2]; out[3] = 1;
        return;
      }
      default: {
        const double a = settings.clear_alpha;
        out[0] = settings.clear_color[0] * a;
        out[1] = settings.clear_color[1] * a;
        out[2] = settings.clear_color[2] * a;
        out[3] = a;
      }
    }
  }
};

// writeTile for one pixel, progressive.ts:295-310. Note that the running sum
// is read back unrounded: `r = sum[d] = sum[d] + r` assigns the double sum to
// r while the Float32Array keeps its rounding.
void encode_pixel(uint8_t* image, const float* data, float* sum, double scale, bool srgb) {
  double r = data[0], g = data[1], b = data[2], a = data[3];
  if (sum) {
    r = static_cast<double>(sum[0]) + r; sum[0] = fround(r);
    g = static_cast<double>(sum[1]) + g; sum[1] = fround(g);
    b = static_cast<double>(sum[2]) + b; sum[2] = fround(b);
    a = static_cast<double>(sum[3]) + a; sum[3] = fround(a);
    r *= scale; g *= scale; b *= scale; a *= scale;
  }
  if (a > 0) {
    r /= a; g /= a; b /= a;
  }
  if (srgb) {
    r = linear_to_srgb(std::max(0.0, r));
    g = linear_to_srgb(std::max(0.0, g));
    b = linear_to_srgb(std::max(0.0, b));
  }
  image[0] = uint8_clamp(r * 255 + 0.5);
  image[1] = uint8_clamp(g * 255 + 0.5);
  image[2] = uint8_clamp(b * 255 + 0.5);
  image[3] = uint8_clamp(a * 255 + 0.5);
}

void add_counters(oracle_counters* into, const oracle_counters& c) {
  if (!into) return;
  into->closest_queries += c.closest_queries;
  into->closest_boxes += c.closest_boxes;
  into->closest_tris += c.closest_tris;
  into->any_queries += c.any_queries;
  into->any_boxes += c.any_boxes;
  into->any_tris += c.any_tris;
  into->samples += c.samples;
}

// Runs fn(index, tracer) for index in [0, count) on `threads` threads.
template <class Fn>
void parallel_pixels(const mcrt_geometry& g, const mcrt_shading& s, const mcrt_settings& st, int32_t count,
                     int threads, oracle_counters* counters, Fn fn) {
  if (threads < 1) threads = 1;
  std::atomic<int32_t> next(0);
  std::vector<oracle_counters> per(threads);
  auto work = [&](int id) {
    oracle_counters c{};
    Tracer tracer(g, s, st, &c);
    for (;;) {
      int32_t begin = next.fetch_add(64);
      if (begin >= count) break;
      int32_t end = std::min(count, begin + 64);
      for (int32_t i = begin; i < end; i++) fn(i, tracer);
    }
    per[id] = c;
  };
  if (threads == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (int i = 0; i < threads; i++) pool.emplace_back(work, i);
    for (auto& th : pool) th.join();
  }
  for (auto& c : per) add_counters(counters, c);
}

}  // namespace

// ------------------------------------------------------------------ C API

extern "C" {

uint32_t oracle_hash(uint32_t x) { return hash32(x); }

void oracle_plant_draw_mistake(int32_t which) { g_planted_draw_mistake = which; }

uint32_t oracle_seed(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  Random r;
  r.seed(a, b, c, d);
  return r.state;
}

double oracle_random_next(uint32_t* state) {
  Random r;
  r.state = *state;
  double v = r.next();
  *state = r.state;
  return v;
}

double oracle_srgb_to_linear(double c) { return srgb_to_linear(c); }
double oracle_linear_to_srgb(double c) { return linear_to_srgb(c); }
double oracle_half_to_float(uint32_t h) { return half_to_float(h); }
void oracle_tone_map(double* c, int mapping, double exposure) { tone_map(c, mapping, exposure); }
uint8_t oracle_uint8_clamp(double v) { return uint8_clamp(v); }

void oracle_dfg(double roughness, double dot_nv, double* out) { dfg(roughness, dot_nv, out); }
double oracle_fresnel_weight(double x) { return fresnel_weight(x); }
double oracle_visibility_ggx(double a, double nl, double nv) { return visibility_ggx(a, nl, nv); }
double oracle_distribution_ggx(double a, double nh) { return distribution_ggx(a, nh); }
double oracle_blinn_phong(double s, double nh) { return blinn_phong(s, nh); }
double oracle_smoothstep(double e0, double e1, double x) { return smoothstep(e0, e1, x); }
double oracle_distance_attenuation(double d, double c, double k) { return distance_attenuation(d, c, k); }

void oracle_sample_texture(const mcrt_texture* texture, double u, double v, double* out4) {
  sample_texture(*texture, u, v, out4);
}

void oracle_sample_environment(const mcrt_environment* env, const mcrt_texture* textures, double dx, double dy,
                               double dz, double* out3) {
  sample_environment(*env, textures, dx, dy, dz, out3);
}

int32_t oracle_build_bvh(const float* triangles, int32_t count, float* bounds, int32_t* nodes, uint32_t* order) {
  return build_bvh(triangles, count, bounds, nodes, order);
}

int32_t oracle_build_bvh_bins(const float* triangles, int32_t count, int32_t bins, float* bounds, int32_t* nodes,
                              uint32_t* order) {
  return build_bvh(triangles, count, bounds, nodes, order, bins);
}

int32_t oracle_intersect_closest(const float* triangles, const uint8_t* sides, const float* bounds,
                                 const int32_t* nodes, int32_t node_count, const double* o, const double* d,
                                 double t_min, double t_max, int32_t cull, oracle_hit* out,
                                 oracle_counters* counters) {
  Bvh bvh{triangles, sides, bounds, nodes, node_count};
  Hit hit;
  int32_t stack[256];
  bool found = intersect_closest(bvh, o[0], o[1], o[2], d[0], d[1], d[2], t_min, t_max, cull != 0, hit, stack,
                                 counters);
  out->triangle = hit.triangle;
  out->front = hit.front;
  out->t = hit.t;
  out->u = hit.u;
  out->v = hit.v;
  return found ? 1 : 0;
}

int32_t oracle_intersect_any_count(const float* triangles, const float* bounds, const int32_t* nodes,
                                   int32_t node_count, const double* o, const double* d, double t_min,
                                   double t_max, oracle_counters* counters) {
  Bvh bvh{triangles, nullptr, bounds, nodes, node_count};
  int32_t stack[256];
  int32_t all = 0;
  intersect_any(bvh, o[0], o[1], o[2], d[0], d[1], d[2], t_min, t_max, stack, counters,
                [&all](int32_t, double, double, double, bool) {
                  all++;
                  return true;
                });
  return all;
}

// compileGeometry, compile.ts:327-403, and writeTangent, compile.ts:406-432.
int32_t oracle_compile_geometry(int32_t count, const double* p, const double* n, const double* uv,
                                const double* colors, const uint8_t* has_color, const uint32_t* materials,
                                const uint8_t* flags, const uint8_t* sides, float* triangles_out,
                                float* normals_out, float* uvs_out, float* tangents_out, float* colors_out,
                                uint32_t* materials_out, uint8_t* flags_out, uint8_t* sides_out,
                                float* bounds_out, int32_t* nodes_out, uint32_t* order_out,
                                int32_t* node_count_out, double* epsilon_out, int32_t* any_colors,
                                int32_t bins) {
  std::vector<float> tris(static_cast<size_t>(count) * 9);
  double max_coordinate = 0;
  bool any = false;
  for (int32_t i = 0; i < count; i++) {
    const double* pi = p + static_cast<size_t>(i) * 9;
    float* t = tris.data() + static_cast<size_t>(i) * 9;
    t[0] = fround(pi[0]); t[1] = fround(pi[1]); t[2] = fround(pi[2]);
    for (int k = 0; k < 3; k++) {
      t[3 + k] = fround(pi[3 + k] - pi[k]);
      t[6 + k] = fround(pi[6 + k] - pi[k]);
    }
    for (int k = 0; k < 9; k++) max_coordinate = std::max(max_coordinate, std::fabs(pi[k]));
    if (has_color && has_color[i]) any = true;
  }
  *any_colors = any ? 1 : 0;
  int32_t node_count = build_bvh(tris.data(), count, bounds_out, nodes_out, order_out, bins > 0 ? bins : kBins);
  *node_count_out = node_count;
  double min_x = kInf, min_y = kInf, min_z = kInf, max_x = -kInf, max_y = -kInf, max_z = -kInf;
  for (int32_t i = 0; i < count; i++) {
    const uint32_t s = order_out[i];
    std::memcpy(triangles_out + static_cast<size_t>(i) * 9, tris.data() + static_cast<size_t>(s) * 9, 9 * sizeof(float));
    for (int k = 0; k < 9; k++) normals_out[static_cast<size_t>(i) * 9 + k] = fround(n[static_cast<size_t>(s) * 9 + k]);
    for (int k = 0; k < 6; k++) uvs_out[static_cast<size_t>(i) * 6 + k] = fround(uv[static_cast<size_t>(s) * 6 + k]);
    if (any) {
      for (int k = 0; k < 12; k++) {
        colors_out[static_cast<size_t>(i) * 12 + k] =
            has_color[s] ? fround(colors[static_cast<size_t>(s) * 12 + k]) : 1.0f;
      }
    }
    materials_out[i] = materials[s];
    flags_out[i] = flags[s];
    sides_out[i] = sides[s];
    const float* o = triangles_out + static_cast<size_t>(i) * 9;
    for (int v = 0; v < 3; v++) {
      double x = static_cast<double>(o[0]) + (v == 1 ? o[3] : v == 2 ? o[6] : 0.0f);
      double y = static_cast<double>(o[1]) + (v == 1 ? o[4] : v == 2 ? o[7] : 0.0f);
      double z = static_cast<double>(o[2]) + (v == 1 ? o[5] : v == 2 ? o[8] : 0.0f);
      if (x < min_x) min_x = x;
      if (y < min_y) min_y = y;
      if (z < min_z) min_z = z;
      if (x > max_x) max_x = x;
      if (y > max_y) max_y = y;
      if (z > max_z) max_z = z;
    }
    // writeTangent
    const float* u6 = uvs_out + static_cast<size_t>(i) * 6;
    double e1x = o[3], e1y = o[4], e1z = o[5];
    double e2x = o[6], e2y = o[7], e2z = o[8];
    double du1 = static_cast<double>(u6[2]) - u6[0], dv1 = static_cast<double>(u6[3]) - u6[1];
    double du2 = static_cast<double>(u6[4]) - u6[0], dv2 = static_cast<double>(u6[5]) - u6[1];
    double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    double d = du1 * dv2 - du2 * dv1;
    double tx, ty, tz, sign = 1;
    if (std::fabs(d) > 1e-20) {
      double r = 1 / d;
      tx = (e1x * dv2 - e2x * dv1) * r; ty = (e1y * dv2 - e2y * dv1) * r; tz = (e1z * dv2 - e2z * dv1) * r;
      double bx = (e2x * du1 - e1x * du2) * r, by = (e2y * du1 - e1y * du2) * r, bz = (e2z * du1 - e1z * du2) * r;
      double cx = ny * tz - nz * ty, cy = nz * tx - nx * tz, cz = nx * ty - ny * tx;
      sign = cx * bx + cy * by + cz * bz < 0 ? -1 : 1;
    } else {
      if (std::fabs(nx) < 0.9 * js_hypot(nx, ny, nz)) {
        tx = 0; ty = -nz; tz = ny;
      } else {
        tx = nz; ty = 0; tz = -nx;
      }
    }
    double length = hypot_or_one(tx, ty, tz);
    float* tg = tangents_out + static_cast<size_t>(i) * 4;
    tg[0] = fround(tx / length); tg[1] = fround(ty / length); tg[2] = fround(tz / length);
    tg[3] = fround(sign);
  }
  double diagonal = count > 0 ? js_hypot(max_x - min_x, max_y - min_y, max_z - min_z) : 1;
  *epsilon_out = std::max(diagonal * 1e-5, std::max(max_coordinate * 2e-6, 1e-7));
  return 0;
}

void oracle_camera_ray(const mcrt_camera* camera, double x, double y, double* out6) {
  camera_ray(*camera, x, y, out6);
}

int32_t oracle_render_tile(const mcrt_geometry* geometry, const mcrt_shading* shading, const mcrt_camera* camera,
                           const mcrt_settings* settings, const mcrt_tile* tile, int32_t width, int32_t height,
                           int32_t pass, int32_t block, float* out, oracle_counters* counters) {
  Tracer tracer(*geometry, *shading, *settings, counters);
  tracer.render_tile(*camera, *tile, width, height, pass, block < 1 ? 1 : block, out);
  return 0;
}

void oracle_encode_tile(uint8_t* image, int32_t width, const mcrt_tile* tile, const float* data, float* sum,
                        int32_t count, int32_t srgb) {
  const double scale = 1.0 / count;
  for (int y = 0; y < tile->height; y++) {
    for (int x = 0; x < tile->width; x++) {
      const size_t s = (static_cast<size_t>(y) * tile->width + x) * 4;
      const size_t d = ((static_cast<size_t>(tile->y) + y) * width + tile->x + x) * 4;
      encode_pixel(image + d, data + s, sum ? sum + d : nullptr, scale, srgb != 0);
    }
  }
}

int32_t oracle_render_pixels(const mcrt_geometry* geometry, const mcrt_shading* shading, const mcrt_camera* camera,
                             const mcrt_settings* settings, int32_t width, int32_t height, int32_t samples,
                             int32_t srgb, int32_t count, const int32_t* px, const int32_t* py,
                             uint8_t* out_rgba, float* out_sum, int32_t threads, oracle_counters* counters) {
  if (samples < 1) samples = 1;
  parallel_pixels(*geometry, *shading, *settings, count, threads, counters, [&](int32_t i, Tracer& tracer) {
    float sum[4] = {0, 0, 0, 0};
    uint8_t rgba[4];
    double sample[4], ray[6];
    for (int pass = 0; pass < samples; pass++) {
      tracer.sample_one(*camera, px[i], py[i], width, height, pass, 1, sample, ray);
      float f[4] = {fround(sample[0]), fround(sample[1]), fround(sample[2]), fround(sample[3])};
      encode_pixel(rgba, f, sum, 1.0 / (pass + 1), srgb != 0);
    }
    std::memcpy(out_rgba + static_cast<size_t>(i) * 4, rgba, 4);
    if (out_sum) std::memcpy(out_sum + static_cast<size_t>(i) * 4, sum, sizeof(sum));
  });
  return 0;
}

int32_t oracle_raytrace(const mcrt_geometry* geometry, const mcrt_shading* shading, const mcrt_camera* camera,
                        const mcrt_settings* settings, int32_t width, int32_t height, int32_t samples,
                        int32_t srgb, uint8_t* out_rgba, int32_t threads, oracle_counters* counters) {
  const int32_t count = width * height;
  std::vector<int32_t> px(count), py(count);
  for (int32_t i = 0; i < count; i++) {
    px[i] = i % width;
    py[i] = i / width;
  }
  return oracle_render_pixels(geometry, shading, camera, settings, width, height, samples, srgb, count, px.data(),
                              py.data(), out_rgba, nullptr, threads, counters);
}

int32_t oracle_trace_primary(const mcrt_geometry* geometry, const mcrt_camera* camera, int32_t width,
                             int32_t height, int32_t pass, uint32_t seed, int32_t count, const int32_t* px,
                             const int32_t* py, int32_t* tri_out, double* t_out, double* u_out, double* v_out,
                             int32_t* front_out, double* rays_out, int32_t threads) {
  mcrt_shading empty{};
  mcrt_settings st{};
  st.seed = seed;
  parallel_pixels(*geometry, empty, st, count, threads, nullptr, [&](int32_t i, Tracer& tracer) {
    tracer.random.seed(static_cast<uint32_t>(px[i]), static_cast<uint32_t>(py[i]), static_cast<uint32_t>(pass), seed);
    double jx = 0.5, jy = 0.5;
    if (pass > 0) {
      jx = tracer.random.next();
      jy = tracer.random.next();
    }
    double sxp = (px[i] + jx) / width, syp = (py[i] + jy) / height;
    double ray[6];
    camera_ray(*camera, sxp * 2 - 1, 1 - syp * 2, ray);
    Hit hit;
    intersect_closest(tracer.bvh, ray[0], ray[1], ray[2], ray[3], ray[4], ray[5], 0, kInf, true, hit, tracer.stack,
                      nullptr);
    tri_out[i] = hit.triangle;
    t_out[i] = hit.t;
    if (u_out) u_out[i] = hit.u;
    if (v_out) v_out[i] = hit.v;
    if (front_out) front_out[i] = hit.front ? 1 : 0;
    if (rays_out) std::memcpy(rays_out + static_cast<size_t>(i) * 6, ray, sizeof(ray));
  });
  return 0;
}

}  // extern "C"
