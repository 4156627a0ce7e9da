/*
 * CPU oracle: a restatement of the reference ray tracer's hot path, for tests.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product calls this library; the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark use
 * it as the checker that the CUDA path is compared against.
 *
 * It follows the reference (VJigouline/MeerCADRaytracer, TypeScript) with
 * JavaScript numeric semantics: every computation in IEEE double, every
 * store into a Float32Array rounded to float, uint32 integer hashing, and
 * Uint8ClampedArray's clamp-then-round-half-to-even. Each function cites the
 * reference file:line it restates. Parity is pinned against the known-answer
 * tests of the reference's own test files (tests/<name>.test.ts), restated in
 * tests/test_oracle_*.py.
 */
#ifndef MCRT_ORACLE_H
#define MCRT_ORACLE_H

#include <stdint.h>
#include "../include/mcrt_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Hit, src/bvh.ts:186-194. */
typedef struct oracle_hit {
  int32_t triangle;
  int32_t front;
  double t;
  double u;
  double v;
} oracle_hit;

/* Work counters: BVH queries and the box / triangle tests they made. */
typedef struct oracle_counters {
  int64_t closest_queries;
  int64_t closest_boxes;
  int64_t closest_tris;
  int64_t any_queries;
  int64_t any_boxes;
  int64_t any_tris;
  int64_t samples;
} oracle_counters;

/* random.ts */
uint32_t oracle_hash(uint32_t x);
uint32_t oracle_seed(uint32_t a, uint32_t b, uint32_t c, uint32_t d);
double oracle_random_next(uint32_t* state);

/* color.ts */
double oracle_srgb_to_linear(double c);
double oracle_linear_to_srgb(double c);
double oracle_half_to_float(uint32_t h);
void oracle_tone_map(double* c, int mapping, double exposure);
uint8_t oracle_uint8_clamp(double v);

/* brdf.ts */
void oracle_dfg(double roughness, double dot_nv, double* out);
double oracle_fresnel_weight(double dot_vh);
double oracle_visibility_ggx(double alpha, double dot_nl, double dot_nv);
double oracle_distribution_ggx(double alpha, double dot_nh);
double oracle_blinn_phong(double shininess, double dot_nh);
double oracle_smoothstep(double e0, double e1, double x);
double oracle_distance_attenuation(double distance, double cutoff, double decay);

/* textures.ts */
void oracle_sample_texture(const mcrt_texture* texture, double u, double v, double* out4);
void oracle_sample_environment(const mcrt_environment* env, const mcrt_texture* textures,
                               double dx, double dy, double dz, double* out3);

/* Test only: plants mistake `which` (1-6, see oracle.cpp) in the order the
 * path loop draws random numbers; 0 restores the reference's order. Process
 * wide: set it only while no render runs. */
void oracle_plant_draw_mistake(int32_t which);

/* bvh.ts. Output arrays hold max(1, 2 * count - 1) nodes; returns nodeCount. */
int32_t oracle_build_bvh(const float* triangles, int32_t count, float* bounds, int32_t* nodes,
                         uint32_t* order);
/* The same build with `bins` bins per axis (bvh.ts:3's BINS; 2 to 64). */
int32_t oracle_build_bvh_bins(const float* triangles, int32_t count, int32_t bins, float* bounds,
                              int32_t* nodes, uint32_t* order);
int32_t oracle_intersect_closest(const float* triangles, const uint8_t* sides, const float* bounds,
                                 const int32_t* nodes, int32_t node_count, const double* origin,
                                 const double* direction, double t_min, double t_max, int32_t cull,
                                 oracle_hit* hit, oracle_counters* counters);
/* Number of hits intersectAny visits between t_min and t_max. */
int32_t oracle_intersect_any_count(const float* triangles, const float* bounds, const int32_t* nodes,
                                   int32_t node_count, const double* origin, const double* direction,
                                   double t_min, double t_max, oracle_counters* counters);

/*
 * compile.ts compileGeometry's sink, reorder, tangents and epsilon
 * (src/compile.ts:327-432), from flattened world-space triangles:
 * p (9 doubles), n (9), uv (6) per triangle, colors (12) per triangle with
 * has_color[k] saying whether triangle k carried vertex colours.
 * Outputs are sized for `count` triangles and max(1, 2 count - 1) nodes;
 * colors_out is written only if any triangle has colours (returned in *any_colors).
 * `bins`: SAH bins per axis of the BVH build (16 as the reference; 0 means 16).
 */
int32_t oracle_compile_geometry(int32_t count, const double* p, const double* n, const double* uv,
                                const double* colors, const uint8_t* has_color,
                                const uint32_t* materials, const uint8_t* flags, const uint8_t* sides,
                                float* triangles_out, float* normals_out, float* uvs_out,
                                float* tangents_out, float* colors_out, uint32_t* materials_out,
                                uint8_t* flags_out, uint8_t* sides_out, float* bounds_out,
                                int32_t* nodes_out, uint32_t* order_out, int32_t* node_count_out,
                                double* epsilon_out, int32_t* any_colors, int32_t bins);

/* tracer.ts cameraRay (src/tracer.ts:705-727): origin then direction. */
void oracle_camera_ray(const mcrt_camera* camera, double x, double y, double* out6);

/* Tracer.renderTile, src/tracer.ts:62-89. out holds tile.width * tile.height * 4 floats. */
int32_t oracle_render_tile(const mcrt_geometry* geometry, const mcrt_shading* shading,
                           const mcrt_camera* camera, const mcrt_settings* settings,
                           const mcrt_tile* tile, int32_t width, int32_t height, int32_t pass,
                           int32_t block, float* out, oracle_counters* counters);

/* writeTile / encodeTile, src/progressive.ts:288-313. `sum` may be NULL. */
void oracle_encode_tile(uint8_t* image, int32_t width, const mcrt_tile* tile, const float* data,
                        float* sum, int32_t count, int32_t srgb);

/*
 * raytraceCompiled (src/raytrace.ts:69-82) restricted to a list of pixels:
 * each pixel gets passes 0 .. samples-1 and the final encode, exactly as the
 * full image would give it (pixels are independent). out_rgba holds 4 bytes
 * and out_sum (may be NULL) 4 floats per listed pixel. Runs on `threads`
 * host threads.
 */
int32_t oracle_render_pixels(const mcrt_geometry* geometry, const mcrt_shading* shading,
                             const mcrt_camera* camera, const mcrt_settings* settings, int32_t width,
                             int32_t height, int32_t samples, int32_t srgb, int32_t count,
                             const int32_t* px, const int32_t* py, uint8_t* out_rgba, float* out_sum,
                             int32_t threads, oracle_counters* counters);

/* raytraceCompiled over the whole image: width * height * 4 bytes. */
int32_t oracle_raytrace(const mcrt_geometry* geometry, const mcrt_shading* shading,
                        const mcrt_camera* camera, const mcrt_settings* settings, int32_t width,
                        int32_t height, int32_t samples, int32_t srgb, uint8_t* out_rgba,
                        int32_t threads, oracle_counters* counters);

/*
 * Closest hit of each listed pixel's camera ray for one pass (the ray
 * renderTile would trace first), culling as samplePixel does. rays_out
 * (6 doubles per pixel, may be NULL) receives the ray.
 */
int32_t oracle_trace_primary(const mcrt_geometry* geometry, const mcrt_camera* camera,
                             int32_t width, int32_t height, int32_t pass, uint32_t seed,
                             int32_t count, const int32_t* px, const int32_t* py, int32_t* tri_out,
                             double* t_out, double* u_out, double* v_out, int32_t* front_out,
                             double* rays_out, int32_t threads);

#ifdef __cplusplus
}
#endif

#endif /* MCRT_ORACLE_H */
