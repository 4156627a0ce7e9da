/*
 * Plain-data form of a compiled scene, as the ray tracer consumes it.
 *
 * Every struct here mirrors a type of the reference's data contract,
 * src/types.ts (file:line cited per struct), field for field and in the same
 * units, so that a compiled scene produced by the reference's compileScene
 * (src/compile.ts:513-527) can be handed over without reinterpretation:
 *   - JavaScript numbers (materials, lights, cameras, settings) are doubles;
 *   - typed arrays (triangles, normals, uvs, BVH) keep their element types
 *     and their per-triangle / per-node strides.
 * Enumerations use the reference's three.js constant values
 * (src/constants.ts:5-44) where the reference uses them, and small integers
 * (documented beside each field) where the reference uses string unions.
 *
 * Pointers are borrowed for the duration of the call they are passed to.
 */
#ifndef MCRT_TYPES_H
#define MCRT_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Triangle flag bits, src/types.ts:133-135. */
#define MCRT_TRI_OPAQUE 1
#define MCRT_TRI_CAST_SHADOW 2
#define MCRT_TRI_RECEIVE_SHADOW 4

/* three.js sides, src/constants.ts:5-7. */
#define MCRT_FRONT_SIDE 0
#define MCRT_BACK_SIDE 1
#define MCRT_DOUBLE_SIDE 2

/* three.js environment combine operations, src/constants.ts:9-11. */
#define MCRT_MULTIPLY_OPERATION 0
#define MCRT_MIX_OPERATION 1
#define MCRT_ADD_OPERATION 2

/* three.js tone mapping constants, src/constants.ts:13-20. */
#define MCRT_NO_TONE_MAPPING 0
#define MCRT_LINEAR_TONE_MAPPING 1
#define MCRT_REINHARD_TONE_MAPPING 2
#define MCRT_CINEON_TONE_MAPPING 3
#define MCRT_ACES_FILMIC_TONE_MAPPING 4
#define MCRT_CUSTOM_TONE_MAPPING 5
#define MCRT_AGX_TONE_MAPPING 6
#define MCRT_NEUTRAL_TONE_MAPPING 7

/* three.js wrapping modes, src/constants.ts:29-31. */
#define MCRT_REPEAT_WRAPPING 1000
#define MCRT_CLAMP_TO_EDGE_WRAPPING 1001
#define MCRT_MIRRORED_REPEAT_WRAPPING 1002

/* CompiledMaterial.model, src/types.ts:41. */
#define MCRT_MODEL_PHYSICAL 0
#define MCRT_MODEL_PHONG 1
#define MCRT_MODEL_LAMBERT 2
#define MCRT_MODEL_TOON 3
#define MCRT_MODEL_BASIC 4

/* CompiledLight.type, src/types.ts:91-113. */
#define MCRT_LIGHT_AMBIENT 0
#define MCRT_LIGHT_HEMISPHERE 1
#define MCRT_LIGHT_DIRECTIONAL 2
#define MCRT_LIGHT_POINT 3
#define MCRT_LIGHT_SPOT 4

/* CompiledBackground.kind, src/types.ts:123-127. */
#define MCRT_BACKGROUND_CLEAR 0
#define MCRT_BACKGROUND_COLOR 1
#define MCRT_BACKGROUND_SCREEN 2
#define MCRT_BACKGROUND_ENVIRONMENT 3

/* CompiledFog.kind, src/types.ts:115-121 (0 stands for `fog: null`). */
#define MCRT_FOG_NONE 0
#define MCRT_FOG_LINEAR 1
#define MCRT_FOG_EXP2 2

/* CompiledEnvironment.kind, src/types.ts:23-39. */
#define MCRT_ENV_CUBE 0
#define MCRT_ENV_EQUIRECT 1

/* TraceSettings.shadows, src/types.ts:195. */
#define MCRT_SHADOWS_ALL 0
#define MCRT_SHADOWS_CAST_SHADOW 1
#define MCRT_SHADOWS_NONE 2

/* Texel formats of CompiledTexture.data, src/types.ts:12. */
#define MCRT_TEXEL_RGBA8 0   /* Uint8Array */
#define MCRT_TEXEL_RGBA32F 1 /* Float32Array */

/* CompiledTexture, src/types.ts:8-21. */
typedef struct mcrt_texture {
  int32_t width;
  int32_t height;
  int32_t format; /* MCRT_TEXEL_* */
  int32_t srgb;
  int32_t flip_y;
  int32_t wrap_s;
  int32_t wrap_t;
  int32_t id; /* TextureRef.id of src/protocol.ts:16; free for direct use */
  double matrix[9]; /* column-major 3 x 3 uv transform */
  const void* data; /* width * height * 4 texels, first row first */
} mcrt_texture;

/* CompiledEnvironment, src/types.ts:23-39. */
typedef struct mcrt_environment {
  int32_t kind; /* MCRT_ENV_* */
  int32_t faces[6]; /* cube: texture indices +x, -x, +y, -y, +z, -z */
  int32_t texture;  /* equirect: texture index */
  int32_t flip_x;   /* cube only */
  double rotation[9];
  double intensity;
} mcrt_environment;

/* CompiledMaterial, src/types.ts:43-89. */
typedef struct mcrt_material {
  int32_t model; /* MCRT_MODEL_* */
  int32_t side;
  double color[3];
  double opacity;
  int32_t transparent;
  int32_t vertex_colors;
  double alpha_test;
  int32_t flat_shading;
  int32_t tone_mapped;
  int32_t map;
  int32_t alpha_map;
  int32_t emissive_map;
  int32_t normal_map;
  int32_t ao_map;
  int32_t roughness_map;
  int32_t metalness_map;
  int32_t physical;
  double emissive[3];
  double normal_scale[2];
  double ao_map_intensity;
  double roughness;
  double metalness;
  double ior;
  double specular_intensity;
  double specular_color[3];
  double transmission;
  double thickness;
  double attenuation[3];
  double shininess;
  double specular[3];
  int32_t env_map;
  int32_t combine;
  double env_map_intensity;
  double reflectivity;
} mcrt_material;

/* CompiledLight, src/types.ts:91-113. Unused fields of a light type are 0. */
typedef struct mcrt_light {
  int32_t type; /* MCRT_LIGHT_* */
  int32_t cast_shadow;
  double color[3];
  double ground_color[3];
  double direction[3];
  double position[3];
  double distance;
  double decay;
  double cone_cos;
  double penumbra_cos;
} mcrt_light;

/* CompiledFog, src/types.ts:115-121. */
typedef struct mcrt_fog {
  int32_t kind; /* MCRT_FOG_* */
  int32_t pad_;
  double color[3];
  double near_;
  double far_;
  double density;
} mcrt_fog;

/* CompiledBackground, src/types.ts:123-127. */
typedef struct mcrt_background {
  int32_t kind; /* MCRT_BACKGROUND_* */
  int32_t texture;
  int32_t environment;
  int32_t pad_;
  double color[3];
  double intensity;
} mcrt_background;

/* CompiledGeometry + CompiledBvh, src/types.ts:137-167. */
typedef struct mcrt_geometry {
  int32_t triangle_count;
  int32_t node_count;
  const float* triangles;    /* 9 per triangle: v0, v1 - v0, v2 - v0 */
  const float* normals;      /* 9 per triangle */
  const float* uvs;          /* 6 per triangle */
  const float* tangents;     /* 4 per triangle */
  const float* colors;       /* 12 per triangle, or NULL when empty */
  const uint32_t* materials; /* 1 per triangle */
  const uint8_t* flags;      /* 1 per triangle, MCRT_TRI_* bits */
  const uint8_t* sides;      /* 1 per triangle, culled side */
  const float* bvh_bounds;   /* 6 per node: min xyz, max xyz */
  const int32_t* bvh_nodes;  /* 3 per node: first, count, axis */
  double epsilon;
} mcrt_geometry;

/* The shading half of CompiledScene (src/types.ts:169-179), as the
 * ShadingPayload of src/protocol.ts:19-27 plus texture pixels. */
typedef struct mcrt_shading {
  int32_t material_count;
  int32_t texture_count;
  int32_t environment_count;
  int32_t light_count;
  const mcrt_material* materials;
  const mcrt_texture* textures;
  const mcrt_environment* environments;
  const mcrt_light* lights;
  mcrt_background background;
  mcrt_fog fog;
  int32_t environment; /* scene.environment index, or -1 */
  int32_t pad_;
} mcrt_shading;

/* CompiledCamera, src/types.ts:181-190. */
typedef struct mcrt_camera {
  double projection_inverse[16]; /* column-major */
  double world[16];              /* column-major */
  int32_t orthographic;
  int32_t pad_;
  double forward[3];
  double position[3];
} mcrt_camera;

/* TraceSettings, src/types.ts:193-204. `seed` is the JavaScript number after
 * ToUint32, which is what the reference's integer hash sees of it. */
typedef struct mcrt_settings {
  int32_t max_bounces;
  int32_t shadows; /* MCRT_SHADOWS_* */
  int32_t global_illumination;
  int32_t tone_mapping;
  double tone_mapping_exposure;
  double clear_color[3];
  double clear_alpha;
  uint32_t seed;
  int32_t pad_;
} mcrt_settings;

/* Tile, src/types.ts:206-211. */
typedef struct mcrt_tile {
  int32_t x;
  int32_t y;
  int32_t width;
  int32_t height;
} mcrt_tile;

#ifdef __cplusplus
}
#endif

#endif /* MCRT_TYPES_H */
