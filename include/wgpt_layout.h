/*
 * Byte layouts of the buffers the drop-in accepts.  They are the reference's own packed layouts,
 * unchanged: the WGSL structs in shader.wgsl / denoiser.wgsl (std430-style storage layout) as
 * filled by tracer.js's packDataFromSchema.  All fields are little-endian 32-bit.
 *
 *   struct                 bytes  WGSL definition            JS packer
 *   wgpt_scene_params        112  shader.wgsl:23-33          tracer.js:2207-2240 (updateUniforms)
 *   wgpt_material            144  shader.wgsl:35-54          tracer.js:258-297   (Material.getSchema)
 *   wgpt_object               96  shader.wgsl:56-63          tracer.js:478-489, 525-536, 672-683,
 *                                                              774-785, 1406-1417 (getSchema)
 *   wgpt_plane                32  shader.wgsl:65-70          tracer.js:902-910
 *   wgpt_mesh_instance        80  shader.wgsl:94-100         tracer.js:1406-1417 packs 96 B (!)
 *   wgpt_bvh_node             32  shader.wgsl:102-107        tracer.js:1592-1618 (TLAS),
 *                                                              tracer.js:1857-1866 (BLAS)
 *   wgpt_triangle            128  shader.wgsl:84-92          tracer.js:1867-1871
 *   wgpt_light                80  shader.wgsl:109-115        tracer.js:1703-1711
 *   wgpt_gbuffer_texel        48  shader.wgsl:2497-2505      (written by gbuf_main)
 *   wgpt_denoise_uniforms     48  denoiser.wgsl:1-14         tracer.js:2560-2581
 */
#ifndef WGPT_LAYOUT_H
#define WGPT_LAYOUT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct wgpt_scene_params {
  float eye[3];
  uint32_t sample_number;
  float ray00[3];
  uint32_t width;
  float ray10[3];
  uint32_t height;
  float ray01[3];
  float exposure;
  float ray11[3];
  uint32_t seed;
  uint32_t sky_width;
  uint32_t sky_height;
  float sky_total_lum;
  float total_light_power;
  uint32_t section[2];
  uint32_t sky_cdf_index;
  float pad0;
} wgpt_scene_params;

typedef struct wgpt_material {
  float color[3];
  float metallic;
  float roughness;
  float ior;
  float specular_tint;
  float anisotropic;
  float aniso_rotation;
  float sheen;
  float sheen_tint;
  float clearcoat;
  float clearcoat_gloss;
  float clearcoat_ior;
  float transmission;
  float concentration;
  float subsurface_tint[3];
  float subsurface;
  float emittance[3];
  int32_t emissive_idx;
  int32_t albedo_idx;
  int32_t normal_idx;
  int32_t height_idx;
  int32_t roughness_idx;
  int32_t metallic_idx;
  float pad1;
  float uv_scale[2];
  float height_params[4];
} wgpt_material;

/* object_type: 0 mesh instance (param0/param1 = bitcast u32 node/tri offsets), 1 sphere, 2 cube,
   3 cylinder (param0 = top radius ratio), 4 torus (param0 = inner radius ratio). */
typedef struct wgpt_object {
  float inv_matrix[16]; /* column-major */
  int32_t material_idx;
  int32_t light_idx;
  int32_t object_type;
  float param0;
  float world_position[3];
  float param1;
} wgpt_object;

typedef struct wgpt_plane {
  float normal[3];
  float d;
  int32_t material_idx;
  float pad[3];
} wgpt_plane;

typedef struct wgpt_mesh_instance {
  float inv_matrix[16];
  int32_t material_idx;
  int32_t pad;
  uint32_t node_offset;
  uint32_t tri_offset;
} wgpt_mesh_instance;

/* num_triangles > 0: leaf.  TLAS leaf: next = object index; TLAS inner: next = right child
   (absolute).  BLAS: next = right child relative to the mesh's node offset, or first triangle
   relative to its triangle offset.  The left child is always the next node (index + 1). */
typedef struct wgpt_bvh_node {
  float aabb_min[3];
  uint32_t num_triangles;
  float aabb_max[3];
  uint32_t next;
} wgpt_bvh_node;

typedef struct wgpt_triangle {
  float v0[3]; float pad0;
  float v1[3]; float pad1;
  float v2[3]; float pad2;
  float n0[3]; float pad3;
  float n1[3]; float pad4;
  float n2[3]; float pad5;
  float uv0[2];
  float uv1[2];
  float uv2[2];
  float pad6[2];
} wgpt_triangle;

typedef struct wgpt_light {
  int32_t obj_idx;
  float area;
  float power;
  float scale;
  float matrix[16];
} wgpt_light;

typedef struct wgpt_gbuffer_texel {
  float normal[3];
  float roughness;
  float albedo[3];
  float metallic;
  float motion[2];
  float transmission;
  float dist;
} wgpt_gbuffer_texel;

typedef struct wgpt_denoise_uniforms {
  uint32_t width;
  uint32_t height;
  uint32_t step_width;
  uint32_t passes;
  float sigma_color;
  float sigma_normal;
  float sigma_depth;
  float sigma_albedo;
  float sigma_material;
  float glossy_protect;
  float exposure;
  uint32_t flags; /* bit 0: 3x3 median prepass, bit 1: albedo demodulation */
} wgpt_denoise_uniforms;

/* Pipeline override constants 1..11 of shader.wgsl:1-12 as bits (constant 0, BOUNCE_LIMIT, is
   passed separately). */
enum {
  WGPT_HAS_SPHERES = 1u << 0,
  WGPT_HAS_CUBES = 1u << 1,
  WGPT_HAS_PLANES = 1u << 2,
  WGPT_HAS_CYLINDERS = 1u << 3,
  WGPT_HAS_TORI = 1u << 4,
  WGPT_HAS_MESHES = 1u << 5,
  WGPT_HAS_LIST_MESHES = 1u << 6,
  WGPT_HAS_HEIGHTMAPS = 1u << 7,
  WGPT_HAS_LIGHTS = 1u << 8,
  WGPT_HAS_SKYBOX = 1u << 9,
  WGPT_MIS_SKYBOX = 1u << 10
};

#define WGPT_STRIDE_MATERIAL 144u
#define WGPT_STRIDE_OBJECT 96u
#define WGPT_STRIDE_PLANE 32u
#define WGPT_STRIDE_MESH_READ 80u   /* what the shader reads */
#define WGPT_STRIDE_MESH_PACKED 96u /* what tracer.js packs */
#define WGPT_STRIDE_NODE 32u
#define WGPT_STRIDE_TRIANGLE 128u
#define WGPT_STRIDE_LIGHT 80u
#define WGPT_STRIDE_GBUFFER 48u

#ifdef __cplusplus
}  /* extern "C" */
static_assert(sizeof(wgpt_scene_params) == 112, "SceneParams is 112 bytes");
static_assert(sizeof(wgpt_material) == 144, "Material is 144 bytes");
static_assert(sizeof(wgpt_object) == 96, "TransformedObject is 96 bytes");
static_assert(sizeof(wgpt_plane) == 32, "Plane is 32 bytes");
static_assert(sizeof(wgpt_mesh_instance) == 80, "MeshInstance is 80 bytes");
static_assert(sizeof(wgpt_bvh_node) == 32, "BVHNode is 32 bytes");
static_assert(sizeof(wgpt_triangle) == 128, "Triangle is 128 bytes");
static_assert(sizeof(wgpt_light) == 80, "Light is 80 bytes");
static_assert(sizeof(wgpt_gbuffer_texel) == 48, "GBufferData is 48 bytes");
static_assert(sizeof(wgpt_denoise_uniforms) == 48, "denoiser Uniforms is 48 bytes");
#endif

#endif /* WGPT_LAYOUT_H */
