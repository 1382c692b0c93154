/*
 * CPU oracle of the path tracer — TEST INFRASTRUCTURE ONLY (see oracle.h for
 * who may call it).
 *
 * Restates CPathIntegrator::Li and direct()
 * (raytracer/include/integrators/path_integrator_impl.hpp:23-247) for surface
 * scenes lit by the environment map, with the reference's materials
 * (material.hpp:67-100, microfacet_brdf.hpp:57-100, microfacet_distribution.hpp:40-141,
 * oren_nayar_brdf.hpp:36-81, fresnel.hpp:28-54), environment sampling
 * (environmentmap.hpp:28-55, distribution_1d.hpp:54-122, distribution_2d.hpp:50-84,
 * environmentmap.cu:16-29) and camera (camera.cu:20-37, pixel_sampler.hpp:36-47),
 * one path at a time, with the same Philox streams as the GPU wavefront.
 */
#ifndef R2_RENDER_ORACLE_H
#define R2_RENDER_ORACLE_H
#include <stdint.h>

#include "oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_mesh {
  const float* positions; /* model space, 3 per vertex */
  uint32_t nverts;
  const uint32_t* indices;
  uint32_t ntris;
  const float* normals;
  float model_to_world[12];
  orc_material material;
  const float* uvs;  /* nullable: 2 texture coordinates per vertex */
  /* texture maps of the material (nullable), CMaterial(aiMaterial*)
   * (material.cu:110-143): map_Kd, map_Ks, map_Bump, map_d */
  const orc_texture* albedo;
  const orc_texture* specular;
  const orc_texture* normal;
  const orc_texture* alpha;
  /* 0: a world-space mesh (flattened into the one-level BVH); k > 0: an
   * instance of mesh asset k, whose geometry, normals, texture coordinates and
   * material are those of the first mesh with this k (two-level scene). */
  uint32_t asset;
} orc_mesh;

typedef struct orc_shape {
  int type; /* 0 sphere, 1 circle */
  float center[3];
  float radius;
  float normal[3];
  orc_material material;
} orc_shape;

/* Medium of a filtered LOD: <path>.nvdb + <path>.brickgrid, placed with
 * T(pos) R(orientation) S(scaling) (sceneobject.cu:50-65). */
typedef struct orc_medium {
  const char* path;
  float sigma_a[3], sigma_s[3];
  float pos[3], orientation[3], scaling[3];
  int hg;  /* 1: Henyey-Greenstein phase function with asymmetry g instead of SGGX */
  float g;
} orc_medium;

typedef struct orc_camera {
  uint32_t width, height;
  float fov_deg;
  float pos[3], look_at[3], up[3];
} orc_camera;

/* Renders pixels [p0, p1) (row-major, row 0 = bottom) with spp samples.
 * rgb_out: 3 floats per pixel, the frame accumulation sum_s L_s / spp;
 * var_out (nullable): per pixel and channel, the unbiased sample variance of
 * L_s.  media (nullable): heterogeneous SGGX media; flags bit 0 selects the
 * brick-grid DDA tracking.  Returns 0 on success. */
int orc_render(const orc_mesh* meshes, uint32_t nmeshes, const orc_shape* shapes, uint32_t nshapes,
               const float* env_rgb, int env_w, int env_h, const orc_camera* cam, uint32_t spp, uint32_t max_depth,
               uint32_t seed, uint32_t p0, uint32_t p1, float* rgb_out, double* var_out, int threads,
               const orc_medium* media, uint32_t nmedia, uint32_t flags);

/* Test hook: while words is not NULL, the Philox blocks of a surface path are
 * taken from words in the order the path asks for them (render one pixel,
 * one sample, one thread); vec2_swap exchanges the GGX lobe's two direction
 * draws.  NULL restores the Philox streams. */
void orc_set_replay(const uint32_t* words, size_t n, int vec2_swap);

/* Natural logarithm of the tracking code (exposed for unit tests). */
float orc_t_log(float x);

/* Log-average tonemap, gamma and bytes of a linear W*H*3 frame (either output nullable). */
void orc_tonemap(const float* rgb, uint32_t W, uint32_t H, float gamma, float* out, uint8_t* bytes);

/* Environment sampling primitives, exposed for unit tests. */
int orc_env_sample(const float* env_rgb, int env_w, int env_h, float u0, float u1, float* dir_out, float* pdf_out,
                   float* le_out);
int orc_env_le(const float* env_rgb, int env_w, int env_h, const float* dir, float* pdf_out, float* le_out);
/* The same with the distributions built once: a handle from orc_env_create. */
void* orc_env_create(const float* env_rgb, int env_w, int env_h);
void orc_env_destroy(void* env);
void orc_env_sample_h(const void* env, float u0, float u1, float* dir_out, float* pdf_out, float* le_out);
void orc_env_le_h(const void* env, const float* dir, float* pdf_out, float* le_out);

#ifdef __cplusplus
}
#endif
#endif
