/*
 * Internal helpers shared by the oracle's translation units (test
 * infrastructure only).  Float expressions keep the device code's order.
 */
#ifndef R2_ORACLE_INTERNAL_H
#define R2_ORACLE_INTERNAL_H
#include <math.h>
#include <stdint.h>

#include "oracle.h"

typedef struct { float x, y, z; } f3;
static inline f3 F3(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 add3(f3 a, f3 b) { return F3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub3(f3 a, f3 b) { return F3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 mul3(f3 a, f3 b) { return F3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline f3 mul3s(f3 a, float s) { return F3(a.x * s, a.y * s, a.z * s); }
static inline f3 div3s(f3 a, float s) { return F3(a.x / s, a.y / s, a.z / s); }
static inline f3 neg3(f3 a) { return F3(-a.x, -a.y, -a.z); }
static inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 cross3(f3 a, f3 b) {
  return F3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline float len3(f3 a) { return sqrtf(dot3(a, a)); }
static inline f3 norm3(f3 a) { return mul3s(a, 1.0f / sqrtf(dot3(a, a))); }
static inline float comp3(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline f3 abs3(f3 a) { return F3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }

/* glm mat4x3 * vec4(p, 1) / vec4(v, 0), left-to-right accumulation. */
static inline f3 xpoint(const float* m, f3 p) {
  return F3(m[0] * p.x + m[3] * p.y + m[6] * p.z + m[9] * 1.0f,
            m[1] * p.x + m[4] * p.y + m[7] * p.z + m[10] * 1.0f,
            m[2] * p.x + m[5] * p.y + m[8] * p.z + m[11] * 1.0f);
}
static inline f3 xvec(const float* m, f3 v) {
  return F3(m[0] * v.x + m[3] * v.y + m[6] * v.z + m[9] * 0.0f,
            m[1] * v.x + m[4] * v.y + m[7] * v.z + m[10] * 0.0f,
            m[2] * v.x + m[5] * v.y + m[8] * v.z + m[11] * 0.0f);
}

typedef struct { float t, b1, b2; int tri; } hit_t;

/* Closest (any_hit = 0) or first found (any_hit = 1) hit in (0, tmax]. */
hit_t oi_trace(const int32_t* nodes, const float* tris, f3 o, f3 d, float tmax, int any_hit);

/* Texture maps: float RGBA texels (4 per texel, row 0 = top), looked up at
 * normalized coordinates with wrap addressing and bilinear weights (the
 * reference's cudaAddressModeWrap + cudaFilterModeLinear texture objects,
 * raytracer/src/texture/texture.cu:176-189, with float weights). */
typedef struct { int W, H; float* texels; } oi_tex;
void oi_tex_lookup(const oi_tex* t, float u, float v, float out[4]);
/* Texel conversions of the reference's CTexture load paths (texture.cu:29-97,
 * 217-271, asset_manager.cu:165-184): rgb / 255 (a = 1); the alpha channel / 255
 * in rgb; the luma of rgb / 255 (luma.hpp:4-6).  Allocates out->texels. */
enum { OI_TEX_COLOR = 0, OI_TEX_ALPHA = 1, OI_TEX_LUMA = 2 };
void oi_tex_from(const orc_texture* src, int kind, oi_tex* out);
/* The texture indices {albedo, glossy, normal, opacity} (-1: none) of a
 * material and its maps (CMaterial(aiMaterial*), material.cu:110-143),
 * appending converted textures to tex[*ntex]. */
void oi_material_maps(const orc_material* m, const orc_texture* albedo, const orc_texture* specular,
                      const orc_texture* normal, const orc_texture* alpha, oi_tex* tex, int* ntex, int out[4]);
/* Albedo, glossy and normal-mapped normal at barycentrics (b1, b2) of a
 * textured triangle: uv6 its 3 texture coordinates, tri12 its 3 world-space
 * vertices (x y z w each), n the interpolated world normal
 * (shaders.optix.cu:61-103, material.hpp:111-155). */
void oi_textured_surface(const oi_tex* tex, int tAlbedo, int tGlossy, int tNormal, const float* uv6,
                         const float* tri12, float b1, float b2, f3* n, f3* diffuse, f3* specular);

/* Alpha test of triangles (__anyhit__mesh, shaders.optix.cu:132-152): per
 * BVH-order triangle its opacity map (-1: opaque) and 3 texture coordinates;
 * a hit where the map's red channel is 0 is ignored. */
typedef struct {
  const int* alpha_tex;
  const float* uv;  /* 6 per triangle */
  const oi_tex* tex;
} oi_alpha;
hit_t oi_trace_alpha(const int32_t* nodes, const float* tris, f3 o, f3 d, float tmax, int any_hit,
                     const oi_alpha* alpha);

static inline float oi_u01(uint32_t b) { return (float)(b >> 8) * (1.0f / 16777216.0f); }

/* 4x4 helpers (m[col][row]) */
typedef struct { float m[4][4]; } m4_t;
m4_t oi_m4_id(void);
m4_t oi_m4_mul(m4_t a, m4_t b);
m4_t oi_m4_inv(m4_t a);
void oi_m4_to43(m4_t a, float* f);

/* NanoVDB Vec4d grid file (volume_reader.c). */
typedef struct {
  uint8_t* buf; /* grid buffer */
  uint64_t size;
  float matF[9], vecF[3];   /* map, row-major */
  double worldBBox[6];
  int32_t indexBBox[6];     /* root bbox (inclusive) */
  uint64_t voxelCount;
  uint64_t rootOff, leafOff;
  uint32_t leafCount, tableSize;
  uint8_t background[32];
} oi_nvdb;
int oi_nvdb_read(const char* path, oi_nvdb* g);
void oi_nvdb_free(oi_nvdb* g);
/* ReadAccessor::getValue by a root/upper/lower/leaf walk (32-byte payload). */
void oi_nvdb_value(const oi_nvdb* g, int x, int y, int z, uint8_t out[32]);
float oi_nvdb_max_density(const oi_nvdb* g);

/* IEEE binary16 conversions: float to half bits, round to nearest even (as
 * glm::detail::toFloat16), and half bits to float (exact). */
uint16_t oi_half_bits(float f);
float oi_half_to_float(uint16_t h);

/* ".brickgrid" file (the reference's cereal PortableBinary layout). */
typedef struct {
  uint32_t nb[3], ad[3], count;
  float minorant, majorant;
  uint32_t *ind, *range, *mips[3];
  uint8_t* atlas;
} oi_bricks;
int oi_bricks_read(const char* path, oi_bricks* b);
void oi_bricks_free(oi_bricks* b);

#endif
