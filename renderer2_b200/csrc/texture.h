// Texture maps of OBJ materials as the reference's CTexture holds them
// (raytracer/src/texture/texture.cu:29-97, 217-271): float RGBA texels,
// row 0 = the file's top row, looked up at normalized coordinates with wrap
// addressing and bilinear filtering (the reference's cudaAddressModeWrap +
// cudaFilterModeLinear texture object, texture.cu:176-189; here the weights
// are full floats where the texture unit uses 8-bit fractions).
#pragma once
#include "r2_core.h"

namespace r2 {

// Kinds of texel conversion (CTexture's load paths).
enum TextureKind : int {
  kTexColor = 0,        // stbi_load with 3 channels: rgb / 255, a = 1 (albedo, specular, normal, map_d maps)
  kTexAlphaChannel = 1, // loadAlpha: the 4th channel / 255 in rgb, a = 1 (albedo with alpha, no map_d)
  kTexLuma = 2,         // specularFromDiffuse: luma of the rgb / 255 texels in rgb
};

struct TexInfo {
  uint32_t offset;  // first texel in the scene's texel array
  int W, H;
  int pad;
};

R2_HD float4 tex_texel(const float4* texels, const TexInfo& t, int x, int y) {
  x %= t.W;
  if (x < 0) x += t.W;
  y %= t.H;
  if (y < 0) y += t.H;
#if defined(__CUDA_ARCH__)
  return __ldg(&texels[t.offset + (size_t)y * t.W + x]);
#else
  return texels[t.offset + (size_t)y * t.W + x];
#endif
}

// tex2D<float4>(obj, u, v) of a wrap / linear / normalized-coordinate texture.
R2_HD float4 tex_lookup(const float4* texels, const TexInfo& t, float u, float v) {
  u = u - floorf(u);
  v = v - floorf(v);
  const float xb = u * (float)t.W - 0.5f, yb = v * (float)t.H - 0.5f;
  const float fx = floorf(xb), fy = floorf(yb);
  const float a = xb - fx, b = yb - fy;
  const int x0 = (int)fx, y0 = (int)fy;
  const float4 t00 = tex_texel(texels, t, x0, y0), t10 = tex_texel(texels, t, x0 + 1, y0);
  const float4 t01 = tex_texel(texels, t, x0, y0 + 1), t11 = tex_texel(texels, t, x0 + 1, y0 + 1);
  const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
  return make_float4(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
                     w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
                     w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z,
                     w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w);
}

// Texture coordinates at barycentrics (b1, b2): (1 - b1 - b2) TC0 + b1 TC1 + b2 TC2
// (shaders.optix.cu:61-66).
R2_HD float2 tex_coord(float2 t0, float2 t1, float2 t2, float b1, float b2) {
  const float b0 = (1.0f - b1) - b2;
  return make_float2(b0 * t0.x + b1 * t1.x + b2 * t2.x, b0 * t0.y + b1 * t1.y + b2 * t2.y);
}

}  // namespace r2
