// Texture maps of a textured triangle's material at a hit, shared by the path
// tracer's shading and the filter's per-hit accumulation.
#pragma once
#include "texture.h"

namespace r2 {

__device__ __forceinline__ V3 tex_rgb(float4 v) { return v3(v.x, v.y, v.z); }

// The maps of a textured triangle's material at the hit (shaders.optix.cu:61-103,
// material.hpp:111-155): albedo and glossy colours, and the shading normal of the
// tangent-space normal map.  The tangent frame is built from the world-space
// triangle (the reference builds it in model space and transforms the mapped
// normal; the two agree for rigid and uniformly scaled objects).
struct TexView {
  const float2* uv;
  const float4* texels;
  const TexInfo* texInfo;
  const float4* tris;
};
struct TexShade {
  V3 n, diffuse, specular;
};
static __device__ __noinline__ TexShade textured_surface(TexView tv, int texAlbedo, int texGlossy, int texNormal, int tri,
                                                         float b1, float b2, V3 n, V3 diffuse, V3 specular) {
  TexShade r;
  r.n = n;
  r.diffuse = diffuse;
  r.specular = specular;
  const float2 t0 = __ldg(&tv.uv[3 * tri]), t1 = __ldg(&tv.uv[3 * tri + 1]), t2 = __ldg(&tv.uv[3 * tri + 2]);
  const float2 tc = tex_coord(t0, t1, t2, b1, b2);
  if (texAlbedo >= 0) r.diffuse = tex_rgb(tex_lookup(tv.texels, tv.texInfo[texAlbedo], tc.x, tc.y));
  if (texGlossy >= 0) r.specular = tex_rgb(tex_lookup(tv.texels, tv.texInfo[texGlossy], tc.x, tc.y));
  if (texNormal >= 0) {
    const V3 P0 = tex_rgb(__ldg(&tv.tris[3 * tri])), P1 = tex_rgb(__ldg(&tv.tris[3 * tri + 1]));
    const V3 P2 = tex_rgb(__ldg(&tv.tris[3 * tri + 2]));
    const float b0 = (1.0f - b1) - b2;
    const V3 P = P0 * b0 + P1 * b1 + P2 * b2;
    const V3 e1 = P1 - P, e2 = P2 - P;
    const float du1 = t1.x - tc.x, dv1 = t1.y - tc.y, du2 = t2.x - tc.x, dv2 = t2.y - tc.y;
    const float den = du1 * dv2 - du2 * dv1;
    if (den != 0.0f) {
      const float f = 1.0f / den;
      const V3 T = v3(f * (dv2 * e1.x - dv1 * e2.x), f * (dv2 * e1.y - dv1 * e2.y), f * (dv2 * e1.z - dv1 * e2.z));
      const V3 B = v3(f * (-du2 * e1.x + du1 * e2.x), f * (-du2 * e1.y + du1 * e2.y), f * (-du2 * e1.z + du1 * e2.z));
      const bool tz = T.x == 0.0f && T.y == 0.0f && T.z == 0.0f, bz = B.x == 0.0f && B.y == 0.0f && B.z == 0.0f;
      if (!tz && !bz) {
        const V3 c = tex_rgb(tex_lookup(tv.texels, tv.texInfo[texNormal], tc.x, tc.y));
        const V3 nt = v3(c.x * 2.0f - 1.0f, c.y * 2.0f - 1.0f, c.z * 2.0f - 1.0f);
        if (!(nt.x == 0.0f && nt.y == 0.0f && nt.z == 0.0f)) {
          const V3 v = normalize(nt);
          r.n = normalize(normalize(T) * v.x + normalize(-B) * v.y + n * v.z);
        }
      }
    }
  }
  return r;
}

}  // namespace r2
