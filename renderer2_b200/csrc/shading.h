// Surface scattering, environment light and camera of the path tracer
// (device + host), restating the reference's DH headers:
//   fresnel.hpp:28-54, microfacet_distribution.hpp:40-141, microfacet_brdf.hpp:57-100,
//   oren_nayar_brdf.hpp:36-81, material.hpp:67-100, brdf_functions.hpp:7-53,
//   objects.hpp:28-76 (CCoordinateFrame), environmentmap.hpp:28-55,
//   distribution_1d.hpp:54-122, distribution_2d.hpp:50-84, pixel_sampler.hpp:36-47,
//   ray.hpp:41-91, functions.hpp:10-27 and 94-126.
// Trigonometry of sampled angles goes through sincos_turns (bit-identical on
// host and device); acos/atan2 appear only in the environment lookup le().
#pragma once
#include <float.h>

#include "r2_core.h"
#include "../../include/r2.h"

namespace r2 {

constexpr float kRayOffset = 1e-4f;   // CRay::OFFSET
constexpr float kDefaultTmax = 1e12f; // CRay::DEFAULT_TMAX
constexpr float kPi = 3.14159265358979323846f;
constexpr double kPiD = 3.14159265358979323846;     // M_PI
constexpr double kInvPiD = 0.318309886183790671538; // M_1_PI

// ---------------------------------------------------------------- brdf_functions.hpp
R2_HD float cos_theta(V3 w) { return w.z; }
R2_HD float cos2_theta(V3 w) { return w.z * w.z; }
R2_HD float abs_cos_theta(V3 w) { return fabsf(w.z); }
R2_HD float sin2_theta(V3 w) { return fmaxf(0.0f, 1.0f - cos2_theta(w)); }
R2_HD float sin_theta(V3 w) { return sqrtf(sin2_theta(w)); }
R2_HD float tan_theta(V3 w) { return sin_theta(w) / cos_theta(w); }
R2_HD float tan2_theta(V3 w) { return sin2_theta(w) / cos2_theta(w); }
R2_HD float cos_phi(V3 w) {
  float s = sin_theta(w);
  return (s == 0.0f) ? 1.0f : clampf(w.x / s, -1.0f, 1.0f);
}
R2_HD float sin_phi(V3 w) {
  float s = sin_theta(w);
  return (s == 0.0f) ? 0.0f : clampf(w.y / s, -1.0f, 1.0f);
}
R2_HD float cos2_phi(V3 w) { float c = cos_phi(w); return c * c; }
R2_HD float sin2_phi(V3 w) { float s = sin_phi(w); return s * s; }
R2_HD bool same_hemisphere(V3 a, V3 b) { return a.z * b.z > 0.0f; }

// ---------------------------------------------------------------- fresnel.hpp
R2_HD float fresnel_dielectric(float etaI0, float etaT0, float cosThetaI) {
  cosThetaI = clampf(cosThetaI, -1.0f, 1.0f);
  float etaI = etaI0, etaT = etaT0;
  if (!(cosThetaI > 0.0f)) {
    etaI = etaT0;
    etaT = etaI0;
    cosThetaI = fabsf(cosThetaI);
  }
  float sinThetaI = sqrtf(fmaxf(0.0f, 1.0f - cosThetaI * cosThetaI));
  float sinThetaT = etaI / etaT * sinThetaI;
  if (sinThetaT >= 1.0f) return 1.0f;
  float cosThetaT = sqrtf(fmaxf(0.0f, 1.0f - sinThetaT * sinThetaT));
  float rPar = ((etaT * cosThetaI) - (etaI * cosThetaT)) / ((etaT * cosThetaI) + (etaI * cosThetaT));
  float rPer = ((etaI * cosThetaI) - (etaT * cosThetaT)) / ((etaI * cosThetaI) + (etaT * cosThetaT));
  return (rPar * rPar + rPer * rPer) / 2.0f;
}

// ---------------------------------------------------------------- microfacet_distribution.hpp (GGX)
struct Ggx {
  float ax, ay;
};

R2_HD float ggx_D(const Ggx& g, V3 h) {
  float t2 = tan2_theta(h);
  if (isinf(t2)) return 0.0f;
  float c2 = cos2_theta(h);
  float c4 = c2 * c2;
  float e = (cos2_phi(h) / (g.ax * g.ax) + sin2_phi(h) / (g.ay * g.ay)) * t2;
  // the reference multiplies by M_PI (double), so the denominator is double
  return (float)(1.0 / (kPiD * (double)g.ax * (double)g.ay * (double)c4 * (double)(1.0f + e) * (double)(1.0f + e)));
}

R2_HD float ggx_lambda(const Ggx& g, V3 w) {
  float absTan = fabsf(tan_theta(w));
  if (isinf(absTan)) return 0.0f;
  float alpha = sqrtf(cos2_phi(w) * g.ax * g.ax + sin2_phi(w) * g.ay * g.ay);
  float a2t2 = (alpha * absTan) * (alpha * absTan);
  return (-1.0f + sqrtf(1.0f + a2t2)) / 2.0f;
}

R2_HD float ggx_G(const Ggx& g, V3 wo, V3 wi) { return 1.0f / (1.0f + ggx_lambda(g, wo) + ggx_lambda(g, wi)); }
R2_HD float ggx_G1(const Ggx& g, V3 w) { return 1.0f / (1.0f + ggx_lambda(g, w)); }

// sample11: slope sampling of the visible normals for a unit-roughness GGX
// (Heitz and d'Eon 2014; the rational fit of the reference, lines 72-112).
R2_HD void ggx_sample11(float cosTheta, float u1, float u2, float* slopeX, float* slopeY) {
  if (cosTheta > 0.9999f) {
    float r = sqrtf(u1 / (1.0f - u1));
    float s, c;
    sincos_turns(u2, &s, &c);
    *slopeX = r * c;
    *slopeY = r * s;
    return;
  }
  float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
  float tanTheta = sinTheta / cosTheta;
  float a = 1.0f / tanTheta;
  float G1 = 2.0f / (1.0f + sqrtf(1.0f + 1.0f / (a * a)));
  float A = 2.0f * u1 / G1 - 1.0f;
  float tmp = 1.0f / (A * A - 1.0f);
  if (tmp > 1e10f) tmp = 1e10f;
  float B = tanTheta;
  float D = sqrtf(fmaxf(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.0f));
  float sx1 = B * tmp - D;
  float sx2 = B * tmp + D;
  *slopeX = (A < 0.0f || sx2 > 1.0f / tanTheta) ? sx1 : sx2;
  float S;
  if (u2 > 0.5f) {
    S = 1.0f;
    u2 = 2.0f * (u2 - 0.5f);
  } else {
    S = -1.0f;
    u2 = 2.0f * (0.5f - u2);
  }
  float z = (u2 * (u2 * (u2 * 0.27385f - 0.73369f) + 0.46341f)) /
            (u2 * (u2 * (u2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
  *slopeY = S * z * sqrtf(1.0f + *slopeX * *slopeX);
}

R2_HD V3 ggx_sample_vis(const Ggx& g, V3 wi, float u1, float u2) {
  V3 ws = normalize(v3(g.ax * wi.x, g.ay * wi.y, wi.z));
  float sx, sy;
  ggx_sample11(cos_theta(ws), u1, u2, &sx, &sy);
  float tmp = cos_phi(ws) * sx - sin_phi(ws) * sy;
  sy = sin_phi(ws) * sx + cos_phi(ws) * sy;
  sx = tmp;
  sx = g.ax * sx;
  sy = g.ay * sy;
  return normalize(v3(-sx, -sy, 1.0f));
}

R2_HD V3 ggx_sample_h(const Ggx& g, V3 wo, float u1, float u2) {
  bool flip = wo.z < 0.0f;
  V3 h = ggx_sample_vis(g, flip ? -wo : wo, u1, u2);
  if (flip) h = -h;
  return h;
}

R2_HD float ggx_pdf(const Ggx& g, V3 wo, V3 wh) {
  return ggx_D(g, wh) * ggx_G1(g, wo) * fabsf(dot(wo, wh)) / abs_cos_theta(wo);
}

R2_HD V3 reflect(V3 i, V3 n) { return i - n * (dot(n, i) * 2.0f); }

// ---------------------------------------------------------------- microfacet_brdf.hpp
struct Material {
  V3 diffuse, specular;  // CMaterial::m_diffuseColor, m_glossyColor
  float onA, onB;        // Oren-Nayar coefficients
  Ggx ggx;
  float etaI, etaT;      // CFresnel of the microfacet BRDF
  int tex[4];            // texture maps: albedo, glossy, normal, opacity (-1: none)
};

R2_HD Material make_material(const r2_material& m) {
  Material r;
  r.diffuse = v3(m.diffuse[0], m.diffuse[1], m.diffuse[2]);
  r.specular = v3(m.specular[0], m.specular[1], m.specular[2]);
  float s2 = m.diffuse_roughness * m.diffuse_roughness;  // COrenNayarBRDF(roughness)
  r.onA = 1.0f - (s2 / (2.0f * (s2 + 0.33f)));
  r.onB = 0.45f * s2 / (s2 + 0.09f);
  r.ggx.ax = m.alpha_x;
  r.ggx.ay = m.alpha_y;
  r.etaI = m.eta_i;
  r.etaT = m.eta_t;
  for (int k = 0; k < 4; ++k) r.tex[k] = -1;
  return r;
}

R2_HD V3 faceforward(V3 v, V3 v2) { return (dot(v, v2) < 0.0f) ? -v : v; }

R2_HD float mf_f(const Material& m, V3 wo, V3 wi) {
  float cO = abs_cos_theta(wo), cI = abs_cos_theta(wi);
  V3 h = wi + wo;
  if (cI == 0.0f || cO == 0.0f) return 0.0f;
  if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return 0.0f;
  h = normalize(h);
  float F = fresnel_dielectric(m.etaI, m.etaT, dot(wi, faceforward(h, v3(0.0f, 0.0f, 1.0f))));
  return ggx_D(m.ggx, h) * ggx_G(m.ggx, wo, wi) * F / (4.0f * cI * cO);
}

R2_HD float mf_pdf(const Material& m, V3 wo, V3 wi) {
  if (!same_hemisphere(wo, wi)) return 0.0f;
  V3 h = normalize(wo + wi);
  return ggx_pdf(m.ggx, wo, h) / (4.0f * dot(wo, h));
}

R2_HD float mf_sample_f(const Material& m, V3 wo, float u1, float u2, V3* wi, float* pdf) {
  if (wo.z == 0.0f) return 0.0f;
  V3 h = ggx_sample_h(m.ggx, wo, u1, u2);
  if (dot(wo, h) < 0.0f) return 0.0f;
  *wi = reflect(-wo, h);
  if (!same_hemisphere(wo, *wi)) return 0.0f;
  *pdf = ggx_pdf(m.ggx, wo, h) / (4.0f * dot(wo, h));
  return mf_f(m, wo, *wi);
}

// ---------------------------------------------------------------- oren_nayar_brdf.hpp
R2_HD float on_f(const Material& m, V3 wo, V3 wi) {
  float sI = sin_theta(wi), sO = sin_theta(wo);
  float maxCos = 0.0f;
  if (sI > 1.0e-4f && sO > 1.0e-4f) {
    float dCos = cos_phi(wi) * cos_phi(wo) + sin_phi(wi) * sin_phi(wo);
    maxCos = fmaxf(0.0f, dCos);
  }
  float sinAlpha, tanBeta;
  if (abs_cos_theta(wi) > abs_cos_theta(wo)) {
    sinAlpha = sO;
    tanBeta = sI / abs_cos_theta(wi);
  } else {
    sinAlpha = sI;
    tanBeta = sO / abs_cos_theta(wo);
  }
  return (float)(kInvPiD * (double)(m.onA + m.onB * maxCos * sinAlpha * tanBeta));
}

// CSampler::cosineHemispherePdf = cosTheta * M_1_PI (double).
R2_HD float on_pdf(V3 wo, V3 wi) {
  return same_hemisphere(wo, wi) ? (float)((double)abs_cos_theta(wi) * kInvPiD) : 0.0f;
}

R2_HD float on_sample_f(const Material& m, V3 wo, float u1, float u2, V3* wi, float* pdf) {
  *wi = cosine_sample_hemisphere(u1, u2);
  if (wo.z < 0.0f) wi->z *= -1.0f;
  *pdf = on_pdf(wo, *wi);
  return on_f(m, wo, *wi);
}

// ---------------------------------------------------------------- material.hpp
R2_HD V3 mat_f(const Material& m, V3 wo, V3 wi) {
  float fd = on_f(m, wo, wi);
  float fg = mf_f(m, wo, wi);
  float w = fresnel_dielectric(m.etaI, m.etaT, abs_cos_theta(wo));
  return m.diffuse * fd * (1.0f - w) + m.specular * fg * w;
}

R2_HD float mat_pdf(const Material& m, V3 wo, V3 wi) {
  float w = fresnel_dielectric(m.etaI, m.etaT, abs_cos_theta(wo));
  return on_pdf(wo, wi) * (1.0f - w) + mf_pdf(m, wo, wi) * w;
}

// CMaterial::sampleF: lobe chosen with probability F(|cos theta_o|); the
// returned value is not divided by that probability (reference behaviour).
R2_HD V3 mat_sample_f(const Material& m, V3 wo, float uSel, float u1, float u2, V3* wi, float* pdf) {
  float p = fresnel_dielectric(m.etaI, m.etaT, abs_cos_theta(wo));
  if (uSel < p) return m.specular * mf_sample_f(m, wo, u1, u2, wi, pdf);
  return m.diffuse * on_sample_f(m, wo, u1, u2, wi, pdf);
}

// ---------------------------------------------------------------- objects.hpp (CCoordinateFrame)
// tangentToWorld = mat3(T, B, N) (columns); worldToTangent is its inverse as
// glm::inverse computes it (cofactors over the determinant), columns W0..W2,
// which differs from the transpose in the last bits.
struct Frame {
  V3 T, B, N;
  V3 W0, W1, W2;
};

R2_HD Frame frame_from_normal(V3 N) {
  Frame f;
  f.N = N;
  f.T = fabsf(N.x) > fabsf(N.y) ? v3(-N.z, 0.0f, N.x) / sqrtf(N.x * N.x + N.z * N.z)
                                : v3(0.0f, N.z, -N.y) / sqrtf(N.y * N.y + N.z * N.z);
  f.B = normalize(cross(N, f.T));
  const V3 T = f.T, B = f.B;
  const float det = T.x * (B.y * N.z - N.y * B.z) - B.x * (T.y * N.z - N.y * T.z) + N.x * (T.y * B.z - B.y * T.z);
  const float inv = 1.0f / det;
  f.W0 = v3(+(B.y * N.z - N.y * B.z) * inv, -(T.y * N.z - N.y * T.z) * inv, +(T.y * B.z - B.y * T.z) * inv);
  f.W1 = v3(-(B.x * N.z - N.x * B.z) * inv, +(T.x * N.z - N.x * T.z) * inv, -(T.x * B.z - B.x * T.z) * inv);
  f.W2 = v3(+(B.x * N.y - N.x * B.y) * inv, -(T.x * N.y - N.x * T.y) * inv, +(T.x * B.y - B.x * T.y) * inv);
  return f;
}
// worldToTangent * v, summed column by column as glm's matrix-vector product.
R2_HD V3 to_local(const Frame& f, V3 v) { return f.W0 * v.x + f.W1 * v.y + f.W2 * v.z; }
R2_HD V3 to_world(const Frame& f, V3 v) { return f.T * v.x + f.B * v.y + f.N * v.z; }

// ---------------------------------------------------------------- ray.hpp / functions.hpp
R2_HD float next_float_up(float v) {
  if (isinf(v) && v > 0.0f) return v;
  if (v == -0.0f) return 0.0f;
  uint32_t ui;
  memcpy(&ui, &v, 4);
  if (v >= 0.0f) ++ui; else --ui;
  float r;
  memcpy(&r, &ui, 4);
  return r;
}
R2_HD float next_float_down(float v) {
  if (isinf(v) && v < 0.0f) return v;
  if (v == 0.0f) return -0.0f;
  uint32_t ui;
  memcpy(&ui, &v, 4);
  if (v > 0.0f) --ui; else ++ui;
  float r;
  memcpy(&r, &ui, 4);
  return r;
}

// CRay::offsetRayOrigin(p, dir): p + (|dir| . 1e-4) dir, then one ulp further.
R2_HD V3 offset_ray_origin(V3 p, V3 dir) {
  float d = dot(vabs(dir), v3(kRayOffset));
  V3 off = dir * d;
  V3 po = p + off;
  if (off.x > 0.0f) po.x = next_float_up(po.x); else if (off.x < 0.0f) po.x = next_float_down(po.x);
  if (off.y > 0.0f) po.y = next_float_up(po.y); else if (off.y < 0.0f) po.y = next_float_down(po.y);
  if (off.z > 0.0f) po.z = next_float_up(po.z); else if (off.z < 0.0f) po.z = next_float_down(po.z);
  return po;
}

// ---------------------------------------------------------------- environment map
// RGB texels (row 0 = top = +Y), the 1D distributions of the reference's
// CDistribution2D (marginal over the quirky sumRows and one conditional per
// row), bilinear texture lookup with wrap (cudaFilterModeLinear + wrap,
// texture.cu:166-189) evaluated in FP32.
struct EnvMap {
  const float4* tex;      // W*H texels (rgb, a=1)
  int W, H;
  const float* margFunc;  // H
  const float* margCdf;   // H+1
  float margFuncInt;
  const float* rowFunc;   // H*W
  const float* rowCdf;    // H*(W+1)
  const float* rowFuncInt;  // H
  int valid;
};

R2_HD float4 env_texel(const EnvMap& e, int x, int y) {
  x %= e.W; if (x < 0) x += e.W;
  y %= e.H; if (y < 0) y += e.H;
#if defined(__CUDA_ARCH__)
  return __ldg(&e.tex[(size_t)y * e.W + x]);
#else
  return e.tex[(size_t)y * e.W + x];
#endif
}

R2_HD V3 env_lookup(const EnvMap& e, float u, float v) {
  float xb = u * (float)e.W - 0.5f, yb = v * (float)e.H - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  float a = xb - fx, b = yb - fy;
  int x0 = (int)fx, y0 = (int)fy;
  float4 t00 = env_texel(e, x0, y0), t10 = env_texel(e, x0 + 1, y0);
  float4 t01 = env_texel(e, x0, y0 + 1), t11 = env_texel(e, x0 + 1, y0 + 1);
  float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
  return v3(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
            w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
            w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z);
}

// findInterval (functions.hpp:10-27) over cdf[0..n] with predicate cdf[i] <= u.
R2_HD int find_interval(const float* cdf, int size, float u) {
  int first = 0, len = size;
  while (len > 0) {
    int half = len >> 1, middle = first + half;
    if (cdf[middle] <= u) {
      first = middle + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  int r = first - 1;
  return r < 0 ? 0 : (r > size - 2 ? size - 2 : r);
}

// CDistribution1D::sampleContinuous (distribution_1d.hpp:54-74).
R2_HD float dist1d_sample(const float* func, const float* cdf, int n, float funcInt, float u, float* pdf, int* off) {
  int o = find_interval(cdf, n + 1, u);
  *off = o;
  float du = u - cdf[o];
  if ((cdf[o + 1] - cdf[o]) > 0.0f) du /= (cdf[o + 1] - cdf[o]);
  *pdf = func[o] / funcInt;
  return ((float)o + du) / (float)n;
}

// CEnvironmentMap::sample (environmentmap.hpp:28-42).
R2_HD V3 env_sample(const EnvMap& e, float u0, float u1, V3* dir, float* pdf) {
  float pdfY, pdfX;
  int row, col;
  float y = dist1d_sample(e.margFunc, e.margCdf, e.H, e.margFuncInt, u0, &pdfY, &row);
  float x = dist1d_sample(e.rowFunc + (size_t)row * e.W, e.rowCdf + (size_t)row * (e.W + 1), e.W,
                          e.rowFuncInt[row], u1, &pdfX, &col);
  *pdf = pdfX * pdfY;
  float sT, cT, sP, cP;
  sincos_turns(y * 0.5f, &sT, &cT);  // theta = y * pi
  sincos_turns(x, &sP, &cP);         // phi = x * 2 pi
  if (sT == 0.0f) *pdf = 0.0f;
  else *pdf = (float)((double)*pdf / ((double)(sT * 2.0f) * kPiD * kPiD));
  *dir = v3(sP * sT, cT, cP * sT);
  return env_lookup(e, x, y);
}

// CDistribution2D::pdf (distribution_2d.hpp:73-84): bilinear over the row
// functions with (W-2)/(H-2) scaling and no normalisation (reference quirk).
R2_HD float dist2d_pdf(const EnvMap& e, float px, float py) {
  int lr = (int)(py * (float)(e.H - 2));
  lr = lr < 0 ? 0 : (lr > e.H - 2 ? e.H - 2 : lr);
  int ur = lr + 1;
  int lc = (int)(px * (float)(e.W - 2));
  lc = lc < 0 ? 0 : (lc > e.W - 2 ? e.W - 2 : lc);
  int uc = lc + 1;
  const float* r0 = e.rowFunc + (size_t)lr * e.W;
  const float* r1 = e.rowFunc + (size_t)ur * e.W;
  float xs = px * ((float)e.W - 2.0f), ys = py * ((float)e.H - 2.0f);
  float lower = r0[lc] * ((float)uc - xs) + r0[uc] * (xs - (float)lc);
  float upper = r1[lc] * ((float)uc - xs) + r1[uc] * (xs - (float)lc);
  return lower * ((float)ur - ys) + upper * (ys - (float)lr);
}

// CEnvironmentMap::le (environmentmap.hpp:44-55).
R2_HD V3 env_le(const EnvMap& e, V3 d, float* pdf) {
  float theta = acosf(clampf(d.y, -1.0f, 1.0f));
  float p = atan2f(d.x, d.z);
  float phi = p < 0.0f ? (float)((double)p + 2.0 * kPiD) : p;
  float x = (float)((double)phi / (2.0 * kPiD)), y = (float)((double)theta / kPiD);
  float st = sinf(theta);
  *pdf = st == 0.0f ? 0.0f : (float)((double)dist2d_pdf(e, x, y) / (2.0 * kPiD * kPiD * (double)st));
  return env_lookup(e, x, y);
}

// ---------------------------------------------------------------- camera (camera.cu:20-37, pixel_sampler.hpp:36-47)
struct Camera {
  M43 viewToWorld;
  float pixelSize, nearPlane;
  int W, H;
};

// View-space ray through pixel (px, py) jittered by u (the reference reuses
// the horizontal jitter for the vertical offset); transformed like CRay::transform.
R2_HD void camera_ray(const Camera& c, int px, int py, float u, V3* o, V3* d) {
  float h = ((float)(px - c.W / 2) + u) * c.pixelSize;
  float v = ((float)(py - c.H / 2) + u) * c.pixelSize;
  V3 dv = normalize(v3(h, v, -c.nearPlane));
  *o = xform_point(c.viewToWorld, v3(0.0f));
  *d = normalize(xform_vector(c.viewToWorld, dv));
}

R2_HD float balance_heuristic(float f, float g) { return (1.0f * f) / (1.0f * f + 1.0f * g); }

}  // namespace r2
