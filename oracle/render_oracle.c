/*
 * CPU oracle of the path tracer — TEST INFRASTRUCTURE ONLY (see
 * render_oracle.h).  Each path runs start to finish like the reference's
 * megakernel; the float expressions follow the same order as the device
 * code so that paths agree sample for sample.
 */
#include "render_oracle.h"

#include <float.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "oracle_internal.h"

#define PI_F 3.14159265358979323846f
#define PI_D 3.14159265358979323846
#define INV_PI_D 0.318309886183790671538
#define RAY_OFFSET 1e-4f
#define DEFAULT_TMAX 1e12f
#define PURPOSE_CAMERA 0xCA3E7Au

static float clampf_(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

/* ------------------------------------------------------------ brdf_functions.hpp */
static float cos2_theta(f3 w) { return w.z * w.z; }
static float abs_cos_theta(f3 w) { return fabsf(w.z); }
static float sin2_theta(f3 w) { return fmaxf(0.0f, 1.0f - cos2_theta(w)); }
static float sin_theta(f3 w) { return sqrtf(sin2_theta(w)); }
static float tan_theta(f3 w) { return sin_theta(w) / w.z; }
static float tan2_theta(f3 w) { return sin2_theta(w) / cos2_theta(w); }
static float cos_phi(f3 w) { float s = sin_theta(w); return (s == 0.0f) ? 1.0f : clampf_(w.x / s, -1.0f, 1.0f); }
static float sin_phi(f3 w) { float s = sin_theta(w); return (s == 0.0f) ? 0.0f : clampf_(w.y / s, -1.0f, 1.0f); }
static float cos2_phi(f3 w) { float c = cos_phi(w); return c * c; }
static float sin2_phi(f3 w) { float s = sin_phi(w); return s * s; }
static int same_hemisphere(f3 a, f3 b) { return a.z * b.z > 0.0f; }

/* ------------------------------------------------------------ fresnel.hpp */
static float fresnel(float etaI0, float etaT0, float c) {
  c = clampf_(c, -1.0f, 1.0f);
  float etaI = etaI0, etaT = etaT0;
  if (!(c > 0.0f)) { etaI = etaT0; etaT = etaI0; c = fabsf(c); }
  float sI = sqrtf(fmaxf(0.0f, 1.0f - c * c));
  float sT = etaI / etaT * sI;
  if (sT >= 1.0f) return 1.0f;
  float cT = sqrtf(fmaxf(0.0f, 1.0f - sT * sT));
  float rPar = ((etaT * c) - (etaI * cT)) / ((etaT * c) + (etaI * cT));
  float rPer = ((etaI * c) - (etaT * cT)) / ((etaI * c) + (etaT * cT));
  return (rPar * rPar + rPer * rPer) / 2.0f;
}

/* ------------------------------------------------------------ GGX */
typedef struct { float ax, ay; } ggx_t;

static float ggx_D(ggx_t g, f3 h) {
  float t2 = tan2_theta(h);
  if (isinf(t2)) return 0.0f;
  float c2 = cos2_theta(h), c4 = c2 * c2;
  float e = (cos2_phi(h) / (g.ax * g.ax) + sin2_phi(h) / (g.ay * g.ay)) * t2;
  return (float)(1.0 / (PI_D * (double)g.ax * (double)g.ay * (double)c4 * (double)(1.0f + e) * (double)(1.0f + e)));
}
static float ggx_lambda(ggx_t g, f3 w) {
  float at = fabsf(tan_theta(w));
  if (isinf(at)) return 0.0f;
  float alpha = sqrtf(cos2_phi(w) * g.ax * g.ax + sin2_phi(w) * g.ay * g.ay);
  float a = (alpha * at) * (alpha * at);
  return (-1.0f + sqrtf(1.0f + a)) / 2.0f;
}
static float ggx_G(ggx_t g, f3 wo, f3 wi) { return 1.0f / (1.0f + ggx_lambda(g, wo) + ggx_lambda(g, wi)); }
static float ggx_G1(ggx_t g, f3 w) { return 1.0f / (1.0f + ggx_lambda(g, w)); }

static void ggx_sample11(float cosTheta, float u1, float u2, float* sx, float* sy) {
  if (cosTheta > 0.9999f) {
    float r = sqrtf(u1 / (1.0f - u1)), s, c;
    orc_sincos_turns(u2, &s, &c);
    *sx = r * c;
    *sy = r * s;
    return;
  }
  float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
  float tanT = sinT / cosTheta;
  float a = 1.0f / tanT;
  float G1 = 2.0f / (1.0f + sqrtf(1.0f + 1.0f / (a * a)));
  float A = 2.0f * u1 / G1 - 1.0f;
  float tmp = 1.0f / (A * A - 1.0f);
  if (tmp > 1e10f) tmp = 1e10f;
  float B = tanT;
  float D = sqrtf(fmaxf(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.0f));
  float s1 = B * tmp - D, s2 = B * tmp + D;
  *sx = (A < 0.0f || s2 > 1.0f / tanT) ? s1 : s2;
  float S;
  if (u2 > 0.5f) { S = 1.0f; u2 = 2.0f * (u2 - 0.5f); }
  else { S = -1.0f; u2 = 2.0f * (0.5f - u2); }
  float z = (u2 * (u2 * (u2 * 0.27385f - 0.73369f) + 0.46341f)) /
            (u2 * (u2 * (u2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
  *sy = S * z * sqrtf(1.0f + *sx * *sx);
}

static f3 ggx_sample_h(ggx_t g, f3 wo, float u1, float u2) {
  int flip = wo.z < 0.0f;
  f3 wi = flip ? neg3(wo) : wo;
  f3 ws = norm3(F3(g.ax * wi.x, g.ay * wi.y, wi.z));
  float sx, sy;
  ggx_sample11(ws.z, u1, u2, &sx, &sy);
  float tmp = cos_phi(ws) * sx - sin_phi(ws) * sy;
  sy = sin_phi(ws) * sx + cos_phi(ws) * sy;
  sx = tmp;
  sx = g.ax * sx;
  sy = g.ay * sy;
  f3 h = norm3(F3(-sx, -sy, 1.0f));
  return flip ? neg3(h) : h;
}
static float ggx_pdf(ggx_t g, f3 wo, f3 wh) {
  return ggx_D(g, wh) * ggx_G1(g, wo) * fabsf(dot3(wo, wh)) / abs_cos_theta(wo);
}
static f3 reflect3(f3 i, f3 n) { return sub3(i, mul3s(n, dot3(n, i) * 2.0f)); }

/* ------------------------------------------------------------ material */
typedef struct {
  f3 diffuse, specular;
  float onA, onB;
  ggx_t ggx;
  float etaI, etaT;
} mat_t;

static mat_t make_mat(const orc_material* m) {
  mat_t r;
  r.diffuse = F3(m->diffuse[0], m->diffuse[1], m->diffuse[2]);
  r.specular = F3(m->specular[0], m->specular[1], m->specular[2]);
  float s2 = m->diffuse_roughness * m->diffuse_roughness;
  r.onA = 1.0f - (s2 / (2.0f * (s2 + 0.33f)));
  r.onB = 0.45f * s2 / (s2 + 0.09f);
  r.ggx.ax = m->alpha_x;
  r.ggx.ay = m->alpha_y;
  r.etaI = m->eta_i;
  r.etaT = m->eta_t;
  return r;
}

static f3 faceforward3(f3 v, f3 v2) { return (dot3(v, v2) < 0.0f) ? neg3(v) : v; }

static float mf_f(const mat_t* m, f3 wo, f3 wi) {
  float cO = abs_cos_theta(wo), cI = abs_cos_theta(wi);
  f3 h = add3(wi, wo);
  if (cI == 0.0f || cO == 0.0f) return 0.0f;
  if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return 0.0f;
  h = norm3(h);
  float F = fresnel(m->etaI, m->etaT, dot3(wi, faceforward3(h, F3(0.0f, 0.0f, 1.0f))));
  return ggx_D(m->ggx, h) * ggx_G(m->ggx, wo, wi) * F / (4.0f * cI * cO);
}
static float mf_pdf(const mat_t* m, f3 wo, f3 wi) {
  if (!same_hemisphere(wo, wi)) return 0.0f;
  f3 h = norm3(add3(wo, wi));
  return ggx_pdf(m->ggx, wo, h) / (4.0f * dot3(wo, h));
}
static float mf_sample_f(const mat_t* m, f3 wo, float u1, float u2, f3* wi, float* pdf) {
  if (wo.z == 0.0f) return 0.0f;
  f3 h = ggx_sample_h(m->ggx, wo, u1, u2);
  if (dot3(wo, h) < 0.0f) return 0.0f;
  *wi = reflect3(neg3(wo), h);
  if (!same_hemisphere(wo, *wi)) return 0.0f;
  *pdf = ggx_pdf(m->ggx, wo, h) / (4.0f * dot3(wo, h));
  return mf_f(m, wo, *wi);
}
static float on_f(const mat_t* m, f3 wo, f3 wi) {
  float sI = sin_theta(wi), sO = sin_theta(wo);
  float maxCos = 0.0f;
  if (sI > 1.0e-4f && sO > 1.0e-4f) {
    float dCos = cos_phi(wi) * cos_phi(wo) + sin_phi(wi) * sin_phi(wo);
    maxCos = fmaxf(0.0f, dCos);
  }
  float sinAlpha, tanBeta;
  if (abs_cos_theta(wi) > abs_cos_theta(wo)) { sinAlpha = sO; tanBeta = sI / abs_cos_theta(wi); }
  else { sinAlpha = sI; tanBeta = sO / abs_cos_theta(wo); }
  return (float)(INV_PI_D * (double)(m->onA + m->onB * maxCos * sinAlpha * tanBeta));
}
static float on_pdf(f3 wo, f3 wi) { return same_hemisphere(wo, wi) ? (float)((double)abs_cos_theta(wi) * INV_PI_D) : 0.0f; }

static f3 cosine_hemisphere(float u1, float u2) {
  float ox = 2.0f * u1 - 1.0f, oy = 2.0f * u2 - 1.0f;
  f3 d;
  if (ox == 0.0f && oy == 0.0f) {
    d = F3(0.0f, 0.0f, 0.0f);
  } else {
    float r, s, c;
    if (fabsf(ox) > fabsf(oy)) {
      r = ox;
      orc_sincos_turns((oy / ox) * 0.125f, &s, &c);
    } else {
      float sa, ca;
      r = oy;
      orc_sincos_turns((ox / oy) * 0.125f, &sa, &ca);
      c = sa;
      s = ca;
    }
    d = F3(r * c, r * s, 0.0f);
  }
  float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
  return F3(d.x, d.y, z);
}

static float on_sample_f(const mat_t* m, f3 wo, float u1, float u2, f3* wi, float* pdf) {
  *wi = cosine_hemisphere(u1, u2);
  if (wo.z < 0.0f) wi->z *= -1.0f;
  *pdf = on_pdf(wo, *wi);
  return on_f(m, wo, *wi);
}
static f3 mat_f(const mat_t* m, f3 wo, f3 wi) {
  float fd = on_f(m, wo, wi), fg = mf_f(m, wo, wi);
  float w = fresnel(m->etaI, m->etaT, abs_cos_theta(wo));
  return add3(mul3s(mul3s(m->diffuse, fd), 1.0f - w), mul3s(mul3s(m->specular, fg), w));
}
static float mat_pdf(const mat_t* m, f3 wo, f3 wi) {
  float w = fresnel(m->etaI, m->etaT, abs_cos_theta(wo));
  return on_pdf(wo, wi) * (1.0f - w) + mf_pdf(m, wo, wi) * w;
}
static f3 mat_sample_f(const mat_t* m, f3 wo, float uSel, float u1, float u2, f3* wi, float* pdf) {
  float p = fresnel(m->etaI, m->etaT, abs_cos_theta(wo));
  if (uSel < p) return mul3s(m->specular, mf_sample_f(m, wo, u1, u2, wi, pdf));
  return mul3s(m->diffuse, on_sample_f(m, wo, u1, u2, wi, pdf));
}

/* ------------------------------------------------------------ frame, ray offset */
typedef struct { f3 T, B, N; } frame_t;
static frame_t frame_from_normal(f3 N) {
  frame_t f;
  f.N = N;
  f.T = fabsf(N.x) > fabsf(N.y) ? div3s(F3(-N.z, 0.0f, N.x), sqrtf(N.x * N.x + N.z * N.z))
                                : div3s(F3(0.0f, N.z, -N.y), sqrtf(N.y * N.y + N.z * N.z));
  f.B = norm3(cross3(N, f.T));
  return f;
}
static f3 to_local(const frame_t* f, f3 v) { return F3(dot3(f->T, v), dot3(f->B, v), dot3(f->N, v)); }
static f3 to_world(const frame_t* f, f3 v) { return add3(add3(mul3s(f->T, v.x), mul3s(f->B, v.y)), mul3s(f->N, v.z)); }

static float next_up(float v) {
  if (isinf(v) && v > 0.0f) return v;
  if (v == -0.0f) return 0.0f;
  uint32_t u;
  memcpy(&u, &v, 4);
  if (v >= 0.0f) ++u; else --u;
  memcpy(&v, &u, 4);
  return v;
}
static float next_down(float v) {
  if (isinf(v) && v < 0.0f) return v;
  if (v == 0.0f) return -0.0f;
  uint32_t u;
  memcpy(&u, &v, 4);
  if (v > 0.0f) --u; else ++u;
  memcpy(&v, &u, 4);
  return v;
}
static f3 offset_origin(f3 p, f3 dir) {
  float d = dot3(abs3(dir), F3(RAY_OFFSET, RAY_OFFSET, RAY_OFFSET));
  f3 off = mul3s(dir, d);
  f3 po = add3(p, off);
  if (off.x > 0.0f) po.x = next_up(po.x); else if (off.x < 0.0f) po.x = next_down(po.x);
  if (off.y > 0.0f) po.y = next_up(po.y); else if (off.y < 0.0f) po.y = next_down(po.y);
  if (off.z > 0.0f) po.z = next_up(po.z); else if (off.z < 0.0f) po.z = next_down(po.z);
  return po;
}

/* ------------------------------------------------------------ environment */
typedef struct {
  int W, H;
  const float* rgb;
  float *margFunc, *margCdf, *rowFunc, *rowCdf, *rowFuncInt;
  float margFuncInt;
} env_t;

static void dist1d(const float* f, int n, float* func, float* cdf, float* funcInt) {
  for (int i = 0; i < n; ++i) func[i] = f[i];
  cdf[0] = 0.0f;
  for (int i = 1; i <= n; ++i) cdf[i] = cdf[i - 1] + func[i - 1] / (float)n;
  *funcInt = cdf[n];
  if (*funcInt == 0.0f) {
    for (int i = 1; i <= n; ++i) cdf[i] = (float)i / (float)n;
  } else {
    for (int i = 1; i <= n; ++i) cdf[i] /= *funcInt;
  }
}

static void env_build(env_t* e, const float* rgb, int W, int H) {
  e->W = W;
  e->H = H;
  e->rgb = rgb;
  float* rad = (float*)malloc(sizeof(float) * (size_t)W * H);
  for (int y = 0; y < H; ++y) {
    double st = sin(PI_D * (double)((float)y + 0.5f) / (double)(float)H);
    for (int x = 0; x < W; ++x) {
      size_t i = (size_t)y * W + x;
      float pr = 0.0f;
      pr += rgb[3 * i];
      pr += rgb[3 * i + 1];
      pr += rgb[3 * i + 2];
      rad[i] = (float)((double)pr * st);
    }
  }
  /* sumRows quirk: push at i % W == 0 */
  float* sums = (float*)malloc(sizeof(float) * (size_t)H);
  int ns = 0;
  float sum = 0.0f;
  for (size_t i = 0; i < (size_t)W * H; ++i) {
    sum += rad[i];
    if (i % (size_t)W == 0) { sums[ns++] = sum; sum = 0.0f; }
  }
  e->margFunc = (float*)malloc(sizeof(float) * (size_t)ns);
  e->margCdf = (float*)malloc(sizeof(float) * (size_t)(ns + 1));
  dist1d(sums, ns, e->margFunc, e->margCdf, &e->margFuncInt);
  e->rowFunc = (float*)malloc(sizeof(float) * (size_t)W * H);
  e->rowCdf = (float*)malloc(sizeof(float) * (size_t)(W + 1) * H);
  e->rowFuncInt = (float*)malloc(sizeof(float) * (size_t)H);
  for (int y = 0; y < H; ++y)
    dist1d(&rad[(size_t)y * W], W, &e->rowFunc[(size_t)y * W], &e->rowCdf[(size_t)y * (W + 1)], &e->rowFuncInt[y]);
  free(rad);
  free(sums);
}

static void env_free(env_t* e) {
  free(e->margFunc); free(e->margCdf); free(e->rowFunc); free(e->rowCdf); free(e->rowFuncInt);
}

static f3 env_texel(const env_t* e, int x, int y) {
  x %= e->W; if (x < 0) x += e->W;
  y %= e->H; if (y < 0) y += e->H;
  const float* t = &e->rgb[3 * ((size_t)y * e->W + x)];
  return F3(t[0], t[1], t[2]);
}

static f3 env_lookup(const env_t* e, float u, float v) {
  float xb = u * (float)e->W - 0.5f, yb = v * (float)e->H - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  float a = xb - fx, b = yb - fy;
  int x0 = (int)fx, y0 = (int)fy;
  f3 t00 = env_texel(e, x0, y0), t10 = env_texel(e, x0 + 1, y0);
  f3 t01 = env_texel(e, x0, y0 + 1), t11 = env_texel(e, x0 + 1, y0 + 1);
  float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
  return F3(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
            w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
            w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z);
}

static int find_interval(const float* cdf, int size, float u) {
  int first = 0, len = size;
  while (len > 0) {
    int half = len >> 1, middle = first + half;
    if (cdf[middle] <= u) { first = middle + 1; len -= half + 1; }
    else len = half;
  }
  int r = first - 1;
  return r < 0 ? 0 : (r > size - 2 ? size - 2 : r);
}

static float dist1d_sample(const float* func, const float* cdf, int n, float funcInt, float u, float* pdf, int* off) {
  int o = find_interval(cdf, n + 1, u);
  *off = o;
  float du = u - cdf[o];
  if ((cdf[o + 1] - cdf[o]) > 0.0f) du /= (cdf[o + 1] - cdf[o]);
  *pdf = func[o] / funcInt;
  return ((float)o + du) / (float)n;
}

static f3 env_sample(const env_t* e, float u0, float u1, f3* dir, float* pdf) {
  float pdfY, pdfX;
  int row, col;
  float y = dist1d_sample(e->margFunc, e->margCdf, e->H, e->margFuncInt, u0, &pdfY, &row);
  float x = dist1d_sample(e->rowFunc + (size_t)row * e->W, e->rowCdf + (size_t)row * (e->W + 1), e->W,
                          e->rowFuncInt[row], u1, &pdfX, &col);
  *pdf = pdfX * pdfY;
  float sT, cT, sP, cP;
  orc_sincos_turns(y * 0.5f, &sT, &cT);
  orc_sincos_turns(x, &sP, &cP);
  if (sT == 0.0f) *pdf = 0.0f;
  else *pdf = (float)((double)*pdf / ((double)(sT * 2.0f) * PI_D * PI_D));
  *dir = F3(sP * sT, cT, cP * sT);
  return env_lookup(e, x, y);
}

static float dist2d_pdf(const env_t* e, float px, float py) {
  int lr = (int)(py * (float)(e->H - 2));
  lr = lr < 0 ? 0 : (lr > e->H - 2 ? e->H - 2 : lr);
  int ur = lr + 1;
  int lc = (int)(px * (float)(e->W - 2));
  lc = lc < 0 ? 0 : (lc > e->W - 2 ? e->W - 2 : lc);
  int uc = lc + 1;
  const float* r0 = e->rowFunc + (size_t)lr * e->W;
  const float* r1 = e->rowFunc + (size_t)ur * e->W;
  float xs = px * ((float)e->W - 2.0f), ys = py * ((float)e->H - 2.0f);
  float lower = r0[lc] * ((float)uc - xs) + r0[uc] * (xs - (float)lc);
  float upper = r1[lc] * ((float)uc - xs) + r1[uc] * (xs - (float)lc);
  return lower * ((float)ur - ys) + upper * (ys - (float)lr);
}

static f3 env_le(const env_t* e, f3 d, float* pdf) {
  float theta = acosf(clampf_(d.y, -1.0f, 1.0f));
  float p = atan2f(d.x, d.z);
  float phi = p < 0.0f ? (float)((double)p + 2.0 * PI_D) : p;
  float x = (float)((double)phi / (2.0 * PI_D)), y = (float)((double)theta / PI_D);
  float st = sinf(theta);
  *pdf = st == 0.0f ? 0.0f : (float)((double)dist2d_pdf(e, x, y) / (2.0 * PI_D * PI_D * (double)st));
  return env_lookup(e, x, y);
}

/* ------------------------------------------------------------ scene */
typedef struct {
  int32_t* nodes;
  float* tris;
  uint32_t* order;
  float* wnrm;      /* per vertex, world space (unnormalised) */
  uint32_t* idx;    /* global indices */
  uint32_t* triMat; /* per original triangle */
  mat_t* mats;
  uint32_t ntris;
  const orc_shape* shapes;
  mat_t* shapeMats;
  uint32_t nshapes;
  env_t env;
  /* camera */
  float v2w[12];
  float pixelSize, nearPlane;
  int W, H;
  uint32_t spp, maxDepth, seed;
} rscene_t;

/* closest: code >= 0 BVH-order triangle, -1 miss, -2 - i shape i */
static int scene_closest(const rscene_t* S, f3 o, f3 d, float tmax, float* tOut, float* b1, float* b2) {
  float t = tmax;
  int code = -1;
  *b1 = *b2 = 0.0f;
  if (S->ntris > 0) {
    hit_t h = oi_trace(S->nodes, S->tris, o, d, tmax, 0);
    if (h.tri >= 0) { t = h.t; *b1 = h.b1; *b2 = h.b2; code = h.tri; }
  }
  for (uint32_t i = 0; i < S->nshapes; ++i) {
    const orc_shape* sh = &S->shapes[i];
    f3 c = F3(sh->center[0], sh->center[1], sh->center[2]);
    float ts = -1.0f;
    if (sh->type == 1) {
      f3 nn = F3(sh->normal[0], sh->normal[1], sh->normal[2]);
      float den = dot3(d, nn);
      if (den != 0.0f) {
        float tc = dot3(sub3(c, o), nn) / den;
        if (tc > 0.0f && tc <= t) {
          f3 p = add3(o, mul3s(d, tc));
          if (len3(sub3(p, c)) < sh->radius) ts = tc;
        }
      }
    } else {
      f3 oc = sub3(o, c);
      float a = dot3(d, d), b = 2.0f * dot3(d, oc), cc = dot3(oc, oc) - sh->radius * sh->radius;
      float disc = b * b - 4.0f * a * cc;
      if (disc == 0.0f) {
        float tc = (-b + sqrtf(disc)) / (2.0f * a);
        if (tc > 0.0f && tc <= t) ts = tc;
      } else if (disc > 0.0f) {
        float sq = sqrtf(disc), den = 1.0f / (2.0f * a);
        float t1 = (-b + sq) * den, t2 = (-b - sq) * den;
        float mn = fminf(t1, t2), mx = fmaxf(t1, t2);
        if (mx > 0.0f) {
          if (mn > 0.0f && mn <= t) ts = mn;
          else if (mn <= 0.0f && mx <= t) ts = mx;
        }
      }
    }
    if (ts > 0.0f && ts < t) { t = ts; code = -2 - (int)i; }
  }
  *tOut = t;
  return code;
}

static int scene_occluded(const rscene_t* S, f3 o, f3 d, float tmax) {
  if (S->ntris > 0) {
    hit_t h = oi_trace(S->nodes, S->tris, o, d, tmax, 1);
    if (h.tri >= 0) return 1;
  }
  if (S->nshapes > 0) {
    rscene_t T = *S;
    T.ntris = 0;
    float t, b1, b2;
    if (scene_closest(&T, o, d, tmax, &t, &b1, &b2) != -1) return 1;
  }
  return 0;
}

static void philox_u(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t ctr[4] = {c0, c1, c2, c3}, key[2] = {k0, k1};
  orc_philox4x32_10(ctr, key, out);
}

static f3 trace_path(const rscene_t* S, uint32_t p, uint32_t s) {
  const int px = (int)(p % (uint32_t)S->W), py = (int)(p / (uint32_t)S->W);
  uint32_t r[4];
  philox_u(s, PURPOSE_CAMERA, 0u, 0u, p, S->seed, r);
  float u = oi_u01(r[0]);
  float hh = ((float)(px - S->W / 2) + u) * S->pixelSize;
  float vv = ((float)(py - S->H / 2) + u) * S->pixelSize;
  f3 dv = norm3(F3(hh, vv, -S->nearPlane));
  f3 o = xpoint(S->v2w, F3(0.0f, 0.0f, 0.0f));
  f3 d = norm3(xvec(S->v2w, dv));
  f3 T = F3(1.0f, 1.0f, 1.0f), L = F3(0.0f, 0.0f, 0.0f);
  for (uint32_t b = 0; b < S->maxDepth; ++b) {
    float t, hb1, hb2;
    int code = scene_closest(S, o, d, DEFAULT_TMAX, &t, &hb1, &hb2);
    if (code == -1) {
      if (b == 0) {
        float lp;
        f3 le = env_le(&S->env, d, &lp);
        L = add3(L, mul3(le, T));
      }
      break;
    }
    f3 pos = add3(o, mul3s(d, t));
    f3 n;
    const mat_t* m;
    if (code >= 0) {
      uint32_t prim = S->order[code];
      const uint32_t* tv = &S->idx[3 * (size_t)prim];
      f3 n0 = F3(S->wnrm[3 * tv[0]], S->wnrm[3 * tv[0] + 1], S->wnrm[3 * tv[0] + 2]);
      f3 n1 = F3(S->wnrm[3 * tv[1]], S->wnrm[3 * tv[1] + 1], S->wnrm[3 * tv[1] + 2]);
      f3 n2 = F3(S->wnrm[3 * tv[2]], S->wnrm[3 * tv[2] + 1], S->wnrm[3 * tv[2] + 2]);
      float b0 = (1.0f - hb1) - hb2;
      n = norm3(add3(add3(mul3s(n0, b0), mul3s(n1, hb1)), mul3s(n2, hb2)));
      m = &S->mats[S->triMat[prim]];
    } else {
      const orc_shape* sh = &S->shapes[-2 - code];
      n = sh->type == 1 ? norm3(F3(sh->normal[0], sh->normal[1], sh->normal[2]))
                        : norm3(sub3(pos, F3(sh->center[0], sh->center[1], sh->center[2])));
      m = &S->shapeMats[-2 - code];
    }
    uint32_t rA[4], rB[4];
    philox_u(s, b, 0u, 1u, p, S->seed, rA);
    philox_u(s, b, 1u, 1u, p, S->seed, rB);
    frame_t fr = frame_from_normal(n);
    f3 wo = neg3(d);
    f3 woT = to_local(&fr, wo);
    f3 offO = offset_origin(pos, n);
    f3 dl = F3(0.0f, 0.0f, 0.0f);
    int anyShadow = 0;
    {
      f3 ldir;
      float lpdf = 0.0f;
      f3 Le = env_sample(&S->env, oi_u01(rA[0]), oi_u01(rA[1]), &ldir, &lpdf);
      if (lpdf > 0.0f) {
        ldir = norm3(ldir);
        f3 lT = norm3(to_local(&fr, ldir));
        f3 f = mul3s(mat_f(m, woT, lT), fabsf(dot3(n, ldir)));
        float spdf = mat_pdf(m, woT, lT);
        float mis = (1.0f * lpdf) / (1.0f * lpdf + 1.0f * spdf);
        f3 pre = mul3(mul3s(f, mis), Le);
        float tr = scene_occluded(S, offO, ldir, DEFAULT_TMAX) ? 0.0f : 1.0f;
        dl = add3(dl, div3s(mul3s(pre, tr), lpdf));
        anyShadow = 1;
      }
    }
    {
      f3 wiT = F3(0.0f, 0.0f, 0.0f);
      float spdf = 0.0f;
      f3 f = mat_sample_f(m, woT, oi_u01(rA[2]), oi_u01(rA[3]), oi_u01(rB[0]), &wiT, &spdf);
      f3 wi = norm3(to_world(&fr, wiT));
      f = mul3s(f, fabsf(dot3(n, wi)));
      if (spdf > 0.0f) {
        wi = norm3(wi);
        float lpdf;
        f3 Le = env_le(&S->env, wi, &lpdf);
        float mis = (1.0f * spdf) / (1.0f * spdf + 1.0f * lpdf);
        f3 pre = mul3(mul3s(f, mis), Le);
        float tr = scene_occluded(S, offO, wi, DEFAULT_TMAX) ? 0.0f : 1.0f;
        dl = add3(dl, div3s(mul3s(pre, tr), spdf));
        anyShadow = 1;
      }
    }
    if (anyShadow) L = add3(L, mul3(dl, T));
    /* continuation */
    f3 dT = norm3(to_local(&fr, d));
    f3 wi = F3(0.0f, 0.0f, 0.0f);
    float pdf = 0.0f;
    f3 f = mat_sample_f(m, neg3(dT), oi_u01(rB[1]), oi_u01(rB[2]), oi_u01(rB[3]), &wi, &pdf);
    if (!(pdf != 0.0f)) break;
    f3 dirW = norm3(to_world(&fr, wi));
    float cosine = fabsf(dot3(n, dirW));
    f3 Tn = mul3(T, div3s(mul3s(f, cosine), pdf));
    if (b > 3) {
      uint32_t rC[4];
      philox_u(s, b, 2u, 1u, p, S->seed, rC);
      float prr = 1.0f - (Tn.x + Tn.y + Tn.z) / 3.0f;
      if (oi_u01(rC[0]) <= prr) break;
      Tn = div3s(Tn, 1.0f - prr);
    }
    if (b + 1 >= S->maxDepth) break;
    o = offO;
    d = dirW;
    T = Tn;
  }
  return L;
}

typedef struct {
  const rscene_t* S;
  uint32_t p0, p1;
  float* rgb;
  double* var;
  int tid, nthreads;
} rjob_t;

static void* render_worker(void* arg) {
  rjob_t* J = (rjob_t*)arg;
  const rscene_t* S = J->S;
  for (uint32_t p = J->p0 + (uint32_t)J->tid; p < J->p1; p += (uint32_t)J->nthreads) {
    float acc[3] = {0.0f, 0.0f, 0.0f};
    double mean[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
    for (uint32_t s = 0; s < S->spp; ++s) {
      f3 L = trace_path(S, p, s);
      if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = F3(0, 0, 0);
      f3 v = div3s(L, (float)S->spp);
      acc[0] += v.x;
      acc[1] += v.y;
      acc[2] += v.z;
      double x[3] = {L.x, L.y, L.z};
      for (int k = 0; k < 3; ++k) {  /* Welford */
        double dlt = x[k] - mean[k];
        mean[k] += dlt / (double)(s + 1);
        m2[k] += dlt * (x[k] - mean[k]);
      }
    }
    size_t o = (size_t)(p - J->p0);
    for (int k = 0; k < 3; ++k) {
      J->rgb[3 * o + k] = acc[k];
      if (J->var) J->var[3 * o + k] = S->spp > 1 ? m2[k] / (double)(S->spp - 1) : 0.0;
    }
  }
  return NULL;
}

static void make_cam(rscene_t* S, const orc_camera* c) {
  S->W = (int)c->width;
  S->H = (int)c->height;
  S->pixelSize = 1e-5f;
  float fov = c->fov_deg * 0.01745329251994329577f;
  float sensorW = (float)c->width * S->pixelSize;
  S->nearPlane = sensorW / (2.0f * tanf(fov / 2.0f));
  f3 eye = F3(c->pos[0], c->pos[1], c->pos[2]);
  f3 ctr = F3(c->look_at[0], c->look_at[1], c->look_at[2]);
  f3 up = F3(c->up[0], c->up[1], c->up[2]);
  f3 f = norm3(sub3(ctr, eye));
  f3 s = norm3(cross3(f, up));
  f3 u = cross3(s, f);
  m4_t view = oi_m4_id();
  view.m[0][0] = s.x; view.m[1][0] = s.y; view.m[2][0] = s.z;
  view.m[0][1] = u.x; view.m[1][1] = u.y; view.m[2][1] = u.z;
  view.m[0][2] = -f.x; view.m[1][2] = -f.y; view.m[2][2] = -f.z;
  view.m[3][0] = -dot3(s, eye);
  view.m[3][1] = -dot3(u, eye);
  view.m[3][2] = dot3(f, eye);
  oi_m4_to43(oi_m4_inv(view), S->v2w);
}

int orc_render(const orc_mesh* meshes, uint32_t nmeshes, const orc_shape* shapes, uint32_t nshapes, const float* env_rgb,
               int env_w, int env_h, const orc_camera* cam, uint32_t spp, uint32_t max_depth, uint32_t seed, uint32_t p0,
               uint32_t p1, float* rgb_out, double* var_out, int threads) {
  if (env_w < 2 || env_h < 2 || spp == 0 || max_depth == 0) return -1;
  rscene_t S;
  memset(&S, 0, sizeof(S));
  uint32_t nv = 0, nt = 0;
  for (uint32_t i = 0; i < nmeshes; ++i) { nv += meshes[i].nverts; nt += meshes[i].ntris; }
  float* wpos = (float*)malloc(sizeof(float) * 3 * (size_t)(nv + 1));
  S.wnrm = (float*)malloc(sizeof(float) * 3 * (size_t)(nv + 1));
  S.idx = (uint32_t*)malloc(sizeof(uint32_t) * 3 * (size_t)(nt + 1));
  S.triMat = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(nt + 1));
  S.mats = (mat_t*)malloc(sizeof(mat_t) * (size_t)(nmeshes + 1));
  uint32_t vb = 0, tb = 0;
  for (uint32_t i = 0; i < nmeshes; ++i) {
    const orc_mesh* M = &meshes[i];
    S.mats[i] = make_mat(&M->material);
    for (uint32_t v = 0; v < M->nverts; ++v) {
      f3 pp = xpoint(M->model_to_world, F3(M->positions[3 * v], M->positions[3 * v + 1], M->positions[3 * v + 2]));
      f3 nn = xvec(M->model_to_world, F3(M->normals[3 * v], M->normals[3 * v + 1], M->normals[3 * v + 2]));
      wpos[3 * (vb + v)] = pp.x; wpos[3 * (vb + v) + 1] = pp.y; wpos[3 * (vb + v) + 2] = pp.z;
      S.wnrm[3 * (vb + v)] = nn.x; S.wnrm[3 * (vb + v) + 1] = nn.y; S.wnrm[3 * (vb + v) + 2] = nn.z;
    }
    for (uint32_t t = 0; t < M->ntris; ++t) {
      for (int k = 0; k < 3; ++k) S.idx[3 * (tb + t) + k] = vb + M->indices[3 * t + k];
      S.triMat[tb + t] = i;
    }
    vb += M->nverts;
    tb += M->ntris;
  }
  S.ntris = nt;
  if (nt > 0) {
    S.nodes = (int32_t*)malloc(64 * (size_t)(nt > 1 ? nt - 1 : 1));
    S.order = (uint32_t*)malloc(4 * (size_t)nt);
    S.tris = (float*)malloc(48 * (size_t)nt);
    int h = orc_build_bvh(wpos, nv, S.idx, nt, S.nodes, S.order, S.tris);
    if (h < 0 || h > 96) return -2;
  }
  S.shapes = shapes;
  S.nshapes = nshapes;
  S.shapeMats = (mat_t*)malloc(sizeof(mat_t) * (size_t)(nshapes + 1));
  for (uint32_t i = 0; i < nshapes; ++i) S.shapeMats[i] = make_mat(&shapes[i].material);
  env_build(&S.env, env_rgb, env_w, env_h);
  make_cam(&S, cam);
  S.spp = spp;
  S.maxDepth = max_depth;
  S.seed = seed;
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  rjob_t* jobs = (rjob_t*)malloc(sizeof(rjob_t) * (size_t)threads);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int t = 0; t < threads; ++t) {
    rjob_t J = {&S, p0, p1, rgb_out, var_out, t, threads};
    jobs[t] = J;
    pthread_create(&th[t], NULL, render_worker, &jobs[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  free(jobs); free(th);
  env_free(&S.env);
  free(wpos); free(S.wnrm); free(S.idx); free(S.triMat); free(S.mats); free(S.shapeMats);
  if (nt > 0) { free(S.nodes); free(S.order); free(S.tris); }
  return 0;
}

int orc_env_sample(const float* env_rgb, int W, int H, float u0, float u1, float* dir, float* pdf, float* le) {
  env_t e;
  env_build(&e, env_rgb, W, H);
  f3 d;
  f3 l = env_sample(&e, u0, u1, &d, pdf);
  dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
  le[0] = l.x; le[1] = l.y; le[2] = l.z;
  env_free(&e);
  return 0;
}

int orc_env_le(const float* env_rgb, int W, int H, const float* dir, float* pdf, float* le) {
  env_t e;
  env_build(&e, env_rgb, W, H);
  f3 l = env_le(&e, F3(dir[0], dir[1], dir[2]), pdf);
  le[0] = l.x; le[1] = l.y; le[2] = l.z;
  env_free(&e);
  return 0;
}

/* ------------------------------------------------------------ unit hooks for the golden-vector tests */

static f3 L3(const float* p) { return F3(p[0], p[1], p[2]); }
static void P3(float* o, f3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

float orc_t_fresnel(float etaI, float etaT, float c) { return fresnel(etaI, etaT, c); }

void orc_t_microfacet(float ax, float ay, float etaI, float etaT, const float* wo, const float* wi, float* out) {
  orc_material om;
  memset(&om, 0, sizeof(om));
  om.alpha_x = ax; om.alpha_y = ay; om.eta_i = etaI; om.eta_t = etaT;
  mat_t m = make_mat(&om);
  out[0] = mf_f(&m, L3(wo), L3(wi));
  out[1] = mf_pdf(&m, L3(wo), L3(wi));
}

void orc_t_microfacet_sample(float ax, float ay, float etaI, float etaT, const float* wo, float u1, float u2,
                             float* out) {
  orc_material om;
  memset(&om, 0, sizeof(om));
  om.alpha_x = ax; om.alpha_y = ay; om.eta_i = etaI; om.eta_t = etaT;
  mat_t m = make_mat(&om);
  f3 wi = F3(0.0f, 0.0f, 0.0f);
  float pdf = 0.0f;
  float f = mf_sample_f(&m, L3(wo), u1, u2, &wi, &pdf);
  P3(out, wi);
  out[3] = pdf;
  out[4] = f;
}

void orc_t_ggx_sample_h(float ax, float ay, const float* wo, float u1, float u2, float* out) {
  ggx_t g = {ax, ay};
  P3(out, ggx_sample_h(g, L3(wo), u1, u2));
}

void orc_t_oren_nayar(float roughness, const float* wo, const float* wi, float* out) {
  orc_material om;
  memset(&om, 0, sizeof(om));
  om.diffuse_roughness = roughness;
  mat_t m = make_mat(&om);
  out[0] = on_f(&m, L3(wo), L3(wi));
  out[1] = on_pdf(L3(wo), L3(wi));
}

void orc_t_oren_nayar_sample(float roughness, const float* wo, float u1, float u2, float* out) {
  orc_material om;
  memset(&om, 0, sizeof(om));
  om.diffuse_roughness = roughness;
  mat_t m = make_mat(&om);
  f3 wi;
  float pdf = 0.0f;
  float f = on_sample_f(&m, L3(wo), u1, u2, &wi, &pdf);
  P3(out, wi);
  out[3] = pdf;
  out[4] = f;
}

void orc_t_warps(float u1, float u2, float* out) {
  float zz = 1.0f - 2.0f * u1, r = sqrtf(fmaxf(0.0f, 1.0f - zz * zz)), s, c;
  orc_sincos_turns(u2, &s, &c);
  P3(out + 0, F3(r * c, r * s, zz));
  float rh = sqrtf(fmaxf(0.0f, 1.0f - u1 * u1));
  P3(out + 3, F3(rh * c, rh * s, u1));
  f3 d = cosine_hemisphere(u1, u2);
  P3(out + 6, F3(d.x, d.y, 0.0f));
  P3(out + 9, d);
}

void orc_t_frame(const float* n, const float* v, float* out) {
  frame_t f = frame_from_normal(L3(n));
  P3(out, f.T);
  P3(out + 3, f.B);
  P3(out + 6, to_local(&f, L3(v)));
}

void orc_t_offset(const float* p, const float* d, float* out) { P3(out, offset_origin(L3(p), L3(d))); }

int orc_t_find_interval(const float* cdf, int size, float u) { return find_interval(cdf, size, u); }

void orc_t_sphere(const float* c, float r, const float* o, const float* d, float tmax, float* out) {
  orc_shape sh;
  memset(&sh, 0, sizeof(sh));
  sh.type = 0;
  sh.center[0] = c[0]; sh.center[1] = c[1]; sh.center[2] = c[2];
  sh.radius = r;
  rscene_t S;
  memset(&S, 0, sizeof(S));
  S.shapes = &sh;
  S.nshapes = 1;
  float t, b1, b2;
  int code = scene_closest(&S, L3(o), L3(d), tmax, &t, &b1, &b2);
  out[0] = code == -2 ? 1.0f : 0.0f;
  out[1] = code == -2 ? t : 0.0f;
}
