/*
 * CPU oracle of the path tracer — TEST INFRASTRUCTURE ONLY (see
 * render_oracle.h).  Each path runs start to finish like the reference's
 * megakernel; the float expressions follow the same order as the device
 * code so that paths agree sample for sample.
 */
#include "render_oracle.h"

#include <float.h>
#include <pthread.h>
#include <stdio.h>
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
  int tex[4]; /* albedo, glossy, normal, opacity texture (-1: none) */
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
  for (int k = 0; k < 4; ++k) r.tex[k] = -1;
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
static int g_replay_swap_lobe = 0;  /* set with the replay: see orc_set_replay */
static f3 mat_sample_f(const mat_t* m, f3 wo, float uSel, float u1, float u2, f3* wi, float* pdf) {
  float p = fresnel(m->etaI, m->etaT, abs_cos_theta(wo));
  if (uSel < p) {
    if (g_replay_swap_lobe) { const float t = u1; u1 = u2; u2 = t; }
    return mul3s(m->specular, mf_sample_f(m, wo, u1, u2, wi, pdf));
  }
  return mul3s(m->diffuse, on_sample_f(m, wo, u1, u2, wi, pdf));
}

/* ------------------------------------------------------------ frame, ray offset */
/* CCoordinateFrame::fromNormal (objects.hpp:31-41): tangentToWorld =
 * mat3(T, B, N) by columns, worldToTangent = glm::inverse of it (cofactors
 * over the determinant), kept as columns W0..W2. */
typedef struct { f3 T, B, N, W0, W1, W2; } frame_t;
static frame_t frame_from_normal(f3 N) {
  frame_t f;
  f.N = N;
  f.T = fabsf(N.x) > fabsf(N.y) ? div3s(F3(-N.z, 0.0f, N.x), sqrtf(N.x * N.x + N.z * N.z))
                                : div3s(F3(0.0f, N.z, -N.y), sqrtf(N.y * N.y + N.z * N.z));
  f.B = norm3(cross3(N, f.T));
  const f3 T = f.T, B = f.B;
  const float det = T.x * (B.y * N.z - N.y * B.z) - B.x * (T.y * N.z - N.y * T.z) + N.x * (T.y * B.z - B.y * T.z);
  const float inv = 1.0f / det;
  f.W0 = F3(+(B.y * N.z - N.y * B.z) * inv, -(T.y * N.z - N.y * T.z) * inv, +(T.y * B.z - B.y * T.z) * inv);
  f.W1 = F3(-(B.x * N.z - N.x * B.z) * inv, +(T.x * N.z - N.x * T.z) * inv, -(T.x * B.z - B.x * T.z) * inv);
  f.W2 = F3(+(B.x * N.y - N.x * B.y) * inv, -(T.x * N.y - N.x * T.y) * inv, +(T.x * B.y - B.x * T.y) * inv);
  return f;
}
/* worldToTangent * v, summed column by column (glm's matrix-vector order) */
static f3 to_local(const frame_t* f, f3 v) {
  return add3(add3(mul3s(f->W0, v.x), mul3s(f->W1, v.y)), mul3s(f->W2, v.z));
}
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

/* ------------------------------------------------------------ media
 * CNVDBMedium / CMediumInstance / SGGX phase function restated from
 * nvdb_medium_impl.hpp:28-320, medium_instance_impl.hpp:7-45,
 * sggx_phase_function.hpp:89-233, device_grid_brick_impl.hpp:9-33 and the
 * bounding-box program shaders.optix.cu:192-236. */
#define MEDIUM_CODE_BASE (-1000000)
#define EV_SCATTER (-2147483647)
#define EV_DEAD (-2147483646)
#define MAX_TRACKING_STEPS (1 << 20)
#define MAX_PASS_THROUGH 4096
#define MAX_SHADOW_SEGMENTS 4096
#define PURPOSE_MEDIUM 0x1000u
#define PURPOSE_SCATTER 0x100u
#define PURPOSE_SHADOW_TR 0x200u

/* log x (x > 0 normal): x = m 2^e with m in [sqrt(1/2), sqrt(2)), then
 * log m = 2 atanh(s) = 2 (s + s^3/3 + ... + s^11/11), s = (m - 1)/(m + 1)
 * (Cody and Waite's reduction); e ln 2 added as 0.693145751953125 + 1.42860682e-6. */
static float oi_log(float x) {
  uint32_t b;
  memcpy(&b, &x, 4);
  int e = (int)((b >> 23) & 0xFFu) - 127;
  uint32_t mb = (b & 0x7FFFFFu) | 0x3F800000u;
  float m;
  memcpy(&m, &mb, 4);
  if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float p = fmaf(s2, 1.0f / 11.0f, 1.0f / 9.0f);
  p = fmaf(s2, p, 1.0f / 7.0f);
  p = fmaf(s2, p, 1.0f / 5.0f);
  p = fmaf(s2, p, 1.0f / 3.0f);
  const float twoS = 2.0f * s;
  const float lm = fmaf(twoS * s2, p, twoS);
  const float fe = (float)e;
  return fmaf(fe, 0.693145751953125f, fmaf(fe, 1.42860682e-6f, lm));
}

/* Sequential uniforms: draw i = word i&3 of Philox((sample, bounce, i>>2, purpose), (pixel, seed)). */
/* replay (nullable, test hooks only): the values to return in order instead of Philox draws */
typedef struct { uint32_t k0, k1, c0, c1, purpose, idx; uint32_t buf[4]; const float* replay; } rng_t;
static rng_t rng_make(uint32_t pixel, uint32_t seed, uint32_t sample, uint32_t bounce, uint32_t purpose) {
  rng_t r;
  memset(&r, 0, sizeof(r));
  r.k0 = pixel; r.k1 = seed; r.c0 = sample; r.c1 = bounce; r.purpose = purpose;
  return r;
}
static float rng_next(rng_t* r) {
  if (r->replay) return r->replay[r->idx++];
  const uint32_t w = r->idx & 3u;
  if (w == 0) {
    uint32_t ctr[4] = {r->c0, r->c1, r->idx >> 2, r->purpose}, key[2] = {r->k0, r->k1};
    orc_philox4x32_10(ctr, key, r->buf);
  }
  r->idx++;
  return oi_u01(r->buf[w]);
}

typedef struct { f3 o, d; float tmax; } ray_t;
static ray_t mkray(f3 o, f3 d, float t) { ray_t r; r.o = o; r.d = d; r.tmax = t; return r; }
/* CRay::transform (direction renormalised) and transform2 (kept). */
static ray_t ray_xf(ray_t r, const float* M) {
  f3 o = xpoint(M, r.o), e = xpoint(M, add3(r.o, mul3s(r.d, r.tmax)));
  return mkray(o, norm3(xvec(M, r.d)), len3(sub3(e, o)));
}
static ray_t ray_xf2(ray_t r, const float* M) {
  f3 o = xpoint(M, r.o), e = xpoint(M, add3(r.o, mul3s(r.d, r.tmax)));
  f3 d = xvec(M, r.d);
  return mkray(o, d, len3(sub3(e, o)) / len3(d));
}
/* CRay::offsetRayOrigin(dir): the origin moves, the end point stays. */
static ray_t ray_off(ray_t r, f3 dir) {
  f3 end = add3(r.o, mul3s(r.d, r.tmax));
  f3 o = offset_origin(r.o, dir);
  return mkray(o, r.d, len3(sub3(end, o)));
}
/* CRay::spawnRay(p0, p1) (ray.hpp:62-69): origin offset from p0 towards p1,
 * direction (p1 - p0) / |p1 - origin|, that length as tmax. */
static ray_t spawn_ray(f3 p0, f3 p1) {
  const f3 off = offset_origin(p0, norm3(sub3(p1, p0)));
  const float tl = len3(sub3(p1, off));
  return mkray(off, div3s(sub3(p1, p0), tl), tl);
}

typedef struct {
  float m2w[12], w2m[12];
  f3 bbMin, bbMax;
  float ratio;
  float i2m[12], m2i[12], u2s[12], s2m[12];
  int ibbMin[3], size[3];
  f3 sigmaS;
  float sigmaT, invMax;
  int hg;
  float hgG;
  oi_nvdb g;
  oi_bricks b;
  float vsF;  /* voxel size of the filtering, from the path */
  int owner;  /* 1: g and b belong to this entry (the first instance of its path) */
} med_t;

typedef struct {
  float density;
  float S[6];
  f3 diffuse, specular, normal;
  float ior;
} fdat;

float oi_half_to_float(uint16_t h) {
  const int e = (h >> 10) & 0x1F, m = h & 0x3FF;
  float v;
  if (e == 0) v = ldexpf((float)m, -24);
  else if (e == 31) v = m ? NAN : INFINITY;
  else v = ldexpf((float)(m | 0x400), e - 25);
  return (h & 0x8000) ? -v : v;
}

/* SFilteredData(const SFilteredDataCompact&) of a 32-byte payload. */
static fdat fd_decode(const uint8_t* c) {
  const float inv16 = 1.0f / 65535.0f, inv8 = 1.0f / 255.0f;
  uint16_t u[6], nn[3], ior;
  fdat d;
  memcpy(&d.density, c, 4);
  memcpy(u, c + 4, 12);
  memcpy(nn, c + 22, 6);
  memcpy(&ior, c + 28, 2);
  const float sx = u[0] * inv16, sy = u[1] * inv16, sz = u[2] * inv16;
  const float rxy = 2.0f * (u[3] * inv16) - 1.0f, rxz = 2.0f * (u[4] * inv16) - 1.0f, ryz = 2.0f * (u[5] * inv16) - 1.0f;
  d.S[0] = sx * sx; d.S[1] = sy * sy; d.S[2] = sz * sz;
  d.S[3] = rxy * sx * sy; d.S[4] = rxz * sx * sz; d.S[5] = ryz * sy * sz;
  d.diffuse = mul3s(F3((float)c[16], (float)c[17], (float)c[18]), inv8);
  d.specular = mul3s(F3((float)c[19], (float)c[20], (float)c[21]), inv8);
  d.normal = norm3(sub3(mul3s(mul3s(F3((float)nn[0], (float)nn[1], (float)nn[2]), 2.0f), inv16), F3(1.0f, 1.0f, 1.0f)));
  d.ior = oi_half_to_float(ior);
  return d;
}

static fdat fd_lerp(float t, const fdat* a, const fdat* b) {
  const float u = 1.0f - t;
  fdat r;
  r.density = u * a->density + t * b->density;
  for (int k = 0; k < 6; ++k) r.S[k] = u * a->S[k] + t * b->S[k];
  r.diffuse = add3(mul3s(a->diffuse, u), mul3s(b->diffuse, t));
  r.specular = add3(mul3s(a->specular, u), mul3s(b->specular, t));
  r.normal = norm3(add3(mul3s(norm3(a->normal), u), mul3s(norm3(b->normal), t)));
  r.ior = u * a->ior + t * b->ior;
  return r;
}

static fdat med_voxel(const med_t* m, int x, int y, int z) {
  uint8_t v[32];
  oi_nvdb_value(&m->g, x, y, z, v);
  return fd_decode(v);
}

/* CNVDBMedium::filteredData: trilinear over 8 payloads at p (unit box). */
static fdat med_filtered(const med_t* m, f3 p) {
  const f3 ps = F3(p.x * (float)m->size[0] + (float)m->ibbMin[0] - 0.5f, p.y * (float)m->size[1] + (float)m->ibbMin[1] - 0.5f,
                   p.z * (float)m->size[2] + (float)m->ibbMin[2] - 0.5f);
  const int ix = (int)floorf(ps.x), iy = (int)floorf(ps.y), iz = (int)floorf(ps.z);
  const f3 d = F3(ps.x - (float)ix, ps.y - (float)iy, ps.z - (float)iz);
  fdat a, b;
  a = med_voxel(m, ix, iy, iz); b = med_voxel(m, ix + 1, iy, iz);
  const fdat d00 = fd_lerp(d.x, &a, &b);
  a = med_voxel(m, ix, iy + 1, iz); b = med_voxel(m, ix + 1, iy + 1, iz);
  const fdat d10 = fd_lerp(d.x, &a, &b);
  a = med_voxel(m, ix, iy, iz + 1); b = med_voxel(m, ix + 1, iy, iz + 1);
  const fdat d01 = fd_lerp(d.x, &a, &b);
  a = med_voxel(m, ix, iy + 1, iz + 1); b = med_voxel(m, ix + 1, iy + 1, iz + 1);
  const fdat d11 = fd_lerp(d.x, &a, &b);
  const fdat d0 = fd_lerp(d.y, &d00, &d10);
  const fdat d1 = fd_lerp(d.y, &d01, &d11);
  return fd_lerp(d.z, &d0, &d1);
}

/* nanovdb::Ray::intersects on the world box; exit t when the origin is strictly inside. */
static float med_box_hit(const med_t* m, f3 o, f3 d) {
  float t0 = 0.0f, t1 = DEFAULT_TMAX;
  const f3 inv = F3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  for (int i = 0; i < 3; ++i) {
    float a = comp3(m->bbMin, i), b = comp3(m->bbMax, i);
    if (a >= b) return -1.0f;
    a = (a - comp3(o, i)) * comp3(inv, i);
    b = (b - comp3(o, i)) * comp3(inv, i);
    if (a > b) { float t = a; a = b; b = t; }
    if (a > t0) t0 = a;
    if (b < t1) t1 = b;
    if (t0 > t1) return -1.0f;
  }
  if (!(t1 < DEFAULT_TMAX)) return -1.0f;
  const int inside = o.x > m->bbMin.x && o.y > m->bbMin.y && o.z > m->bbMin.z && o.x < m->bbMax.x &&
                     o.y < m->bbMax.y && o.z < m->bbMax.z;
  return inside ? t1 : t0;
}

static uint32_t brick_word(const uint32_t* a, int nx, int ny, int nz, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0u;
  return a[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny];
}
static float brick_majorant(const med_t* m, f3 ip, int mip) {
  const int bx = (int)floorf(ip.x) >> 3, by = (int)floorf(ip.y) >> 3, bz = (int)floorf(ip.z) >> 3;
  const int nx = (int)m->b.nb[0], ny = (int)m->b.nb[1], nz = (int)m->b.nb[2];
  uint32_t w;
  if (mip <= 0) w = brick_word(m->b.range, nx, ny, nz, bx, by, bz);
  else w = brick_word(m->b.mips[mip - 1], nx >> mip, ny >> mip, nz >> mip, bx >> mip, by >> mip, bz >> mip);
  return oi_half_to_float((uint16_t)(w >> 16));
}
static float brick_density(const med_t* m, f3 ip) {
  const int ix = (int)floorf(ip.x), iy = (int)floorf(ip.y), iz = (int)floorf(ip.z);
  const int nx = (int)m->b.nb[0], ny = (int)m->b.nb[1], nz = (int)m->b.nb[2];
  const uint32_t ptr = brick_word(m->b.ind, nx, ny, nz, ix >> 3, iy >> 3, iz >> 3);
  const uint32_t rw = brick_word(m->b.range, nx, ny, nz, ix >> 3, iy >> 3, iz >> 3);
  const int ax = (int)((ptr >> 22) & 1023u) * 8 + (ix & 7);
  const int ay = (int)((ptr >> 12) & 1023u) * 8 + (iy & 7);
  const int az = (int)((ptr >> 2) & 1023u) * 8 + (iz & 7);
  uint8_t v = 0;
  if (ax < (int)m->b.ad[0] && ay < (int)m->b.ad[1] && az < (int)m->b.ad[2])
    v = m->b.atlas[(size_t)ax + (size_t)ay * m->b.ad[0] + (size_t)az * m->b.ad[0] * m->b.ad[1]];
  const float lo = oi_half_to_float((uint16_t)(rw & 0xFFFFu)), hi = oi_half_to_float((uint16_t)(rw >> 16));
  return lo + (float)v * (1.0f / 255.0f) * (hi - lo);
}
static float step_dda(f3 pos, f3 inv, int mip) {
  const float dim = (float)(8 << mip);
  const float ox = inv.x >= 0.0f ? dim + 0.5f : -0.5f;
  const float oy = inv.y >= 0.0f ? dim + 0.5f : -0.5f;
  const float oz = inv.z >= 0.0f ? dim + 0.5f : -0.5f;
  const float tx = (floorf(pos.x * (1.0f / dim)) * dim + ox - pos.x) * inv.x;
  const float ty = (floorf(pos.y * (1.0f / dim)) * dim + oy - pos.y) * inv.y;
  const float tz = (floorf(pos.z * (1.0f / dim)) * dim + oz - pos.z) * inv.z;
  return fminf(tx, fminf(ty, tz));
}

typedef struct { int hit; f3 pos, normal; float S[6]; float ior; } mev_t;

static f3 scatter_albedo(const med_t* m, const fdat* fd, f3 dirModel) {
  const f3 n = norm3(fd->normal);
  const float w = fresnel(1.0f, fd->ior, fabsf(dot3(norm3(neg3(dirModel)), n)));
  const f3 a = add3(mul3s(fd->diffuse, 1.0f - w), mul3s(fd->specular, w));
  return F3(a.x * m->sigmaS.x / m->sigmaT, a.y * m->sigmaS.y / m->sigmaT, a.z * m->sigmaS.z / m->sigmaT);
}
static void fill_event(mev_t* ev, ray_t w, const fdat* fd) {
  ev->hit = 1;
  ev->pos = add3(w.o, mul3s(w.d, w.tmax));
  ev->normal = norm3(fd->normal);
  for (int k = 0; k < 6; ++k) ev->S[k] = fd->S[k];
  ev->ior = fd->ior;
}
static float inv_majorant(const med_t* m) { return 1.0f / (m->ratio / m->invMax); }

static f3 med_sample_internal(const med_t* m, ray_t rm, rng_t* rng, mev_t* ev, int* err) {
  ray_t ray = ray_xf2(rm, m->m2i);
  const float invMax = inv_majorant(m);
  if (!(invMax < INFINITY)) return F3(1.0f, 1.0f, 1.0f);
  float t = 0.0f;
  for (int it = 0; it < MAX_TRACKING_STEPS; ++it) {
    t -= oi_log(1.0f - rng_next(rng)) * invMax / m->sigmaT;
    if (t >= ray.tmax) return F3(1.0f, 1.0f, 1.0f);
    const fdat fd = med_filtered(m, add3(ray.o, mul3s(ray.d, t)));
    if (m->ratio * fd.density * invMax > rng_next(rng)) {
      ray.tmax = t;
      const ray_t w = ray_xf2(ray, m->i2m);
      fill_event(ev, w, &fd);
      return scatter_albedo(m, &fd, w.d);
    }
  }
  *err = 1;
  return F3(0.0f, 0.0f, 0.0f);
}

static f3 med_sample_dda(const med_t* m, ray_t rm, rng_t* rng, mev_t* ev, int* err) {
  ray_t iray = ray_xf2(rm, m->u2s);
  const f3 ri = F3(1.0f / iray.d.x, 1.0f / iray.d.y, 1.0f / iray.d.z);
  float t = 0.0f;
  float tau = -oi_log(1.0f - rng_next(rng));
  float mip = 3.0f;
  for (int it = 0; it < MAX_TRACKING_STEPS; ++it) {
    if (!(t < iray.tmax)) return F3(1.0f, 1.0f, 1.0f);
    const f3 curr = add3(iray.o, mul3s(iray.d, t));
    const int mi = (int)roundf(mip);
    const float majorant = m->ratio * brick_majorant(m, curr, mi);
    const float dt = step_dda(curr, ri, mi);
    const float prevT = t;
    t += dt / m->sigmaT;
    if (t == prevT) return F3(1.0f, 1.0f, 1.0f);
    tau -= majorant * dt;
    mip = fminf(mip + 0.25f, 3.0f);
    if (tau > 0.0f) continue;
    t += tau / (majorant * m->sigmaT);
    if (t >= iray.tmax) return F3(1.0f, 1.0f, 1.0f);
    const float jx = rng_next(rng);
    const float jy = rng_next(rng);
    const float jz = rng_next(rng);
    const float d = brick_density(m, sub3(add3(add3(iray.o, mul3s(iray.d, t)), F3(jx, jy, jz)), F3(0.5f, 0.5f, 0.5f)));
    if (rng_next(rng) * majorant < d * m->ratio) {
      iray.tmax = t;
      const f3 ip = add3(iray.o, mul3s(iray.d, t));
      const f3 pos = F3((ip.x - (float)m->ibbMin[0]) / (float)m->size[0], (ip.y - (float)m->ibbMin[1]) / (float)m->size[1],
                        (ip.z - (float)m->ibbMin[2]) / (float)m->size[2]);
      const fdat fd = med_filtered(m, pos);
      const ray_t w = ray_xf2(iray, m->s2m);
      fill_event(ev, w, &fd);
      return scatter_albedo(m, &fd, w.d);
    }
    tau = -oi_log(1.0f - rng_next(rng));
    mip = fmaxf(0.0f, mip - 2.0f);
  }
  *err = 1;
  return F3(0.0f, 0.0f, 0.0f);
}

static float med_tr_internal(const med_t* m, ray_t rm, rng_t* rng, int* err) {
  const ray_t ray = ray_xf2(rm, m->m2i);
  const float invMax = inv_majorant(m);
  if (!(invMax < INFINITY)) return 1.0f;
  float tr = 1.0f, t = 0.0f;
  for (int it = 0; it < MAX_TRACKING_STEPS; ++it) {
    t -= oi_log(1.0f - rng_next(rng)) * invMax / m->sigmaT;
    if (t >= ray.tmax) return tr;
    const float d = med_filtered(m, add3(ray.o, mul3s(ray.d, t))).density;
    tr *= 1.0f - fmaxf(0.0f, m->ratio * d * invMax);
    if (tr < 1.0f) {
      const float p = 1.0f - tr;
      if (rng_next(rng) < p) return 0.0f;
      tr /= 1.0f - p;
    }
  }
  *err = 1;
  return 0.0f;
}

static float med_tr_dda(const med_t* m, ray_t rm, rng_t* rng, int* err) {
  const ray_t iray = ray_xf2(rm, m->u2s);
  const f3 ri = F3(1.0f / iray.d.x, 1.0f / iray.d.y, 1.0f / iray.d.z);
  float tr = 1.0f, t = 0.0f;
  const float volMajorant = 1.0f / inv_majorant(m);
  float tau = -oi_log(1.0f - rng_next(rng));
  float mip = 3.0f;
  for (int it = 0; it < MAX_TRACKING_STEPS; ++it) {
    if (!(t < iray.tmax)) return tr;
    const f3 curr = add3(iray.o, mul3s(iray.d, t));
    const int mi = (int)roundf(mip);
    const float majorant = m->ratio * brick_majorant(m, curr, mi);
    const float dt = step_dda(curr, ri, mi);
    const float prevT = t;
    t += dt / m->sigmaT;
    if (t == prevT) return tr;
    tau -= majorant * dt;
    mip = fminf(mip + 0.25f, 3.0f);
    if (tau > 0.0f) continue;
    t += tau / (majorant * m->sigmaT);
    if (t >= iray.tmax) return tr;
    const float jx = rng_next(rng);
    const float jy = rng_next(rng);
    const float jz = rng_next(rng);
    const float d = brick_density(m, sub3(add3(add3(iray.o, mul3s(iray.d, t)), F3(jx, jy, jz)), F3(0.5f, 0.5f, 0.5f)));
    if (rng_next(rng) * majorant < d * m->ratio) {
      tr *= fmaxf(0.0f, 1.0f - volMajorant / majorant);
      if (tr < 0.1f) {
        const float prob = 1.0f - tr;
        if (rng_next(rng) < prob) return 0.0f;
        tr /= 1.0f - prob;
      }
    }
    tau = -oi_log(1.0f - rng_next(rng));
    mip = fmaxf(0.0f, mip - 2.0f);
  }
  *err = 1;
  return 0.0f;
}

static f3 inst_sample(const med_t* m, ray_t rw, int dda, rng_t* rng, mev_t* ev, int* err) {
  const ray_t rm = ray_xf2(rw, m->w2m);
  ev->hit = 0;
  const f3 a = dda ? med_sample_dda(m, rm, rng, ev, err) : med_sample_internal(m, rm, rng, ev, err);
  if (ev->hit) {
    ev->pos = xpoint(m->m2w, ev->pos);
    ev->normal = norm3(xvec(m->m2w, ev->normal));
  }
  return a;
}
static float inst_tr(const med_t* m, ray_t rw, int dda, rng_t* rng, int* err) {
  const ray_t rm = ray_xf2(rw, m->w2m);
  return dda ? med_tr_dda(m, rm, rng, err) : med_tr_internal(m, rm, rng, err);
}

/* CNVDBMedium::moveToVoxelBorder and CMediumInstance::moveToVoxelBorder. */
static ray_t med_move(const med_t* m, ray_t rm) {
  const ray_t ri = ray_xf(rm, m->m2i);
  const f3 ibb = F3((float)m->ibbMin[0], (float)m->ibbMin[1], (float)m->ibbMin[2]);
  const f3 sz = F3((float)m->size[0], (float)m->size[1], (float)m->size[2]);
  const f3 ip = F3(ri.o.x * sz.x + ibb.x, ri.o.y * sz.y + ibb.y, ri.o.z * sz.z + ibb.z);
  const f3 vlo = F3((floorf(ip.x) - ibb.x) / sz.x, (floorf(ip.y) - ibb.y) / sz.y, (floorf(ip.z) - ibb.z) / sz.z);
  const f3 vhi = F3((ceilf(ip.x) - ibb.x) / sz.x, (ceilf(ip.y) - ibb.y) / sz.y, (ceilf(ip.z) - ibb.z) / sz.z);
  const float eps = FLT_EPSILON;
  const float gamma = (3.0f * eps) / (1.0f - 3.0f * eps);
  float t1 = ri.tmax;
  for (int i = 0; i < 3; ++i) {
    const float inv = 1.0f / comp3(ri.d, i);
    float tn = (comp3(vlo, i) - comp3(ri.o, i)) * inv;
    float tf = (comp3(vhi, i) - comp3(ri.o, i)) * inv;
    if (tn > tf) { float tt = tn; tn = tf; tf = tt; }
    tf *= 1.0f + 2.0f * gamma;
    t1 = tf < t1 ? tf : t1;
  }
  t1 *= (1.0f - RAY_OFFSET);
  const ray_t moved = mkray(add3(ri.o, mul3s(ri.d, t1)), ri.d, ri.tmax - t1);
  return ray_off(ray_xf(moved, m->i2m), neg3(rm.d));
}
static ray_t inst_move(const med_t* m, ray_t rw) {
  const ray_t rm = ray_xf(rw, m->w2m);
  const ray_t moved = med_move(m, rm);
  return ray_off(ray_xf(moved, m->m2w), neg3(rw.d));
}

/* SGGX microflake distribution and phase function. */
typedef struct { float S[6]; float inv[9]; f3 normal; } sggx_t;
static float s_at(const float* S, int r, int c) {
  if (r == c) return S[r];
  const int a = r < c ? r : c, b = r < c ? c : r;
  return (a == 0 && b == 1) ? S[3] : ((a == 0) ? S[4] : S[5]);
}
static float det3s(const float* S) {
  return s_at(S, 0, 0) * (s_at(S, 1, 1) * s_at(S, 2, 2) - s_at(S, 2, 1) * s_at(S, 1, 2)) -
         s_at(S, 1, 0) * (s_at(S, 0, 1) * s_at(S, 2, 2) - s_at(S, 2, 1) * s_at(S, 0, 2)) +
         s_at(S, 2, 0) * (s_at(S, 0, 1) * s_at(S, 1, 2) - s_at(S, 1, 1) * s_at(S, 0, 2));
}
static f3 smul(const float* S, f3 w) {
  return F3(s_at(S, 0, 0) * w.x + s_at(S, 1, 0) * w.y + s_at(S, 2, 0) * w.z,
            s_at(S, 0, 1) * w.x + s_at(S, 1, 1) * w.y + s_at(S, 2, 1) * w.z,
            s_at(S, 0, 2) * w.x + s_at(S, 1, 2) * w.y + s_at(S, 2, 2) * w.z);
}
static sggx_t make_sggx(const float* S, f3 n) {
  sggx_t g;
  float m[3][3];
  for (int k = 0; k < 6; ++k) g.S[k] = S[k];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) m[c][r] = s_at(S, r, c);
  const float o = 1.0f / (m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                          m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
                          m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]));
  g.inv[0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * o;
  g.inv[3] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * o;
  g.inv[6] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * o;
  g.inv[1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * o;
  g.inv[4] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * o;
  g.inv[7] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * o;
  g.inv[2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * o;
  g.inv[5] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * o;
  g.inv[8] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * o;
  g.normal = n;
  return g;
}
static float sggx_D(const sggx_t* g, f3 w) {
  const f3 iw = F3(g->inv[0] * w.x + g->inv[3] * w.y + g->inv[6] * w.z, g->inv[1] * w.x + g->inv[4] * w.y + g->inv[7] * w.z,
                   g->inv[2] * w.x + g->inv[5] * w.y + g->inv[8] * w.z);
  const float v = dot3(w, iw);
  return (float)(1.0 / (PI_D * (double)sqrtf(fabsf(det3s(g->S))) * (double)v * (double)v));
}
static float sggx_sigma(const sggx_t* g, f3 w) { return sqrtf(fmaxf(dot3(w, smul(g->S, w)), 0.0f)); }
static f3 sggx_vndf(const sggx_t* g, float u1, float u2) {
  const f3 N = g->normal;
  f3 T, B;
  if (N.z < -0.9999999f) {
    T = F3(0.0f, -1.0f, 0.0f);
    B = F3(-1.0f, 0.0f, 0.0f);
  } else {
    const float a = 1.0f / (1.0f + N.z);
    const float b = -N.x * N.y * a;
    T = norm3(F3(1.0f - N.x * N.x * a, b, -N.x));
    B = norm3(F3(b, 1.0f - N.y * N.y * a, -N.y));
  }
  const f3 wk = B, wj = T, wi = N;
  const float Skk = dot3(wk, smul(g->S, wk)), Skj = dot3(wk, smul(g->S, wj)), Ski = dot3(wk, smul(g->S, wi));
  const float Sjj = dot3(wj, smul(g->S, wj)), Sji = dot3(wj, smul(g->S, wi)), Sii = dot3(wi, smul(g->S, wi));
  const float P[6] = {Skk, Sjj, Sii, Skj, Ski, Sji};
  const float temp = sqrtf(Sjj * Sii - Sji * Sji);
  const f3 Mk = F3(sqrtf(fabsf(det3s(P))) / temp, 0.0f, 0.0f);
  const float scaling = 1.0f / sqrtf(Sii);
  const f3 Mj = mul3s(F3(-(Ski * Sji - Skj * Sii) / temp, temp, 0.0f), scaling);
  const f3 Mi = mul3s(F3(Ski, Sji, Sii), scaling);
  const float sq = sqrtf(u1);
  float sn, cs;
  orc_sincos_turns(u2, &sn, &cs);
  const float u = sq * cs, v = sq * sn;
  const float w = sqrtf(1.0f - u * u - v * v);
  const f3 wm = norm3(add3(add3(mul3s(Mk, u), mul3s(Mj, v)), mul3s(Mi, w)));
  return norm3(add3(add3(mul3s(wk, wm.x), mul3s(wj, wm.y)), mul3s(wi, wm.z)));
}
static float sggx_p_spec(const sggx_t* g, f3 wo, f3 wi) {
  const f3 wh = norm3(add3(wi, wo));
  return sggx_D(g, wh) / (4.0f * sggx_sigma(g, wo));
}
static float sggx_p(const sggx_t* g, float ior, f3 wo, f3 wi, rng_t* rng) {
  const float w = fresnel(1.0f, ior, fabsf(dot3(norm3(wo), g->normal)));
  const float a = rng_next(rng);
  const float b = rng_next(rng);
  const f3 wm = sggx_vndf(g, a, b);
  const float pd = (float)((double)fmaxf(dot3(wi, wm), 0.0f) / PI_D);
  return pd * (1.0f - w) + sggx_p_spec(g, wo, wi) * w;
}
static float sggx_sample_p(const sggx_t* g, float ior, f3 wo, f3* wi, rng_t* rng) {
  const float w = fresnel(1.0f, ior, fabsf(dot3(norm3(wo), g->normal)));
  if (rng_next(rng) < w) {
    const float a = rng_next(rng);
    const float b = rng_next(rng);
    const f3 wm = sggx_vndf(g, a, b);
    *wi = reflect3(neg3(wo), wm);
    return sggx_p_spec(g, wo, *wi);
  }
  const float a = rng_next(rng);
  const float b = rng_next(rng);
  const f3 wn = sggx_vndf(g, a, b);
  const frame_t fr = frame_from_normal(wn);
  const float c1 = rng_next(rng);
  const float c2 = rng_next(rng);
  *wi = norm3(to_world(&fr, cosine_hemisphere(c1, c2)));
  return (float)((double)fmaxf(dot3(*wi, wn), 0.0f) / PI_D);
}

/* Henyey-Greenstein (henyey_greenstein_phase_function.hpp:22-50). */
static float phase_hg(float cosTheta, float g) {
  const float denom = 1.0f + g * g + 2.0f * g * cosTheta;
  return (float)((double)(1.0f - g * g) / (4.0 * PI_D * (double)denom * (double)sqrtf(denom)));
}
static float hg_sample_p(float g, f3 wo, f3* wi, rng_t* rng) {
  const float u1 = rng_next(rng);
  const float u2 = rng_next(rng);
  float cosTheta;
  if (fabsf(g) < 1e-3f) {
    cosTheta = 1.0f - 2.0f * u1;
  } else {
    const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
    cosTheta = (1.0f + g * g - sq * sq) / (2.0f * g);
  }
  const float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
  float s, c;
  orc_sincos_turns(u2, &s, &c);
  const f3 v1 = fabsf(wo.x) > fabsf(wo.y) ? div3s(F3(-wo.z, 0.0f, wo.x), sqrtf(wo.x * wo.x + wo.z * wo.z))
                                          : div3s(F3(0.0f, wo.z, -wo.y), sqrtf(wo.y * wo.y + wo.z * wo.z));
  const f3 v2 = cross3(wo, v1);
  *wi = add3(add3(mul3s(v1, sinTheta * c), mul3s(v2, sinTheta * s)), mul3s(neg3(wo), cosTheta));
  return phase_hg(-cosTheta, g);
}

/* getRotation (functions.hpp:128-142): +Y to `n`, entries rounded. */
static m4_t rot_from_normal(f3 n) {
  m4_t r = oi_m4_id();
  const float c = dot3(n, F3(0.0f, 1.0f, 0.0f));
  if (c == 1.0f) return r;
  if (c == -1.0f) { r.m[0][0] = r.m[1][1] = r.m[2][2] = -1.0f; return r; }
  const float angle = acosf(c);
  const f3 ax = norm3(cross3(n, F3(0.0f, 1.0f, 0.0f)));
  const float cs = cosf(angle), sn = sinf(angle);
  const f3 tp = mul3s(ax, 1.0f - cs);
  r.m[0][0] = cs + tp.x * ax.x; r.m[0][1] = tp.x * ax.y + sn * ax.z; r.m[0][2] = tp.x * ax.z - sn * ax.y;
  r.m[1][0] = tp.y * ax.x - sn * ax.z; r.m[1][1] = cs + tp.y * ax.y; r.m[1][2] = tp.y * ax.z + sn * ax.x;
  r.m[2][0] = tp.z * ax.x + sn * ax.y; r.m[2][1] = tp.z * ax.y - sn * ax.x; r.m[2][2] = cs + tp.z * ax.z;
  for (int c2 = 0; c2 < 4; ++c2)
    for (int i = 0; i < 4; ++i) r.m[c2][i] = roundf(r.m[c2][i]);
  return r;
}
static m4_t affine4(m4_t a) {
  for (int c = 0; c < 4; ++c) a.m[c][3] = c == 3 ? 1.0f : 0.0f;
  return a;
}

/* CNVDBMedium::getVoxelSizeFiltering: trailing \d+\.\d+ of the path. */
static int voxel_size_from_path(const char* path, float* out) {
  size_t n = strlen(path), i = n;
  while (i > 0 && path[i - 1] >= '0' && path[i - 1] <= '9') --i;
  if (i == n || i == 0 || path[i - 1] != '.') return -1;
  size_t k = i - 1;
  while (k > 0 && path[k - 1] >= '0' && path[k - 1] <= '9') --k;
  if (k == i - 1) return -1;
  *out = strtof(path + k, NULL);
  return 0;
}

/* Placement of one instance: T(pos) R(orientation) S(scaling), the world box
   from the model box's two corners, the filter/render voxel ratio
   (sceneobject.cu:50-65, 108-114; aabb.hpp:9-13). */
static void med_place(med_t* m, const orc_medium* om) {
  m4_t T = oi_m4_id(), Sc = oi_m4_id();
  for (int k = 0; k < 3; ++k) { T.m[3][k] = om->pos[k]; Sc.m[k][k] = om->scaling[k]; }
  const m4_t m2w = oi_m4_mul(oi_m4_mul(T, rot_from_normal(F3(om->orientation[0], om->orientation[1], om->orientation[2]))), Sc);
  oi_m4_to43(m2w, m->m2w);
  oi_m4_to43(oi_m4_inv(m2w), m->w2m);
  const f3 bmin = F3((float)m->g.worldBBox[0], (float)m->g.worldBBox[1], (float)m->g.worldBBox[2]);
  const f3 bmax = F3((float)m->g.worldBBox[3], (float)m->g.worldBBox[4], (float)m->g.worldBBox[5]);
  const f3 a = xpoint(m->m2w, bmin), b = xpoint(m->m2w, bmax);
  m->bbMin = F3(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z);
  m->bbMax = F3(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z);
  m->ratio = m->vsF / ((m->bbMax.x - m->bbMin.x) / (float)m->size[0]);
}

static int med_load(med_t* m, const orc_medium* om) {
  memset(m, 0, sizeof(*m));
  char buf[4096];
  float vsF;
  if (voxel_size_from_path(om->path, &vsF)) return -1;
  m->vsF = vsF;
  snprintf(buf, sizeof(buf), "%s.nvdb", om->path);
  if (oi_nvdb_read(buf, &m->g)) return -2;
  snprintf(buf, sizeof(buf), "%s.brickgrid", om->path);
  if (oi_bricks_read(buf, &m->b)) { oi_nvdb_free(&m->g); return -3; }
  for (int k = 0; k < 3; ++k) {
    const int lo = m->g.voxelCount == 0 ? 0 : m->g.indexBBox[k];
    const int hi = m->g.voxelCount == 0 ? 0 : m->g.indexBBox[3 + k];
    m->ibbMin[k] = lo;
    m->size[k] = hi - lo + 1;
  }
  m4_t nano = oi_m4_id(), toNano = oi_m4_id();
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) nano.m[c][r] = m->g.matF[3 * r + c];
  for (int r = 0; r < 3; ++r) nano.m[3][r] = m->g.vecF[r];
  for (int k = 0; k < 3; ++k) { toNano.m[k][k] = (float)m->size[k]; toNano.m[3][k] = (float)m->ibbMin[k]; }
  const m4_t i2m = affine4(oi_m4_mul(nano, toNano));
  const m4_t m2i = affine4(oi_m4_inv(i2m));
  const m4_t s2i = affine4(oi_m4_inv(toNano));
  oi_m4_to43(i2m, m->i2m);
  oi_m4_to43(m2i, m->m2i);
  oi_m4_to43(oi_m4_mul(toNano, m2i), m->u2s);
  oi_m4_to43(oi_m4_mul(i2m, s2i), m->s2m);
  m->hg = om->hg;
  m->hgG = om->g;
  m->sigmaS = F3(om->sigma_s[0], om->sigma_s[1], om->sigma_s[2]);
  m->sigmaT = fmaxf(om->sigma_a[0] + om->sigma_s[0], fmaxf(om->sigma_a[1] + om->sigma_s[1], om->sigma_a[2] + om->sigma_s[2]));
  m->invMax = 1.0f / oi_nvdb_max_density(&m->g);
  m->owner = 1;
  med_place(m, om);
  return 0;
}
static void med_free(med_t* m) {
  if (!m->owner) return;
  oi_nvdb_free(&m->g);
  oi_bricks_free(&m->b);
}

/* ------------------------------------------------------------ scene */
/* Two-level scenes: a mesh asset in model space with its own BVH and
 * per-BVH-order shading data, and its instances (the GPU's BvhInstance). */
typedef struct {
  int32_t* nodes;
  uint32_t* order;
  float* tris;
  uint32_t ntris;
  const float* nrm;     /* per vertex, model space */
  const uint32_t* idx;  /* local vertex indices */
  int mat;              /* index into the scene's materials */
  float* triUV;         /* per BVH-order triangle, 6 each; null without coordinates */
  int* triAlpha;
  oi_alpha alpha;       /* alpha.alpha_tex null: no alpha test */
} asset_t;
typedef struct {
  int asset;
  float m2w[12];  /* object -> world, glm mat4x3 column order */
  float w2o[12];  /* world -> object, three rows of (3x3 | translation) */
  uint32_t code;  /* hit code of the asset's BVH-order triangle 0 */
} oinst_t;

typedef struct {
  int32_t* nodes;
  float* tris;
  uint32_t* order;
  float* wnrm;      /* per vertex, world space (unnormalised) */
  uint32_t* idx;    /* global indices */
  uint32_t* triMat; /* per original triangle */
  mat_t* mats;
  float* uv;        /* per vertex (global), 2 each; null without texture coordinates */
  oi_tex* tex;      /* texture table */
  int ntex;
  oi_alpha alpha;   /* alpha.alpha_tex null: no alpha test */
  int* triAlpha;    /* per BVH-order triangle */
  float* triUV;     /* per BVH-order triangle, 6 each */
  uint32_t ntris;
  asset_t* assets;  /* two-level: codes from ntris on belong to instances */
  oinst_t* insts;
  uint32_t ninst;
  const orc_shape* shapes;
  mat_t* shapeMats;
  uint32_t nshapes;
  med_t* media;
  uint32_t nmedia;
  int dda;
  env_t env;
  /* camera */
  float v2w[12];
  float pixelSize, nearPlane;
  int W, H;
  uint32_t spp, maxDepth, seed;
} rscene_t;

/* The object-space ray of instance I (the GPU's inst_point / inst_vector). */
static void inst_ray(const oinst_t* I, f3 o, f3 d, f3* oo, f3* od) {
  const float* w = I->w2o;
  *oo = F3(w[0] * o.x + w[1] * o.y + w[2] * o.z + w[3], w[4] * o.x + w[5] * o.y + w[6] * o.z + w[7],
           w[8] * o.x + w[9] * o.y + w[10] * o.z + w[11]);
  *od = F3(w[0] * d.x + w[1] * d.y + w[2] * d.z, w[4] * d.x + w[5] * d.y + w[6] * d.z,
           w[8] * d.x + w[9] * d.y + w[10] * d.z);
}

/* Closest triangle over the world-space meshes and every instance: the hit
 * code (world: BVH-order triangle; instance: its code + the asset's
 * BVH-order triangle), -1 on a miss; ties in t go to the lower code. */
static int tris_closest(const rscene_t* S, f3 o, f3 d, float tmax, hit_t* out) {
  hit_t best;
  best.t = tmax;
  best.b1 = best.b2 = 0.0f;
  best.tri = -1;
  if (S->ntris > 0) {
    hit_t h = oi_trace_alpha(S->nodes, S->tris, o, d, tmax, 0, S->alpha.alpha_tex ? &S->alpha : NULL);
    if (h.tri >= 0) best = h;
  }
  for (uint32_t i = 0; i < S->ninst; ++i) {
    const oinst_t* I = &S->insts[i];
    const asset_t* A = &S->assets[I->asset];
    f3 oo, od;
    inst_ray(I, o, d, &oo, &od);
    hit_t h = oi_trace_alpha(A->nodes, A->tris, oo, od, best.t, 0, A->alpha.alpha_tex ? &A->alpha : NULL);
    if (h.tri < 0) continue;
    const int code = (int)(I->code + (uint32_t)h.tri);
    if (best.tri < 0 || h.t < best.t || (h.t == best.t && code < best.tri)) {
      best = h;
      best.tri = code;
    }
  }
  *out = best;
  return best.tri;
}

static int tris_occluded(const rscene_t* S, f3 o, f3 d, float tmax) {
  if (S->ntris > 0) {
    hit_t h = oi_trace_alpha(S->nodes, S->tris, o, d, tmax, 1, S->alpha.alpha_tex ? &S->alpha : NULL);
    if (h.tri >= 0) return 1;
  }
  for (uint32_t i = 0; i < S->ninst; ++i) {
    const oinst_t* I = &S->insts[i];
    const asset_t* A = &S->assets[I->asset];
    f3 oo, od;
    inst_ray(I, o, d, &oo, &od);
    hit_t h = oi_trace_alpha(A->nodes, A->tris, oo, od, tmax, 1, A->alpha.alpha_tex ? &A->alpha : NULL);
    if (h.tri >= 0) return 1;
  }
  return 0;
}

/* closest: code >= 0 BVH-order triangle, -1 miss, -2 - i shape i */
static int scene_closest(const rscene_t* S, f3 o, f3 d, float tmax, float* tOut, float* b1, float* b2) {
  float t = tmax;
  int code = -1;
  *b1 = *b2 = 0.0f;
  if (S->ntris > 0 || S->ninst > 0) {
    hit_t h;
    if (tris_closest(S, o, d, tmax, &h) >= 0) { t = h.t; *b1 = h.b1; *b2 = h.b2; code = h.tri; }
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
    if (ts > 0.0f && ts < t) { t = ts; *b1 = *b2 = 0.0f; code = -2 - (int)i; }
  }
  *tOut = t;
  return code;
}

/* closest including the medium boxes: code MEDIUM_CODE_BASE - m for medium m */
static int scene_closest_media(const rscene_t* S, f3 o, f3 d, float tmax, float* tOut, float* b1, float* b2) {
  int code = scene_closest(S, o, d, tmax, tOut, b1, b2);
  for (uint32_t m = 0; m < S->nmedia; ++m) {
    const float tm = med_box_hit(&S->media[m], o, d);
    if (tm >= 0.0f && tm <= tmax && tm < *tOut) {
      *tOut = tm;
      *b1 = *b2 = 0.0f;
      code = MEDIUM_CODE_BASE - (int)m;
    }
  }
  return code;
}

static int scene_occluded(const rscene_t* S, f3 o, f3 d, float tmax) {
  if (tris_occluded(S, o, d, tmax)) return 1;
  if (S->nshapes > 0) {
    rscene_t T = *S;
    T.ntris = 0;
    T.ninst = 0;
    float t, b1, b2;
    if (scene_closest(&T, o, d, tmax, &t, &b1, &b2) != -1) return 1;
  }
  return 0;
}

/* Replay of trace_path's draws (test hook, orc_set_replay): while set, each
 * Philox block of a surface path (camera, per bounce the shading blocks and
 * the roulette block) is the next four words of the list, in the order the
 * path asks for them; g_replay_swap exchanges the two direction draws of the
 * GGX lobe, for a build that evaluates glm::vec2(u(), u()) right to left. */
static const uint32_t* g_replay = NULL;
static size_t g_replay_n = 0, g_replay_pos = 0;
static int g_replay_swap = 0;

void orc_set_replay(const uint32_t* words, size_t n, int vec2_swap) {
  g_replay = words;
  g_replay_n = n;
  g_replay_pos = 0;
  g_replay_swap = vec2_swap;
  g_replay_swap_lobe = words ? vec2_swap : 0;
}

static void philox_u(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[4]) {
  if (g_replay) {
    for (int k = 0; k < 4; ++k) out[k] = g_replay_pos < g_replay_n ? g_replay[g_replay_pos++] : 0x80000000u;
    return;
  }
  uint32_t ctr[4] = {c0, c1, c2, c3}, key[2] = {k0, k1};
  orc_philox4x32_10(ctr, key, out);
}

/* intersectTr as direct() uses it: 0 when the walk ends on a surface, else
 * the product of the media's ratio-tracking estimates along the segments. */
static float shadow_tr(const rscene_t* S, f3 o, f3 d, float tmax, int med, rng_t* rng, int* err) {
  f3 p0 = o;
  const f3 p1 = add3(o, mul3s(d, tmax));
  const ray_t r0 = spawn_ray(p0, p1);
  if (scene_occluded(S, r0.o, r0.d, r0.tmax)) return 0.0f;
  float tr = 1.0f;
  if (S->nmedia == 0) return tr;
  int cur = med;
  for (int k = 0; k < MAX_SHADOW_SEGMENTS; ++k) {
    const f3 off = offset_origin(p0, norm3(sub3(p1, p0)));
    const float tl = len3(sub3(p1, off));
    const f3 dir = div3s(sub3(p1, p0), tl);
    float best = tl;
    int hitM = -1;
    for (uint32_t m = 0; m < S->nmedia; ++m) {
      const float tm = med_box_hit(&S->media[m], off, dir);
      if (tm >= 0.0f && tm <= tl && tm < best) { best = tm; hitM = (int)m; }
    }
    if (hitM < 0) return tr;
    if (cur >= 0 && hitM == cur) tr *= inst_tr(&S->media[cur], mkray(off, dir, best), S->dda, rng, err);
    p0 = add3(off, mul3s(dir, best));
    cur = cur < 0 ? hitM : -1;
  }
  *err = 1;
  return 0.0f;
}

/* The medium part of Li (path_integrator_impl.hpp:127-192) up to the event
 * the bounce shades; updates the ray, its medium, and the throughput. */
static int extend_media(const rscene_t* S, uint32_t p, uint32_t s, uint32_t b, f3* o, f3* d, int* med, float* tmax,
                        f3* T, float* tHit, float* hb1, float* hb2, mev_t* ev, int* evMed, int* err) {
  int j;
  for (j = 0; j < MAX_PASS_THROUGH; ++j) {
    const int c = scene_closest_media(S, *o, *d, *tmax, tHit, hb1, hb2);
    int dead = 0;
    ev->hit = 0;
    if (c <= MEDIUM_CODE_BASE) {
      const int mi = MEDIUM_CODE_BASE - c;
      rng_t rs = rng_make(p, S->seed, s, b, PURPOSE_MEDIUM + (uint32_t)j);
      if (*med >= 0) {
        if (mi != *med) dead = 1;
        else { *T = mul3(*T, inst_sample(&S->media[*med], mkray(*o, *d, *tHit), S->dda, &rs, ev, err)); *evMed = *med; }
      } else {
        const ray_t mr = ray_off(mkray(add3(*o, mul3s(*d, *tHit)), norm3(*d), DEFAULT_TMAX), *d);
        float te, e1, e2;
        const int ce = scene_closest_media(S, mr.o, mr.d, mr.tmax, &te, &e1, &e2);
        if (ce != -1) {
          if (ce <= MEDIUM_CODE_BASE && MEDIUM_CODE_BASE - ce != mi) dead = 1;
          else { *T = mul3(*T, inst_sample(&S->media[mi], mkray(mr.o, mr.d, te), S->dda, &rs, ev, err)); *evMed = mi; }
        }
      }
      if (*err) dead = 1;
      if (!dead && (T->x == 0.0f || T->y == 0.0f || T->z == 0.0f)) dead = 1;
    }
    if (dead) return EV_DEAD;
    if (ev->hit) return EV_SCATTER;
    if (c <= MEDIUM_CODE_BASE) {
      const ray_t nr = ray_off(mkray(add3(*o, mul3s(*d, *tHit)), norm3(*d), DEFAULT_TMAX), *d);
      *o = nr.o;
      *d = nr.d;
      *tmax = nr.tmax;
      *med = *med < 0 ? MEDIUM_CODE_BASE - c : -1;
      continue;
    }
    return c;
  }
  *err = 1;
  return EV_DEAD;
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
  int med = -1;
  float tmax = DEFAULT_TMAX;
  for (uint32_t b = 0; b < S->maxDepth; ++b) {
    float t, hb1, hb2;
    int code;
    mev_t ev;
    int evMed = -1, err = 0;
    if (S->nmedia == 0) code = scene_closest(S, o, d, DEFAULT_TMAX, &t, &hb1, &hb2);
    else code = extend_media(S, p, s, b, &o, &d, &med, &tmax, &T, &t, &hb1, &hb2, &ev, &evMed, &err);
    if (code == -1) {
      if (b == 0) {
        float lp;
        f3 le = env_le(&S->env, d, &lp);
        L = add3(L, mul3(le, T));
      }
      break;
    }
    if (code == EV_DEAD) break;
    if (code == EV_SCATTER) {
      /* direct() with the phase function, then the phase-sampled continuation */
      const med_t* M = &S->media[evMed];
      const sggx_t g = make_sggx(ev.S, ev.normal);
      const f3 wo = neg3(d);
      rng_t rs = rng_make(p, S->seed, s, b, PURPOSE_SCATTER);
      f3 dl = F3(0.0f, 0.0f, 0.0f);
      int anyShadow = 0;
      {
        f3 ldir;
        float lpdf = 0.0f;
        const float u0 = rng_next(&rs);
        const float u1 = rng_next(&rs);
        const f3 Le = env_sample(&S->env, u0, u1, &ldir, &lpdf);
        if (lpdf > 0.0f) {
          ldir = norm3(ldir);
          const ray_t lr = inst_move(M, ray_off(mkray(ev.pos, ldir, DEFAULT_TMAX), ev.normal));
          const float sp = M->hg ? phase_hg(dot3(wo, ldir), M->hgG) : sggx_p(&g, ev.ior, wo, ldir, &rs);
          const float mis = (1.0f * lpdf) / (1.0f * lpdf + 1.0f * sp);
          const f3 pre = mul3(mul3s(F3(sp, sp, sp), mis), Le);
          rng_t rt = rng_make(p, S->seed, s, b, PURPOSE_SHADOW_TR + 0u);
          const float tr = shadow_tr(S, lr.o, lr.d, lr.tmax, evMed, &rt, &err);
          dl = add3(dl, div3s(mul3s(pre, tr), lpdf));
          anyShadow = 1;
        }
      }
      {
        f3 wi = F3(0.0f, 0.0f, 0.0f);
        const float sp = M->hg ? hg_sample_p(M->hgG, wo, &wi, &rs) : sggx_sample_p(&g, ev.ior, wo, &wi, &rs);
        if (sp > 0.0f) {
          wi = norm3(wi);
          const ray_t br = inst_move(M, ray_off(mkray(ev.pos, wi, DEFAULT_TMAX), ev.normal));
          float lpdf;
          const f3 Le = env_le(&S->env, wi, &lpdf);
          const float mis = (1.0f * sp) / (1.0f * sp + 1.0f * lpdf);
          const f3 pre = mul3(mul3s(F3(sp, sp, sp), mis), Le);
          rng_t rt = rng_make(p, S->seed, s, b, PURPOSE_SHADOW_TR + 1u);
          const float tr = shadow_tr(S, br.o, br.d, br.tmax, evMed, &rt, &err);
          dl = add3(dl, div3s(mul3s(pre, tr), sp));
          anyShadow = 1;
        }
      }
      if (anyShadow) L = add3(L, mul3(dl, T));
      f3 wc = F3(0.0f, 0.0f, 0.0f);
      if (M->hg) hg_sample_p(M->hgG, wo, &wc, &rs);
      else sggx_sample_p(&g, ev.ior, wo, &wc, &rs);
      const ray_t cr = inst_move(M, ray_off(mkray(ev.pos, norm3(wc), DEFAULT_TMAX), wc));
      f3 Tn = T;
      if (b > 3) {
        uint32_t rC[4];
        philox_u(s, b, 2u, 1u, p, S->seed, rC);
        float prr = 1.0f - (Tn.x + Tn.y + Tn.z) / 3.0f;
        if (oi_u01(rC[0]) <= prr) break;
        Tn = div3s(Tn, 1.0f - prr);
      }
      if (b + 1 >= S->maxDepth) break;
      o = cr.o;
      d = cr.d;
      tmax = cr.tmax;
      med = evMed;
      T = Tn;
      continue;
    }
    f3 pos = add3(o, mul3s(d, t));
    f3 n;
    const mat_t* m;
    mat_t mt;
    if (code >= 0 && (uint32_t)code < S->ntris) {
      uint32_t prim = S->order[code];
      const uint32_t* tv = &S->idx[3 * (size_t)prim];
      f3 n0 = F3(S->wnrm[3 * tv[0]], S->wnrm[3 * tv[0] + 1], S->wnrm[3 * tv[0] + 2]);
      f3 n1 = F3(S->wnrm[3 * tv[1]], S->wnrm[3 * tv[1] + 1], S->wnrm[3 * tv[1] + 2]);
      f3 n2 = F3(S->wnrm[3 * tv[2]], S->wnrm[3 * tv[2] + 1], S->wnrm[3 * tv[2] + 2]);
      float b0 = (1.0f - hb1) - hb2;
      n = norm3(add3(add3(mul3s(n0, b0), mul3s(n1, hb1)), mul3s(n2, hb2)));
      m = &S->mats[S->triMat[prim]];
      if (S->triUV && (m->tex[0] >= 0 || m->tex[1] >= 0 || m->tex[2] >= 0)) {
        mt = *m;
        oi_textured_surface(S->tex, mt.tex[0], mt.tex[1], mt.tex[2], &S->triUV[6 * (size_t)code],
                            &S->tris[12 * (size_t)code], hb1, hb2, &n, &mt.diffuse, &mt.specular);
        m = &mt;
      }
    } else if (code >= 0) {  /* an instance: model-space normal, then the instance's transform */
      uint32_t k = 0;
      while (k + 1 < S->ninst && S->insts[k + 1].code <= (uint32_t)code) ++k;
      const oinst_t* I = &S->insts[k];
      const asset_t* A = &S->assets[I->asset];
      const uint32_t tri = (uint32_t)code - I->code, prim = A->order[tri];
      const uint32_t* tv = &A->idx[3 * (size_t)prim];
      f3 n0 = F3(A->nrm[3 * tv[0]], A->nrm[3 * tv[0] + 1], A->nrm[3 * tv[0] + 2]);
      f3 n1 = F3(A->nrm[3 * tv[1]], A->nrm[3 * tv[1] + 1], A->nrm[3 * tv[1] + 2]);
      f3 n2 = F3(A->nrm[3 * tv[2]], A->nrm[3 * tv[2] + 1], A->nrm[3 * tv[2] + 2]);
      float b0 = (1.0f - hb1) - hb2;
      n = norm3(add3(add3(mul3s(n0, b0), mul3s(n1, hb1)), mul3s(n2, hb2)));
      m = &S->mats[A->mat];
      if (A->triUV && (m->tex[0] >= 0 || m->tex[1] >= 0 || m->tex[2] >= 0)) {
        mt = *m;
        oi_textured_surface(S->tex, mt.tex[0], mt.tex[1], mt.tex[2], &A->triUV[6 * (size_t)tri],
                            &A->tris[12 * (size_t)tri], hb1, hb2, &n, &mt.diffuse, &mt.specular);
        m = &mt;
      }
      n = norm3(xvec(I->m2w, n));
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
        const ray_t lr = ray_off(mkray(pos, ldir, DEFAULT_TMAX), n);
        rng_t rt = rng_make(p, S->seed, s, b, PURPOSE_SHADOW_TR + 0u);
        const float tr = shadow_tr(S, offO, ldir, lr.tmax, med, &rt, &err);
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
        const ray_t br = ray_off(mkray(pos, wi, DEFAULT_TMAX), n);
        rng_t rt = rng_make(p, S->seed, s, b, PURPOSE_SHADOW_TR + 1u);
        const float tr = shadow_tr(S, offO, wi, br.tmax, med, &rt, &err);
        dl = add3(dl, div3s(mul3s(pre, tr), spdf));
        anyShadow = 1;
      }
    }
    if (anyShadow) L = add3(L, mul3(dl, T));
    /* continuation */
    /* CRay::transform through the mat4x3 widening: + 0 * (zero column) */
    f3 dT = norm3(add3(to_local(&fr, d), F3(0.0f, 0.0f, 0.0f)));
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
    tmax = S->nmedia == 0 ? DEFAULT_TMAX : ray_off(mkray(pos, dirW, DEFAULT_TMAX), n).tmax;
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
               uint32_t p1, float* rgb_out, double* var_out, int threads, const orc_medium* media, uint32_t nmedia,
               uint32_t flags) {
  if (env_w < 2 || env_h < 2 || spp == 0 || max_depth == 0) return -1;
  med_t* meds = NULL;
  if (nmedia > 0) {
    meds = (med_t*)calloc(nmedia, sizeof(med_t));
    for (uint32_t i = 0; i < nmedia; ++i) {
      /* one load per path; later instances of the path share its grid and
         its coefficients (CAssetManager::loadMedium, asset_manager.cu:114-137) */
      uint32_t j = 0;
      while (j < i && strcmp(media[j].path, media[i].path) != 0) ++j;
      if (j < i) {
        meds[i] = meds[j];
        meds[i].owner = 0;
        med_place(&meds[i], &media[i]);
        continue;
      }
      if (med_load(&meds[i], &media[i]) != 0) {
        for (uint32_t k = 0; k < i; ++k) med_free(&meds[k]);
        free(meds);
        return -3;
      }
    }
  }
  rscene_t S;
  memset(&S, 0, sizeof(S));
  uint32_t nv = 0, nt = 0;
  for (uint32_t i = 0; i < nmeshes; ++i)
    if (meshes[i].asset == 0) { nv += meshes[i].nverts; nt += meshes[i].ntris; }
  float* wpos = (float*)malloc(sizeof(float) * 3 * (size_t)(nv + 1));
  S.wnrm = (float*)malloc(sizeof(float) * 3 * (size_t)(nv + 1));
  S.idx = (uint32_t*)malloc(sizeof(uint32_t) * 3 * (size_t)(nt + 1));
  S.triMat = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(nt + 1));
  S.mats = (mat_t*)malloc(sizeof(mat_t) * (size_t)(nmeshes + 1));
  uint32_t vb = 0, tb = 0;
  int anyUV = 0;
  for (uint32_t i = 0; i < nmeshes; ++i) anyUV = anyUV || (meshes[i].asset == 0 && meshes[i].uvs != NULL);
  if (anyUV) S.uv = (float*)calloc(2 * (size_t)(nv + 1), sizeof(float));
  S.tex = (oi_tex*)calloc(5 * (size_t)(nmeshes + 1), sizeof(oi_tex));
  /* asset k's first mesh (its geometry and material) */
  int* firstOf = (int*)malloc(sizeof(int) * (size_t)(nmeshes + 1));
  int* assetOf = (int*)malloc(sizeof(int) * (size_t)(nmeshes + 1));
  uint32_t nassets = 0, ninst = 0;
  for (uint32_t i = 0; i < nmeshes; ++i) {
    assetOf[i] = -1;
    if (meshes[i].asset == 0) continue;
    ++ninst;
    for (uint32_t a = 0; a < nassets; ++a)
      if (meshes[firstOf[a]].asset == meshes[i].asset) assetOf[i] = (int)a;
    if (assetOf[i] < 0) {
      firstOf[nassets] = (int)i;
      assetOf[i] = (int)nassets++;
    }
  }
  for (uint32_t i = 0; i < nmeshes; ++i) {
    const orc_mesh* M = &meshes[i];
    S.mats[i] = make_mat(&M->material);
    const int owner = M->asset == 0 || firstOf[assetOf[i]] == (int)i;
    /* CMaterial(aiMaterial*) (material.cu:110-143); maps without texture coordinates are unused */
    if (M->uvs && owner)
      oi_material_maps(&M->material, M->albedo, M->specular, M->normal, M->alpha, S.tex, &S.ntex, S.mats[i].tex);
    if (M->asset != 0) continue;
    if (M->uvs) memcpy(&S.uv[2 * (size_t)vb], M->uvs, sizeof(float) * 2 * (size_t)M->nverts);
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
    if (anyUV) {  /* per BVH-order triangle: texture coordinates and opacity map */
      S.triUV = (float*)malloc(sizeof(float) * 6 * (size_t)nt);
      S.triAlpha = (int*)malloc(sizeof(int) * (size_t)nt);
      int anyAlpha = 0;
      for (uint32_t i = 0; i < nt; ++i) {
        const uint32_t prim = S.order[i];
        for (int k = 0; k < 3; ++k) {
          const uint32_t v = S.idx[3 * (size_t)prim + k];
          S.triUV[6 * (size_t)i + 2 * k] = S.uv[2 * (size_t)v];
          S.triUV[6 * (size_t)i + 2 * k + 1] = S.uv[2 * (size_t)v + 1];
        }
        S.triAlpha[i] = S.mats[S.triMat[prim]].tex[3];
        anyAlpha = anyAlpha || S.triAlpha[i] >= 0;
      }
      if (anyAlpha) {
        S.alpha.alpha_tex = S.triAlpha;
        S.alpha.uv = S.triUV;
        S.alpha.tex = S.tex;
      }
    }
  }
  /* two-level: the assets' model-space BVHs and the instances, numbered after the world triangles */
  S.assets = (asset_t*)calloc((size_t)nassets + 1, sizeof(asset_t));
  S.insts = (oinst_t*)calloc((size_t)ninst + 1, sizeof(oinst_t));
  for (uint32_t a = 0; a < nassets; ++a) {
    const orc_mesh* M = &meshes[firstOf[a]];
    asset_t* A = &S.assets[a];
    A->ntris = M->ntris;
    A->nrm = M->normals;
    A->idx = M->indices;
    A->mat = firstOf[a];
    A->nodes = (int32_t*)malloc(64 * (size_t)(M->ntris > 1 ? M->ntris - 1 : 1));
    A->order = (uint32_t*)malloc(4 * (size_t)M->ntris);
    A->tris = (float*)malloc(48 * (size_t)M->ntris);
    int h = orc_build_bvh(M->positions, M->nverts, M->indices, M->ntris, A->nodes, A->order, A->tris);
    if (h < 0 || h > 96) return -2;
    if (M->uvs) {
      A->triUV = (float*)malloc(sizeof(float) * 6 * (size_t)M->ntris);
      A->triAlpha = (int*)malloc(sizeof(int) * (size_t)M->ntris);
      for (uint32_t i = 0; i < M->ntris; ++i) {
        const uint32_t prim = A->order[i];
        for (int k = 0; k < 3; ++k) {
          const uint32_t v = M->indices[3 * (size_t)prim + k];
          A->triUV[6 * (size_t)i + 2 * k] = M->uvs[2 * (size_t)v];
          A->triUV[6 * (size_t)i + 2 * k + 1] = M->uvs[2 * (size_t)v + 1];
        }
        A->triAlpha[i] = S.mats[A->mat].tex[3];
      }
      if (S.mats[A->mat].tex[3] >= 0) {
        A->alpha.alpha_tex = A->triAlpha;
        A->alpha.uv = A->triUV;
        A->alpha.tex = S.tex;
      }
    }
  }
  {
    uint32_t code = nt, k = 0;
    for (uint32_t i = 0; i < nmeshes; ++i) {
      if (meshes[i].asset == 0) continue;
      oinst_t* I = &S.insts[k++];
      I->asset = assetOf[i];
      memcpy(I->m2w, meshes[i].model_to_world, sizeof(I->m2w));
      m4_t M4 = oi_m4_id();
      for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 3; ++r) M4.m[c][r] = I->m2w[3 * c + r];
      float w43[12];
      oi_m4_to43(oi_m4_inv(M4), w43);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) I->w2o[4 * r + c] = w43[3 * c + r];
      I->code = code;
      code += S.assets[I->asset].ntris;
    }
    S.ninst = ninst;
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
  S.media = meds;
  S.nmedia = nmedia;
  S.dda = (flags & 1u) ? 1 : 0;
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
  free(S.uv); free(S.triUV); free(S.triAlpha);
  for (int k = 0; k < S.ntex; ++k) free(S.tex[k].texels);
  free(S.tex);
  if (nt > 0) { free(S.nodes); free(S.order); free(S.tris); }
  for (uint32_t a = 0; a < nassets; ++a) {
    free(S.assets[a].nodes); free(S.assets[a].order); free(S.assets[a].tris);
    free(S.assets[a].triUV); free(S.assets[a].triAlpha);
  }
  free(S.assets); free(S.insts); free(firstOf); free(assetOf);
  for (uint32_t i = 0; i < nmedia; ++i) med_free(&meds[i]);
  free(meds);
  return 0;
}

float orc_t_log(float x) { return oi_log(x); }

/* Raytracer's output stage (raytracer.cu:33-127): column sums of
 * log(r+g+b+FLT_MIN)/(3WH) in row order, their sum in column order,
 * L = exp(sum) - WH FLT_MIN, c/(c+L), ^(1/gamma), round(255 c). */
void orc_tonemap(const float* rgb, uint32_t W, uint32_t H, float gamma, float* out, uint8_t* bytes) {
  const float divisor = (float)(H * W * 3);
  float total = 0.0f;
  for (uint32_t x = 0; x < W; ++x) {
    float acc = 0.0f;
    for (uint32_t y = 0; y < H; ++y) {
      const float* p = rgb + 3 * ((size_t)y * W + x);
      acc += logf(p[0] + p[1] + p[2] + FLT_MIN) / divisor;
    }
    total += acc;
  }
  const float L = expf(total) - (float)(W * H) * FLT_MIN;
  const float invGamma = 1.0f / gamma;
  for (size_t i = 0; i < (size_t)W * H * 3; ++i) {
    const float c = rgb[i];
    const float t = powf(c / (c + L), invGamma);
    if (out) out[i] = t;
    if (bytes) bytes[i] = (uint8_t)roundf(t * 255.0f);
  }
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

/* An environment map with its distributions built once (for callers that
 * query it per path). */
void* orc_env_create(const float* env_rgb, int W, int H) {
  env_t* e = (env_t*)malloc(sizeof(env_t));
  if (e) env_build(e, env_rgb, W, H);
  return e;
}
void orc_env_destroy(void* h) {
  if (!h) return;
  env_free((env_t*)h);
  free(h);
}
void orc_env_sample_h(const void* h, float u0, float u1, float* dir, float* pdf, float* le) {
  f3 d;
  f3 l = env_sample((const env_t*)h, u0, u1, &d, pdf);
  dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
  le[0] = l.x; le[1] = l.y; le[2] = l.z;
}
void orc_env_le_h(const void* h, const float* dir, float* pdf, float* le) {
  f3 l = env_le((const env_t*)h, F3(dir[0], dir[1], dir[2]), pdf);
  le[0] = l.x; le[1] = l.y; le[2] = l.z;
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

/* SGGX microflake distribution of S (xx yy zz xy xz yz) and normal n:
 * out = D(wi), sigma(wi), sampleVNDF(u1, u2) (3), specular p(wo, wi). */
void orc_t_sggx(const float* S6, const float* n, const float* wo, const float* wi, float u1, float u2, float* out) {
  const sggx_t g = make_sggx(S6, L3(n));
  out[0] = sggx_D(&g, L3(wi));
  out[1] = sggx_sigma(&g, L3(wi));
  P3(out + 2, sggx_vndf(&g, u1, u2));
  out[5] = sggx_p_spec(&g, L3(wo), L3(wi));
}

/* CSGGXPhaseFunction::sampleP with the uniforms u (consumed in order:
 * lobe choice, VNDF pair, and for the diffuse lobe the cosine pair):
 * out = wi (3), p, draws consumed. */
void orc_t_sggx_sample(const float* S6, const float* n, float ior, const float* wo, const float* u, float* out) {
  const sggx_t g = make_sggx(S6, L3(n));
  rng_t r;
  memset(&r, 0, sizeof(r));
  r.replay = u;
  f3 wi;
  out[3] = sggx_sample_p(&g, ior, L3(wo), &wi, &r);
  P3(out, wi);
  out[4] = (float)r.idx;
}

/* getRotation(n): 16 floats, column major. */
void orc_t_get_rotation(const float* n, float* out) {
  const m4_t m = rot_from_normal(L3(n));
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < 4; ++i) out[4 * c + i] = m.m[c][i];
}

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
