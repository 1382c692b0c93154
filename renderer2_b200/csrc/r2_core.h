// Core math shared by every sm_100a kernel and the host runtime of the
// Renderer2 hot paths: small vector/matrix types with glm's column-major
// semantics, the Philox4x32-10 counter-based generator that keys every random
// draw by (voxel|pixel, sample, bounce, draw), and the sampling warps of the
// reference's CSampler (raytracer/include/sampling/sampler.hpp:50-93).
//
// Floating-point discipline: the library is compiled with -fmad=false (device)
// and -ffp-contract=off (host) so that every expression below rounds the same
// way on the GPU and on the host; fused multiply-adds appear only where they
// are written out as fmaf().  Division and sqrt are IEEE (no fast-math).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define R2_HD __host__ __device__ __forceinline__
#define R2_D __device__ __forceinline__
#else
#define R2_HD inline
#define R2_D inline
#endif

namespace r2 {

// ---------------------------------------------------------------------------
// vec3 / vec2
// ---------------------------------------------------------------------------
struct V3 {
  float x, y, z;
};
struct V2 {
  float x, y;
};

R2_HD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
R2_HD V3 v3(float s) { return v3(s, s, s); }
R2_HD V2 v2(float x, float y) { V2 r; r.x = x; r.y = y; return r; }
R2_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
R2_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
R2_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
R2_HD V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
R2_HD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
R2_HD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
R2_HD V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
R2_HD V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
R2_HD V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
R2_HD V3& operator*=(V3& a, V3 b) { a = a * b; return a; }
R2_HD V3& operator*=(V3& a, float s) { a = a * s; return a; }
R2_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
R2_HD V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
R2_HD float length(V3 a) { return sqrtf(dot(a, a)); }
// glm::normalize: v * inversesqrt(dot(v, v)) with inversesqrt = 1 / sqrt.
R2_HD V3 normalize(V3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
R2_HD V3 vmin(V3 a, V3 b) { return v3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
R2_HD V3 vmax(V3 a, V3 b) { return v3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
R2_HD V3 vabs(V3 a) { return v3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
R2_HD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
R2_HD float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// glm::mat4x3: four column vectors; M * vec4(p, w) = c0*p.x + c1*p.y + c2*p.z + c3*w,
// accumulated left to right per component exactly like glm's operator*.
struct M43 {
  V3 c[4];
};
R2_HD V3 xform_point(const M43& m, V3 p) {
  return v3(m.c[0].x * p.x + m.c[1].x * p.y + m.c[2].x * p.z + m.c[3].x * 1.0f,
            m.c[0].y * p.x + m.c[1].y * p.y + m.c[2].y * p.z + m.c[3].y * 1.0f,
            m.c[0].z * p.x + m.c[1].z * p.y + m.c[2].z * p.z + m.c[3].z * 1.0f);
}
R2_HD V3 xform_vector(const M43& m, V3 v) {
  return v3(m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z + m.c[3].x * 0.0f,
            m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z + m.c[3].y * 0.0f,
            m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z + m.c[3].z * 0.0f);
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).  Counter = 4 x u32, key = 2 x u32, ten rounds.
// ---------------------------------------------------------------------------
struct U4 {
  uint32_t x, y, z, w;
};

R2_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
#if defined(__CUDA_ARCH__)
  *lo = a * b;
  *hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *lo = (uint32_t)p;
  *hi = (uint32_t)(p >> 32);
#endif
}

R2_HD U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, ctr.x, &hi0, &lo0);
    mulhilo32(M1, ctr.z, &hi1, &lo1);
    U4 n;
    n.x = hi1 ^ ctr.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ ctr.w ^ k1;
    n.w = lo0;
    ctr = n;
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

R2_HD U4 u4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
  U4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r;
}

// Uniform float in [0, 1 - 2^-24]: the top 24 bits, exact in binary32.
R2_HD float u01(uint32_t bits) { return (float)(bits >> 8) * (1.0f / 16777216.0f); }

// ---------------------------------------------------------------------------
// sin/cos of a fraction of a turn, written from the Taylor series of sin and
// cos on [-pi/4, pi/4] with quadrant reduction.  The reduction u - q/4 is exact
// (Sterbenz), so host and device produce identical bits.  Truncation error of
// the series is below 2e-9 on the reduced interval.
// ---------------------------------------------------------------------------
R2_HD void sincos_turns(float u, float* s, float* c) {
  float q = rintf(u * 4.0f);
  float r = u - q * 0.25f;
  float t = r * 6.28318548f;  // 2*pi rounded to binary32
  float t2 = t * t;
  // sin t = t - t^3/3! + t^5/5! - t^7/7! + t^9/9!
  float ps = fmaf(t2, 2.75573192e-6f, -1.98412698e-4f);
  ps = fmaf(t2, ps, 8.33333333e-3f);
  ps = fmaf(t2, ps, -1.66666667e-1f);
  float sn = fmaf(t * t2, ps, t);
  // cos t = 1 - t^2/2! + t^4/4! - t^6/6! + t^8/8! - t^10/10!
  float pc = fmaf(t2, -2.75573192e-7f, 2.48015873e-5f);
  pc = fmaf(t2, pc, -1.38888889e-3f);
  pc = fmaf(t2, pc, 4.16666667e-2f);
  pc = fmaf(t2, pc, -0.5f);
  float cs = fmaf(t2, pc, 1.0f);
  int qi = ((int)q) & 3;
  if (qi == 0) { *s = sn; *c = cs; }
  else if (qi == 1) { *s = cs; *c = -sn; }
  else if (qi == 2) { *s = -sn; *c = -cs; }
  else { *s = -cs; *c = sn; }
}

// ---------------------------------------------------------------------------
// Natural logarithm of a positive normal float, written from the series
// log m = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + ...), s = (m - 1)/(m + 1), after
// the classical reduction x = m 2^e with m in [sqrt(1/2), sqrt(2)) (Cody and
// Waite, "Software Manual for the Elementary Functions", 1980).  |s| <= 0.1716,
// the series stops after s^11 (truncation below 1e-10 relative), and e ln 2 is
// added in two parts (0.693145751953125 + 1.42860682e-6).  Every step is an
// IEEE operation or an explicit fmaf, so host and device give identical bits.
// Used for the free-flight distances of delta and ratio tracking.
// ---------------------------------------------------------------------------
R2_HD float log_r2(float x) {
  uint32_t b;
  memcpy(&b, &x, 4);
  int e = (int)((b >> 23) & 0xFFu) - 127;
  uint32_t mb = (b & 0x7FFFFFu) | 0x3F800000u;
  float m;
  memcpy(&m, &mb, 4);
  if (m > 1.41421354f) {
    m = m * 0.5f;
    e += 1;
  }
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

// CSampler::uniformSampleSphere (sampler.hpp:86-94): z = 1 - 2u1, phi = 2 pi u2.
R2_HD V3 uniform_sample_sphere(float u1, float u2) {
  float z = 1.0f - 2.0f * u1;
  float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float s, c;
  sincos_turns(u2, &s, &c);
  return v3(r * c, r * s, z);
}

// CSampler::uniformSampleHemisphere (sampler.hpp:39-46).
R2_HD V3 uniform_sample_hemisphere(float u1, float u2) {
  float r = sqrtf(fmaxf(0.0f, 1.0f - u1 * u1));
  float s, c;
  sincos_turns(u2, &s, &c);
  return v3(r * c, r * s, u1);
}

// CSampler::concentricSampleDisk (sampler.hpp:52-74).  theta = pi/4 * (y/x)
// or pi/2 - pi/4 * (x/y); both are evaluated through sincos_turns of (ratio/8).
R2_HD V3 concentric_sample_disk(float u1, float u2) {
  float ox = 2.0f * u1 - 1.0f;
  float oy = 2.0f * u2 - 1.0f;
  if (ox == 0.0f && oy == 0.0f) return v3(0.0f);
  float r, s, c;
  if (fabsf(ox) > fabsf(oy)) {
    r = ox;
    sincos_turns((oy / ox) * 0.125f, &s, &c);
  } else {
    r = oy;
    float sa, ca;
    sincos_turns((ox / oy) * 0.125f, &sa, &ca);
    c = sa;  // cos(pi/2 - a) = sin a
    s = ca;  // sin(pi/2 - a) = cos a
  }
  return v3(r * c, r * s, 0.0f);
}

// CSampler::cosineSampleHemisphere (sampler.hpp:76-80).
R2_HD V3 cosine_sample_hemisphere(float u1, float u2) {
  V3 d = concentric_sample_disk(u1, u2);
  float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
  return v3(d.x, d.y, z);
}

// ---------------------------------------------------------------------------
// IEEE half conversion (round to nearest even), used for the ior field of the
// 32-byte voxel payload (filtered_data.hpp:44) and the optional FP16 payload.
// ---------------------------------------------------------------------------
R2_HD uint16_t f32_to_f16_bits(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t mag = x & 0x7FFFFFFFu;
  if (mag >= 0x7F800000u) {  // inf or nan
    return (uint16_t)(sign | 0x7C00u | (mag > 0x7F800000u ? 0x200u : 0u));
  }
  if (mag >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);  // rounds to inf
  if (mag < 0x38800000u) {  // subnormal half or zero
    if (mag < 0x33000000u) return (uint16_t)sign;  // below half of the smallest subnormal
    uint32_t e = mag >> 23;
    uint32_t m = (mag & 0x7FFFFFu) | 0x800000u;
    uint32_t shift = 126u - e;  // 14 + (112 - e) ... places the value in units of 2^-24
    uint32_t v = m >> shift;
    uint32_t rem = m & ((1u << shift) - 1u);
    uint32_t half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (v & 1u))) ++v;
    return (uint16_t)(sign | v);
  }
  uint32_t v = ((mag - 0x38000000u) >> 13);
  uint32_t rem = mag & 0x1FFFu;
  if (rem > 0x1000u || (rem == 0x1000u && (v & 1u))) ++v;
  return (uint16_t)(sign | v);
}

R2_HD float f16_bits_to_f32(uint16_t h) {
#if defined(__CUDA_ARCH__)
  float f;  // half -> float is exact: the conversion instruction gives the same bits
  asm("cvt.f32.f16 %0, %1;" : "=f"(f) : "h"(h));
  return f;
#else
  uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1Fu;
  uint32_t m = h & 0x3FFu;
  uint32_t x;
  if (e == 0) {
    if (m == 0) {
      x = sign;
    } else {
      // subnormal: value = m * 2^-24
      float f = (float)m * (1.0f / 16777216.0f);
      memcpy(&x, &f, 4);
      x |= sign;
    }
  } else if (e == 31) {
    x = sign | 0x7F800000u | (m << 13);
  } else {
    x = sign | ((e + 112u) << 23) | (m << 13);
  }
  float f;
  memcpy(&f, &x, 4);
  return f;
#endif
}

}  // namespace r2
