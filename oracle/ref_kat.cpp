// Host build of the reference's own math headers (TEST INFRASTRUCTURE ONLY).
//
// Compiled in place from the reference tree (-I .../raytracer/include) against
// the from-scratch shims in oracle/refshim/ (glm subset, OptiX/NanoVDB type
// stand-ins, a cuRAND stand-in that replays queued draws).  The exported
// functions evaluate the reference implementation on given inputs; the golden
// vectors they produce (tests/golden/make_golden.py) pin the oracle's
// restatement.  Nothing of the product links this file.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <glm/glm.hpp>
#include "utility/qualifiers.hpp"
// sampler.hpp's uniformSample01 reads cuRAND only when compiled for the
// device; expose that branch so the queued draws reach the sampling code.
#define __CUDA_ARCH__ 860
#include "sampling/sampler.hpp"
#undef __CUDA_ARCH__
#include "filtering/filtered_data.hpp"
#include "integrators/objects.hpp"
#include "intersect/ray.hpp"
#include "material/fresnel.hpp"
#include "material/microfacet_brdf.hpp"
#include "material/oren_nayar_brdf.hpp"
#include "medium/sggx_phase_function.hpp"
#include "shapes/sphere.hpp"
#include "utility/functions.hpp"

namespace r2ref {
static std::vector<float> g_queue;
static size_t g_pos = 0;
float next_curand() { return g_pos < g_queue.size() ? g_queue[g_pos++] : 0.5f; }
}  // namespace r2ref

static void feed(const float* c, int n) {
  r2ref::g_queue.assign(c, c + n);
  r2ref::g_pos = 0;
}
static glm::vec3 V(const float* p) { return glm::vec3(p[0], p[1], p[2]); }
static void put(float* o, const glm::vec3& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

extern "C" {

// Number of queued draws consumed by the last call.
int ref_draws_used() { return (int)r2ref::g_pos; }

// CSampler::uniformSample01 for a queued cuRAND value.
float ref_u01(float c) {
  feed(&c, 1);
  rt::CSampler s;
  return s.uniformSample01();
}

// Evaluation order of a two-argument constructor's arguments in this build
// (glm::vec2(a(), b())): 0 = left to right, 1 = right to left.
int ref_vec2_arg_order() {
  float c[2] = {0.25f, 0.75f};
  feed(c, 2);
  rt::CSampler s;
  glm::vec2 v(s.uniformSample01(), s.uniformSample01());
  return v.x < v.y ? 0 : 1;
}

// CSampler warps: out = sphere(3) hemisphere(3) disk(3) cosine(3), each from
// a fresh queue [c0, c1].
void ref_warps(const float* c, float* out) {
  rt::CSampler s;
  feed(c, 2); put(out + 0, s.uniformSampleSphere());
  feed(c, 2); put(out + 3, s.uniformSampleHemisphere());
  feed(c, 2); put(out + 6, s.concentricSampleDisk());
  feed(c, 2); put(out + 9, s.cosineSampleHemisphere());
}

// CSGGXMicroflakeDistribution::buildS -> xx yy zz xy xz yz
void ref_build_s(const float* n, float sigma, float* out) {
  glm::mat3 S = rt::CSGGXMicroflakeDistribution::buildS(V(n), sigma);
  out[0] = S[0][0]; out[1] = S[1][1]; out[2] = S[2][2];
  out[3] = S[0][1]; out[4] = S[0][2]; out[5] = S[1][2];
}

// SFilteredDataCompact(SFilteredData): in = density, S(6), diffuse(3),
// specular(3), normal(3), ior -> 32 bytes.
void ref_encode(const float* in, unsigned char* out32) {
  filter::SFilteredData d;
  d.density = in[0];
  float xx = in[1], yy = in[2], zz = in[3], xy = in[4], xz = in[5], yz = in[6];
  d.S = glm::mat3(xx, xy, xz, xy, yy, yz, xz, yz, zz);
  d.diffuseColor = V(in + 7);
  d.specularColor = V(in + 10);
  d.normal = V(in + 13);
  d.ior = in[16];
  filter::SFilteredDataCompact c(d);
  static_assert(sizeof(c) == 32, "payload size");
  std::memcpy(out32, &c, 32);
}

// SFilteredData(SFilteredDataCompact): 32 bytes -> density, S(6), diffuse,
// specular, normal, ior.
void ref_decode(const unsigned char* in32, float* out) {
  filter::SFilteredDataCompact c;
  std::memcpy(&c, in32, 32);
  filter::SFilteredData d(c);
  out[0] = d.density;
  out[1] = d.S[0][0]; out[2] = d.S[1][1]; out[3] = d.S[2][2];
  out[4] = d.S[0][1]; out[5] = d.S[0][2]; out[6] = d.S[1][2];
  put(out + 7, d.diffuseColor);
  put(out + 10, d.specularColor);
  put(out + 13, d.normal);
  out[16] = d.ior;
}

float ref_fresnel(float etaI, float etaT, float c) { return rt::CFresnel(etaI, etaT).evaluate(c); }

// Microfacet BRDF (GGX + Fresnel): out = f(wo,wi), pdf(wo,wi).
void ref_microfacet(float ax, float ay, float etaI, float etaT, const float* wo, const float* wi, float* out) {
  rt::CMicrofacetBRDF b(ax, ay, etaI, etaT);
  out[0] = b.f(V(wo), V(wi));
  out[1] = b.pdf(V(wo), V(wi));
}

// CMicrofacetBRDF::sampleF with queued draws: out = wi(3), pdf, f.
void ref_microfacet_sample(float ax, float ay, float etaI, float etaT, const float* wo, const float* c, float* out) {
  rt::CMicrofacetBRDF b(ax, ay, etaI, etaT);
  feed(c, 2);
  rt::CSampler s;
  glm::vec3 wi(0.f);
  float pdf = 0.f;
  float f = b.sampleF(V(wo), &wi, s, &pdf);
  put(out, wi);
  out[3] = pdf;
  out[4] = f;
}

// CMicrofacetDistribution::sampleH with an explicit u.
void ref_ggx_sample_h(float ax, float ay, const float* wo, float u1, float u2, float* out) {
  rt::CMicrofacetDistribution d(ax, ay);
  put(out, d.sampleH(V(wo), glm::vec2(u1, u2)));
}

// Oren-Nayar: out = f, pdf.
void ref_oren_nayar(float roughness, const float* wo, const float* wi, float* out) {
  rt::COrenNayarBRDF b(roughness);
  out[0] = b.f(V(wo), V(wi));
  out[1] = b.pdf(V(wo), V(wi));
}

// COrenNayarBRDF::sampleF with queued draws: out = wi(3), pdf, f.
void ref_oren_nayar_sample(float roughness, const float* wo, const float* c, float* out) {
  rt::COrenNayarBRDF b(roughness);
  feed(c, 2);
  rt::CSampler s;
  glm::vec3 wi(0.f);
  float pdf = 0.f;
  float f = b.sampleF(V(wo), &wi, s, &pdf);
  put(out, wi);
  out[3] = pdf;
  out[4] = f;
}

// CCoordinateFrame::fromNormal: out = T, B, worldToTangent * v.
void ref_frame(const float* n, const float* v, float* out) {
  rt::CCoordinateFrame f = rt::CCoordinateFrame::fromNormal(V(n));
  put(out, f.T());
  put(out + 3, f.B());
  put(out + 6, f.worldToTangent() * V(v));
}

// CRay::offsetRayOrigin(p, dir)
void ref_offset(const float* p, const float* d, float* out) { put(out, rt::CRay::offsetRayOrigin(V(p), V(d))); }

// Sphere(center, radius, normal).intersect(ray): out = hit, t.
void ref_sphere(const float* c, float r, const float* n, const float* o, const float* d, float tmax, float* out) {
  rt::Sphere s(V(c), r, V(n));
  rt::SHitInformation h = s.intersect(rt::CRay(V(o), V(d), tmax));
  out[0] = h.hit ? 1.f : 0.f;
  out[1] = h.hit ? h.t : 0.f;
}

// findInterval over a cdf with predicate cdf[i] <= u.
int ref_find_interval(const float* cdf, int size, float u) {
  return rt::findInterval(size, [&](int i) { return cdf[i] <= u; });
}

// SGGX phase function: out = D(w), sigma(w), sampleVNDF(wi, U)(3), specular p(wo, wi)
void ref_sggx(const float* S6, const float* normal, const float* wo, const float* wi, float u1, float u2, float* out) {
  glm::mat3 S(S6[0], S6[3], S6[4], S6[3], S6[1], S6[5], S6[4], S6[5], S6[2]);
  rt::CSGGXMicroflakeDistribution d(S, V(normal));
  out[0] = d.D(V(wi));
  out[1] = d.sigma(V(wi));
  put(out + 2, d.sampleVNDF(V(wo), glm::vec2(u1, u2)));
  rt::CSGGXSpecularPhaseFunction sp(d);
  out[5] = sp.p(V(wo), V(wi));
}

// CSGGXPhaseFunction::sampleP with queued draws: out = wi(3), p.
void ref_sggx_sample(const float* S6, const float* normal, float ior, const float* wo, const float* c, int nc,
                     float* out) {
  glm::mat3 S(S6[0], S6[3], S6[4], S6[3], S6[1], S6[5], S6[4], S6[5], S6[2]);
  rt::CSGGXPhaseFunction ph(S, V(normal), ior);
  feed(c, nc);
  rt::CSampler s;
  glm::vec3 wi(0.f);
  float p = ph.sampleP(V(wo), &wi, s);
  put(out, wi);
  out[3] = p;
}

// getRotation(normal) rounded rotation: 16 floats column major.
void ref_get_rotation(const float* n, float* out) {
  glm::mat4 m = rt::getRotation(V(n));
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) out[4 * c + r] = m[c][r];
}

}  // extern "C"
