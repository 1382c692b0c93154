// Host build of the reference's own math headers (TEST INFRASTRUCTURE ONLY).
//
// Compiled in place from the reference tree (-I .../raytracer/include) against
// the from-scratch shims in oracle/refshim/ (glm subset, OptiX/NanoVDB type
// stand-ins, a cuRAND stand-in that replays queued draws, and a scene,
// scene-object and material stand-in whose closest hit is the oracle's BVH
// trace, so that CMeshFilter::run compiles and runs as written).  The exported
// functions evaluate the reference implementation on given inputs; the golden
// vectors they produce (tests/golden/make_golden.py) pin the oracle's
// restatement.  Nothing of the product links this file.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "r2_host_texfetch.h"
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
// CMeshFilter and CPathIntegrator with the scene and scene-object shims of
// refshim/; the oracle's BVH and closest-hit trace stand in for OptiX, the
// oracle's environment map for CEnvironmentMap (whose CDistribution2D g++
// cannot compile), and camera.cu is compiled from the reference's sources.
#include "filtering/mesh_filter.hpp"
#include "integrators/path_integrator_impl.hpp"
#include "camera/camera.cu"
#include "oracle.h"
#include "render_oracle.h"

// The CMaterial constructors and destructor live in material.cu with the
// assimp material import; the plain ones initialise the members as written
// there (material.cu:8-53, 68-72), and nothing here owns a mesh path.
namespace rt {
CMaterial::CMaterial(const glm::vec3& diffuseColor, const glm::vec3& glossyColor, const COrenNayarBRDF& diffuse,
                     const CMicrofacetBRDF& glossy)
    : m_deviceObject(false), m_Le(0.f), m_diffuseColor(diffuseColor), m_glossyColor(glossyColor),
      m_orenNayarBRDF(diffuse), m_microfacetBRDF(glossy), m_albedoTexture(nullptr), m_glossyTexture(nullptr),
      m_normalTexture(nullptr), m_alphaTexture(nullptr), m_pathLength(0), m_meshPath(nullptr), m_submeshId(0) {}
CMaterial::~CMaterial() {}
}  // namespace rt

namespace r2ref {
// Draws of the current thread: the queued cuRAND values first; then, when a
// generator is started (timing runs), Philox4x32-10 words keyed by the path
// mapped to (0, 1] as curand_uniform's range; else 0.5.
struct DrawGen {
  uint32_t key[2], ctr[4], buf[4];
  int left;
  bool on;
};
static thread_local std::vector<float> g_queue;
static thread_local size_t g_pos = 0;
static thread_local DrawGen g_gen = {};
float next_curand() {
  if (g_pos < g_queue.size()) return g_queue[g_pos++];
  if (g_gen.on) {
    if (g_gen.left == 0) {
      orc_philox4x32_10(g_gen.ctr, g_gen.key, g_gen.buf);
      ++g_gen.ctr[1];
      g_gen.left = 4;
    }
    const uint32_t w = g_gen.buf[4 - g_gen.left--];
    return (float)((w >> 8) + 1u) * (1.0f / 16777216.0f);
  }
  return 0.5f;
}
static void gen_start(uint32_t a, uint32_t b, uint32_t c) {
  g_queue.clear();
  g_pos = 0;
  g_gen = DrawGen{};
  g_gen.on = true;
  g_gen.key[0] = a;
  g_gen.key[1] = b;
  g_gen.ctr[0] = c;
}

// Scene of the CDeviceScene shim: the oracle's BVH over world-space
// triangles, model-space vertex normals, per triangle its object (transform)
// and material; the environment map (row 0 = top, RGB) for NEE and misses.
struct HookScene {
  std::vector<int32_t> nodes;
  std::vector<uint32_t> order, idx, triObj;
  std::vector<float> tris, nrm;
  std::vector<glm::mat4x3> m2w;
  std::vector<std::unique_ptr<rt::CMaterial>> mats;  // per object
  std::vector<float> env;
  int envW = 0, envH = 0;
  void* envH_ = nullptr;  // the oracle's environment map with its distributions, built once
  unsigned int mask = 0;  // visibility of the objects (ESceneobjectMask)
  bool ready = false;
};
static HookScene g_fs;

// __closesthit__ch (shaders.optix.cu:28-130) for untextured meshes: the hit
// position o + t d, the normal interpolated from the vertex normals with the
// hit's barycentrics and normalised, taken to world space by the object's
// transform and normalised; the object's material and its ior.
void scene_intersect(const rt::CRay& ray, rt::SInteraction* si, unsigned int mask) {
  si->hitInformation.hit = false;
  if (!(mask & g_fs.mask) || !g_fs.ready) return;
  float t = 0.f, b1 = 0.f, b2 = 0.f;
  const int tri = orc_trace(g_fs.nodes.data(), g_fs.tris.data(), ray.m_origin.x, ray.m_origin.y, ray.m_origin.z,
                            ray.m_direction.x, ray.m_direction.y, ray.m_direction.z, ray.m_t_max, &t, &b1, &b2);
  if (tri < 0) return;
  const uint32_t prim = g_fs.order[tri];
  const uint32_t* v = &g_fs.idx[3 * (size_t)prim];
  const uint32_t obj = g_fs.triObj[prim];
  auto N = [&](uint32_t k) { return glm::vec3(g_fs.nrm[3 * k], g_fs.nrm[3 * k + 1], g_fs.nrm[3 * k + 2]); };
  glm::vec3 n = glm::normalize((1.f - b1 - b2) * N(v[0]) + b1 * N(v[1]) + b2 * N(v[2]));
  n = glm::normalize(g_fs.m2w[obj] * glm::vec4(n, 0.f));
  si->hitInformation.hit = true;
  si->hitInformation.pos = glm::vec3(ray.m_origin.x + t * ray.m_direction.x, ray.m_origin.y + t * ray.m_direction.y,
                                     ray.m_origin.z + t * ray.m_direction.z);
  si->hitInformation.normal = n;
  si->hitInformation.normalG = n;
  si->hitInformation.tc = glm::vec2(0.f);
  si->hitInformation.ior = g_fs.mats[obj]->ior();
  si->hitInformation.t = t;
  si->material = g_fs.mats[obj].get();
}

glm::vec3 scene_sample_light(float u0, float u1, glm::vec3* dir, float* pdf) {
  float d[3], le[3];
  orc_env_sample_h(g_fs.envH_, u0, u1, d, pdf, le);
  *dir = glm::vec3(d[0], d[1], d[2]);
  return glm::vec3(le[0], le[1], le[2]);
}

glm::vec3 scene_le(const glm::vec3& dir, float* pdf) {
  const float d[3] = {dir.x, dir.y, dir.z};
  float le[3];
  orc_env_le_h(g_fs.envH_, d, pdf, le);
  return glm::vec3(le[0], le[1], le[2]);
}
}  // namespace r2ref

glm::vec3 rt::CDeviceScene::sampleLightSources(CSampler& sampler, glm::vec3* direction, float* pdf) const {
  const float u0 = sampler.uniformSample01();  // CDistribution2D::sampleContinuous: the marginal's draw first
  const float u1 = sampler.uniformSample01();
  return r2ref::scene_sample_light(u0, u1, direction, pdf);
}

static void feed(const float* c, int n) {
  r2ref::g_queue.assign(c, c + n);
  r2ref::g_pos = 0;
  r2ref::g_gen.on = false;
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

// Evaluation order of a three-argument constructor's arguments in this build
// (glm::vec3(a(), b(), c())): 0 = left to right, 1 = right to left.
int ref_vec3_arg_order() {
  float c[3] = {0.25f, 0.5f, 0.75f};
  feed(c, 3);
  rt::CSampler s;
  glm::vec3 v(s.uniformSample01(), s.uniformSample01(), s.uniformSample01());
  return v.x < v.z ? 0 : 1;
}

static glm::mat4x3 M43(const float* m) {
  return glm::mat4x3(glm::vec3(m[0], m[1], m[2]), glm::vec3(m[3], m[4], m[5]), glm::vec3(m[6], m[7], m[8]),
                     glm::vec3(m[9], m[10], m[11]));
}

// Scene of ref_mesh_filter_voxel: world-space vertices (the oracle's BVH is
// built over them), indices, model-space vertex normals, the object's
// model-to-world transform (12 floats, glm mat4x3) and the material (Kd, Ks,
// GGX alpha, ior).  Returns the BVH height, negative on failure.
int ref_filter_scene(const float* wpos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* nrm,
                     const float* m2w, const float* kd, const float* ks, float alpha, float ior) {
  r2ref::HookScene& fs = r2ref::g_fs;
  fs.nodes.assign(16 * (size_t)(ntris > 1 ? ntris - 1 : 1), 0);
  fs.order.assign(ntris, 0);
  fs.tris.assign(12 * (size_t)ntris, 0.f);
  fs.idx.assign(idx, idx + 3 * (size_t)ntris);
  fs.triObj.assign(ntris, 0u);
  fs.nrm.assign(nrm, nrm + 3 * (size_t)nverts);
  fs.m2w.assign(1, M43(m2w));
  fs.mats.clear();
  fs.mats.emplace_back(new rt::CMaterial(V(kd), V(ks), rt::COrenNayarBRDF(0.f),
                                         rt::CMicrofacetBRDF(alpha, alpha, 1.f, ior)));
  fs.mask = rt::ESceneobjectMask::FILTER;
  const int h = orc_build_bvh_filter(wpos, nverts, idx, ntris, fs.nodes.data(), fs.order.data(), fs.tris.data());
  fs.ready = h >= 0;
  return h;
}

// Timing run of the reference's filter on the scene of ref_filter_scene:
// CMeshFilter::run for voxels [v0, v1) (ids x + y*nx + z*nx*ny) of the grid,
// draws from a Philox generator per voxel (voxel, seed), `threads` host
// threads taking every threads-th voxel; out32: the payloads.
int ref_filter_voxels(const float* i2m, const float* m2i, const float* m2w, const float* w2m, const int32_t* nv,
                      const float* bbmin, const float* bbmax, float sigma_t, uint32_t iters, float alpha, int clip,
                      uint32_t spv, uint32_t seed, uint64_t v0, uint64_t v1, unsigned char* out32, int threads) {
  if (!r2ref::g_fs.ready || v1 <= v0 || spv > 1000) return -1;
  if (threads < 1) threads = 1;
  const glm::mat4x3 indexToModel = M43(i2m), modelToIndex = M43(m2i), modelToWorld = M43(m2w),
                    worldToModel = M43(w2m);
  const glm::ivec3 numVoxels(nv[0], nv[1], nv[2]);
  const rt::SAABB bb{V(bbmin), V(bbmax)};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([=, &bb]() {
      for (uint64_t v = v0 + (uint64_t)t; v < v1; v += (uint64_t)threads) {
        const glm::ivec3 cv((int)(v % (uint64_t)nv[0]), (int)((v / (uint64_t)nv[0]) % (uint64_t)nv[1]),
                            (int)(v / ((uint64_t)nv[0] * (uint64_t)nv[1])));
        r2ref::gen_start((uint32_t)v, seed, 0u);
        rt::CSampler sampler;
        filter::CMeshFilter f(cv, indexToModel, modelToIndex, modelToWorld, worldToModel, numVoxels, bb, sampler,
                              sigma_t, iters, alpha, clip != 0, 1.0f);
        rt::CDeviceScene scene;
        const filter::SFilteredDataCompact out = f.run(scene, spv);
        std::memcpy(out32 + 32 * (size_t)(v - v0), &out, 32);
      }
      r2ref::g_gen.on = false;
    });
  }
  for (auto& th : pool) th.join();
  return 0;
}

// Render scene of ref_path_li: world-space vertices and indices of all
// meshes, model-space vertex normals, the object of each triangle, per object
// its transform (12 floats) and material (Kd, Ks, GGX alpha, ior; Oren-Nayar
// roughness 0 as for OBJ materials, material.cu:95), and the environment map.
int ref_render_scene(const float* wpos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* nrm,
                     const uint32_t* triObj, uint32_t nobj, const float* m2w12, const float* mat8, const float* env,
                     int envW, int envH) {
  r2ref::HookScene& fs = r2ref::g_fs;
  fs.nodes.assign(16 * (size_t)(ntris > 1 ? ntris - 1 : 1), 0);
  fs.order.assign(ntris, 0);
  fs.tris.assign(12 * (size_t)ntris, 0.f);
  fs.idx.assign(idx, idx + 3 * (size_t)ntris);
  fs.triObj.assign(triObj, triObj + ntris);
  fs.nrm.assign(nrm, nrm + 3 * (size_t)nverts);
  fs.m2w.clear();
  fs.mats.clear();
  for (uint32_t o = 0; o < nobj; ++o) {
    fs.m2w.push_back(M43(m2w12 + 12 * o));
    const float* m = mat8 + 8 * o;
    fs.mats.emplace_back(new rt::CMaterial(V(m), V(m + 3), rt::COrenNayarBRDF(0.f),
                                           rt::CMicrofacetBRDF(m[6], m[6], 1.f, m[7])));
  }
  fs.env.assign(env, env + 3 * (size_t)envW * envH);
  fs.envW = envW;
  fs.envH = envH;
  orc_env_destroy(fs.envH_);
  fs.envH_ = orc_env_create(fs.env.data(), envW, envH);
  fs.mask = rt::ESceneobjectMask::ALL;
  const int h = orc_build_bvh(wpos, nverts, idx, ntris, fs.nodes.data(), fs.order.data(), fs.tris.data());
  fs.ready = h >= 0;
  return h;
}

// One sample of CPathIntegrator::Li (path_integrator_impl.hpp:120-247, with
// direct(), :23-118) for pixel (px, py) of the camera CCamera(W, H, fov, pos,
// lookAt, up) (camera.cu:20-31), the pixel sampled by CPixelSampler
// (pixel_sampler.hpp:36-47), every draw taken from the queued cuRAND values c.
// L3 receives Li() (NaN or infinite radiance becomes 0; one sample per pixel).
// Returns the draws consumed.
int ref_path_li(uint32_t W, uint32_t H, float fov, const float* pos, const float* lookAt, const float* up,
                uint32_t px, uint32_t py, const float* c, int nc, float* L3) {
  rt::CCamera cam((uint16_t)W, (uint16_t)H, fov, V(pos), V(lookAt), V(up));
  feed(c, nc);
  rt::CSampler sampler;
  rt::CPixelSampler ps(&cam, (uint16_t)px, (uint16_t)py, &sampler);
  rt::CDeviceScene scene;
  rt::CPathIntegrator li(&scene, &ps, &sampler, 1, false, rt::EDebugMode::NONE);
  put(L3, li.Li());
  return ref_draws_used();
}

// Timing run of the reference's integrator on the scene of ref_render_scene:
// for pixels [p0, p1) of the camera, spp samples of CPathIntegrator::Li each
// (its own bounce cap of 50 and roulette from bounce 4), draws from a Philox
// generator per path (pixel, seed, sample), `threads` host threads taking
// every threads-th pixel.  rgb_out: the mean per pixel (3 floats).
int ref_render_paths(uint32_t W, uint32_t H, float fov, const float* pos, const float* lookAt, const float* up,
                     uint32_t spp, uint32_t seed, uint32_t p0, uint32_t p1, float* rgb_out, int threads) {
  if (!r2ref::g_fs.ready || p1 <= p0 || p1 > W * H || spp == 0) return -1;
  if (threads < 1) threads = 1;
  const glm::vec3 P = V(pos), A = V(lookAt), U = V(up);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([=]() {
      rt::CCamera cam((uint16_t)W, (uint16_t)H, fov, P, A, U);
      for (uint32_t p = p0 + (uint32_t)t; p < p1; p += (uint32_t)threads) {
        glm::vec3 acc(0.f);
        for (uint32_t s = 0; s < spp; ++s) {
          r2ref::gen_start(p, seed, s);
          rt::CSampler sampler;
          rt::CPixelSampler ps(&cam, (uint16_t)(p % W), (uint16_t)(p / W), &sampler);
          rt::CDeviceScene scene;
          rt::CPathIntegrator li(&scene, &ps, &sampler, 1, false, rt::EDebugMode::NONE);
          acc += li.Li();
        }
        put(rgb_out + 3 * (size_t)(p - p0), acc / (float)spp);
      }
      r2ref::g_gen.on = false;
    });
  }
  for (auto& th : pool) th.join();
  return 0;
}

// CMeshFilter(voxel, grid...).run(scene, spv) (mesh_filter.hpp:24-122): the
// reference's sampling, closest-hit accumulation, estimateDensity (:182-204,
// 216-226) and payload compaction for one voxel, with the queued draws c (nc
// of them; generateRay takes five per sample).  The grid is the filter's
// launch description (COpenvdbBackend::setupGrid): indexToModel, modelToIndex,
// modelToWorld, worldToModel (12 floats each), numVoxels and the world box.
// out32: the SFilteredDataCompact bytes.  Returns the draws consumed.
int ref_mesh_filter_voxel(const int32_t* voxel, const float* i2m, const float* m2i, const float* m2w,
                          const float* w2m, const int32_t* nv, const float* bbmin, const float* bbmax, float sigma_t,
                          uint32_t iters, float alpha, int clip, uint32_t spv, const float* c, int nc,
                          unsigned char* out32) {
  if (spv > 1000) return -1;  // rayTs[1000] of CMeshFilter::run
  const glm::ivec3 cv(voxel[0], voxel[1], voxel[2]);
  const glm::mat4x3 indexToModel = M43(i2m), modelToIndex = M43(m2i), modelToWorld = M43(m2w),
                    worldToModel = M43(w2m);
  const glm::ivec3 numVoxels(nv[0], nv[1], nv[2]);
  const rt::SAABB bb{V(bbmin), V(bbmax)};
  feed(c, nc);
  rt::CSampler sampler;
  filter::CMeshFilter f(cv, indexToModel, modelToIndex, modelToWorld, worldToModel, numVoxels, bb, sampler, sigma_t,
                        iters, alpha, clip != 0, 1.0f);
  rt::CDeviceScene scene;
  filter::SFilteredDataCompact out = f.run(scene, spv);
  std::memcpy(out32, &out, 32);
  return ref_draws_used();
}

}  // extern "C"
