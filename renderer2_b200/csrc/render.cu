// Wavefront path tracer for sm_100a.
//
// Reference: OptiX megakernel __raygen__rg (raytracer/src/backend/shaders.optix.cu:240-256)
// running CPathIntegrator::Li (raytracer/include/integrators/path_integrator_impl.hpp:120-247)
// with direct() (23-118) once per spp launch (raytracer/raytracer.cu:161-210).
//
// Here one wave is one sample of every pixel.  Per bounce:
//   k_extend  closest hit of every live path (BVH + analytic shapes, and in
//             scenes with media the medium boxes: entering / traversing a
//             medium runs delta tracking, and material-less medium hits are
//             passed through inside the kernel without counting a bounce,
//             exactly like the reference's `--bounces; continue`);
//   k_shade   miss / surface or medium-collision shading: next-event
//             estimation from the environment map and the BSDF- or
//             phase-sampled MIS ray become two shadow records; the
//             continuation ray, Russian roulette and the push of the surviving
//             path into the next queue (warp ballot + popc);
//   k_shadow  transmittance of every shadow record (any-hit against surfaces,
//             then ratio tracking through the media boxes along the ray);
//   k_accum   L += (L_light * tr + L_bsdf * tr) * T for the bounce.
// All kernels are grid-stride over a live count read on the device, so a
// wave is a fixed launch sequence (graph-capturable, no host round trips).
// Random numbers: Philox4x32-10 keyed by (pixel, seed), counter (sample,
// bounce, block, purpose) — independent of queue position and batching.
#include "render.cuh"

namespace r2 {
namespace {

constexpr uint32_t kPurposeCamera = 0xCA3E7Au;
constexpr uint32_t kPurposeMedium = 0x10u;     // + pass-through index within the bounce
constexpr uint32_t kPurposeScatter = 0x100u;   // phase-function and light draws at a collision
constexpr uint32_t kPurposeShadowTr = 0x200u;  // + shadow slot (0 light, 1 BSDF)
constexpr int kMaxPassThrough = 64;            // medium boundaries crossed within one bounce
constexpr int kMaxShadowSegments = 256;        // medium boundaries along one shadow ray

__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ V3 xyz(float4 v) { return v3(v.x, v.y, v.z); }

// Closest hit over triangles, analytic shapes and (kMedia) medium boxes.
// Code: >= 0 triangle, -1 miss, -2 - i shape i, kMediumCodeBase - m medium m.
template <bool kMedia>
__device__ __forceinline__ float4 scene_closest(const SceneView& S, V3 o, V3 d, float tmax) {
  float t = tmax, b1 = 0.0f, b2 = 0.0f;
  int code = -1;
  if (S.hasTris) {
    Hit h = bvh_trace<false>(S.bvh, o, d, tmax);
    if (h.tri >= 0) {
      t = h.t;
      b1 = h.b1;
      b2 = h.b2;
      code = h.tri;
    }
  }
  for (int i = 0; i < S.nshapes; ++i) {
    const Shape& sh = S.shapes[i];
    float ts = -1.0f;
    if (sh.type == kShapeCircle) {
      float den = dot(d, sh.normal);
      if (den != 0.0f) {
        float tc = dot(sh.center - o, sh.normal) / den;
        if (tc > 0.0f && tc <= t) {
          V3 p = o + d * tc;
          if (length(p - sh.center) < sh.radius) ts = tc;
        }
      }
    } else {
      V3 oc = o - sh.center;
      float a = dot(d, d), b = 2.0f * dot(d, oc), c = dot(oc, oc) - sh.radius * sh.radius;
      float disc = b * b - 4.0f * a * c;
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
    if (ts > 0.0f && ts < t) {
      t = ts;
      b1 = b2 = 0.0f;
      code = -2 - i;
    }
  }
  if (kMedia) {
    for (int m = 0; m < S.nmedia; ++m) {
      const float tm = medium_box_hit(S.media[m], o, d);
      if (tm >= 0.0f && tm <= tmax && tm < t) {
        t = tm;
        b1 = b2 = 0.0f;
        code = kMediumCodeBase - m;
      }
    }
  }
  return make_float4(t, b1, b2, __int_as_float(code));
}

// Any surface (triangle or shape) along the ray.
__device__ __forceinline__ bool scene_occluded(const SceneView& S, V3 o, V3 d, float tmax) {
  if (S.hasTris) {
    Hit h = bvh_trace<true>(S.bvh, o, d, tmax);
    if (h.tri >= 0) return true;
  }
  if (S.nshapes > 0) {
    SceneView noTris = S;
    noTris.hasTris = 0;
    const float4 r = scene_closest<false>(noTris, o, d, tmax);
    if (__float_as_int(r.w) != -1) return true;
  }
  return false;
}

// CDeviceScene::intersectTr seen from direct(): the result is 0 when the walk
// ends on a surface (materials do not emit), else the product of the media's
// ratio-tracking estimates.  A surface anywhere on the ray ends the walk
// there, so the any-hit test decides that case; without one the walk visits
// only medium boxes, segment by segment through CRay::spawnRay towards the
// fixed far point p1, multiplying Tr when a segment leaves the current medium.
__device__ float shadow_transmittance(const SceneView& S, V3 o, V3 d, float tmax, int med, bool dda, RngStream& rng,
                                      int* err) {
  if (scene_occluded(S, o, d, tmax)) return 0.0f;
  float tr = 1.0f;
  if (S.nmedia == 0) return tr;
  V3 p0 = o;
  const V3 p1 = o + d * tmax;
  int cur = med;
  for (int k = 0; k < kMaxShadowSegments; ++k) {
    const V3 off = offset_ray_origin(p0, normalize(p1 - p0));
    const float tl = length(p1 - off);
    const V3 dir = (p1 - p0) / tl;
    float best = tl;
    int hitM = -1;
    for (int m = 0; m < S.nmedia; ++m) {
      const float tm = medium_box_hit(S.media[m], off, dir);
      if (tm >= 0.0f && tm <= tl && tm < best) {
        best = tm;
        hitM = m;
      }
    }
    if (hitM < 0) return tr;
    if (cur >= 0 && hitM == cur) tr *= instance_tr(S.media[cur], make_ray(off, dir, best), dda, rng, err);
    p0 = off + dir * best;
    cur = cur < 0 ? hitM : -1;
  }
  *err = 1;
  return 0.0f;
}

__device__ __forceinline__ uint32_t push_queue(uint32_t* q, uint32_t* count, bool pred, uint32_t value) {
  const unsigned full = __activemask();
  const unsigned m = __ballot_sync(full, pred);
  if (m == 0) return 0;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(full, base, leader);
  if (pred) q[base + __popc(m & ((1u << lane) - 1u))] = value;
  return 1;
}

__global__ void __launch_bounds__(256) k_camera(RenderLaunch L) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < L.npix; p += stride) {
    const int px = (int)(p % (uint32_t)L.cam.W), py = (int)(p / (uint32_t)L.cam.W);
    const U4 r = philox4x32_10(u4(L.sample, kPurposeCamera, 0u, 0u), p, L.seed);
    V3 o, d;
    camera_ray(L.cam, px, py, u01(r.x), &o, &d);
    L.st.rayO[p] = f4(o, __int_as_float(-1));
    L.st.rayD[p] = f4(d, kDefaultTmax);
    L.st.T[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    L.st.L[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    L.st.q[0][p] = p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) L.st.counts[0] = L.npix;
}

__global__ void __launch_bounds__(128) k_extend(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = L.st.q[L.bounce & 1];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t p = q[i];
    const V3 o = xyz(L.st.rayO[p]), d = xyz(L.st.rayD[p]);
    L.st.hit[p] = scene_closest<false>(L.scene, o, d, kDefaultTmax);
  }
}

// The medium part of Li (path_integrator_impl.hpp:127-192) up to the event
// that the bounce shades: a surface hit, a medium collision, a miss, or the
// end of the path by a medium rule.
__global__ void __launch_bounds__(128) k_extend_media(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = L.st.q[L.bounce & 1];
  const uint32_t stride = gridDim.x * blockDim.x;
  const SceneView& S = L.scene;
  const bool dda = L.dda != 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t p = q[i];
    const float4 ro = L.st.rayO[p], rd = L.st.rayD[p];
    V3 o = xyz(ro), d = xyz(rd);
    int med = __float_as_int(ro.w);
    float tmax = rd.w;
    V3 T = xyz(L.st.T[p]);
    float4 hr = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(kEventDead));
    int err = 0;
    int j = 0;
    for (; j < kMaxPassThrough; ++j) {
      hr = scene_closest<true>(S, o, d, tmax);
      const int c = __float_as_int(hr.w);
      MediumEvent ev;
      ev.hit = 0;
      int evMed = -1;
      bool dead = false;
      if (c <= kMediumCodeBase) {
        const int mi = kMediumCodeBase - c;
        RngStream rs = rng_stream(p, L.seed, L.sample, L.bounce, kPurposeMedium + (uint32_t)j);
        if (med >= 0) {  // origin inside a medium: track to the hit
          if (mi != med) {
            dead = true;
          } else {
            T = T * instance_sample(S.media[med], make_ray(o, d, hr.x), dda, rs, &ev, &err);
            evMed = med;
          }
        } else {  // entering: find the far side, track through
          const Ray mr = ray_offset(make_ray(o + d * hr.x, normalize(d), kDefaultTmax), d);
          const float4 he = scene_closest<true>(S, mr.o, mr.d, mr.tmax);
          const int ce = __float_as_int(he.w);
          if (ce != -1) {
            if (ce <= kMediumCodeBase && kMediumCodeBase - ce != mi) {
              dead = true;
            } else {
              T = T * instance_sample(S.media[mi], make_ray(mr.o, mr.d, he.x), dda, rs, &ev, &err);
              evMed = mi;
            }
          }
        }
        if (err) dead = true;
        if (!dead && (T.x == 0.0f || T.y == 0.0f || T.z == 0.0f)) dead = true;
      }
      if (dead) {
        hr.w = __int_as_float(kEventDead);
        break;
      }
      if (ev.hit) {
        L.st.evA[p] = f4(ev.pos, ev.ior);
        L.st.evB[p] = f4(ev.normal, __int_as_float(evMed));
        L.st.evC[p] = make_float4(ev.S[0], ev.S[1], ev.S[2], ev.S[3]);
        L.st.evD[p] = make_float2(ev.S[4], ev.S[5]);
        hr.w = __int_as_float(kEventScatter);
        break;
      }
      if (c <= kMediumCodeBase) {  // material-less hit: continue from it without counting a bounce
        const Ray nr = ray_offset(make_ray(o + d * hr.x, normalize(d), kDefaultTmax), d);
        o = nr.o;
        d = nr.d;
        tmax = nr.tmax;
        med = med < 0 ? kMediumCodeBase - c : -1;
        hr.w = __int_as_float(kEventDead);  // stays so if the pass-through bound is reached
        continue;
      }
      break;  // surface hit or miss
    }
    if (j == kMaxPassThrough) err = 1;
    if (err) atomicAdd(L.bound, 1u);
    L.st.rayO[p] = f4(o, __int_as_float(med));
    L.st.rayD[p] = f4(d, tmax);
    L.st.T[p] = f4(T, 0.0f);
    L.st.hit[p] = hr;
  }
}

// Surface shading: direct() at a surface and the sampleF continuation
// (path_integrator_impl.hpp:23-118, 196-222).
template <bool kMedia>
__device__ __forceinline__ bool shade_surface(const RenderLaunch& L, uint32_t i, uint32_t p, int code, float4 hr,
                                              V3 o, V3 d, int med, V3 T) {
  const V3 pos = o + d * hr.x;
  V3 n;
  Material m;
  if (code >= 0) {
    const float4 n0 = __ldg(&L.scene.triN[3 * code]);
    const float4 n1 = __ldg(&L.scene.triN[3 * code + 1]);
    const float4 n2 = __ldg(&L.scene.triN[3 * code + 2]);
    const float b0 = (1.0f - hr.y) - hr.z;
    n = normalize(xyz(n0) * b0 + xyz(n1) * hr.y + xyz(n2) * hr.z);
    m = L.scene.mats[__ldg(&L.scene.triMat[code])];
  } else {
    const Shape& sh = L.scene.shapes[-2 - code];
    // __closesthit__ch normalises the reported shape normal (shaders.optix.cu:110-114)
    n = sh.type == kShapeCircle ? normalize(sh.normal) : normalize(pos - sh.center);
    m = L.scene.mats[sh.material];
  }
  const U4 rA = philox4x32_10(u4(L.sample, L.bounce, 0u, 1u), p, L.seed);
  const U4 rB = philox4x32_10(u4(L.sample, L.bounce, 1u, 1u), p, L.seed);
  const Frame fr = frame_from_normal(n);
  const V3 wo = -d;
  const V3 woT = to_local(fr, wo);
  const V3 offO = offset_ray_origin(pos, n);
  float4 shO0 = make_float4(0, 0, 0, 0), shO1 = shO0, shD0 = shO0, shD1 = shO0, pre0 = shO0, pre1 = shO0;
  // --- direct(): light sample (path_integrator_impl.hpp:31-71)
  {
    V3 ldir;
    float lpdf = 0.0f;
    const V3 Le = env_sample(L.scene.env, u01(rA.x), u01(rA.y), &ldir, &lpdf);
    if (lpdf > 0.0f) {
      ldir = normalize(ldir);
      const V3 lT = normalize(to_local(fr, ldir));
      const V3 f = mat_f(m, woT, lT) * fabsf(dot(n, ldir));
      const float spdf = mat_pdf(m, woT, lT);
      const float mis = balance_heuristic(lpdf, spdf);
      shO0 = f4(offO, lpdf);
      shD0 = f4(ldir, 0.0f);
      pre0 = f4((f * mis) * Le, 0.0f);
      if (kMedia) {
        const Ray lr = ray_offset(make_ray(pos, ldir, kDefaultTmax), n);
        L.st.shX[2 * i] = make_float2(lr.tmax, __int_as_float(med));
      }
    }
  }
  // --- direct(): BSDF sample (path_integrator_impl.hpp:74-113)
  {
    V3 wiT = v3(0.0f);
    float spdf = 0.0f;
    V3 f = mat_sample_f(m, woT, u01(rA.z), u01(rA.w), u01(rB.x), &wiT, &spdf);
    V3 wi = normalize(to_world(fr, wiT));
    f = f * fabsf(dot(n, wi));
    if (spdf > 0.0f) {
      wi = normalize(wi);
      float lpdf;
      const V3 Le = env_le(L.scene.env, wi, &lpdf);
      const float mis = balance_heuristic(spdf, lpdf);
      shO1 = f4(offO, spdf);
      shD1 = f4(wi, 0.0f);
      pre1 = f4((f * mis) * Le, 0.0f);
      if (kMedia) {
        const Ray br = ray_offset(make_ray(pos, wi, kDefaultTmax), n);
        L.st.shX[2 * i + 1] = make_float2(br.tmax, __int_as_float(med));
      }
    }
  }
  L.st.shO[2 * i] = shO0;
  L.st.shO[2 * i + 1] = shO1;
  L.st.shD[2 * i] = shD0;
  L.st.shD[2 * i + 1] = shD1;
  L.st.shPre[2 * i] = pre0;
  L.st.shPre[2 * i + 1] = pre1;
  L.st.shT[i] = f4(T, 0.0f);
  // --- continuation (path_integrator_impl.hpp:200-232)
  const V3 dT = normalize(to_local(fr, d));
  V3 wi = v3(0.0f);
  float pdf = 0.0f;
  const V3 f = mat_sample_f(m, -dT, u01(rB.y), u01(rB.z), u01(rB.w), &wi, &pdf);
  if (pdf == 0.0f) return false;
  const V3 dirW = normalize(to_world(fr, wi));
  const float cosine = fabsf(dot(n, dirW));
  V3 Tn = T * ((f * cosine) / pdf);
  if (L.bounce > 3) {
    const U4 rC = philox4x32_10(u4(L.sample, L.bounce, 2u, 1u), p, L.seed);
    const float prr = 1.0f - (Tn.x + Tn.y + Tn.z) / 3.0f;
    if (u01(rC.x) <= prr) return false;
    Tn = Tn / (1.0f - prr);
  }
  if (L.bounce + 1 >= L.maxDepth) return false;
  L.st.rayO[p] = f4(offO, __int_as_float(med));
  // CRay(pos, dir, DEFAULT_TMAX).offsetRayOrigin(n): the end point stays at pos + 1e12 dir
  L.st.rayD[p] = f4(dirW, kMedia ? ray_offset(make_ray(pos, dirW, kDefaultTmax), n).tmax : kDefaultTmax);
  L.st.T[p] = f4(Tn, 0.0f);
  return true;
}

// Collision shading: direct() with the SGGX phase function, then the
// phase-sampled continuation moved to the voxel border
// (path_integrator_impl.hpp:164-173, 23-118).
__device__ __forceinline__ bool shade_scatter(const RenderLaunch& L, uint32_t i, uint32_t p, V3 d, V3 T) {
  const float4 a = L.st.evA[p], b = L.st.evB[p], c = L.st.evC[p];
  const float2 e = L.st.evD[p];
  const V3 pos = xyz(a), n = xyz(b);
  const float ior = a.w;
  const int med = __float_as_int(b.w);
  const MediumView& M = L.scene.media[med];
  const float S[6] = {c.x, c.y, c.z, c.w, e.x, e.y};
  const Sggx g = make_sggx(S, n);
  const V3 wo = -d;
  RngStream rs = rng_stream(p, L.seed, L.sample, L.bounce, kPurposeScatter);
  float4 shO0 = make_float4(0, 0, 0, 0), shO1 = shO0, shD0 = shO0, shD1 = shO0, pre0 = shO0, pre1 = shO0;
  {
    V3 ldir;
    float lpdf = 0.0f;
    const float u0 = rs.next();
    const float u1 = rs.next();
    const V3 Le = env_sample(L.scene.env, u0, u1, &ldir, &lpdf);
    if (lpdf > 0.0f) {
      ldir = normalize(ldir);
      const Ray lr = instance_move_to_voxel_border(M, ray_offset(make_ray(pos, ldir, kDefaultTmax), n));
      const float sp = M.hg ? phase_hg(dot(wo, ldir), M.g) : sggx_p(g, ior, wo, ldir, rs);
      const float mis = balance_heuristic(lpdf, sp);
      shO0 = f4(lr.o, lpdf);
      shD0 = f4(lr.d, 0.0f);
      L.st.shX[2 * i] = make_float2(lr.tmax, __int_as_float(med));
      pre0 = f4((v3(sp) * mis) * Le, 0.0f);
    }
  }
  {
    V3 wi = v3(0.0f);
    const float sp = M.hg ? hg_sample_p(M.g, wo, &wi, rs) : sggx_sample_p(g, ior, wo, &wi, rs);
    if (sp > 0.0f) {
      wi = normalize(wi);
      const Ray br = instance_move_to_voxel_border(M, ray_offset(make_ray(pos, wi, kDefaultTmax), n));
      float lpdf;
      const V3 Le = env_le(L.scene.env, wi, &lpdf);
      const float mis = balance_heuristic(sp, lpdf);
      shO1 = f4(br.o, sp);
      shD1 = f4(br.d, 0.0f);
      L.st.shX[2 * i + 1] = make_float2(br.tmax, __int_as_float(med));
      pre1 = f4((v3(sp) * mis) * Le, 0.0f);
    }
  }
  L.st.shO[2 * i] = shO0;
  L.st.shO[2 * i + 1] = shO1;
  L.st.shD[2 * i] = shD0;
  L.st.shD[2 * i + 1] = shD1;
  L.st.shPre[2 * i] = pre0;
  L.st.shPre[2 * i + 1] = pre1;
  L.st.shT[i] = f4(T, 0.0f);
  V3 wi = v3(0.0f);
  if (M.hg) hg_sample_p(M.g, wo, &wi, rs);
  else sggx_sample_p(g, ior, wo, &wi, rs);
  const Ray cr = instance_move_to_voxel_border(M, ray_offset(make_ray(pos, normalize(wi), kDefaultTmax), wi));
  V3 Tn = T;
  if (L.bounce > 3) {
    const U4 rC = philox4x32_10(u4(L.sample, L.bounce, 2u, 1u), p, L.seed);
    const float prr = 1.0f - (Tn.x + Tn.y + Tn.z) / 3.0f;
    if (u01(rC.x) <= prr) return false;
    Tn = Tn / (1.0f - prr);
  }
  if (L.bounce + 1 >= L.maxDepth) return false;
  L.st.rayO[p] = f4(cr.o, __int_as_float(med));
  L.st.rayD[p] = f4(cr.d, cr.tmax);
  L.st.T[p] = f4(Tn, 0.0f);
  return true;
}

template <bool kMedia>
__global__ void __launch_bounds__(128) k_shade(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = L.st.q[L.bounce & 1];
  uint32_t* qn = L.st.q[(L.bounce + 1) & 1];
  uint32_t* cn = &L.st.counts[L.bounce + 1];
  const uint32_t stride = gridDim.x * blockDim.x;
  // uniform trip count per warp so the ballot below sees the whole warp
  const uint32_t nRound = (n + 31u) & ~31u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nRound; i += stride) {
    bool cont = false;
    uint32_t p = 0;
    if (i < n) {
      p = q[i];
      const float4 hr = L.st.hit[p];
      const int code = __float_as_int(hr.w);
      const float4 ro = L.st.rayO[p];
      const V3 o = xyz(ro), d = xyz(L.st.rayD[p]);
      const V3 T = xyz(L.st.T[p]);
      if (code == -1 || code == kEventDead) {
        if (code == -1 && L.bounce == 0) {
          float lp;
          const V3 le = env_le(L.scene.env, d, &lp);
          L.st.L[p] = f4(xyz(L.st.L[p]) + le * T, 0.0f);
        }
        const float4 z = make_float4(0, 0, 0, 0);
        L.st.shO[2 * i] = z;
        L.st.shO[2 * i + 1] = z;
      } else if (kMedia && code == kEventScatter) {
        cont = shade_scatter(L, i, p, d, T);
      } else {
        cont = shade_surface<kMedia>(L, i, p, code, hr, o, d, __float_as_int(ro.w), T);
      }
    }
    push_queue(qn, cn, cont, p);
  }
}

template <bool kMedia>
__global__ void __launch_bounds__(128) k_shadow(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = L.st.q[L.bounce & 1];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < 2 * n; j += stride) {
    const float4 o = L.st.shO[j];
    float tr = 0.0f;
    const bool traced = o.w > 0.0f;
    if (traced) {
      const float4 d = L.st.shD[j];
      if (kMedia) {
        const float2 x = L.st.shX[j];
        RngStream rs = rng_stream(q[j >> 1], L.seed, L.sample, L.bounce, kPurposeShadowTr + (j & 1u));
        int err = 0;
        tr = shadow_transmittance(L.scene, xyz(o), xyz(d), x.x, __float_as_int(x.y), L.dda != 0, rs, &err);
        if (err) atomicAdd(L.bound, 1u);
      } else {
        tr = scene_occluded(L.scene, xyz(o), xyz(d), kDefaultTmax) ? 0.0f : 1.0f;
      }
    }
    L.st.shTr[j] = tr;
    if (L.stats) {
      const unsigned m = __ballot_sync(__activemask(), traced);
      if ((threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1) && m)
        atomicAdd(&L.stats[1], (unsigned long long)__popc(m));
    }
  }
  if (L.stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&L.stats[0], (unsigned long long)n);
}

__global__ void __launch_bounds__(256) k_accum(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = L.st.q[L.bounce & 1];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float4 o0 = L.st.shO[2 * i], o1 = L.st.shO[2 * i + 1];
    if (!(o0.w > 0.0f) && !(o1.w > 0.0f)) continue;
    const uint32_t p = q[i];
    V3 dl = v3(0.0f);
    if (o0.w > 0.0f) dl = dl + (xyz(L.st.shPre[2 * i]) * L.st.shTr[2 * i]) / o0.w;
    if (o1.w > 0.0f) dl = dl + (xyz(L.st.shPre[2 * i + 1]) * L.st.shTr[2 * i + 1]) / o1.w;
    const V3 Lp = xyz(L.st.L[p]);
    L.st.L[p] = f4(Lp + dl * xyz(L.st.shT[i]), 0.0f);
  }
}

__global__ void __launch_bounds__(256) k_finish(RenderLaunch L) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < L.npix; p += stride) {
    V3 v = xyz(L.st.L[p]);
    if (isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z)) v = v3(0.0f);
    else v = v / (float)L.spp;
    L.frame[3 * p] += v.x;
    L.frame[3 * p + 1] += v.y;
    L.frame[3 * p + 2] += v.z;
  }
}

}  // namespace

void launch_render_wave(const RenderLaunch& L0, int nblocks, cudaStream_t s, WaveTimer* tm) {
  RenderLaunch L = L0;
  const bool media = L.scene.nmedia > 0;
  int ev = 0;
  auto mark = [&](int kind) {
    if (!tm) return;
    R2_CUDA(cudaEventRecord(tm->ev[ev], s));
    tm->kind[ev] = kind;
    ++ev;
  };
  R2_CUDA(cudaMemsetAsync(L.st.counts, 0, sizeof(uint32_t) * (L.maxDepth + 2), s));
  mark(-1);
  k_camera<<<nblocks, 256, 0, s>>>(L);
  mark(0);
  for (uint32_t b = 0; b < L.maxDepth; ++b) {
    L.bounce = b;
    if (media) {
      k_extend_media<<<nblocks * 2, 128, 0, s>>>(L);
      mark(1);
      k_shade<true><<<nblocks * 2, 128, 0, s>>>(L);
      mark(2);
      k_shadow<true><<<nblocks * 2, 128, 0, s>>>(L);
    } else {
      k_extend<<<nblocks * 2, 128, 0, s>>>(L);
      mark(1);
      k_shade<false><<<nblocks * 2, 128, 0, s>>>(L);
      mark(2);
      k_shadow<false><<<nblocks * 2, 128, 0, s>>>(L);
    }
    mark(3);
    k_accum<<<nblocks, 256, 0, s>>>(L);
    mark(4);
  }
  k_finish<<<nblocks, 256, 0, s>>>(L);
  mark(5);
  if (tm) tm->n = ev;
  R2_CUDA(cudaGetLastError());
}

}  // namespace r2
