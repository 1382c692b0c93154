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
#include <algorithm>

#include <map>
#include <mutex>

#include "render.cuh"
#include "texture_shade.cuh"

namespace r2 {
namespace {

constexpr uint32_t kPurposeCamera = 0xCA3E7Au;
constexpr uint32_t kPurposeMedium = 0x1000u;   // + pass-through index within the bounce
constexpr uint32_t kPurposeScatter = 0x100u;   // phase-function and light draws at a collision
constexpr uint32_t kPurposeShadowTr = 0x200u;  // + shadow slot (0 light, 1 BSDF)
constexpr int kMaxPassThrough = 4096;          // medium boundaries crossed within one bounce
constexpr int kMaxShadowSegments = 4096;       // medium boundaries along one shadow ray (per round)

__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
// Sample index of the wave: a kernel parameter, or the device counter of a
// captured wave that is replayed once per sample.
__device__ __forceinline__ uint32_t wave_sample(const RenderLaunch& L) {
  return L.sampleDev ? *(volatile const uint32_t*)L.sampleDev : L.sample;
}
// Pixel and sample of path p of the wave (waves group consecutive samples).
__device__ __forceinline__ uint32_t path_pixel(const RenderLaunch& L, uint32_t p) {
  return L.waveSpp == 1u ? p : p % L.npix;
}
__device__ __forceinline__ uint32_t path_sample(const RenderLaunch& L, uint32_t p) {
  return wave_sample(L) + (L.waveSpp == 1u ? 0u : p / L.npix);
}
__device__ __forceinline__ V3 xyz(float4 v) { return v3(v.x, v.y, v.z); }
// Entries of the kernel parameter's pointer pairs, picked with selects: a
// dynamic index into an array inside the parameter makes the compiler copy the
// whole launch description to local memory.
__device__ __forceinline__ uint32_t* pick(uint32_t* const (&a)[2], uint32_t i) { return i ? a[1] : a[0]; }
__device__ __forceinline__ uint32_t* path_queue(const RenderLaunch& L, uint32_t b) { return pick(L.st.q, b & 1u); }
// Events of the bounce (surface hits, then medium collisions) and the path of event i.
__device__ __forceinline__ uint32_t event_count(const RenderLaunch& L) {
  return *(volatile uint32_t*)&L.st.counts[kHitCounters + L.bounce] +
         *(volatile uint32_t*)&L.st.counts[kScatterCounters + L.bounce];
}
__device__ __forceinline__ uint32_t event_path(const RenderLaunch& L, uint32_t i) {
  const uint32_t nh = *(volatile uint32_t*)&L.st.counts[kHitCounters + L.bounce];
  return i < nh ? L.st.qh[i] : L.st.qs[i - nh];
}

// Entry distance of a ray into a BVH node's child box, or INFINITY when the
// ray misses it: the slab arithmetic and comparisons of medium_box_hit, so
// with the builder's boxes padded around the instances' boxes an instance
// the ray hits is never culled and its distance is >= the entry returned here.
__device__ __forceinline__ float media_box_enter(float lx, float hx, float ly, float hy, float lz, float hz, V3 o,
                                                 V3 inv) {
  float t0 = 0.0f, t1 = kDefaultTmax;
  const float lo[3] = {lx, ly, lz}, hi[3] = {hx, hy, hz};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float a = (lo[i] - comp(o, i)) * comp(inv, i);
    float b = (hi[i] - comp(o, i)) * comp(inv, i);
    if (a > b) {
      const float t = a;
      a = b;
      b = t;
    }
    if (a > t0) t0 = a;
    if (b < t1) t1 = b;
  }
  return t0 > t1 ? INFINITY : t0;
}

// First medium-box boundary along a ray: the smallest medium_box_hit in
// [0, limit] over the instances, the lowest instance index among equal
// distances (what a loop over the instances in order with a strict `<`
// keeps).  Returns the instance (-1: none) and its distance in *tOut.
__device__ __forceinline__ int media_first(const SceneView& S, V3 o, V3 d, float limit, float* tOut) {
  float best = INFINITY;
  int bestM = -1;
  if (S.mediaNodes == nullptr) {
    for (int m = 0; m < S.nmedia; ++m) {
      const float tm = medium_box_hit(S.media[m], o, d);
      if (tm >= 0.0f && tm <= limit && tm < best) {
        best = tm;
        bestM = m;
      }
    }
    *tOut = best;
    return bestM;
  }
  const V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  int stack[R2_BVH_STACK];
  float stackT[R2_BVH_STACK];
  int sp = 0;
  int ref = 0;  // the root node
  float refT = 0.0f;
  for (;;) {
    if (refT <= best && refT <= limit) {
      if (ref < 0) {
        const int first = bvh_leaf_first(ref), count = bvh_leaf_count(ref);
        for (int k = 0; k < count; ++k) {
          const int m = (int)__ldg(&S.mediaOrder[first + k]);
          const float tm = medium_box_hit(S.media[m], o, d);
          if (tm >= 0.0f && tm <= limit && (tm < best || (tm == best && m < bestM))) {
            best = tm;
            bestM = m;
          }
        }
      } else {
        const BvhNode* nd = S.mediaNodes + ref;
        const float4 b0 = __ldg(&nd->b0), b1 = __ldg(&nd->b1), bz = __ldg(&nd->bz);
        const int4 ch = __ldg(&nd->ch);
        const float t0 = media_box_enter(b0.x, b0.y, b0.z, b0.w, bz.x, bz.y, o, inv);
        const float t1 = ch.y == R2_BVH_NONE ? INFINITY : media_box_enter(b1.x, b1.y, b1.z, b1.w, bz.z, bz.w, o, inv);
        const bool h0 = t0 <= best && t0 <= limit, h1 = t1 <= best && t1 <= limit;
        if (h0 && h1) {
          const bool near0 = t0 <= t1;
          stack[sp] = near0 ? ch.y : ch.x;
          stackT[sp] = near0 ? t1 : t0;
          ++sp;
          ref = near0 ? ch.x : ch.y;
          refT = near0 ? t0 : t1;
          continue;
        }
        if (h0 || h1) {
          ref = h0 ? ch.x : ch.y;
          refT = h0 ? t0 : t1;
          continue;
        }
      }
    }
    if (sp == 0) break;
    --sp;
    ref = stack[sp];
    refT = stackT[sp];
  }
  *tOut = best;
  return bestM;
}

// Closest hit over triangles, analytic shapes and (kMedia) medium boxes.
// Code: >= 0 triangle, -1 miss, -2 - i shape i, kMediumCodeBase - m medium m.
// scene_closest_after finishes the query from the triangles' result h.
template <bool kMedia>
__device__ __forceinline__ float4 scene_closest_after(const SceneView& S, V3 o, V3 d, float tmax, const Hit& h) {
  float t = tmax, b1 = 0.0f, b2 = 0.0f;
  int code = -1;
  if (h.tri >= 0) {
    t = h.t;
    b1 = h.b1;
    b2 = h.b2;
    code = h.tri;
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
  if (kMedia && S.nmedia > 0) {
    float tm;
    const int m = media_first(S, o, d, tmax, &tm);
    if (m >= 0 && tm < t) {
      t = tm;
      b1 = b2 = 0.0f;
      code = kMediumCodeBase - m;
    }
  }
  return make_float4(t, b1, b2, __int_as_float(code));
}

template <bool kMedia>
__device__ __forceinline__ float4 scene_closest(const SceneView& S, V3 o, V3 d, float tmax) {
  Hit h;
  h.tri = -1;
  if (S.hasTris) h = bvh_trace<false>(S.bvh, o, d, tmax);
  return scene_closest_after<kMedia>(S, o, d, tmax, h);
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
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < L.wavePaths; p += stride) {
    const uint32_t pix = path_pixel(L, p);
    const int px = (int)(pix % (uint32_t)L.cam.W), py = (int)(pix / (uint32_t)L.cam.W);
    const U4 r = philox4x32_10(u4(path_sample(L, p), kPurposeCamera, 0u, 0u), pix, L.seed);
    V3 o, d;
    camera_ray(L.cam, px, py, u01(r.x), &o, &d);
    L.st.rayO[p] = f4(o, __int_as_float(-1));
    L.st.rayD[p] = f4(d, kDefaultTmax);
    L.st.T[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    L.st.L[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    L.st.q[0][p] = p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) L.st.counts[0] = L.wavePaths;
}

// Out-of-line copies of the large shading routines.  k_shade's lanes diverge
// between lobes and events, and with every routine inlined at each call site
// the kernel's code outgrew the instruction cache (warps stalled on
// instruction fetch); one copy of each keeps the working set small.  The
// arithmetic is the same, so results do not change.
struct BsdfSample {
  V3 f, wi;
  float pdf;
};
__device__ __noinline__ BsdfSample bsdf_sample_nc(Material m, V3 wo, float uSel, float u1, float u2) {
  BsdfSample r;
  r.wi = v3(0.0f);
  r.pdf = 0.0f;
  r.f = mat_sample_f(m, wo, uSel, u1, u2, &r.wi, &r.pdf);
  return r;
}
struct BsdfEval {
  V3 f;
  float pdf;
};
__device__ __noinline__ BsdfEval bsdf_eval_nc(Material m, V3 wo, V3 wi) {
  BsdfEval r;
  r.f = mat_f(m, wo, wi);
  r.pdf = mat_pdf(m, wo, wi);
  return r;
}
struct EnvSample {
  V3 Le, dir;
  float pdf;
};
__device__ __noinline__ EnvSample env_sample_nc(EnvMap e, float u0, float u1) {
  EnvSample r;
  r.dir = v3(0.0f);
  r.pdf = 0.0f;
  r.Le = env_sample(e, u0, u1, &r.dir, &r.pdf);
  return r;
}
struct EnvEval {
  V3 Le;
  float pdf;
};
__device__ __noinline__ EnvEval env_le_nc(EnvMap e, V3 d) {
  EnvEval r;
  r.pdf = 0.0f;
  r.Le = env_le(e, d, &r.pdf);
  return r;
}
__device__ __noinline__ U4 philox_nc(U4 ctr, uint32_t k0, uint32_t k1) { return philox4x32_10(ctr, k0, k1); }

// Phase functions of a medium collision (SGGX, or Henyey-Greenstein for media
// with "G"); the stream is passed through by value.
struct PhaseEval {
  float p;
  RngStream rs;
};
__device__ __noinline__ PhaseEval phase_eval_nc(const MediumView* M, Sggx g, float ior, V3 wo, V3 wi, RngStream rs) {
  PhaseEval r;
  r.p = M->hg ? phase_hg(dot(wo, wi), M->g) : sggx_p(g, ior, wo, wi, rs);
  r.rs = rs;
  return r;
}
struct PhaseSample {
  V3 wi;
  float p;
  RngStream rs;
};
__device__ __noinline__ PhaseSample phase_sample_nc(const MediumView* M, Sggx g, float ior, V3 wo, RngStream rs) {
  PhaseSample r;
  r.wi = v3(0.0f);
  r.p = M->hg ? hg_sample_p(M->g, wo, &r.wi, rs) : sggx_sample_p(g, ior, wo, &r.wi, rs);
  r.rs = rs;
  return r;
}
__device__ __noinline__ Ray voxel_border_nc(const MediumView* M, Ray r) { return instance_move_to_voxel_border(*M, r); }

// Persistent BVH traversal with dynamic ray fetch (Aila and Laine,
// "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009): the
// lanes of a warp run their rays in rounds of `visits` node/leaf visits, and
// as soon as `refill` lanes have finished (or all of them) the warp takes as
// many new items from the queue with one atomic, so that lanes do not idle
// behind the warp's longest ray.  begin(k, s, &item) starts item k (false: it
// needed no traversal and is done); end(item, s) consumes a finished query.
// Results do not depend on visits or refill.
// A ray still unfinished after kMaxTraceVisits visits (a correct traversal
// visits each node at most once) is ended as a miss and counted in *bound.
constexpr int kMaxTraceVisits = 1 << 26;

template <bool kAnyHit, bool kAlpha, bool kInst, bool kTop, class Begin, class End>
__device__ __forceinline__ void trace_persistent(const BvhView& bvh, uint32_t n, uint32_t* taken, int visits,
                                                 int refill, unsigned int* bound, Begin begin, End end) {
  int stack[R2_BVH_STACK];
  float stackT[R2_BVH_STACK];
  TraceState s;
  uint32_t item = 0;
  int spent = 0;  // visits of the lane's current ray
  bool active = false;
  bool more = true;  // warp-uniform: the queue may still hold items
  const int lane = threadIdx.x & 31;
  while (true) {
    if (more) {
      const unsigned idle = __ballot_sync(0xffffffffu, !active);
      const int nIdle = __popc(idle);
      if (nIdle >= refill || idle == 0xffffffffu) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(taken, (uint32_t)nIdle);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base + (uint32_t)nIdle >= n) more = false;
        if (!active) {
          const uint32_t k = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
          if (k < n) {
            active = begin(k, s, &item);
            spent = 0;
          }
        }
      }
    }
    if (__ballot_sync(0xffffffffu, active) == 0) {
      if (!more) break;
      continue;
    }
    if (active) {
      bool done = trace_advance<kAnyHit, false, kAlpha, kInst, kTop>(bvh, s, stack, stackT, visits);
      spent += visits;
      if (!done && spent >= kMaxTraceVisits) {
        s.best.tri = -1;
        atomicAdd(bound, 1u);
        done = true;
      }
      if (done) {
        if (!kInst) {  // one level: the traversal ray is the world ray (keeps wo/wd out of the live state)
          s.wo = s.r.o;
          s.wd = s.r.d;
        }
        end(item, s);
        active = false;
      }
    }
  }
}

__device__ __forceinline__ int trav_visits(const RenderLaunch& L) { return (int)max(1u, L.travVisits); }
__device__ __forceinline__ int trav_refill(const RenderLaunch& L) { return (int)min(32u, max(1u, L.travRefill)); }

// The persistent traversal of the scene's BVH (kAlpha: alpha-tested
// triangles; kInst: two levels).  kTop: the block first copies BVH nodes
// 0 .. L.topNodes-1 (the host keeps the count within the tree and
// kMaxTopNodes) into its dynamic shared memory and reads them from there.
// Every thread of the block calls this once.
template <bool kAnyHit, bool kAlpha, bool kInst, bool kTop, class Begin, class End>
__device__ __forceinline__ void trace_scene(const RenderLaunch& L, uint32_t n, uint32_t* taken, Begin begin, End end) {
  BvhView bvh = L.scene.bvh;
  if (kTop) {
    extern __shared__ BvhNode sTop[];
    const int ntop = (int)L.topNodes;
    for (int k = threadIdx.x; k < ntop; k += blockDim.x) sTop[k] = bvh.nodes[k];
    __syncthreads();
    bvh.top = sTop;
    bvh.ntop = ntop;
  }
  trace_persistent<kAnyHit, kAlpha, kInst, kTop>(bvh, n, taken, trav_visits(L), trav_refill(L), L.bound, begin, end);
}

// ------------------------------------------------------------------ ray order
// Coherence order of a bounce's rays (tuning sort_rays): the path queue is
// reordered by an 8-bit key — direction octant (3 bits), dominant axis
// (2 bits) and the origin's octant of the scene box (3 bits) — with a counting
// sort: block histograms, one scan of the 256 bins, a scatter.  Positions
// within a bin depend on atomic order; no result depends on the order of the
// rays (each path keeps its own random streams and the frame adds samples per
// pixel in sample order).
__device__ __forceinline__ uint32_t ray_key(V3 o, V3 d, V3 mid) {
  const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  const V3 a = vabs(d);
  const uint32_t axis = a.x >= a.y ? (a.x >= a.z ? 0u : 2u) : (a.y >= a.z ? 1u : 2u);
  const uint32_t cell = (o.x < mid.x ? 0u : 1u) | (o.y < mid.y ? 0u : 2u) | (o.z < mid.z ? 0u : 4u);
  return (cell << 5) | (axis << 3) | oct;
}

__device__ __forceinline__ V3 scene_mid(const SceneView& S) {
  const BvhNode nd = S.bvh.nodes[0];
  const bool two = nd.ch.y != R2_BVH_NONE;
  const V3 lo = two ? v3(fminf(nd.b0.x, nd.b1.x), fminf(nd.b0.z, nd.b1.z), fminf(nd.bz.x, nd.bz.z))
                    : v3(nd.b0.x, nd.b0.z, nd.bz.x);
  const V3 hi = two ? v3(fmaxf(nd.b0.y, nd.b1.y), fmaxf(nd.b0.w, nd.b1.w), fmaxf(nd.bz.y, nd.bz.w))
                    : v3(nd.b0.y, nd.b0.w, nd.bz.y);
  return (lo + hi) * 0.5f;
}

__global__ void __launch_bounds__(256) k_sort_hist(RenderLaunch L) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = path_queue(L, L.bounce);
  const V3 mid = scene_mid(L.scene);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = q[i];
    atomicAdd(&h[ray_key(xyz(L.st.rayO[p]), xyz(L.st.rayD[p]), mid)], 1u);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&L.st.sortBins[threadIdx.x], h[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_sort_scan(RenderLaunch L) {
  __shared__ uint32_t w[8];
  const uint32_t v = L.st.sortBins[threadIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) w[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  for (int k = 0; k < warp; ++k) before += w[k];
  L.st.sortBins[threadIdx.x] = before + x - v;  // exclusive: the bin's first position
}

// Each block takes its keys' positions from the bins' cursors with one atomic
// per bin, then places its rays with shared-memory cursors.
__global__ void __launch_bounds__(256) k_sort_scatter(RenderLaunch L) {
  __shared__ uint32_t h[256], base[256];
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = path_queue(L, L.bounce);
  const V3 mid = scene_mid(L.scene);
  for (uint32_t b0 = blockIdx.x * blockDim.x; b0 < n; b0 += gridDim.x * blockDim.x) {
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = b0 + threadIdx.x;
    uint32_t p = 0, key = 0, rank = 0;
    if (i < n) {
      p = q[i];
      key = ray_key(xyz(L.st.rayO[p]), xyz(L.st.rayD[p]), mid);
      rank = atomicAdd(&h[key], 1u);
    }
    __syncthreads();
    if (h[threadIdx.x]) base[threadIdx.x] = atomicAdd(&L.st.sortBins[threadIdx.x], h[threadIdx.x]);
    __syncthreads();
    if (i < n) L.st.qs[base[key] + rank] = p;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_sort_copy(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  uint32_t* q = path_queue(L, L.bounce);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) q[i] = L.st.qs[i];
}

// Closest hit of every live path (scenes without media).  A path that hits a
// surface goes to the bounce's hit queue (shading, shadow rays and
// accumulation then run over hits only); a miss ends the path here with the
// environment term of the first bounce (k_shade's miss rule).
__device__ __forceinline__ void extend_result(const RenderLaunch& L, uint32_t p, V3 d, float4 h) {
  if (__float_as_int(h.w) == -1) {
    if (L.bounce == 0) {
      const V3 le = env_le_nc(L.scene.env, d).Le;
      L.st.L[p] = f4(xyz(L.st.L[p]) + le * xyz(L.st.T[p]), 0.0f);
    }
  } else {
    L.st.hit[p] = h;
  }
  push_queue(L.st.qh, &L.st.counts[kHitCounters + L.bounce], __float_as_int(h.w) != -1, p);
}

// One instantiation per traversal variant (no triangles; alpha test, two
// levels, shared top nodes), each with its own register allocation.
template <bool kTris, bool kAlpha, bool kInst, bool kTop>
__global__ void __launch_bounds__(128, 10) k_extend(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = path_queue(L, L.bounce);
  if constexpr (!kTris) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const uint32_t p = q[i];
      const V3 d = xyz(L.st.rayD[p]);
      extend_result(L, p, d, scene_closest<false>(L.scene, xyz(L.st.rayO[p]), d, kDefaultTmax));
    }
  } else {
    auto begin = [&](uint32_t k, TraceState& s, uint32_t* item) {
      const uint32_t p = q[k];
      *item = p;
      trace_begin(s, xyz(L.st.rayO[p]), xyz(L.st.rayD[p]), kDefaultTmax);
      return true;
    };
    auto end = [&](uint32_t p, const TraceState& s) {
      extend_result(L, p, s.wd, scene_closest_after<false>(L.scene, s.wo, s.wd, kDefaultTmax, s.best));
    };
    trace_scene<false, kAlpha, kInst, kTop>(L, n, &L.st.counts[kTravCounters + 2 * L.bounce], begin, end);
  }
}

// ------------------------------------------------------------------ media: path extension
// The medium part of Li (path_integrator_impl.hpp:127-192) up to the event
// that the bounce shades: a surface hit, a medium collision, a miss, or the
// end of the path by a medium rule; material-less medium hits are passed
// through without counting a bounce (the reference's `--bounces; continue`).
//
// Tracking runs apart from the closest-hit work: a resolve round takes a path
// up to its first segment that needs tracking and queues that segment; the
// persistent k_track resolves queued segments, refilling a lane as soon as its
// segment ends, and either ends the path's bounce (collision, dead path) or
// passes the path to the next round, which continues from the segment's far
// boundary.  The last round tracks inline.  Every segment draws from its own
// stream (purpose kPurposeMedium + j, j = medium boundaries met in the bounce)
// and the steps repeat the loop's operations, so the split changes no result.

// Reserves one slot per calling lane of a warp-aggregated counter.
__device__ __forceinline__ uint32_t warp_reserve(uint32_t* counter) {
  const unsigned m = __activemask();
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(m, base, leader);
  return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// A stream positioned at draw idx.
__device__ __forceinline__ RngStream rng_resume(uint32_t pixel, uint32_t seed, uint32_t sample, uint32_t bounce,
                                                uint32_t purpose, uint32_t idx) {
  RngStream r = rng_stream(pixel, seed, sample, bounce, purpose);
  r.idx = idx;
  if (idx & 3u) r.buf = philox4x32_10(u4(sample, bounce, idx >> 2, purpose), pixel, seed);
  return r;
}

template <bool kInline>
__device__ __forceinline__ void resolve_path(const RenderLaunch& L, uint32_t p, bool fresh, uint32_t* jobCounter) {
  const SceneView& S = L.scene;
  const float4 ro = L.st.rayO[p], rd = L.st.rayD[p];
  V3 o = xyz(ro), d = xyz(rd);
  int med = __float_as_int(ro.w);
  float tmax = rd.w;
  V3 T = xyz(L.st.T[p]);
  int j = 0;
  if (!fresh) {  // k_track passed the segment that ends at the pending boundary hit
    const float4 h = L.st.hit[p];
    const int mi = kMediumCodeBase - __float_as_int(h.w);
    const Ray nr = ray_offset(make_ray(o + d * h.x, normalize(d), kDefaultTmax), d);
    o = nr.o;
    d = nr.d;
    tmax = nr.tmax;
    med = med < 0 ? mi : -1;
    j = (int)L.st.pj[p] + 1;
  }
  float4 hr = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(kEventDead));
  int err = 0;
  for (; j < kMaxPassThrough; ++j) {
    hr = scene_closest<true>(S, o, d, tmax);
    const int c = __float_as_int(hr.w);
    MediumEvent ev;
    ev.hit = 0;
    int evMed = -1;
    bool dead = false;
    if (c <= kMediumCodeBase) {
      const int mi = kMediumCodeBase - c;
      Ray seg = make_ray(o, d, hr.x);
      int segMed = -1;
      if (med >= 0) {  // origin inside a medium: track to the hit
        if (mi != med) dead = true;
        else segMed = med;
      } else {  // entering: find the far side, track through
        const Ray mr = ray_offset(make_ray(o + d * hr.x, normalize(d), kDefaultTmax), d);
        const float4 he = scene_closest<true>(S, mr.o, mr.d, mr.tmax);
        const int ce = __float_as_int(he.w);
        if (ce != -1) {
          if (ce <= kMediumCodeBase && kMediumCodeBase - ce != mi) {
            dead = true;
          } else {
            seg = make_ray(mr.o, mr.d, he.x);
            segMed = mi;
          }
        }
      }
      if (segMed >= 0) {
        if (kInline) {
          RngStream rs = rng_stream(path_pixel(L, p), L.seed, path_sample(L, p), L.bounce,
                                    kPurposeMedium + (uint32_t)j);
          T = T * instance_sample(S.media[segMed], seg, L.dda != 0, rs, &ev, &err, (int)L.trackLimit);
          evMed = segMed;
          if (err) dead = true;
        } else {  // queue the segment; the path waits at this boundary hit
          const uint32_t k = warp_reserve(jobCounter);
          L.st.jO[k] = f4(seg.o, seg.tmax);
          L.st.jD[k] = f4(seg.d, __int_as_float(segMed));
          L.st.jM[k] = make_uint2(p, (uint32_t)j);
          L.st.rayO[p] = f4(o, __int_as_float(med));
          L.st.rayD[p] = f4(d, tmax);
          L.st.hit[p] = hr;
          L.st.pj[p] = (uint32_t)j;
          return;
        }
      }
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

// Round `round` of path extension: round 0 takes the bounce's live paths,
// later rounds the paths k_track passed; kInline tracks instead of queueing.
template <bool kFirst, bool kInline>
__global__ void __launch_bounds__(128) k_resolve(RenderLaunch L, int round) {
  uint32_t* mc = L.st.mc + kCountersPerBounce * L.bounce;
  const uint32_t n = kFirst ? *(volatile uint32_t*)&L.st.counts[L.bounce] : *(volatile uint32_t*)&mc[3 * (round - 1) + 2];
  const uint32_t* list = kFirst ? path_queue(L, L.bounce) : pick(L.st.rl, (uint32_t)(round - 1) & 1u);
  uint32_t* jobs = &mc[3 * round];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) resolve_path<kInline>(L, list[i], kFirst, jobs);
}

// End of a tracked path segment without a collision: a pass (or an error).
__device__ __forceinline__ void finish_pass(const RenderLaunch& L, uint32_t p, int st, uint32_t* nextCount,
                                            uint32_t* nextList) {
  const V3 T = xyz(L.st.T[p]);
  bool dead = false;
  if (st == kTrackError) {
    atomicAdd(L.bound, 1u);
    dead = true;
  }
  if (!dead && (T.x == 0.0f || T.y == 0.0f || T.z == 0.0f)) dead = true;
  if (dead) {
    float4 h = L.st.hit[p];
    h.w = __int_as_float(kEventDead);
    L.st.hit[p] = h;
  } else {
    nextList[warp_reserve(nextCount)] = p;
  }
}

// A collision: the tracking-space ray and parameter are parked in evA/evB and
// the path joins the collision list that k_collide resolves.
__device__ __forceinline__ void finish_collide(const RenderLaunch& L, uint32_t p, int med, const TrackState& s) {
  uint32_t* mc = L.st.mc + kCountersPerBounce * L.bounce;
  L.st.evA[p] = f4(s.o, s.t);
  L.st.evB[p] = f4(s.d, __int_as_float(med));
  L.st.cl[warp_reserve(&mc[kCollideCounter])] = p;
}

// Collision events of the bounce's queued segments (sampleInternal /
// sampleDDA on acceptance), the albedo weight, and the dead-path rule.
template <bool kDDA>
__global__ void __launch_bounds__(128) k_collide(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.mc[kCountersPerBounce * L.bounce + kCollideCounter];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t p = L.st.cl[i];
    const float4 a = L.st.evA[p], b = L.st.evB[p];
    const int med = __float_as_int(b.w);
    MediumEvent ev;
    const V3 albedo = track_collision<kDDA>(L.scene.media[med], xyz(a), xyz(b), a.w, &ev);
    const V3 T = xyz(L.st.T[p]) * albedo;
    L.st.T[p] = f4(T, 0.0f);
    float4 h = L.st.hit[p];
    if (T.x == 0.0f || T.y == 0.0f || T.z == 0.0f) {
      h.w = __int_as_float(kEventDead);
    } else {
      L.st.evA[p] = f4(ev.pos, ev.ior);
      L.st.evB[p] = f4(ev.normal, __int_as_float(med));
      L.st.evC[p] = make_float4(ev.S[0], ev.S[1], ev.S[2], ev.S[3]);
      L.st.evD[p] = make_float2(ev.S[4], ev.S[5]);
      h.w = __int_as_float(kEventScatter);
    }
    L.st.hit[p] = h;
  }
}

// End of a tracked shadow segment: the walk's transmittance absorbs it.
__device__ __forceinline__ void finish_tr(const RenderLaunch& L, uint32_t slot, int st, const TrackState& s,
                                          uint32_t* nextCount, uint32_t* nextList) {
  if (st == kTrackError) {
    atomicAdd(L.bound, 1u);
    L.st.shTr[slot] = 0.0f;
    return;
  }
  const float4 w = L.st.swP[slot];
  const float tr = w.w * s.tr;
  if (tr == 0.0f) {
    L.st.shTr[slot] = 0.0f;
    return;
  }
  L.st.swP[slot] = make_float4(w.x, w.y, w.z, tr);
  L.st.swM[slot] = make_int2(L.st.swM[slot].x, (int)s.rng.idx);
  nextList[warp_reserve(nextCount)] = slot;
}

// Persistent tracking of the queued segments of round `round`: every lane
// holds one segment, advances it L.trackSteps steps at a time, and takes the
// next queued segment as soon as its own ends.  With the brick-grid DDA a
// lane that reaches a tentative collision holds it (pending) while the other
// lanes keep stepping across majorant cells, and the pending collisions are
// tested together once they are at least half of the warp's running lanes:
// the test (Philox draws, indirection and atlas lookups) is the long branch
// of a step, and divergent tests left most lanes idle.
template <bool kDDA, bool kSample>
__global__ void __launch_bounds__(128) k_track(RenderLaunch L, int round) {
  uint32_t* mc = L.st.mc + kCountersPerBounce * L.bounce + (kSample ? 0 : kShadowCounters);
  const uint32_t njobs = *(volatile uint32_t*)&mc[3 * round];
  uint32_t* taken = &mc[3 * round + 1];
  uint32_t* nextCount = &mc[3 * round + 2];
  uint32_t* nextList = kSample ? pick(L.st.rl, (uint32_t)round & 1u) : pick(L.st.sl, (uint32_t)round & 1u);
  const int lane = threadIdx.x & 31;
  TrackState s;
  uint32_t owner = 0;
  int med = 0;
  bool active = false, drained = false, pending = false;
  for (;;) {
    const bool need = !active && !drained;
    const unsigned want = __ballot_sync(0xffffffffu, need);
    if (want) {
      const int leader = __ffs(want) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(taken, (uint32_t)__popc(want));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (base + (uint32_t)__popc(want) >= njobs) drained = true;  // warp-uniform
      if (need) {
        const uint32_t k = base + (uint32_t)__popc(want & ((1u << lane) - 1u));
        if (k < njobs) {
          const float4 jo = L.st.jO[k], jd = L.st.jD[k];
          const uint2 jm = L.st.jM[k];
          owner = jm.x;
          med = __float_as_int(jd.w);
          if (kSample) {
            s.rng = rng_stream(path_pixel(L, owner), L.seed, path_sample(L, owner), L.bounce, kPurposeMedium + jm.y);
          } else {
            const uint32_t op = event_path(L, owner >> 1);
            s.rng = rng_resume(path_pixel(L, op), L.seed, path_sample(L, op), L.bounce,
                               kPurposeShadowTr + (owner & 1u), jm.y);
          }
          const int st = track_init<kDDA, kSample>(L.scene.media[med], make_ray(xyz(jo), xyz(jd), jo.w), &s,
                                                     (int)L.trackLimit);
          if (st == kTrackRunning) {
            active = true;
          } else if (kSample) {
            finish_pass(L, owner, st, nextCount, nextList);
          } else {
            finish_tr(L, owner, st, s, nextCount, nextList);
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (drained) break;
      continue;
    }
    if (kDDA) {
      for (uint32_t k = 0; k < L.trackSteps; ++k) {
        if (!__any_sync(0xffffffffu, active)) break;
        int st = kTrackRunning;
        if (active && !pending) {
          st = track_dda_advance<kSample>(L.scene.media[med], s);
          if (st == kTrackPending) {
            pending = true;
            st = kTrackRunning;
          }
        }
        const unsigned held = __ballot_sync(0xffffffffu, pending);
        const unsigned running = __ballot_sync(0xffffffffu, active && st == kTrackRunning);
        if (held && 2 * __popc(held) >= __popc(running) && pending) {
          st = track_dda_collide<kSample>(L.scene.media[med], s);
          pending = false;
        }
        if (active && st != kTrackRunning) {
          if (kSample && st == kTrackCollide) finish_collide(L, owner, med, s);
          else if (kSample) finish_pass(L, owner, st, nextCount, nextList);
          else finish_tr(L, owner, st, s, nextCount, nextList);
          active = false;
        }
      }
    } else {
      for (uint32_t k = 0; k < L.trackSteps && active; ++k) {
        const int st = track_step<kDDA, kSample>(L.scene.media[med], s);
        if (st != kTrackRunning) {
          if (kSample && st == kTrackCollide) finish_collide(L, owner, med, s);
          else if (kSample) finish_pass(L, owner, st, nextCount, nextList);
          else finish_tr(L, owner, st, s, nextCount, nextList);
          active = false;
        }
      }
    }
  }
}

// Surface shading: direct() at a surface and the sampleF continuation
// (path_integrator_impl.hpp:23-118, 196-222).
// kTex: the scene has texture coordinates; kInst: two levels (otherwise those
// branches are compiled out of the instantiation).
template <bool kMedia, bool kTex, bool kInst>
__device__ __forceinline__ bool shade_surface(const RenderLaunch& L, uint32_t i, uint32_t p, int code, float4 hr,
                                              V3 o, V3 d, int med, V3 T) {
  const V3 pos = o + d * hr.x;
  V3 n;
  Material m;
  if (code >= 0) {
    int tri = code, inst = -1;
    if (kInst && L.scene.bvh.inst) {  // the instance of the code, and the triangle's BVH-order index
      int lo = 0, hi = L.scene.ninst - 1;
      while (lo < hi) {  // last instance whose first code is <= code
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&L.scene.instCode[mid]) <= code) lo = mid; else hi = mid - 1;
      }
      inst = lo;
      tri = code - __ldg(&L.scene.bvh.inst[inst].vdelta);
      if (__ldg(&L.scene.bvh.inst[inst].identity)) inst = -1;
    }
    const float4 n0 = __ldg(&L.scene.triN[3 * tri]);
    const float4 n1 = __ldg(&L.scene.triN[3 * tri + 1]);
    const float4 n2 = __ldg(&L.scene.triN[3 * tri + 2]);
    const float b0 = (1.0f - hr.y) - hr.z;
    n = normalize(xyz(n0) * b0 + xyz(n1) * hr.y + xyz(n2) * hr.z);
    m = L.scene.mats[__ldg(&L.scene.triMat[tri])];
    if (kTex && L.scene.triUV && (m.tex[0] >= 0 || m.tex[1] >= 0 || m.tex[2] >= 0)) {
      const TexView tv = {L.scene.triUV, L.scene.texels, L.scene.texInfo, L.scene.bvh.tris};
      const TexShade ts = textured_surface(tv, m.tex[0], m.tex[1], m.tex[2], tri, hr.y, hr.z, n, m.diffuse, m.specular);
      n = ts.n;
      m.diffuse = ts.diffuse;
      m.specular = ts.specular;
    }
    if (inst >= 0) {  // __closesthit__ch: normalize(modelToWorld * vec4(n, 0)) in glm's column order
      const float4 r0 = __ldg(&L.scene.instO2W[3 * inst]), r1 = __ldg(&L.scene.instO2W[3 * inst + 1]);
      const float4 r2 = __ldg(&L.scene.instO2W[3 * inst + 2]);
      n = normalize(v3(r0.x * n.x + r0.y * n.y + r0.z * n.z + r0.w * 0.0f,
                       r1.x * n.x + r1.y * n.y + r1.z * n.z + r1.w * 0.0f,
                       r2.x * n.x + r2.y * n.y + r2.z * n.z + r2.w * 0.0f));
    }
  } else {
    const Shape& sh = L.scene.shapes[-2 - code];
    // __closesthit__ch normalises the reported shape normal (shaders.optix.cu:110-114)
    n = sh.type == kShapeCircle ? normalize(sh.normal) : normalize(pos - sh.center);
    m = L.scene.mats[sh.material];
  }
  const uint32_t pix = path_pixel(L, p), smp = path_sample(L, p);
  const U4 rA = philox_nc(u4(smp, L.bounce, 0u, 1u), pix, L.seed);
  const U4 rB = philox_nc(u4(smp, L.bounce, 1u, 1u), pix, L.seed);
  const Frame fr = frame_from_normal(n);
  const V3 wo = -d;
  const V3 woT = to_local(fr, wo);
  const V3 offO = offset_ray_origin(pos, n);
  float4 shO0 = make_float4(0, 0, 0, 0), shO1 = shO0, shD0 = shO0, shD1 = shO0, pre0 = shO0, pre1 = shO0;
  // --- direct(): light sample (path_integrator_impl.hpp:31-71)
  {
    const EnvSample es = env_sample_nc(L.scene.env, u01(rA.x), u01(rA.y));
    const V3 Le = es.Le;
    const float lpdf = es.pdf;
    if (lpdf > 0.0f) {
      const V3 ldir = normalize(es.dir);
      const V3 lT = normalize(to_local(fr, ldir));
      const BsdfEval be = bsdf_eval_nc(m, woT, lT);
      const V3 f = be.f * fabsf(dot(n, ldir));
      const float spdf = be.pdf;
      const float mis = balance_heuristic(lpdf, spdf);
      // offsetRayOrigin(n) of the ray (pos, ldir, DEFAULT_TMAX): origin offO, end point kept
      const float t1 = length((pos + ldir * kDefaultTmax) - offO);
      shO0 = f4(offO, lpdf);
      shD0 = f4(ldir, t1);  // intersectTr walks towards offO + ldir * t1
      pre0 = f4((f * mis) * Le, 0.0f);
      if (kMedia) L.st.shX[2 * i] = make_float2(t1, __int_as_float(med));
    }
  }
  // --- direct(): BSDF sample (path_integrator_impl.hpp:74-113)
  {
    const BsdfSample bs = bsdf_sample_nc(m, woT, u01(rA.z), u01(rA.w), u01(rB.x));
    const float spdf = bs.pdf;
    V3 wi = normalize(to_world(fr, bs.wi));
    const V3 f = bs.f * fabsf(dot(n, wi));
    if (spdf > 0.0f) {
      wi = normalize(wi);
      const EnvEval ee = env_le_nc(L.scene.env, wi);
      const V3 Le = ee.Le;
      const float lpdf = ee.pdf;
      const float mis = balance_heuristic(spdf, lpdf);
      const float t1 = length((pos + wi * kDefaultTmax) - offO);
      shO1 = f4(offO, spdf);
      shD1 = f4(wi, t1);
      pre1 = f4((f * mis) * Le, 0.0f);
      if (kMedia) L.st.shX[2 * i + 1] = make_float2(t1, __int_as_float(med));
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
  // CRay::transform(worldToTangent) widens the matrix to mat4x3 with a zero
  // fourth column: the direction gains a + 0 term (-0 becomes +0).
  const V3 dT = normalize(to_local(fr, d) + v3(0.0f));
  const BsdfSample cs = bsdf_sample_nc(m, -dT, u01(rB.y), u01(rB.z), u01(rB.w));
  const V3 wi = cs.wi, f = cs.f;
  const float pdf = cs.pdf;
  if (pdf == 0.0f) return false;
  const V3 dirW = normalize(to_world(fr, wi));
  const float cosine = fabsf(dot(n, dirW));
  V3 Tn = T * ((f * cosine) / pdf);
  if (L.bounce > 3) {
    const U4 rC = philox_nc(u4(smp, L.bounce, 2u, 1u), pix, L.seed);
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
  RngStream rs = rng_stream(path_pixel(L, p), L.seed, path_sample(L, p), L.bounce, kPurposeScatter);
  float4 shO0 = make_float4(0, 0, 0, 0), shO1 = shO0, shD0 = shO0, shD1 = shO0, pre0 = shO0, pre1 = shO0;
  {
    const float u0 = rs.next();
    const float u1 = rs.next();
    const EnvSample es = env_sample_nc(L.scene.env, u0, u1);
    const V3 Le = es.Le;
    const float lpdf = es.pdf;
    if (lpdf > 0.0f) {
      const V3 ldir = normalize(es.dir);
      const Ray lr = voxel_border_nc(&M, ray_offset(make_ray(pos, ldir, kDefaultTmax), n));
      const PhaseEval pe = phase_eval_nc(&M, g, ior, wo, ldir, rs);
      rs = pe.rs;
      const float sp = pe.p;
      const float mis = balance_heuristic(lpdf, sp);
      shO0 = f4(lr.o, lpdf);
      shD0 = f4(lr.d, 0.0f);
      L.st.shX[2 * i] = make_float2(lr.tmax, __int_as_float(med));
      pre0 = f4((v3(sp) * mis) * Le, 0.0f);
    }
  }
  {
    const PhaseSample ps = phase_sample_nc(&M, g, ior, wo, rs);
    rs = ps.rs;
    const float sp = ps.p;
    if (sp > 0.0f) {
      const V3 wi = normalize(ps.wi);
      const Ray br = voxel_border_nc(&M, ray_offset(make_ray(pos, wi, kDefaultTmax), n));
      const EnvEval ee = env_le_nc(L.scene.env, wi);
      const V3 Le = ee.Le;
      const float lpdf = ee.pdf;
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
  const V3 wi = phase_sample_nc(&M, g, ior, wo, rs).wi;
  const Ray cr = voxel_border_nc(&M, ray_offset(make_ray(pos, normalize(wi), kDefaultTmax), wi));
  V3 Tn = T;
  if (L.bounce > 3) {
    const U4 rC = philox_nc(u4(path_sample(L, p), L.bounce, 2u, 1u), path_pixel(L, p), L.seed);
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

// Media scenes: sorts the bounce's outcomes after the extension phase.  A miss
// ends the path with the environment term of the first bounce (the
// reference's miss rule, path_integrator_impl.hpp:176-182), a path ended by a
// medium rule is dropped, surface hits and medium collisions go to their own
// queues, so that shading runs over coherent warps of one kind of event.
__global__ void __launch_bounds__(256) k_events(RenderLaunch L) {
  const uint32_t n = *(volatile uint32_t*)&L.st.counts[L.bounce];
  const uint32_t* q = path_queue(L, L.bounce);
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t nRound = (n + 31u) & ~31u;  // whole warps reach the pushes
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nRound; i += stride) {
    int code = kEventDead;
    uint32_t p = 0;
    if (i < n) {
      p = q[i];
      code = __float_as_int(L.st.hit[p].w);
      if (code == -1 && L.bounce == 0) {
        const V3 le = env_le_nc(L.scene.env, xyz(L.st.rayD[p])).Le;
        L.st.L[p] = f4(xyz(L.st.L[p]) + le * xyz(L.st.T[p]), 0.0f);
      }
    }
    push_queue(L.st.qs, &L.st.counts[kScatterCounters + L.bounce], code == kEventScatter, p);
    push_queue(L.st.qh, &L.st.counts[kHitCounters + L.bounce], code != -1 && code != kEventDead && code != kEventScatter,
               p);
  }
}

// Register caps (64 a thread without media): the few spilled values of the
// rare branches cost less than the warps gained (16-sample wave of the
// 327,680-triangle scene: shading 5.8 -> 4.7 ms).
template <bool kMedia, bool kTex, bool kInst>
__global__ void __launch_bounds__(128, kMedia ? 6 : 8) k_shade(RenderLaunch L) {
  // the bounce's events: misses and ended paths were finished by k_extend / k_events
  const uint32_t n = event_count(L);
  uint32_t* qn = path_queue(L, L.bounce + 1);
  uint32_t* cn = &L.st.counts[L.bounce + 1];
  const uint32_t stride = gridDim.x * blockDim.x;
  // uniform trip count per warp so the ballot below sees the whole warp
  const uint32_t nRound = (n + 31u) & ~31u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nRound; i += stride) {
    bool cont = false;
    uint32_t p = 0;
    if (i < n) {
      p = event_path(L, i);
      const float4 hr = L.st.hit[p];
      const int code = __float_as_int(hr.w);
      const float4 ro = L.st.rayO[p];
      const V3 o = xyz(ro), d = xyz(L.st.rayD[p]);
      const V3 T = xyz(L.st.T[p]);
      if (code == -1 || code == kEventDead) {
        if (code == -1 && L.bounce == 0) {
          const V3 le = env_le_nc(L.scene.env, d).Le;
          L.st.L[p] = f4(xyz(L.st.L[p]) + le * T, 0.0f);
        }
        const float4 z = make_float4(0, 0, 0, 0);
        L.st.shO[2 * i] = z;
        L.st.shO[2 * i + 1] = z;
      } else if (kMedia && code == kEventScatter) {
        cont = shade_scatter(L, i, p, d, T);
      } else {
        cont = shade_surface<kMedia, kTex, kInst>(L, i, p, code, hr, o, d, __float_as_int(ro.w), T);
      }
    }
    push_queue(qn, cn, cont, p);
  }
}

// The first segment of CDeviceScene::intersectTr for a shadow record: the
// record holds the normal-offset origin o and direction d with the offset
// ray's length t1, and intersectTr traces CRay::spawnRay(o, o + d * t1).
__device__ __forceinline__ Ray shadow_ray(float4 o, float4 d) {
  const V3 p0 = xyz(o);
  return spawn_ray(p0, p0 + xyz(d) * d.w);
}

// Visibility of every shadow record of a scene without media.
template <bool kTris, bool kAlpha, bool kInst, bool kTop>
__global__ void __launch_bounds__(128, 10) k_shadow_surfaces(RenderLaunch L) {
  const uint32_t n = event_count(L);
  uint32_t traced = 0;
  if constexpr (!kTris) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < 2 * n; j += stride) {
      const float4 o = L.st.shO[j];
      float tr = 0.0f;
      if (o.w > 0.0f) {
        const Ray r = shadow_ray(o, L.st.shD[j]);
        tr = scene_occluded(L.scene, r.o, r.d, r.tmax) ? 0.0f : 1.0f;
        ++traced;
      }
      L.st.shTr[j] = tr;
    }
  } else {
    auto begin = [&](uint32_t j, TraceState& s, uint32_t* item) {
      const float4 o = L.st.shO[j];
      *item = j;
      if (!(o.w > 0.0f)) {  // no ray for this record
        L.st.shTr[j] = 0.0f;
        return false;
      }
      ++traced;
      const Ray r = shadow_ray(o, L.st.shD[j]);
      trace_begin(s, r.o, r.d, r.tmax);
      return true;
    };
    auto end = [&](uint32_t j, const TraceState& s) {
      bool occluded = s.best.tri >= 0;
      if (!occluded && L.scene.nshapes > 0) {
        SceneView noTris = L.scene;
        noTris.hasTris = 0;
        Hit none;
        none.tri = -1;
        occluded = __float_as_int(scene_closest_after<false>(noTris, s.wo, s.wd, s.best.t, none).w) != -1;
      }
      L.st.shTr[j] = occluded ? 0.0f : 1.0f;
    };
    trace_scene<true, kAlpha, kInst, kTop>(L, 2 * n, &L.st.counts[kTravCounters + 2 * L.bounce + 1], begin, end);
  }
  if (L.stats) {
    for (int o = 16; o > 0; o >>= 1) traced += __shfl_down_sync(0xffffffffu, traced, o);
    if ((threadIdx.x & 31) == 0 && traced) atomicAdd(&L.stats[1], (unsigned long long)traced);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&L.stats[0], (unsigned long long)L.st.counts[L.bounce]);
  }
}

// ------------------------------------------------------------------ media: shadow transmittance
// CDeviceScene::intersectTr as direct() uses it: 0 when the walk ends on a
// surface (materials do not emit), else the product of the media's
// ratio-tracking estimates.  A surface anywhere on the ray ends the walk there,
// so the any-hit test decides that case; without one the walk visits only
// medium boxes, segment by segment through CRay::spawnRay towards the fixed
// far point p1, multiplying Tr when a segment leaves the current medium.  As
// for path extension, segments that need tracking are queued for k_track and
// the walk resumes after them; the last round tracks inline.  The slot's
// stream (purpose kPurposeShadowTr + slot parity) continues across segments.
template <bool kInline>
__device__ __forceinline__ void shadow_walk(const RenderLaunch& L, uint32_t slot, bool fresh, uint32_t* jobCounter) {
  const SceneView& S = L.scene;
  const float4 o4 = L.st.shO[slot], d4 = L.st.shD[slot];
  const float2 x = L.st.shX[slot];
  const V3 o = xyz(o4), d = xyz(d4);
  V3 p0;
  int cur;
  float tr;
  uint32_t idx;
  if (fresh) {
    const Ray r0 = spawn_ray(o, o + d * x.x);
    if (scene_occluded(S, r0.o, r0.d, r0.tmax)) {
      L.st.shTr[slot] = 0.0f;
      return;
    }
    p0 = o;
    cur = __float_as_int(x.y);
    tr = 1.0f;
    idx = 0;
  } else {
    const float4 w = L.st.swP[slot];
    const int2 m = L.st.swM[slot];
    p0 = xyz(w);
    tr = w.w;
    cur = m.x;
    idx = (uint32_t)m.y;
  }
  const V3 p1 = o + d * x.x;
  RngStream rs;
  if (kInline) {
    const uint32_t op = event_path(L, slot >> 1);
    rs = rng_resume(path_pixel(L, op), L.seed, path_sample(L, op), L.bounce, kPurposeShadowTr + (slot & 1u), idx);
  }
  int err = 0;
  for (int k = 0; k < kMaxShadowSegments; ++k) {
    const V3 off = offset_ray_origin(p0, normalize(p1 - p0));
    const float tl = length(p1 - off);
    const V3 dir = (p1 - p0) / tl;
    float best;
    int hitM = media_first(S, off, dir, tl, &best);
    if (hitM >= 0 && !(best < tl)) hitM = -1;
    if (hitM < 0) {
      L.st.shTr[slot] = tr;
      if (err) atomicAdd(L.bound, 1u);
      return;
    }
    if (cur >= 0 && hitM == cur) {
      if (kInline) {
        tr *= instance_tr(S.media[cur], make_ray(off, dir, best), L.dda != 0, rs, &err, (int)L.trackLimit);
      } else {
        const uint32_t k2 = warp_reserve(jobCounter);
        L.st.jO[k2] = f4(off, best);
        L.st.jD[k2] = f4(dir, __int_as_float(cur));
        L.st.jM[k2] = make_uint2(slot, idx);
        L.st.swP[slot] = f4(off + dir * best, tr);
        L.st.swM[slot] = make_int2(-1, (int)idx);
        return;
      }
    }
    p0 = off + dir * best;
    cur = cur < 0 ? hitM : -1;
  }
  atomicAdd(L.bound, 1u);
  L.st.shTr[slot] = 0.0f;
}

template <bool kFirst, bool kInline>
__global__ void __launch_bounds__(128) k_shadow_resolve(RenderLaunch L, int round) {
  uint32_t* mc = L.st.mc + kCountersPerBounce * L.bounce + kShadowCounters;
  const uint32_t n = kFirst ? 2 * event_count(L) : *(volatile uint32_t*)&mc[3 * (round - 1) + 2];
  const uint32_t* list = kFirst ? nullptr : pick(L.st.sl, (uint32_t)(round - 1) & 1u);
  uint32_t* jobs = &mc[3 * round];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t slot = kFirst ? i : list[i];
    if (kFirst) {
      const bool traced = L.st.shO[slot].w > 0.0f;
      if (L.stats) {
        const unsigned m = __ballot_sync(__activemask(), traced);
        if ((threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1) && m)
          atomicAdd(&L.stats[1], (unsigned long long)__popc(m));
      }
      if (!traced) {
        L.st.shTr[slot] = 0.0f;
        continue;
      }
    }
    shadow_walk<kInline>(L, slot, kFirst, jobs);
  }
  if (kFirst && L.stats && blockIdx.x == 0 && threadIdx.x == 0)
    atomicAdd(&L.stats[0], (unsigned long long)L.st.counts[L.bounce]);
}

__global__ void __launch_bounds__(256) k_accum(RenderLaunch L) {
  const uint32_t n = event_count(L);  // the shadow records of the bounce's events
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float4 o0 = L.st.shO[2 * i], o1 = L.st.shO[2 * i + 1];
    if (!(o0.w > 0.0f) && !(o1.w > 0.0f)) continue;
    const uint32_t p = event_path(L, i);
    V3 dl = v3(0.0f);
    if (o0.w > 0.0f) dl = dl + (xyz(L.st.shPre[2 * i]) * L.st.shTr[2 * i]) / o0.w;
    if (o1.w > 0.0f) dl = dl + (xyz(L.st.shPre[2 * i + 1]) * L.st.shTr[2 * i + 1]) / o1.w;
    const V3 Lp = xyz(L.st.L[p]);
    L.st.L[p] = f4(Lp + dl * xyz(L.st.shT[i]), 0.0f);
  }
}

// Adds the wave's samples to the frame pixel by pixel in sample order, the
// same additions as one wave per sample.
__global__ void __launch_bounds__(256) k_finish(RenderLaunch L) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < L.npix; p += stride) {
    float fx = L.frame[3 * p], fy = L.frame[3 * p + 1], fz = L.frame[3 * p + 2];
    for (uint32_t k = 0; k < L.waveSpp; ++k) {
      V3 v = xyz(L.st.L[p + k * L.npix]);
      if (isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z)) v = v3(0.0f);
      else v = v / (float)L.spp;
      fx += v.x;
      fy += v.y;
      fz += v.z;
    }
    L.frame[3 * p] = fx;
    L.frame[3 * p + 1] = fy;
    L.frame[3 * p + 2] = fz;
  }
}

template <typename K>
int resident_blocks(K kernel, int threads, size_t smem = 0) {
  int n = 0;
  R2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem));
  return std::max(1, n) * sm_count();
}

int g_trackBlocks[4] = {0, 0, 0, 0};  // resident blocks of k_track<dda, sample>, by dda + 2 sample

int g_travBlocks[2] = {0, 0};  // resident blocks of k_extend, k_shadow_surfaces

// The surface traversal kernels by variant: alpha + 2 * two-level + 4 * top
// nodes; 8: a scene without triangles.
using RenderKernel = void (*)(RenderLaunch);
const RenderKernel kExtendVariants[9] = {
    k_extend<true, false, false, false>, k_extend<true, true, false, false>, k_extend<true, false, true, false>,
    k_extend<true, true, true, false>,   k_extend<true, false, false, true>, k_extend<true, true, false, true>,
    k_extend<true, false, true, true>,   k_extend<true, true, true, true>,   k_extend<false, false, false, false>};
const RenderKernel kShadowVariants[9] = {
    k_shadow_surfaces<true, false, false, false>, k_shadow_surfaces<true, true, false, false>,
    k_shadow_surfaces<true, false, true, false>,  k_shadow_surfaces<true, true, true, false>,
    k_shadow_surfaces<true, false, false, true>,  k_shadow_surfaces<true, true, false, true>,
    k_shadow_surfaces<true, false, true, true>,   k_shadow_surfaces<true, true, true, true>,
    k_shadow_surfaces<false, false, false, false>};

// k_shade by variant: 4 * media + textured + 2 * two-level.
const RenderKernel kShadeVariants[8] = {k_shade<false, false, false>, k_shade<false, true, false>,
                                        k_shade<false, false, true>,  k_shade<false, true, true>,
                                        k_shade<true, false, false>,  k_shade<true, true, false>,
                                        k_shade<true, false, true>,   k_shade<true, true, true>};

int shade_variant(const RenderLaunch& L) {
  return (L.scene.triUV ? 1 : 0) + (L.scene.bvh.inst ? 2 : 0);
}

int trav_variant(const RenderLaunch& L) {
  if (!L.scene.hasTris) return 8;
  return (L.scene.bvh.alpha.alphaTex ? 1 : 0) + (L.scene.bvh.inst ? 2 : 0) + (L.topNodes ? 4 : 0);
}

// Resident blocks of a surface traversal kernel (0: k_extend, 1:
// k_shadow_surfaces) of a variant with topNodes BVH nodes of dynamic shared memory.
int trav_blocks(int which, int variant, uint32_t topNodes) {
  static std::mutex mu;
  static std::map<std::pair<int, uint32_t>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const int key = which * 9 + variant;
  auto it = cache.find({key, topNodes});
  if (it != cache.end()) return it->second;
  const size_t smem = topNodes * sizeof(BvhNode);
  const RenderKernel k = which == 0 ? kExtendVariants[variant] : kShadowVariants[variant];
  const int n = resident_blocks(k, 128, smem);
  cache[{key, topNodes}] = n;
  return n;
}

void query_track_blocks() {
  if (g_trackBlocks[0] != 0) return;
  g_travBlocks[0] = resident_blocks(kExtendVariants[0], 128);
  g_travBlocks[1] = resident_blocks(kShadowVariants[0], 128);
  g_trackBlocks[1] = resident_blocks(k_track<true, false>, 128);
  g_trackBlocks[2] = resident_blocks(k_track<false, true>, 128);
  g_trackBlocks[3] = resident_blocks(k_track<true, true>, 128);
  g_trackBlocks[0] = resident_blocks(k_track<false, false>, 128);
}

__global__ void k_advance_sample(uint32_t* sample, uint32_t n) { *sample += n; }

void launch_track(const RenderLaunch& L, bool sample, int round, cudaStream_t s) {
  query_track_blocks();
  const int which = (L.dda ? 1 : 0) + (sample ? 2 : 0);
  // all resident blocks, or L.trackBlocks per SM (fewer warps per SM can
  // reuse L1 better: a tuning choice)
  int b[4];
  for (int i = 0; i < 4; ++i)
    b[i] = L.trackBlocks ? std::max(1, std::min(g_trackBlocks[i], (int)L.trackBlocks * sm_count())) : g_trackBlocks[i];
  switch (which) {
    case 0: k_track<false, false><<<b[0], 128, 0, s>>>(L, round); break;
    case 1: k_track<true, false><<<b[1], 128, 0, s>>>(L, round); break;
    case 2: k_track<false, true><<<b[2], 128, 0, s>>>(L, round); break;
    default: k_track<true, true><<<b[3], 128, 0, s>>>(L, round); break;
  }
}

}  // namespace

void launch_render_wave(const RenderLaunch& L0, int nblocks, cudaStream_t s, WaveTimer* tm) {
  RenderLaunch L = L0;
  if (L.trackSteps == 0) L.trackSteps = kDefaultTrackSteps;
  if (L.travVisits == 0) L.travVisits = kDefaultTravVisits;
  if (L.travRefill == 0) L.travRefill = kDefaultTravRefill;
  if (L.mediaRounds == 0) L.mediaRounds = kDefaultMediaRounds;
  const int rounds = (int)std::min<uint32_t>(L.mediaRounds, kMaxMediaRounds);
  query_track_blocks();
  const bool media = L.scene.nmedia > 0;
  int ev = 0;
  auto mark = [&](int kind) {
    if (!tm) return;
    R2_CUDA(cudaEventRecord(tm->ev[ev], s));
    tm->kind[ev] = kind;
    ++ev;
  };
  R2_CUDA(cudaMemsetAsync(L.st.counts, 0, sizeof(uint32_t) * kCountsSize, s));
  if (media) R2_CUDA(cudaMemsetAsync(L.st.mc, 0, sizeof(uint32_t) * kCountersPerBounce * L.maxDepth, s));
  mark(-1);
  k_camera<<<nblocks, 256, 0, s>>>(L);
  mark(0);
  for (uint32_t b = 0; b < L.maxDepth; ++b) {
    L.bounce = b;
    if (media) {
      k_resolve<true, false><<<nblocks * 2, 128, 0, s>>>(L, 0);
      for (int r = 0; r < rounds; ++r) {
        launch_track(L, true, r, s);
        if (r + 1 < rounds) k_resolve<false, false><<<nblocks * 2, 128, 0, s>>>(L, r + 1);
        else k_resolve<false, true><<<nblocks * 2, 128, 0, s>>>(L, r + 1);
      }
      if (L.dda) k_collide<true><<<nblocks * 2, 128, 0, s>>>(L);
      else k_collide<false><<<nblocks * 2, 128, 0, s>>>(L);
      k_events<<<nblocks, 256, 0, s>>>(L);
      mark(1);
      kShadeVariants[4 + shade_variant(L)]<<<nblocks * 2, 128, 0, s>>>(L);
      mark(2);
      k_shadow_resolve<true, false><<<nblocks * 2, 128, 0, s>>>(L, 0);
      for (int r = 0; r < rounds; ++r) {
        launch_track(L, false, r, s);
        if (r + 1 < rounds) k_shadow_resolve<false, false><<<nblocks * 2, 128, 0, s>>>(L, r + 1);
        else k_shadow_resolve<false, true><<<nblocks * 2, 128, 0, s>>>(L, r + 1);
      }
    } else {
      if (L.sortRays && b > 0) {
        R2_CUDA(cudaMemsetAsync(L.st.sortBins, 0, 256 * sizeof(uint32_t), s));
        k_sort_hist<<<nblocks, 256, 0, s>>>(L);
        k_sort_scan<<<1, 256, 0, s>>>(L);
        k_sort_scatter<<<nblocks, 256, 0, s>>>(L);
        k_sort_copy<<<nblocks, 256, 0, s>>>(L);
      }
      const int tv = trav_variant(L);
      kExtendVariants[tv]<<<std::min(nblocks * 2, trav_blocks(0, tv, L.topNodes)), 128,
                            L.topNodes * sizeof(BvhNode), s>>>(L);
      mark(1);
      kShadeVariants[shade_variant(L)]<<<nblocks * 2, 128, 0, s>>>(L);
      mark(2);
      kShadowVariants[tv]<<<std::min(nblocks * 2, trav_blocks(1, tv, L.topNodes)), 128,
                            L.topNodes * sizeof(BvhNode), s>>>(L);
    }
    mark(3);
    k_accum<<<nblocks, 256, 0, s>>>(L);
    mark(4);
  }
  k_finish<<<nblocks, 256, 0, s>>>(L);
  mark(5);
  if (L.sampleDev) k_advance_sample<<<1, 1, 0, s>>>(L.sampleDev, L.waveSpp);
  if (tm) tm->n = ev;
  R2_CUDA(cudaGetLastError());
}

void prepare_render_launches() {
  query_track_blocks();
  sm_count();
}

}  // namespace r2
