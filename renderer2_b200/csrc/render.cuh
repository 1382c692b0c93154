// Wavefront path tracer: launch description shared by the kernels (render.cu)
// and the host runtime (render_host.cu).
#pragma once
#include "bvh_build.cuh"
#include "media.cuh"

namespace r2 {

// Analytic scene objects of the reference's scene description (Circle,
// Sphere; include/shapes/circle.hpp:35-60, sphere.hpp:33-90).
enum ShapeType : int { kShapeSphere = 0, kShapeCircle = 1 };

struct Shape {
  int type;
  int material;
  float radius;
  float pad;
  V3 center;
  V3 normal;
};

// Device view of a committed scene.
struct SceneView {
  BvhView bvh;
  const float4* triN;      // 3 per BVH-order triangle: world-space vertex normals
  const uint32_t* triMat;  // per BVH-order triangle: material index
  const Material* mats;
  const Shape* shapes;
  int nshapes;
  int hasTris;
  const MediumView* media;  // medium instances (device array), nullable
  int nmedia;
  const BvhNode* mediaNodes;    // BVH over the instances' world boxes (more than kMediaLinearMax), nullable
  const uint32_t* mediaOrder;   // BVH leaf position -> instance index
  EnvMap env;
  const float2* triUV;      // 3 texture coordinates per BVH-order triangle, nullable
  const float4* texels;     // texture maps of the materials (TexInfo offsets), nullable
  const TexInfo* texInfo;
  // two-level scenes (bvh.inst set): per instance the first hit code (ascending)
  // and the object-to-world 3x3 | translation rows that take its normals to world space
  const int* instCode;
  const float4* instO2W;
  int ninst;
};

// Per-path SoA state of one wave (one sample of every pixel).
struct PathState {
  float4* rayO;     // origin, .w = current medium index as int bits (-1: none)
  float4* rayD;     // direction, .w = ray tmax
  float4* T;        // throughput
  float4* L;        // radiance
  float4* hit;      // t, b1, b2, event code (int bits: >= 0 triangle, -1 miss, -2 - i shape i,
                    // kEventScatter medium collision, kEventDead path ended by a medium rule)
  uint32_t* q[2];   // ping-pong queues of live path ids
  uint32_t* qh;     // paths of the bounce that hit a surface (k_extend, or k_events with media)
  uint32_t* qs;     // media: paths of the bounce with a medium collision (k_events); surfaces: ray sort output
  uint32_t* sortBins;  // 256 key counters of the ray sort
  uint32_t* counts; // [bounce] live path count entering the bounce; from kTravCounters on,
                    // per bounce the rays taken by the persistent surface traversals
  // shadow records, two per queue slot (0: light sample, 1: BSDF sample)
  float4* shO;      // origin.xyz, pdf (0 = no ray)
  float4* shD;      // direction.xyz, unused
  float4* shPre;    // (mis * f) * Le
  float4* shT;      // throughput at the bounce (one per slot pair)
  float* shTr;      // transmittance of each shadow ray (0 or 1 without media)
  // media scenes only
  float2* shX;      // shadow ray tmax, medium index (int bits)
  float4* evA;      // collision position, ior
  float4* evB;      // collision normal, medium index (int bits)
  float4* evC;      // SGGX S xx yy zz xy
  float2* evD;      // SGGX S xz yz
  uint32_t* mc;     // per-bounce counters of the tracking rounds
  uint32_t* pj;     // per path: medium boundaries met in the bounce when its segment was queued
  float4* jO;       // queued segments: origin, tmax
  float4* jD;       //                  direction, medium (int bits)
  uint2* jM;        //                  owner (path or shadow slot), stream purpose / draw index
  uint32_t* rl[2];  // paths resumed in the next round (round r writes list r & 1)
  uint32_t* sl[2];  // shadow slots resumed in the next round
  uint32_t* cl;     // paths whose queued segment ended in a collision
  float4* swP;      // shadow walk: next origin, transmittance so far
  int2* swM;        // shadow walk: current medium, draw index of the slot's stream
};

// Most BVH nodes the surface traversals stage in shared memory (16 KB per block).
constexpr uint32_t kMaxTopNodes = 256;
// Launch tuning defaults (RenderLaunch::trackSteps, travVisits, travRefill);
// no result depends on them.
constexpr uint32_t kDefaultTrackSteps = 8;   // tracking steps a lane takes between refills
constexpr uint32_t kDefaultTravVisits = 32;  // BVH visits between refill checks
constexpr uint32_t kDefaultTravRefill = 8;   // finished lanes that trigger a refill
constexpr uint32_t kDefaultWavePaths = 1u << 22;  // paths per wave a frame's samples are grouped to
constexpr uint32_t kDefaultMediaRounds = 2;       // queued medium-boundary rounds per bounce
constexpr uint32_t kMaxMediaRounds = 32;
// Media counters of a bounce (PathState::mc): [3r] segments queued in round r,
// [3r+1] segments taken, [3r+2] entries of list r + 1; path extension from 0,
// shadow rays from kShadowCounters, then the collision list's entries.
constexpr int kShadowCounters = 3 * (kMaxMediaRounds + 1);
constexpr int kCollideCounter = 2 * kShadowCounters;
constexpr int kCountersPerBounce = (kCollideCounter + 4) & ~3;

// PathState::counts layout: [0, 64) live paths per bounce, then two counters
// per bounce (extension rays taken, shadow records taken), then the surface
// hits and the medium collisions per bounce.  Shading, shadow records and
// accumulation run over the bounce's events: item i < hits is qh[i], the
// others qs[i - hits].
constexpr int kTravCounters = 64;
constexpr int kHitCounters = kTravCounters + 2 * 64;
constexpr int kScatterCounters = kHitCounters + 64;
constexpr int kCountsSize = kScatterCounters + 64;

// Scenes with at most this many medium instances test every box along a ray;
// larger ones walk the instance BVH (same result either way).
constexpr int kMediaLinearMax = 8;
constexpr size_t kMaxMediumInstances = size_t(1) << 22;

constexpr int kEventScatter = -2147483647;  // INT_MIN + 1
constexpr int kEventDead = -2147483646;     // INT_MIN + 2

struct RenderLaunch {
  SceneView scene;
  Camera cam;
  PathState st;
  float* frame;       // W*H*3 linear RGB, row 0 = bottom (SFrame layout)
  uint32_t npix;      // pixels of the frame
  uint32_t waveSpp;   // samples per wave (>= 1): path p is pixel p % npix, sample `sample` + p / npix
  uint32_t wavePaths; // npix * waveSpp
  uint32_t sample;    // first sample index of the wave
  uint32_t* sampleDev;  // nullable: device sample counter of a captured wave (read instead of `sample`)
  uint32_t spp;
  uint32_t maxDepth;
  uint32_t seed;
  uint32_t bounce;
  uint32_t dda;       // brick-grid DDA tracking (UseBrickGrid) instead of the global majorant
  uint32_t trackSteps;  // tracking steps a lane takes between refills (tuning, >= 1)
  uint32_t travVisits;  // BVH visits a lane takes between refill checks of the surface kernels (tuning, >= 1)
  uint32_t travRefill;  // finished lanes of a warp that trigger a refill (tuning, 1..32)
  uint32_t mediaRounds; // queued medium-boundary rounds per bounce (tuning, 1..kMaxMediaRounds)
  uint32_t trackBlocks; // persistent tracker blocks per SM (tuning; 0: every resident block)
  uint32_t trackLimit;  // steps of one tracking loop after which the path ends (1..kMaxTrackingSteps)
  uint32_t topNodes;    // BVH nodes staged in shared memory by the surface traversals (0: none, <= kMaxTopNodes)
  uint32_t sortRays;    // surface scenes: reorder each bounce's rays by a coherence key before k_extend
  unsigned long long* stats;  // nullable: [0] path segments traced, [1] shadow rays traced
  unsigned int* bound;        // paths and shadow rays ended by a loop bound (tracking steps, boundaries)
};

// Optional per-kernel timing of one wave: events recorded after each launch;
// kind: -1 start, 0 camera, 1 extend, 2 shade, 3 shadow, 4 accum, 5 finish.
struct WaveTimer {
  static constexpr int kMax = 6 + 4 * 64;
  cudaEvent_t ev[kMax];
  int kind[kMax];
  int n = 0;
};

// One wave (L.waveSpp consecutive samples of every pixel).  With L.sampleDev
// the last launch advances the device sample counter by L.waveSpp, so a
// captured wave replays as the next samples.
void launch_render_wave(const RenderLaunch& L, int nblocks, cudaStream_t s, WaveTimer* tm = nullptr);
// Occupancy queries of the persistent kernels, done before any capture.
void prepare_render_launches();

}  // namespace r2
