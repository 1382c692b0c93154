// Host side of the wavefront path tracer.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "asset_io.h"
#include "host_math.h"
#include "render_host.h"

namespace r2 {

Camera make_camera(const r2_camera& c) {
  Camera cam;
  cam.W = (int)c.width;
  cam.H = (int)c.height;
  cam.pixelSize = 1e-5f;
  float fov = c.fov_deg * 0.01745329251994329577f;  // glm::radians
  float sensorW = (float)c.width * cam.pixelSize;
  cam.nearPlane = sensorW / (2.0f * tanf(fov / 2.0f));
  // glm::lookAt (right handed): rows s, u, -f; viewToWorld is its inverse
  V3 eye = v3(c.pos[0], c.pos[1], c.pos[2]);
  V3 ctr = v3(c.look_at[0], c.look_at[1], c.look_at[2]);
  V3 up = v3(c.up[0], c.up[1], c.up[2]);
  V3 f = normalize(ctr - eye);
  V3 s = normalize(cross(f, up));
  V3 u = cross(s, f);
  M4 view = m4_identity();
  view.m[0][0] = s.x; view.m[1][0] = s.y; view.m[2][0] = s.z;
  view.m[0][1] = u.x; view.m[1][1] = u.y; view.m[2][1] = u.z;
  view.m[0][2] = -f.x; view.m[1][2] = -f.y; view.m[2][2] = -f.z;
  view.m[3][0] = -dot(s, eye);
  view.m[3][1] = -dot(u, eye);
  view.m[3][2] = dot(f, eye);
  cam.viewToWorld = m4_to_m43(m4_inverse(view));
  return cam;
}

// CDistribution1D(std::vector<float>&) (distribution_1d.cu:6-39).
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

void build_env(const float* rgb, int W, int H, EnvHost* e) {
  e->W = W;
  e->H = H;
  e->tex.resize((size_t)W * H);
  std::vector<float> rad((size_t)W * H);
  for (int y = 0; y < H; ++y) {
    // radiancePerPixel: (r + g + b) * sin(pi (row + 0.5) / H) in double
    double st = sin(3.14159265358979323846 * (double)((float)y + 0.5f) / (double)(float)H);
    for (int x = 0; x < W; ++x) {
      size_t i = (size_t)y * W + x;
      float r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
      e->tex[i] = make_float4(r, g, b, 1.0f);
      float pr = 0.0f;
      pr += r;
      pr += g;
      pr += b;
      rad[i] = (float)((double)pr * st);
    }
  }
  // sumRows (distribution_2d.hpp:59-71): pushes the running sum when i % W == 0,
  // so entry 0 is texel 0 alone and entry r >= 1 sums texels (r-1)W+1 .. rW.
  std::vector<float> sums;
  sums.reserve(H);
  float sum = 0.0f;
  for (size_t i = 0; i < (size_t)W * H; ++i) {
    sum += rad[i];
    if (i % (size_t)W == 0) {
      sums.push_back(sum);
      sum = 0.0f;
    }
  }
  int nm = (int)sums.size();
  e->margFunc.resize(nm);
  e->margCdf.resize(nm + 1);
  dist1d(sums.data(), nm, e->margFunc.data(), e->margCdf.data(), &e->margFuncInt);
  e->rowFunc.resize((size_t)W * H);
  e->rowCdf.resize((size_t)(W + 1) * H);
  e->rowFuncInt.resize(H);
  for (int y = 0; y < H; ++y)
    dist1d(&rad[(size_t)y * W], W, &e->rowFunc[(size_t)y * W], &e->rowCdf[(size_t)y * (W + 1)], &e->rowFuncInt[y]);
}

RenderContext::RenderContext() {
  R2_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  R2_CUDA(cudaEventCreate(&ev0));
  R2_CUDA(cudaEventCreate(&ev1));
  bound.alloc(1);
  sampleDev.alloc(1);
}

RenderContext::~RenderContext() {
  if (stream) cudaStreamSynchronize(stream);
  if (timer)
    for (int i = 0; i < WaveTimer::kMax; ++i) cudaEventDestroy(timer->ev[i]);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (stream) cudaStreamDestroy(stream);
}

RenderScene::RenderScene() {
  memset(&view_, 0, sizeof(view_));
  auto env = [](const char* name, long lo, long hi) -> uint32_t {
    const char* e = getenv(name);
    return e ? (uint32_t)std::max(lo, std::min(hi, atol(e))) : 0u;
  };
  tuning_.track_steps = env("R2_TRACK_STEPS", 1, 1024);
  tuning_.trav_visits = env("R2_TRAV_VISITS", 1, 1 << 20);
  tuning_.trav_refill = env("R2_TRAV_REFILL", 1, 32);
  tuning_.media_rounds = env("R2_MEDIA_ROUNDS", 1, kMaxMediaRounds);
  tuning_.track_blocks = env("R2_TRACK_BLOCKS", 1, 64);
}

RenderScene::~RenderScene() {}

void RenderScene::add_mesh(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* nrm,
                           const r2_material& mat, const float* m2w, uint32_t mask, const float* uv,
                           const r2_material_maps* maps) {
  R2_REQUIRE(pos && idx && nrm && m2w, R2_ERR_INVALID_ARGUMENT, "null mesh array");
  R2_REQUIRE(nverts > 0 && ntris > 0, R2_ERR_INVALID_ARGUMENT, "empty mesh");
  // render rays carry visibility mask 255 (device_scene.hpp:17): every object
  // with a nonzero mask is visible, FILTER-only ones included
  if (mask == 0) return;
  M43 M = m43_from_floats(m2w);
  uint32_t base = (uint32_t)(hPos_.size() / 3);
  uint32_t matId = (uint32_t)hMats_.size();
  Material hm = make_material(mat);
  if (maps && uv) {  // without texture coordinates the maps are not used (shaders.optix.cu:60-61)
    textures_.material_maps(mat, maps, hm.tex);
  }
  hMats_.push_back(hm);
  if (uv && !anyUV_) {  // earlier meshes get coordinates (0, 0)
    anyUV_ = true;
    hUV_.assign(2 * (size_t)base, 0.0f);
  }
  for (uint32_t v = 0; v < nverts; ++v) {
    V3 p = xform_point(M, v3(pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]));
    V3 n = xform_vector(M, v3(nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2]));
    hPos_.push_back(p.x); hPos_.push_back(p.y); hPos_.push_back(p.z);
    hNrm_.push_back(n.x); hNrm_.push_back(n.y); hNrm_.push_back(n.z);
    if (anyUV_) {
      hUV_.push_back(uv ? uv[2 * v] : 0.0f);
      hUV_.push_back(uv ? uv[2 * v + 1] : 0.0f);
    }
  }
  for (uint32_t t = 0; t < ntris; ++t) {
    for (int k = 0; k < 3; ++k) {
      R2_REQUIRE(idx[3 * t + k] < nverts, R2_ERR_INVALID_ARGUMENT, "triangle index out of range");
      hIdx_.push_back(base + idx[3 * t + k]);
    }
    hTriMat_.push_back(matId);
  }
  committed_ = false;
}

uint32_t RenderScene::add_mesh_asset(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris,
                                     const float* nrm, const r2_material& mat, const float* uv,
                                     const r2_material_maps* maps) {
  R2_REQUIRE(pos && idx && nrm, R2_ERR_INVALID_ARGUMENT, "null mesh array");
  R2_REQUIRE(nverts > 0 && ntris > 0, R2_ERR_INVALID_ARGUMENT, "empty mesh");
  auto a = std::make_unique<MeshAsset>();
  a->matId = (uint32_t)hMats_.size();
  Material hm = make_material(mat);
  if (maps && uv) textures_.material_maps(mat, maps, hm.tex);
  hMats_.push_back(hm);
  a->pos.assign(pos, pos + 3 * (size_t)nverts);
  a->nrm.assign(nrm, nrm + 3 * (size_t)nverts);
  if (uv) {
    a->hasUV = true;
    a->uv.assign(uv, uv + 2 * (size_t)nverts);
  }
  a->idx.assign(idx, idx + 3 * (size_t)ntris);
  for (uint32_t k = 0; k < 3 * ntris; ++k)
    R2_REQUIRE(idx[k] < nverts, R2_ERR_INVALID_ARGUMENT, "triangle index out of range");
  assets_.push_back(std::move(a));
  committed_ = false;
  return (uint32_t)(assets_.size() - 1);
}

void RenderScene::add_mesh_instance(uint32_t asset, const float* m2w, uint32_t mask) {
  R2_REQUIRE(asset < assets_.size(), R2_ERR_INVALID_ARGUMENT, "unknown mesh asset");
  R2_REQUIRE(m2w, R2_ERR_INVALID_ARGUMENT, "null transform");
  if (mask == 0) return;  // invisible to render rays, as add_mesh
  meshInstances_.push_back(MeshInstanceHost{asset, m43_from_floats(m2w)});
  committed_ = false;
}

void RenderScene::add_shape(int type, const float* center, float radius, const float* normal, const r2_material& mat,
                            uint32_t mask) {
  R2_REQUIRE(type == kShapeSphere || type == kShapeCircle, R2_ERR_INVALID_ARGUMENT, "unknown shape type");
  if (mask == 0) return;
  Shape s;
  memset(&s, 0, sizeof(s));
  s.type = type;
  s.material = (int)hMats_.size();
  hMats_.push_back(make_material(mat));
  s.radius = radius;
  s.center = v3(center[0], center[1], center[2]);
  s.normal = normal ? v3(normal[0], normal[1], normal[2]) : v3(0.0f, 1.0f, 0.0f);
  hShapes_.push_back(s);
  committed_ = false;
}

void RenderScene::set_envmap(const float* rgb, int W, int H) {
  R2_REQUIRE(rgb && W >= 2 && H >= 2, R2_ERR_INVALID_ARGUMENT, "environment map must be at least 2x2");
  build_env(rgb, W, H, &env_);
  committed_ = false;
}

void RenderScene::add_medium(const char* path, const float* sigmaA, const float* sigmaS, const float* pos,
                             const float* orientation, const float* scaling, uint32_t mask, bool hg, float g) {
  R2_REQUIRE(path && sigmaA && sigmaS && pos && orientation && scaling, R2_ERR_INVALID_ARGUMENT, "null medium argument");
  R2_REQUIRE(media_.size() < kMaxMediumInstances, R2_ERR_UNSUPPORTED, "too many media in one scene");
  auto it = mediaByPath_.find(path);
  if (it == mediaByPath_.end())
    it = mediaByPath_.emplace(std::string(path), load_medium(path, sigmaA, sigmaS, hg, g)).first;
  if (mask == 0) return;  // render rays (mask 255) never see objects with mask NONE
  media_.push_back(MediumInstance{it->second.get(), v3(pos[0], pos[1], pos[2]),
                                  v3(orientation[0], orientation[1], orientation[2]),
                                  v3(scaling[0], scaling[1], scaling[2])});
  committed_ = false;
}

namespace {
// Per BVH-order triangle: vertex normals, material, texture coordinates and
// opacity map of the scene-order triangle order[i].
__global__ void k_gather_shading(const uint32_t* __restrict__ order, uint32_t n, const uint32_t* __restrict__ idx,
                                 const float* __restrict__ nrm, const uint32_t* __restrict__ matIn,
                                 const float* __restrict__ uv, const int* __restrict__ alphaIn,
                                 float4* __restrict__ triN, uint32_t* __restrict__ triMat,
                                 float2* __restrict__ triUV, int* __restrict__ triAlpha) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = order[i];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = idx[3 * p + k];
    triN[3 * i + k] = make_float4(nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2], 0.0f);
    if (triUV) triUV[3 * i + k] = make_float2(uv[2 * v], uv[2 * v + 1]);
  }
  triMat[i] = matIn[p];
  if (triAlpha) triAlpha[i] = alphaIn[p];
}

// A bottom-level BVH copied into the global node array: inner references
// move by nodeOff, leaf ranges by triOff, parents by nodeOff.
__global__ void k_rebase_nodes(const BvhNode* __restrict__ src, uint32_t n, int nodeOff, int triOff,
                               BvhNode* __restrict__ dst) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BvhNode nd = src[i];
  auto move = [&](int c) {
    if (c == R2_BVH_NONE) return c;
    if (c >= 0) return c + nodeOff;
    return bvh_leaf_ref(bvh_leaf_first(c) + triOff, bvh_leaf_count(c));
  };
  nd.ch.x = move(nd.ch.x);
  nd.ch.y = move(nd.ch.y);
  if (nd.ch.z >= 0) nd.ch.z += nodeOff;
  dst[i] = nd;
}

// The top level (one box per leaf) with its leaves turned into instance
// references: ~instance, a leaf reference with count 0.
__global__ void k_top_level_nodes(const BvhNode* __restrict__ src, uint32_t n, const uint32_t* __restrict__ order,
                                  BvhNode* __restrict__ dst) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BvhNode nd = src[i];
  auto inst = [&](int c) {
    if (c == R2_BVH_NONE || c >= 0) return c;
    return bvh_leaf_ref((int)order[bvh_leaf_first(c)], 0);
  };
  nd.ch.x = inst(nd.ch.x);
  nd.ch.y = inst(nd.ch.y);
  dst[i] = nd;
}
}  // namespace

void RenderScene::rebuild(cudaStream_t s) {
  if (!s) s = ctx_.stream;
  if (two_level()) {
    build_two_level(s);
    return;
  }
  const uint32_t nt = (uint32_t)(hIdx_.size() / 3);
  R2_REQUIRE(nt > 0 && dIdx_.get(), R2_ERR_INVALID_ARGUMENT, "scene has no committed triangles");
  builder_.build(dPos_.get(), dIdx_.get(), nt, &bvh_, s);
  bvhNodes_ = bvh_.nnodes;
  bvhHeight_ = bvh_.height;
  buildLaunches_ = builder_.launches() + 1;
  triN_.reserve((size_t)3 * nt);
  triMat_.reserve(nt);
  if (anyUV_) triUV_.reserve((size_t)3 * nt);
  if (dTriAlphaIn_.get()) triAlpha_.reserve(nt);
  k_gather_shading<<<(nt + 255) / 256, 256, 0, s>>>(bvh_.order.get(), nt, dIdx_.get(), dNrm_.get(), dTriMatIn_.get(),
                                                    anyUV_ ? dUV_.get() : nullptr, dTriAlphaIn_.get(), triN_.get(),
                                                    triMat_.get(), anyUV_ ? triUV_.get() : nullptr,
                                                    dTriAlphaIn_.get() ? triAlpha_.get() : nullptr);
  R2_CUDA(cudaGetLastError());
  const BvhAlpha alpha = view_.bvh.alpha;
  view_.bvh = bvh_.view();
  view_.bvh.alpha = alpha;
}

// Device inputs and bottom-level BVHs of the mesh assets (once per commit:
// their geometry does not change afterwards).
void RenderScene::upload_assets(cudaStream_t s) {
  for (auto& ap : assets_) {
    MeshAsset& a = *ap;
    const uint32_t nt = (uint32_t)(a.idx.size() / 3);
    a.dPos.upload(a.pos.data(), a.pos.size(), s);
    a.dNrm.upload(a.nrm.data(), a.nrm.size(), s);
    a.dIdx.upload(a.idx.data(), a.idx.size(), s);
    std::vector<uint32_t> mat(nt, a.matId);
    a.dTriMat.upload(mat.data(), mat.size(), s);
    if (a.hasUV) a.dUV.upload(a.uv.data(), a.uv.size(), s);
    const int alphaTex = a.hasUV ? hMats_[a.matId].tex[3] : -1;
    if (alphaTex >= 0) {
      std::vector<int> al(nt, alphaTex);
      a.dAlphaIn.upload(al.data(), al.size(), s);
    }
    builder_.build(a.dPos.get(), a.dIdx.get(), nt, &a.bvh, s);
  }
}

// The two-level structure: the world-space meshes' BVH (rebuilt from the
// resident triangles), the top level over the instances' world boxes, the
// global node array [top level | world meshes | assets] and triangle array
// [world meshes | assets] with per-triangle shading data in the same order.
// Instance 0 is the world-space meshes (identity) when there are any.
void RenderScene::build_two_level(cudaStream_t s) {
  const uint32_t nw = (uint32_t)(hIdx_.size() / 3);
  int launches = 0;
  if (nw > 0) {
    builder_.build(dPos_.get(), dIdx_.get(), nw, &bvh_, s);
    launches += builder_.launches();
  }
  // triangle and node offsets of the pools (0: world meshes, 1 + a: asset a)
  const size_t npool = 1 + assets_.size();
  std::vector<uint32_t> triOff(npool), ntri(npool), nnode(npool), height(npool);
  ntri[0] = nw;
  nnode[0] = nw ? bvh_.nnodes : 0;
  height[0] = nw ? bvh_.height : 0;
  for (size_t a = 0; a < assets_.size(); ++a) {
    ntri[1 + a] = (uint32_t)(assets_[a]->idx.size() / 3);
    nnode[1 + a] = assets_[a]->bvh.nnodes;
    height[1 + a] = assets_[a]->bvh.height;
  }
  uint64_t totalTris = 0;
  for (size_t k = 0; k < npool; ++k) {
    triOff[k] = (uint32_t)totalTris;
    totalTris += ntri[k];
  }
  R2_REQUIRE(totalTris < (1u << 26), R2_ERR_UNSUPPORTED, "two-level scene with 2^26 or more distinct triangles");
  // instances: boxes (padded so that rounding never culls a hit), transforms, codes
  struct Inst {
    size_t pool;
    M43 m;
    bool identity;
  };
  std::vector<Inst> insts;
  if (nw > 0) insts.push_back(Inst{0, M43{}, true});
  for (const MeshInstanceHost& mi : meshInstances_) insts.push_back(Inst{1 + mi.asset, mi.m2w, false});
  const uint32_t ninst = (uint32_t)insts.size();
  std::vector<float4> lo(ninst), hi(ninst), o2w(3 * (size_t)ninst);
  std::vector<BvhInstance> hin(ninst);
  std::vector<int> code(ninst);
  auto pad = [](float x) { return 1e-5f * (fabsf(x) + 1.0f); };
  uint64_t nextCode = 0;
  for (uint32_t i = 0; i < ninst; ++i) {
    const Inst& in = insts[i];
    const std::vector<float>& P = in.pool == 0 ? hPos_ : assets_[in.pool - 1]->pos;
    V3 mlo = v3(INFINITY), mhi = v3(-INFINITY);
    for (size_t v = 0; v < P.size(); v += 3) {
      const V3 p = v3(P[v], P[v + 1], P[v + 2]);
      mlo = vmin(mlo, p);
      mhi = vmax(mhi, p);
    }
    V3 wlo = mlo, whi = mhi;
    BvhInstance& b = hin[i];
    memset(&b, 0, sizeof(b));
    if (in.identity) {
      b.identity = 1;
      b.w2o[0] = make_float4(1, 0, 0, 0);
      b.w2o[1] = make_float4(0, 1, 0, 0);
      b.w2o[2] = make_float4(0, 0, 1, 0);
      for (int r = 0; r < 3; ++r) o2w[3 * i + r] = b.w2o[r];
    } else {
      wlo = v3(INFINITY);
      whi = v3(-INFINITY);
      for (int c = 0; c < 8; ++c) {
        const V3 p = xform_point(in.m, v3(c & 1 ? mhi.x : mlo.x, c & 2 ? mhi.y : mlo.y, c & 4 ? mhi.z : mlo.z));
        wlo = vmin(wlo, p);
        whi = vmax(whi, p);
      }
      const M4 inv = m4_inverse(m43_to_m4(in.m));  // double elimination, rounded to float
      for (int r = 0; r < 3; ++r) {
        b.w2o[r] = make_float4(inv.m[0][r], inv.m[1][r], inv.m[2][r], inv.m[3][r]);
        o2w[3 * i + r] = make_float4(comp(in.m.c[0], r), comp(in.m.c[1], r), comp(in.m.c[2], r), comp(in.m.c[3], r));
      }
    }
    lo[i] = make_float4(wlo.x - pad(wlo.x), wlo.y - pad(wlo.y), wlo.z - pad(wlo.z), 0.0f);
    hi[i] = make_float4(whi.x + pad(whi.x), whi.y + pad(whi.y), whi.z + pad(whi.z), 0.0f);
    code[i] = (int)nextCode;
    b.vdelta = (int)((int64_t)nextCode - (int64_t)triOff[in.pool]);
    nextCode += ntri[in.pool];
    R2_REQUIRE(nextCode < 0x7FFFFFFFull, R2_ERR_UNSUPPORTED, "two-level scene with 2^31 or more instanced triangles");
  }
  dInstLo_.upload(lo.data(), ninst, s);
  dInstHi_.upload(hi.data(), ninst, s);
  builder_.build_boxes(dInstLo_.get(), dInstHi_.get(), ninst, &tlas_, s, 1);
  launches += builder_.launches();
  const uint32_t ntl = tlas_.nnodes;
  std::vector<uint32_t> nodeOff(npool);
  uint64_t totalNodes = ntl;
  uint32_t maxHeight = 0;
  for (size_t k = 0; k < npool; ++k) {
    nodeOff[k] = (uint32_t)totalNodes;
    totalNodes += nnode[k];
    maxHeight = std::max(maxHeight, height[k]);
  }
  R2_REQUIRE(tlas_.height + maxHeight + 2 <= R2_BVH_STACK, R2_ERR_UNSUPPORTED,
             "two-level BVH deeper than the traversal stack");
  for (uint32_t i = 0; i < ninst; ++i) hin[i].root = (int)nodeOff[insts[i].pool];
  dInst_.upload(hin.data(), ninst, s);
  dInstCode_.upload(code.data(), ninst, s);
  dInstO2W_.upload(o2w.data(), o2w.size(), s);
  gNodes_.reserve(totalNodes);
  gTris_.reserve(3 * totalTris);
  triN_.reserve(3 * totalTris);
  triMat_.reserve(totalTris);
  bool sceneUV = anyUV_;
  for (auto& a : assets_) sceneUV = sceneUV || a->hasUV;
  if (sceneUV) triUV_.reserve(3 * totalTris);
  if (anyAlpha_) triAlpha_.reserve(totalTris);
  k_top_level_nodes<<<(ntl + 255) / 256, 256, 0, s>>>(tlas_.nodes.get(), ntl, tlas_.order.get(), gNodes_.get());
  ++launches;
  for (size_t k = 0; k < npool; ++k) {
    if (ntri[k] == 0) continue;
    const DeviceBvh& b = k == 0 ? bvh_ : assets_[k - 1]->bvh;
    k_rebase_nodes<<<(nnode[k] + 255) / 256, 256, 0, s>>>(b.nodes.get(), nnode[k], (int)nodeOff[k], (int)triOff[k],
                                                          gNodes_.get() + nodeOff[k]);
    R2_CUDA(cudaMemcpyAsync(gTris_.get() + 3 * (size_t)triOff[k], b.tris.get(), sizeof(float4) * 3 * ntri[k],
                            cudaMemcpyDeviceToDevice, s));
    const uint32_t o = triOff[k], n = ntri[k];
    if (k == 0) {
      k_gather_shading<<<(n + 255) / 256, 256, 0, s>>>(
          b.order.get(), n, dIdx_.get(), dNrm_.get(), dTriMatIn_.get(), sceneUV ? dUV_.get() : nullptr,
          anyAlpha_ ? dTriAlphaIn_.get() : nullptr, triN_.get() + 3 * (size_t)o, triMat_.get() + o,
          sceneUV ? triUV_.get() + 3 * (size_t)o : nullptr, anyAlpha_ ? triAlpha_.get() + o : nullptr);
    } else {
      MeshAsset& a = *assets_[k - 1];
      k_gather_shading<<<(n + 255) / 256, 256, 0, s>>>(
          b.order.get(), n, a.dIdx.get(), a.dNrm.get(), a.dTriMat.get(), sceneUV ? a.dUV.get() : nullptr,
          anyAlpha_ ? a.dAlphaIn.get() : nullptr, triN_.get() + 3 * (size_t)o, triMat_.get() + o,
          sceneUV ? triUV_.get() + 3 * (size_t)o : nullptr, anyAlpha_ ? triAlpha_.get() + o : nullptr);
    }
    launches += 2;
  }
  R2_CUDA(cudaGetLastError());
  const BvhAlpha alpha = view_.bvh.alpha;
  memset(&view_.bvh, 0, sizeof(view_.bvh));
  view_.bvh.nodes = gNodes_.get();
  view_.bvh.tris = gTris_.get();
  view_.bvh.ntris = (uint32_t)totalTris;
  view_.bvh.alpha = alpha;
  view_.bvh.inst = dInst_.get();
  view_.instCode = dInstCode_.get();
  view_.instO2W = dInstO2W_.get();
  view_.ninst = (int)ninst;
  bvhNodes_ = (uint32_t)totalNodes;
  bvhHeight_ = tlas_.height + maxHeight;
  buildLaunches_ = launches;
  R2_CUDA(cudaStreamSynchronize(s));  // the host vectors above are freed on return
}

void RenderScene::set_vertices(const float* pos, const float* nrm, uint32_t nverts, cudaStream_t s) {
  if (!s) s = ctx_.stream;
  R2_REQUIRE((size_t)nverts * 3 == hPos_.size() && nverts > 0, R2_ERR_INVALID_ARGUMENT,
             "vertex count differs from the scene's (" + std::to_string(hPos_.size() / 3) + ")");
  memcpy(hPos_.data(), pos, hPos_.size() * sizeof(float));
  R2_CUDA(cudaMemcpyAsync(dPos_.get(), pos, hPos_.size() * sizeof(float), cudaMemcpyHostToDevice, s));
  if (nrm) {
    memcpy(hNrm_.data(), nrm, hNrm_.size() * sizeof(float));
    R2_CUDA(cudaMemcpyAsync(dNrm_.get(), nrm, hNrm_.size() * sizeof(float), cudaMemcpyHostToDevice, s));
  }
}

void RenderScene::commit() {
  R2_REQUIRE(env_.W > 0, R2_ERR_INVALID_CONFIG, "scene has no environment map");
  cudaStream_t s = ctx_.stream;
  uint32_t nt = (uint32_t)(hIdx_.size() / 3);
  memset(&view_, 0, sizeof(view_));
  const bool twoLevel = two_level();
  bool sceneUV = anyUV_;
  if (twoLevel)
    for (auto& a : assets_) sceneUV = sceneUV || a->hasUV;
  if (sceneUV && !anyUV_) hUV_.assign(2 * (hPos_.size() / 3), 0.0f);  // world meshes without coordinates: (0, 0)
  anyAlpha_ = false;
  if (nt > 0) {
    dPos_.upload(hPos_.data(), hPos_.size(), s);
    dNrm_.upload(hNrm_.data(), hNrm_.size(), s);
    dIdx_.upload(hIdx_.data(), hIdx_.size(), s);
    dTriMatIn_.upload(hTriMat_.data(), hTriMat_.size(), s);
    if (sceneUV) {  // texture coordinates and opacity maps per triangle
      dUV_.upload(hUV_.data(), hUV_.size(), s);
      std::vector<int> alphaIn(nt);
      for (uint32_t t = 0; t < nt; ++t) {
        alphaIn[t] = hMats_[hTriMat_[t]].tex[3];
        anyAlpha_ = anyAlpha_ || alphaIn[t] >= 0;
      }
      if (anyAlpha_ || twoLevel) dTriAlphaIn_.upload(alphaIn.data(), alphaIn.size(), s);
    }
  }
  if (twoLevel) {
    for (auto& a : assets_) anyAlpha_ = anyAlpha_ || (a->hasUV && hMats_[a->matId].tex[3] >= 0);
    if (anyAlpha_)  // every pool needs its opacity-map input
      for (auto& a : assets_)
        if (!(a->hasUV && hMats_[a->matId].tex[3] >= 0)) {
          std::vector<int> al(a->idx.size() / 3, -1);
          a->dAlphaIn.upload(al.data(), al.size(), s);
        }
    for (auto& a : assets_)
      if (sceneUV && !a->hasUV) {
        std::vector<float> z(2 * (a->pos.size() / 3), 0.0f);
        a->dUV.upload(z.data(), z.size(), s);
      }
    if (anyAlpha_ && nt > 0 && !dTriAlphaIn_.get()) {
      std::vector<int> al(nt, -1);
      dTriAlphaIn_.upload(al.data(), al.size(), s);
    }
    upload_assets(s);
  }
  if (nt > 0 || twoLevel) {
    rebuild(s);
    if (sceneUV) view_.triUV = triUV_.get();
    if (anyAlpha_) {
      view_.bvh.alpha.alphaTex = triAlpha_.get();
      view_.bvh.alpha.uv = triUV_.get();
    }
    view_.triN = triN_.get();
    view_.triMat = triMat_.get();
    view_.hasTris = 1;
  }
  mats_.upload(hMats_.data(), hMats_.size(), s);
  view_.mats = mats_.get();
  if (textures_.upload(&texels_, &texInfo_, s)) {
    view_.texels = texels_.get();
    view_.texInfo = texInfo_.get();
    view_.bvh.alpha.texels = view_.texels;
    view_.bvh.alpha.texInfo = view_.texInfo;
  }
  if (!hShapes_.empty()) shapes_.upload(hShapes_.data(), hShapes_.size(), s);
  view_.shapes = shapes_.get();
  view_.nshapes = (int)hShapes_.size();
  if (!media_.empty()) {
    std::vector<MediumView> mv;
    mv.reserve(media_.size());
    for (const MediumInstance& m : media_) {
      if (!m.medium->uploaded) m.medium->upload(s);
      mv.push_back(place_medium(*m.medium, m.pos, m.orientation, m.scaling));
    }
    mediaViews_.upload(mv.data(), mv.size(), s);
    if (mv.size() > (size_t)kMediaLinearMax) {
      // instance BVH over the world boxes, padded so that rounding in the
      // node tests never culls a box that a ray hits
      std::vector<float4> lo(mv.size()), hi(mv.size());
      for (size_t i = 0; i < mv.size(); ++i) {
        const V3 a = mv[i].aabbMin, b = mv[i].aabbMax;
        auto pad = [](float x) { return 1e-5f * (fabsf(x) + 1.0f); };
        lo[i] = make_float4(a.x - pad(a.x), a.y - pad(a.y), a.z - pad(a.z), 0.0f);
        hi[i] = make_float4(b.x + pad(b.x), b.y + pad(b.y), b.z + pad(b.z), 0.0f);
      }
      DBuf<float4> dlo, dhi;
      dlo.upload(lo.data(), lo.size(), s);
      dhi.upload(hi.data(), hi.size(), s);
      build_box_bvh(dlo.get(), dhi.get(), (uint32_t)mv.size(), &mediaBvh_, s);
      view_.mediaNodes = mediaBvh_.nodes.get();
      view_.mediaOrder = mediaBvh_.order.get();
    }
  }
  view_.media = mediaViews_.get();
  view_.nmedia = (int)media_.size();
  // environment: texels + one float buffer for all distribution arrays
  envTex_.upload(env_.tex.data(), env_.tex.size(), s);
  std::vector<float> buf;
  size_t oMF = buf.size(); buf.insert(buf.end(), env_.margFunc.begin(), env_.margFunc.end());
  size_t oMC = buf.size(); buf.insert(buf.end(), env_.margCdf.begin(), env_.margCdf.end());
  size_t oRF = buf.size(); buf.insert(buf.end(), env_.rowFunc.begin(), env_.rowFunc.end());
  size_t oRC = buf.size(); buf.insert(buf.end(), env_.rowCdf.begin(), env_.rowCdf.end());
  size_t oRI = buf.size(); buf.insert(buf.end(), env_.rowFuncInt.begin(), env_.rowFuncInt.end());
  envBuf_.upload(buf.data(), buf.size(), s);
  EnvMap& e = view_.env;
  e.tex = envTex_.get();
  e.W = env_.W;
  e.H = env_.H;
  e.margFunc = envBuf_.get() + oMF;
  e.margCdf = envBuf_.get() + oMC;
  e.margFuncInt = env_.margFuncInt;
  e.rowFunc = envBuf_.get() + oRF;
  e.rowCdf = envBuf_.get() + oRC;
  e.rowFuncInt = envBuf_.get() + oRI;
  e.valid = 1;
  R2_CUDA(cudaStreamSynchronize(s));
  committed_ = true;
}

uint32_t RenderContext::capacity_for(uint32_t n) {
  uint64_t c = 1u << 16;
  while (c < n) c <<= 1;
  return (uint32_t)std::min<uint64_t>(c, 0x80000000ull);
}

void RenderContext::ensure(uint32_t n, bool media) {
  n = capacity_for(n);
  if (n > cap_) {
    rayO_.alloc(n); rayD_.alloc(n); T_.alloc(n); L_.alloc(n); hit_.alloc(n);
    shO_.alloc(2 * (size_t)n); shD_.alloc(2 * (size_t)n); shPre_.alloc(2 * (size_t)n); shT_.alloc(n);
    q0_.alloc(n); q1_.alloc(n); qh_.alloc(n); qs_.alloc(n); shTr_.alloc(2 * (size_t)n);
    counts_.alloc(kCountsSize);
    sortBins_.alloc(256);
    cap_ = n;
  }
  if (media && n > mediaCap_) {
    shX_.alloc(2 * (size_t)n);
    evA_.alloc(n); evB_.alloc(n); evC_.alloc(n); evD_.alloc(n);
    mc_.alloc((size_t)kCountersPerBounce * 64);
    pj_.alloc(n); rl0_.alloc(n); rl1_.alloc(n); cl_.alloc(n);
    sl0_.alloc(2 * (size_t)n); sl1_.alloc(2 * (size_t)n);
    jO_.alloc(2 * (size_t)n); jD_.alloc(2 * (size_t)n); jM_.alloc(2 * (size_t)n);
    swP_.alloc(2 * (size_t)n); swM_.alloc(2 * (size_t)n);
    mediaCap_ = n;
  }
}

size_t RenderContext::bytes_for(uint32_t n, bool media) {
  n = capacity_for(n);
  // per path: 5 float4 state + 3 x 2 float4 records + float4 throughput + 4 queue ids + 2 transmittances
  size_t b = (size_t)n * (5 * 16 + 6 * 16 + 16 + 16 + 8) + kCountsSize * 4;
  // media: records (4 float4 + float2), shadow tmax/medium, round queues and walk state
  if (media) b += (size_t)n * (16 + 48 + 8 + 16 + 16 + 64 + 16 + 32 + 16) + 16 * 64 * 4;
  return b + (size_t)n * 12;  // frame
}

void RenderContext::fill(PathState* st) const {
  st->rayO = rayO_.get(); st->rayD = rayD_.get(); st->T = T_.get(); st->L = L_.get(); st->hit = hit_.get();
  st->q[0] = q0_.get(); st->q[1] = q1_.get(); st->qh = qh_.get(); st->qs = qs_.get(); st->counts = counts_.get();
  st->sortBins = sortBins_.get();
  st->shO = shO_.get(); st->shD = shD_.get(); st->shPre = shPre_.get(); st->shT = shT_.get();
  st->shTr = shTr_.get();
  if (mediaCap_ > 0) {
    st->shX = shX_.get();
    st->evA = evA_.get(); st->evB = evB_.get(); st->evC = evC_.get(); st->evD = evD_.get();
    st->mc = mc_.get(); st->pj = pj_.get();
    st->rl[0] = rl0_.get(); st->rl[1] = rl1_.get(); st->cl = cl_.get();
    st->sl[0] = sl0_.get(); st->sl[1] = sl1_.get();
    st->jO = jO_.get(); st->jD = jD_.get(); st->jM = jM_.get();
    st->swP = swP_.get(); st->swM = swM_.get();
  }
}

uint32_t RenderContext::bound_hits(cudaStream_t s) {
  unsigned int b = 0;
  bound.download(&b, 1, s);
  R2_CUDA(cudaStreamSynchronize(s));
  return b;
}

void RenderScene::check_params(const r2_camera& c, const r2_render_params& p, const float* d_frame) {
  R2_REQUIRE(d_frame, R2_ERR_INVALID_ARGUMENT, "null frame");
  R2_REQUIRE(c.width > 0 && c.height > 0, R2_ERR_INVALID_ARGUMENT, "empty frame");
  R2_REQUIRE((uint64_t)c.width * c.height < (1ull << 31), R2_ERR_UNSUPPORTED, "frame too large");
  R2_REQUIRE(p.spp > 0, R2_ERR_INVALID_ARGUMENT, "spp must be positive");
  R2_REQUIRE(p.max_depth > 0 && p.max_depth <= 60, R2_ERR_UNSUPPORTED, "max_depth must be in [1, 60]");
  R2_REQUIRE((p.flags & ~R2_RENDER_BRICK_GRID) == 0, R2_ERR_INVALID_ARGUMENT, "unknown render flags");
}

uint32_t RenderScene::wave_spp(uint32_t npix, uint32_t spp, uint32_t maxWavePaths) const {
  uint64_t target = tuning_.wave_paths ? tuning_.wave_paths : kDefaultWavePaths;
  if (maxWavePaths && maxWavePaths < target) target = maxWavePaths;
  uint32_t best = 1;
  for (uint32_t k = 2; k <= spp; ++k)
    if (spp % k == 0 && (uint64_t)k * npix <= target && (uint64_t)k * npix < (1ull << 31)) best = k;
  return best;
}

RenderLaunch RenderScene::make_launch(const RenderContext& ctx, const r2_camera& c, const r2_render_params& p,
                                      float* d_frame, uint32_t waveSpp) {
  RenderLaunch L;
  memset(&L, 0, sizeof(L));
  L.scene = view_;
  L.cam = make_camera(c);
  ctx.fill(&L.st);
  L.frame = d_frame;
  L.npix = c.width * c.height;
  L.waveSpp = waveSpp;
  L.wavePaths = L.npix * waveSpp;
  L.spp = p.spp;
  L.maxDepth = p.max_depth;
  L.seed = p.seed;
  L.dda = (p.flags & R2_RENDER_BRICK_GRID) ? 1u : 0u;
  L.trackSteps = tuning_.track_steps;
  L.travVisits = tuning_.trav_visits;
  L.travRefill = tuning_.trav_refill;
  L.mediaRounds = tuning_.media_rounds;
  L.trackBlocks = tuning_.track_blocks;
  L.trackLimit = tuning_.track_limit ? tuning_.track_limit : (uint32_t)kMaxTrackingSteps;
  // shared-memory top nodes: surface scenes only, within the tree
  L.topNodes = media_.empty() && view_.hasTris ? std::min(tuning_.top_nodes, bvhNodes_) : 0u;
  L.sortRays = media_.empty() && view_.hasTris && tuning_.sort_rays ? 1u : 0u;
  L.bound = ctx.bound.get();
  return L;
}

static int wave_blocks(uint32_t npix) { return std::max(1, std::min((int)((npix + 255) / 256), sm_count() * 8)); }

void RenderScene::render(const r2_camera& c, const r2_render_params& p, float* d_frame, cudaStream_t s,
                         double* stats) {
  check_params(c, p, d_frame);
  if (!committed_) commit();
  RenderContext& ctx = ctx_;
  if (!s) s = ctx.stream;
  const uint32_t npix = c.width * c.height;
  const uint32_t S = wave_spp(npix, p.spp);
  ctx.ensure(npix * S, !media_.empty());
  RenderLaunch L = make_launch(ctx, c, p, d_frame, S);
  R2_CUDA(cudaMemsetAsync(ctx.bound.get(), 0, sizeof(unsigned int), s));
  const int nblocks = wave_blocks(npix * S);
  R2_CUDA(cudaMemsetAsync(d_frame, 0, sizeof(float) * 3 * (size_t)npix, s));
  if (stats) {
    ctx.statBuf.reserve(2);
    R2_CUDA(cudaMemsetAsync(ctx.statBuf.get(), 0, 2 * sizeof(unsigned long long), s));
    L.stats = ctx.statBuf.get();
    if (!ctx.timer) {
      ctx.timer.reset(new WaveTimer());
      for (int i = 0; i < WaveTimer::kMax; ++i) R2_CUDA(cudaEventCreate(&ctx.timer->ev[i]));
    }
  }
  R2_CUDA(cudaEventRecord(ctx.ev0, s));
  for (uint32_t smp = 0; smp < p.spp; smp += S) {
    L.sample = smp;
    // the middle wave of a frame is timed kernel by kernel when statistics are requested
    const bool timed = stats && smp <= p.spp / 2 && p.spp / 2 < smp + S;
    launch_render_wave(L, nblocks, s, timed ? ctx.timer.get() : nullptr);
  }
  R2_CUDA(cudaEventRecord(ctx.ev1, s));
  if (stats) {
    R2_CUDA(cudaEventSynchronize(ctx.ev1));
    float ms = 0.0f;
    R2_CUDA(cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1));
    unsigned long long cnt[2] = {0, 0};
    R2_CUDA(cudaMemcpy(cnt, ctx.statBuf.get(), sizeof(cnt), cudaMemcpyDeviceToHost));
    double kms[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 1; i < ctx.timer->n; ++i) {
      float d = 0.0f;
      R2_CUDA(cudaEventElapsedTime(&d, ctx.timer->ev[i - 1], ctx.timer->ev[i]));
      int k = ctx.timer->kind[i];
      if (k >= 0 && k < 6) kms[k] += d;
    }
    stats[0] = (double)npix * p.spp;
    stats[1] = ms;
    stats[2] = (double)cnt[0];
    stats[3] = (double)cnt[1];
    for (int k = 1; k <= 4; ++k) stats[3 + k] = kms[k];  // one wave: extend, shade, shadow, accum
  }
}

void RenderScene::render_graph(RenderContext& ctx, const r2_camera& c, const r2_render_params& p, float* d_frame,
                               cudaStream_t s, uint32_t maxWavePaths) {
  const uint32_t npix = c.width * c.height;
  const uint32_t S = wave_spp(npix, p.spp, maxWavePaths);
  RenderLaunch L = prepare(ctx, c, p, d_frame, S);
  R2_CUDA(cudaMemsetAsync(ctx.bound.get(), 0, sizeof(unsigned int), s));
  R2_CUDA(cudaMemsetAsync(ctx.sampleDev.get(), 0, sizeof(uint32_t), s));
  R2_CUDA(cudaMemsetAsync(d_frame, 0, sizeof(float) * 3 * (size_t)npix, s));
  prepare_render_launches();  // occupancy queries stay outside the capture
  // one wave (reading its first sample index from the device counter, which
  // its last node advances), captured once and replayed spp / S times
  cudaStream_t cap = nullptr;
  R2_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  struct Guard {
    cudaStream_t s;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~Guard() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(s);
    }
  } guard{cap};
  R2_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  try {
    launch_render_wave(L, wave_blocks(npix * S), cap, nullptr);
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(cap, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  R2_CUDA(cudaStreamEndCapture(cap, &guard.g));
  R2_CUDA(cudaGraphInstantiate(&guard.e, guard.g, 0));
  for (uint32_t smp = 0; smp < p.spp; smp += S) R2_CUDA(cudaGraphLaunch(guard.e, s));
  // the executable graph may be destroyed while its launches are pending
}

RenderLaunch RenderScene::prepare(RenderContext& ctx, const r2_camera& c, const r2_render_params& p, float* d_frame,
                                  uint32_t waveSpp) {
  check_params(c, p, d_frame);
  R2_REQUIRE(committed_, R2_ERR_INVALID_ARGUMENT, "scene not committed");
  R2_REQUIRE(waveSpp >= 1 && p.spp % waveSpp == 0, R2_ERR_INVALID_ARGUMENT, "samples per wave must divide spp");
  ctx.ensure(c.width * c.height * waveSpp, !media_.empty());
  RenderLaunch L = make_launch(ctx, c, p, d_frame, waveSpp);
  L.sampleDev = ctx.sampleDev.get();
  return L;
}

void RenderScene::set_tuning(const r2_render_tuning& t) {
  R2_REQUIRE(t.track_steps <= 1024 && t.trav_refill <= 32 && t.wave_paths < (1u << 31) &&
                 t.media_rounds <= kMaxMediaRounds && t.track_blocks <= 64 &&
                 t.track_limit <= (uint32_t)kMaxTrackingSteps && t.top_nodes <= kMaxTopNodes && t.sort_rays <= 1,
             R2_ERR_INVALID_ARGUMENT,
             "tuning out of range (track_steps <= 1024, trav_refill <= 32, wave_paths < 2^31, media_rounds <= 32, "
             "track_blocks <= 64, track_limit <= 2^20, top_nodes <= 256, sort_rays <= 1)");
  tuning_ = t;
}

r2_render_tuning RenderScene::autotune(const r2_camera& c, const r2_render_params& p) {
  R2_REQUIRE(c.width > 0 && c.height > 0 && (uint64_t)c.width * c.height < (1ull << 31), R2_ERR_INVALID_ARGUMENT,
             "frame size out of range");
  const uint32_t npix = c.width * c.height;
  DBuf<float> frame((size_t)npix * 3);  // the tuner's own frame
  check_params(c, p, frame.get());
  if (!committed_) commit();
  RenderContext& ctx = ctx_;
  cudaStream_t s = ctx.stream;
  prepare_render_launches();
  const r2_render_tuning saved = tuning_;
  // milliseconds per path of the frame's first wave under tuning t, the faster of two runs
  auto time_wave = [&](const r2_render_tuning& t) {
    tuning_ = t;
    const uint32_t S = wave_spp(npix, p.spp);
    RenderLaunch L = prepare(ctx, c, p, frame.get(), S);
    L.sampleDev = nullptr;
    L.sample = 0;
    float best = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      R2_CUDA(cudaEventRecord(ctx.ev0, s));
      launch_render_wave(L, wave_blocks(npix * S), s, nullptr);
      R2_CUDA(cudaEventRecord(ctx.ev1, s));
      R2_CUDA(cudaEventSynchronize(ctx.ev1));
      float ms = 0.0f;
      R2_CUDA(cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1));
      best = std::min(best, ms);
    }
    return best / ((float)S * (float)npix);
  };
  r2_render_tuning cur{kDefaultTrackSteps, kDefaultTravVisits, kDefaultTravRefill, kDefaultWavePaths,
                       kDefaultMediaRounds, 0, saved.track_limit, 0, 0};  // the step bound is kept, never tuned
  try {
    R2_CUDA(cudaMemsetAsync(ctx.bound.get(), 0, sizeof(unsigned int), s));
    time_wave(cur);  // warm-up
    float curT = time_wave(cur);
    auto sweep = [&](uint32_t r2_render_tuning::*field, const uint32_t* cand, int n) {
      const r2_render_tuning base = cur;
      for (int i = 0; i < n; ++i) {
        r2_render_tuning t = base;
        t.*field = cand[i];
        if (field == &r2_render_tuning::wave_paths) {  // skip settings that give the same waves
          tuning_ = t;
          const uint32_t S = wave_spp(npix, p.spp);
          tuning_ = cur;
          if (S == wave_spp(npix, p.spp)) continue;
        }
        const float ms = time_wave(t);
        if (ms < curT * 0.98f) {
          cur = t;
          curT = ms;
        }
      }
    };
    static const uint32_t wavePaths[] = {1u << 20, 1u << 21, 1u << 23, 1u << 24};
    static const uint32_t refills[] = {2, 4, 16, 32};
    static const uint32_t visits[] = {8, 16, 64, 256};
    static const uint32_t steps[] = {2, 4, 16, 32};
    static const uint32_t rounds[] = {1, 4, 8, 16};
    static const uint32_t trackBlocks[] = {2, 3, 4, 6};
    static const uint32_t topNodes[] = {64, 128, 256};
    static const uint32_t sortRays[] = {1};
    sweep(&r2_render_tuning::wave_paths, wavePaths, 4);
    if (media_.empty()) {  // the persistent surface traversals run in scenes without media
      sweep(&r2_render_tuning::trav_refill, refills, 4);
      sweep(&r2_render_tuning::trav_visits, visits, 4);
      sweep(&r2_render_tuning::top_nodes, topNodes, 3);
      sweep(&r2_render_tuning::sort_rays, sortRays, 1);
    } else {
      sweep(&r2_render_tuning::media_rounds, rounds, 4);
      sweep(&r2_render_tuning::track_steps, steps, 4);
      sweep(&r2_render_tuning::track_blocks, trackBlocks, 4);
    }
  } catch (...) {
    tuning_ = saved;
    throw;
  }
  tuning_ = cur;
  return cur;
}

RenderBatch::RenderBatch(const std::vector<RenderScene*>& scenes, const std::vector<r2_camera>& cams,
                         const std::vector<r2_render_params>& params, const std::vector<float*>& frames) {
  const size_t n = scenes.size();
  R2_REQUIRE(n > 0 && cams.size() == n && params.size() == n && frames.size() == n, R2_ERR_INVALID_ARGUMENT,
             "batch arrays must have one entry per frame");
  spp_ = params[0].spp;
  std::vector<RenderLaunch> Ls;
  for (size_t i = 0; i < n; ++i) {
    R2_REQUIRE(scenes[i], R2_ERR_INVALID_ARGUMENT, "null scene in batch");
    R2_REQUIRE(params[i].spp == spp_, R2_ERR_INVALID_ARGUMENT, "all frames of a batch share the sample count");
    ctx_.emplace_back(new RenderContext());
    // one sample per wave: the batch's frames together fill the GPU
    Ls.push_back(scenes[i]->prepare(*ctx_.back(), cams[i], params[i], frames[i], 1));
    frames_.push_back(frames[i]);
    npix_.push_back((size_t)cams[i].width * cams[i].height);
  }
  prepare_render_launches();  // occupancy queries stay outside the capture
  R2_CUDA(cudaEventCreate(&ev0_));
  R2_CUDA(cudaEventCreate(&ev1_));
  // one wave of every frame: the capture stream forks into the contexts'
  // streams (each frame a branch of its own) and joins them again
  cudaStream_t cap = nullptr;
  R2_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  std::vector<cudaEvent_t> evs(n + 1, nullptr);
  struct Guard {
    cudaStream_t s;
    std::vector<cudaEvent_t>& evs;
    ~Guard() {
      for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
      cudaStreamDestroy(s);
    }
  } guard{cap, evs};
  for (auto& e : evs) R2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  R2_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  try {
    R2_CUDA(cudaEventRecord(evs[n], cap));
    for (size_t i = 0; i < n; ++i) {
      cudaStream_t b = ctx_[i]->stream;
      R2_CUDA(cudaStreamWaitEvent(b, evs[n], 0));
      launch_render_wave(Ls[i], wave_blocks((uint32_t)npix_[i]), b, nullptr);
      R2_CUDA(cudaEventRecord(evs[i], b));
      R2_CUDA(cudaStreamWaitEvent(cap, evs[i], 0));
    }
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(cap, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  R2_CUDA(cudaStreamEndCapture(cap, &graph_));
  R2_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
}

RenderBatch::~RenderBatch() {
  if (ev1_) cudaEventSynchronize(ev1_);  // the last run's samples, before the buffers go
  if (exec_) cudaGraphExecDestroy(exec_);
  if (graph_) cudaGraphDestroy(graph_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
}

double RenderBatch::run(cudaStream_t s, bool timing) {
  for (size_t i = 0; i < ctx_.size(); ++i) {
    R2_CUDA(cudaMemsetAsync(ctx_[i]->bound.get(), 0, sizeof(unsigned int), s));
    R2_CUDA(cudaMemsetAsync(ctx_[i]->sampleDev.get(), 0, sizeof(uint32_t), s));
    R2_CUDA(cudaMemsetAsync(frames_[i], 0, sizeof(float) * 3 * npix_[i], s));
  }
  R2_CUDA(cudaEventRecord(ev0_, s));
  for (uint32_t smp = 0; smp < spp_; ++smp) R2_CUDA(cudaGraphLaunch(exec_, s));
  R2_CUDA(cudaEventRecord(ev1_, s));
  if (!timing) return 0.0;
  R2_CUDA(cudaEventSynchronize(ev1_));
  float ms = 0.0f;
  R2_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  return ms;
}

uint32_t RenderBatch::bound_hits(cudaStream_t s) {
  std::vector<unsigned int> b(ctx_.size(), 0);
  for (size_t i = 0; i < ctx_.size(); ++i) ctx_[i]->bound.download(&b[i], 1, s);
  R2_CUDA(cudaStreamSynchronize(s));
  uint32_t t = 0;
  for (unsigned int v : b) t += v;
  return t;
}

}  // namespace r2
