// Host side of the wavefront path tracer.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

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

RenderScene::RenderScene() {
  R2_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  R2_CUDA(cudaEventCreate(&ev0_));
  R2_CUDA(cudaEventCreate(&ev1_));
  memset(&view_, 0, sizeof(view_));
  if (const char* e = getenv("R2_TRACK_STEPS")) trackSteps_ = (uint32_t)std::max(1l, std::min(1024l, atol(e)));
}

RenderScene::~RenderScene() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (timer_)
    for (int i = 0; i < WaveTimer::kMax; ++i) cudaEventDestroy(timer_->ev[i]);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

void RenderScene::add_mesh(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* nrm,
                           const r2_material& mat, const float* m2w, uint32_t mask) {
  R2_REQUIRE(pos && idx && nrm && m2w, R2_ERR_INVALID_ARGUMENT, "null mesh array");
  R2_REQUIRE(nverts > 0 && ntris > 0, R2_ERR_INVALID_ARGUMENT, "empty mesh");
  // render rays carry visibility mask 255 (device_scene.hpp:17): every object
  // with a nonzero mask is visible, FILTER-only ones included
  if (mask == 0) return;
  M43 M = m43_from_floats(m2w);
  uint32_t base = (uint32_t)(hPos_.size() / 3);
  uint32_t matId = (uint32_t)hMats_.size();
  hMats_.push_back(make_material(mat));
  for (uint32_t v = 0; v < nverts; ++v) {
    V3 p = xform_point(M, v3(pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]));
    V3 n = xform_vector(M, v3(nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2]));
    hPos_.push_back(p.x); hPos_.push_back(p.y); hPos_.push_back(p.z);
    hNrm_.push_back(n.x); hNrm_.push_back(n.y); hNrm_.push_back(n.z);
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
  R2_REQUIRE(media_.size() < 4096, R2_ERR_UNSUPPORTED, "too many media in one scene");
  std::unique_ptr<MediumHost> m = load_medium(path, sigmaA, sigmaS, v3(pos[0], pos[1], pos[2]),
                                              v3(orientation[0], orientation[1], orientation[2]),
                                              v3(scaling[0], scaling[1], scaling[2]), hg, g);
  if (mask == 0) return;  // render rays (mask 255) never see objects with mask NONE
  media_.push_back(std::move(m));
  committed_ = false;
}

void RenderScene::commit() {
  R2_REQUIRE(env_.W > 0, R2_ERR_INVALID_CONFIG, "scene has no environment map");
  cudaStream_t s = stream_;
  uint32_t nt = (uint32_t)(hIdx_.size() / 3);
  memset(&view_, 0, sizeof(view_));
  if (nt > 0) {
    DBuf<float> dpos;
    DBuf<uint32_t> didx;
    dpos.upload(hPos_.data(), hPos_.size(), s);
    didx.upload(hIdx_.data(), hIdx_.size(), s);
    build_bvh(dpos.get(), didx.get(), nt, &bvh_, s);
    std::vector<uint32_t> order(nt);
    bvh_.order.download(order.data(), nt, s);
    R2_CUDA(cudaStreamSynchronize(s));
    std::vector<float4> triN((size_t)3 * nt);
    std::vector<uint32_t> triMat(nt);
    for (uint32_t i = 0; i < nt; ++i) {
      uint32_t p = order[i];
      for (int k = 0; k < 3; ++k) {
        uint32_t v = hIdx_[3 * p + k];
        triN[3 * i + k] = make_float4(hNrm_[3 * v], hNrm_[3 * v + 1], hNrm_[3 * v + 2], 0.0f);
      }
      triMat[i] = hTriMat_[p];
    }
    triN_.upload(triN.data(), triN.size(), s);
    triMat_.upload(triMat.data(), triMat.size(), s);
    view_.bvh = bvh_.view();
    view_.triN = triN_.get();
    view_.triMat = triMat_.get();
    view_.hasTris = 1;
  }
  mats_.upload(hMats_.data(), hMats_.size(), s);
  view_.mats = mats_.get();
  if (!hShapes_.empty()) shapes_.upload(hShapes_.data(), hShapes_.size(), s);
  view_.shapes = shapes_.get();
  view_.nshapes = (int)hShapes_.size();
  if (!media_.empty()) {
    std::vector<MediumView> mv;
    for (auto& m : media_) {
      m->upload(s);
      mv.push_back(m->view);
    }
    mediaViews_.upload(mv.data(), mv.size(), s);
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

void RenderScene::ensure_state(uint32_t n) {
  if (n > cap_) {
    rayO_.alloc(n); rayD_.alloc(n); T_.alloc(n); L_.alloc(n); hit_.alloc(n);
    shO_.alloc(2 * (size_t)n); shD_.alloc(2 * (size_t)n); shPre_.alloc(2 * (size_t)n); shT_.alloc(n);
    q0_.alloc(n); q1_.alloc(n); shTr_.alloc(2 * (size_t)n);
    counts_.alloc(64);
    bound_.alloc(1);
    cap_ = n;
  }
  if (!media_.empty() && n > mediaCap_) {
    shX_.alloc(2 * (size_t)n);
    evA_.alloc(n); evB_.alloc(n); evC_.alloc(n); evD_.alloc(n);
    mc_.alloc(16 * 64);
    pj_.alloc(n); rl0_.alloc(n); rl1_.alloc(n); cl_.alloc(n);
    sl0_.alloc(2 * (size_t)n); sl1_.alloc(2 * (size_t)n);
    jO_.alloc(2 * (size_t)n); jD_.alloc(2 * (size_t)n); jM_.alloc(2 * (size_t)n);
    swP_.alloc(2 * (size_t)n); swM_.alloc(2 * (size_t)n);
    mediaCap_ = n;
  }
}

void RenderScene::render(const r2_camera& c, const r2_render_params& p, float* d_frame, cudaStream_t s,
                         double* stats) {
  R2_REQUIRE(d_frame, R2_ERR_INVALID_ARGUMENT, "null frame");
  R2_REQUIRE(c.width > 0 && c.height > 0, R2_ERR_INVALID_ARGUMENT, "empty frame");
  R2_REQUIRE(p.spp > 0, R2_ERR_INVALID_ARGUMENT, "spp must be positive");
  R2_REQUIRE(p.max_depth > 0 && p.max_depth <= 60, R2_ERR_UNSUPPORTED, "max_depth must be in [1, 60]");
  R2_REQUIRE((p.flags & ~R2_RENDER_BRICK_GRID) == 0, R2_ERR_INVALID_ARGUMENT, "unknown render flags");
  if (!committed_) commit();
  if (!s) s = stream_;
  const uint32_t npix = c.width * c.height;
  ensure_state(npix);
  RenderLaunch L;
  memset(&L, 0, sizeof(L));
  L.scene = view_;
  L.cam = make_camera(c);
  L.st.rayO = rayO_.get(); L.st.rayD = rayD_.get(); L.st.T = T_.get(); L.st.L = L_.get(); L.st.hit = hit_.get();
  L.st.q[0] = q0_.get(); L.st.q[1] = q1_.get(); L.st.counts = counts_.get();
  L.st.shO = shO_.get(); L.st.shD = shD_.get(); L.st.shPre = shPre_.get(); L.st.shT = shT_.get();
  L.st.shTr = shTr_.get();
  if (!media_.empty()) {
    L.st.shX = shX_.get();
    L.st.evA = evA_.get(); L.st.evB = evB_.get(); L.st.evC = evC_.get(); L.st.evD = evD_.get();
    L.st.mc = mc_.get(); L.st.pj = pj_.get();
    L.st.rl[0] = rl0_.get(); L.st.rl[1] = rl1_.get(); L.st.cl = cl_.get(); L.st.sl[0] = sl0_.get(); L.st.sl[1] = sl1_.get();
    L.st.jO = jO_.get(); L.st.jD = jD_.get(); L.st.jM = jM_.get();
    L.st.swP = swP_.get(); L.st.swM = swM_.get();
  }
  L.frame = d_frame;
  L.npix = npix;
  L.spp = p.spp;
  L.maxDepth = p.max_depth;
  L.seed = p.seed;
  L.dda = (p.flags & R2_RENDER_BRICK_GRID) ? 1u : 0u;
  L.trackSteps = trackSteps_;
  L.bound = bound_.get();
  R2_CUDA(cudaMemsetAsync(bound_.get(), 0, sizeof(unsigned int), s));
  int nblocks = std::max(1, std::min((int)((npix + 255) / 256), sm_count() * 8));
  R2_CUDA(cudaMemsetAsync(d_frame, 0, sizeof(float) * 3 * (size_t)npix, s));
  if (stats) {
    statBuf_.reserve(2);
    R2_CUDA(cudaMemsetAsync(statBuf_.get(), 0, 2 * sizeof(unsigned long long), s));
    L.stats = statBuf_.get();
    if (!timer_) {
      timer_.reset(new WaveTimer());
      for (int i = 0; i < WaveTimer::kMax; ++i) R2_CUDA(cudaEventCreate(&timer_->ev[i]));
    }
  }
  R2_CUDA(cudaEventRecord(ev0_, s));
  for (uint32_t smp = 0; smp < p.spp; ++smp) {
    L.sample = smp;
    // the middle wave of a frame is timed kernel by kernel when statistics are requested
    launch_render_wave(L, nblocks, s, (stats && smp == p.spp / 2) ? timer_.get() : nullptr);
  }
  R2_CUDA(cudaEventRecord(ev1_, s));
  if (stats) {
    R2_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0.0f;
    R2_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    unsigned long long cnt[2] = {0, 0};
    R2_CUDA(cudaMemcpy(cnt, statBuf_.get(), sizeof(cnt), cudaMemcpyDeviceToHost));
    double kms[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 1; i < timer_->n; ++i) {
      float d = 0.0f;
      R2_CUDA(cudaEventElapsedTime(&d, timer_->ev[i - 1], timer_->ev[i]));
      int k = timer_->kind[i];
      if (k >= 0 && k < 6) kms[k] += d;
    }
    stats[0] = (double)npix * p.spp;
    stats[1] = ms;
    stats[2] = (double)cnt[0];
    stats[3] = (double)cnt[1];
    for (int k = 1; k <= 4; ++k) stats[3 + k] = kms[k];  // one wave: extend, shade, shadow, accum
  }
}

uint32_t RenderScene::bound_hits(cudaStream_t s) {
  if (!bound_.get()) return 0;
  unsigned int b = 0;
  bound_.download(&b, 1, s ? s : stream_);
  R2_CUDA(cudaStreamSynchronize(s ? s : stream_));
  return b;
}

}  // namespace r2
