// Host side of the path tracer: scene assembly (meshes flattened to world
// space, analytic shapes, media, environment map with the reference's
// distributions), camera setup, per-render state and the per-sample wave loop.
#pragma once
#include <map>
#include <string>
#include <memory>
#include <vector>

#include "medium_host.h"
#include "render.cuh"
#include "texture_host.h"

namespace r2 {

// CCamera (raytracer/src/camera/camera.cu:20-37): 10 um pixels, near plane
// from the horizontal field of view, view matrix glm::lookAt.
Camera make_camera(const r2_camera& c);

// Environment map distributions built exactly like CEnvironmentMap
// (src/scene/environmentmap.cu:11-29) and CDistribution1D/2D
// (src/sampling/distribution_1d.cu:6-39, distribution_2d.cu:7-14, .hpp:59-71).
struct EnvHost {
  int W = 0, H = 0;
  std::vector<float4> tex;
  std::vector<float> margFunc, margCdf, rowFunc, rowCdf, rowFuncInt;
  float margFuncInt = 0.0f;
};
void build_env(const float* rgb, int W, int H, EnvHost* e);

// The state of one render in flight: wave buffers (grown on demand), the
// device sample counter of captured waves, the loop-bound counter, statistics
// buffers and timers.  Renders that run concurrently use separate contexts.
class RenderContext {
 public:
  RenderContext();
  ~RenderContext();
  RenderContext(const RenderContext&) = delete;
  RenderContext& operator=(const RenderContext&) = delete;

  // Buffers for at least npix paths (media: the tracking-round state too),
  // grown to a power of two so that renders of varying size reallocate rarely.
  void ensure(uint32_t npix, bool media);
  void fill(PathState* st) const;
  // Device bytes a render of npix paths needs (buffers as ensure grows them + frame).
  static size_t bytes_for(uint32_t npix, bool media);
  static uint32_t capacity_for(uint32_t npix);
  // Paths and shadow rays of the last render that a loop bound ended (waits for s).
  uint32_t bound_hits(cudaStream_t s);

  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DBuf<unsigned int> bound;
  DBuf<uint32_t> sampleDev;
  DBuf<unsigned long long> statBuf;
  std::unique_ptr<WaveTimer> timer;

 private:
  uint32_t cap_ = 0, mediaCap_ = 0;
  DBuf<float4> rayO_, rayD_, T_, L_, hit_, shO_, shD_, shPre_, shT_;
  DBuf<uint32_t> q0_, q1_, qh_, qs_, counts_, sortBins_;
  DBuf<float> shTr_;
  DBuf<float2> shX_, evD_;
  DBuf<float4> evA_, evB_, evC_;
  DBuf<uint32_t> mc_, pj_, rl0_, rl1_, sl0_, sl1_, cl_;
  DBuf<float4> jO_, jD_, swP_;
  DBuf<uint2> jM_;
  DBuf<int2> swM_;
};

class RenderScene {
 public:
  RenderScene();
  ~RenderScene();
  RenderScene(const RenderScene&) = delete;
  RenderScene& operator=(const RenderScene&) = delete;

  // uv (nullable): 2 texture coordinates per vertex; maps (nullable): the
  // material's texture files (unused without texture coordinates).
  void add_mesh(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* nrm,
                const r2_material& mat, const float* modelToWorld, uint32_t mask, const float* uv = nullptr,
                const r2_material_maps* maps = nullptr);
  // Two-level scenes (the reference's GAS per mesh asset and IAS over scene
  // objects, scene.cu:188-256): a mesh kept in model space with its own BVH,
  // placed by any number of instances.  Returns the asset's index.
  uint32_t add_mesh_asset(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* nrm,
                          const r2_material& mat, const float* uv = nullptr, const r2_material_maps* maps = nullptr);
  void add_mesh_instance(uint32_t asset, const float* modelToWorld, uint32_t mask);
  void add_shape(int type, const float* center, float radius, const float* normal, const r2_material& mat,
                 uint32_t mask);
  void set_envmap(const float* rgb, int W, int H);
  // Medium of a filtered LOD: <path>.nvdb + <path>.brickgrid placed with T(pos) R(orientation) S(scaling).
  void add_medium(const char* path, const float* sigmaA, const float* sigmaS, const float* pos,
                  const float* orientation, const float* scaling, uint32_t mask, bool hg = false, float g = 0.0f);
  void commit();
  // Rebuilds the triangle BVH from the device-resident triangles and
  // re-gathers the per-triangle shading data in the new order, on stream s
  // (the scene's own when null): the per-frame BVH build of a scene whose
  // geometry stays on the device.  Same tree as the commit's; allocates
  // nothing after the first build; waits for the build's end.
  void rebuild(cudaStream_t s);
  // The surface BVH: inner nodes, height and the kernels its last build launched
  // (BVH builds, shading gathers and, two-level, the node copies).
  uint32_t bvh_nodes() const { return bvhNodes_; }
  uint32_t bvh_height() const { return bvhHeight_; }
  int bvh_build_launches() const { return buildLaunches_; }
  bool two_level() const { return !meshInstances_.empty(); }
  // Replaces the world-space vertex positions (and normals when given) of the
  // committed scene from host memory, on stream s (the scene's own when null).
  void set_vertices(const float* pos, const float* nrm, uint32_t nverts, cudaStream_t s);
  // Device frame of r2_render_host, kept between calls.
  DBuf<float>& host_frame() { return hostFrame_; }
  bool committed() const { return committed_; }
  bool has_media() const { return !media_.empty(); }
  // One frame: spp / wave_spp waves accumulated into d_frame (W*H*3 floats,
  // cleared here), on the scene's own context.
  void render(const r2_camera& cam, const r2_render_params& p, float* d_frame, cudaStream_t s, double* stats);
  // The same frame on a caller's context and stream, one wave captured as a
  // CUDA graph and replayed spp / wave_spp times (the scene must be committed).
  // maxWavePaths (0: the tuning's) caps the paths per wave.
  void render_graph(RenderContext& ctx, const r2_camera& cam, const r2_render_params& p, float* d_frame,
                    cudaStream_t s, uint32_t maxWavePaths = 0);
  // The launch description of a frame on ctx with waveSpp samples per wave
  // (a divisor of p.spp; the context's buffers grown to fit).
  RenderLaunch prepare(RenderContext& ctx, const r2_camera& cam, const r2_render_params& p, float* d_frame,
                       uint32_t waveSpp);
  // Samples per wave of a frame: the largest divisor of spp whose wave stays
  // within the tuning's paths per wave, or maxWavePaths if smaller and nonzero
  // (at least one sample).
  uint32_t wave_spp(uint32_t npix, uint32_t spp, uint32_t maxWavePaths = 0) const;
  // Launch tuning (0 fields: the defaults) and the autotuner that sets it.
  void set_tuning(const r2_render_tuning& t);
  r2_render_tuning tuning() const { return tuning_; }
  r2_render_tuning autotune(const r2_camera& cam, const r2_render_params& p);
  // Paths and shadow rays of the last render() that a loop bound ended (waits for the stream).
  uint32_t bound_hits(cudaStream_t s) { return ctx_.bound_hits(s ? s : ctx_.stream); }
  cudaStream_t stream() const { return ctx_.stream; }
  uint32_t ntris() const { return (uint32_t)(hIdx_.size() / 3); }
  const DeviceBvh& bvh() const { return bvh_; }

 private:
  RenderLaunch make_launch(const RenderContext& ctx, const r2_camera& c, const r2_render_params& p, float* d_frame,
                           uint32_t waveSpp);
  static void check_params(const r2_camera& c, const r2_render_params& p, const float* d_frame);
  RenderContext ctx_;
  bool committed_ = false;
  std::vector<float> hPos_, hNrm_, hUV_;
  bool anyUV_ = false;
  TextureSet textures_;
  DBuf<float2> triUV_;
  DBuf<int> triAlpha_;
  DBuf<float4> texels_;
  DBuf<TexInfo> texInfo_;
  std::vector<uint32_t> hIdx_, hTriMat_;
  std::vector<Material> hMats_;
  std::vector<Shape> hShapes_;
  // media loaded once per path (the first load's coefficients, like
  // CAssetManager::loadMedium, asset_manager.cu:114-137) and their instances
  struct MediumInstance {
    MediumHost* medium;
    V3 pos, orientation, scaling;
  };
  std::map<std::string, std::unique_ptr<MediumHost>> mediaByPath_;
  std::vector<MediumInstance> media_;
  DBuf<MediumView> mediaViews_;
  DeviceBvh mediaBvh_;
  EnvHost env_;
  DeviceBvh bvh_;
  BvhBuilder builder_;
  // two-level scenes: mesh assets in model space, their instances, the top
  // level over the instances' world boxes and the concatenated node and
  // triangle arrays (top level, then the world-space meshes, then the assets)
  struct MeshAsset {
    std::vector<float> pos, nrm, uv;
    std::vector<uint32_t> idx;
    uint32_t matId = 0;
    bool hasUV = false;
    DBuf<float> dPos, dNrm, dUV;
    DBuf<uint32_t> dIdx, dTriMat;
    DBuf<int> dAlphaIn;
    DeviceBvh bvh;
  };
  struct MeshInstanceHost {
    uint32_t asset;
    M43 m2w;
  };
  std::vector<std::unique_ptr<MeshAsset>> assets_;
  std::vector<MeshInstanceHost> meshInstances_;
  DeviceBvh tlas_;
  DBuf<BvhNode> gNodes_;
  DBuf<float4> gTris_;
  DBuf<BvhInstance> dInst_;
  DBuf<int> dInstCode_;
  DBuf<float4> dInstO2W_, dInstLo_, dInstHi_;
  uint32_t bvhNodes_ = 0, bvhHeight_ = 0;
  int buildLaunches_ = 0;
  bool anyAlpha_ = false;
  void upload_assets(cudaStream_t s);
  void build_two_level(cudaStream_t s);
  // device-resident triangle inputs in scene order (kept for rebuilds)
  DBuf<float> dPos_, dNrm_, dUV_;
  DBuf<uint32_t> dIdx_, dTriMatIn_;
  DBuf<int> dTriAlphaIn_;
  DBuf<float4> triN_;
  DBuf<uint32_t> triMat_;
  DBuf<Material> mats_;
  DBuf<Shape> shapes_;
  DBuf<float4> envTex_;
  DBuf<float> envBuf_;
  DBuf<float> hostFrame_;
  SceneView view_;
  r2_render_tuning tuning_{0, 0, 0, 0, 0, 0, 0, 0, 0};  // 0 fields: the kernels' defaults
};

// Frames of several committed scenes rendered by one captured CUDA graph: the
// graph holds one wave of every scene, each on its own branch (forked capture
// streams), and is replayed once per sample (waves of one sample: the frames
// together fill the GPU).  Frames, cameras and parameters
// are fixed at construction; all entries share the sample count.
class RenderBatch {
 public:
  RenderBatch(const std::vector<RenderScene*>& scenes, const std::vector<r2_camera>& cams,
              const std::vector<r2_render_params>& params, const std::vector<float*>& frames);
  ~RenderBatch();
  RenderBatch(const RenderBatch&) = delete;
  RenderBatch& operator=(const RenderBatch&) = delete;
  // All frames (cleared first); returns the device milliseconds between the
  // first clear and the last wave when timing is requested (waits).
  double run(cudaStream_t s, bool timing);
  // Paths and shadow rays of the last run that a loop bound ended (waits for s).
  uint32_t bound_hits(cudaStream_t s);

 private:
  std::vector<std::unique_ptr<RenderContext>> ctx_;
  std::vector<float*> frames_;
  std::vector<size_t> npix_;
  uint32_t spp_ = 0;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
};

}  // namespace r2
