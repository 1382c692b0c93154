// Device-resident filter scene: the FILTER-masked mesh of one object, its BVH,
// per-triangle shading data and materials.  Mirrors the state CFilter keeps
// between LODs (raytracer/filter.hpp:13-44).
#pragma once
#include "bvh_build.cuh"
#include "texture_host.h"

namespace r2 {

r2_filter_grid setup_grid(V3 minWorld, V3 maxWorld, const M43& worldToModel, float voxelSize);
void world_aabb(V3 mlo, V3 mhi, const M43& modelToWorld, V3* wlo, V3* whi);

class FilterScene {
 public:
  // uvs (nullable): 2 texture coordinates per vertex; maps (nullable): the
  // texture files of each material (nmaterials entries).
  FilterScene(const float* positions, uint32_t nverts, const uint32_t* indices, uint32_t ntris,
              const float* normals, const r2_material* materials, uint32_t nmaterials,
              const uint32_t* triMaterial, const float* modelToWorld, const float* uvs = nullptr,
              const r2_material_maps* maps = nullptr);
  ~FilterScene();
  FilterScene(const FilterScene&) = delete;
  FilterScene& operator=(const FilterScene&) = delete;

  r2_filter_grid grid(float voxelSize) const;
  // One LOD.  d_work/d_counters (nullable) override the scene-owned work list
  // (nx*ny*nz words) and counters (2 words).  d_ops (nullable, 3 zeroed words)
  // selects the counting build of the sampling kernel, which adds the rays
  // traced, inner nodes visited and triangles tested.
  // d_eig (nullable): 12 floats per voxel, the FP64 eigendecomposition of the mean S.
  void run(const r2_filter_grid& g, const r2_filter_params& p, uint32_t lod, r2_voxel* d_out,
           float* d_wide, uint16_t* d_fp16, cudaStream_t s, double* stats,
           uint32_t* d_work = nullptr, uint32_t* d_counters = nullptr, unsigned long long* d_ops = nullptr,
           float* d_eig = nullptr);

  const DeviceBvh& bvh() const { return bvh_; }
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }
  V3 worldLo() const { return worldLo_; }
  V3 worldHi() const { return worldHi_; }

 private:
  cudaStream_t stream_ = nullptr;
  int device_ = 0;  // the device current when the scene was created; its buffers live there
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  M43 modelToWorld_, worldToModel_;
  V3 modelLo_, modelHi_, worldLo_, worldHi_;
  uint32_t ntris_ = 0;
  DeviceBvh bvh_;
  DBuf<float4> triN_;
  DBuf<uint32_t> triMat_;
  DBuf<r2_material> mats_;
  DBuf<uint32_t> work_;
  DBuf<uint32_t> counters_;
  TextureSet textures_;
  DBuf<float2> triUV_;
  DBuf<int> triAlpha_;
  DBuf<float4> texels_;
  DBuf<TexInfo> texInfo_;
  DBuf<int4> matTex_;
};

}  // namespace r2
