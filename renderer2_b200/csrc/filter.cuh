// SGGX mesh-to-volume filter: device kernels and their launch description.
#pragma once
#include "bvh_build.cuh"

namespace r2 {

constexpr uint32_t kFilterMaxSpv = 1024;  // per-voxel sample cap (reference: rayTs[1000])
constexpr int kWideFloats = 20;           // floats per voxel of the wide (pre-quantisation) output

// Everything the per-voxel kernels read.  Passed by value (kernel parameter
// space), so each launch is self-contained and graph-capturable.
struct FilterLaunch {
  M43 indexToWorld;   // mat4(modelToWorld) * mat4(indexToModel)
  M43 indexToModel;   // voxel index -> model space (COpenvdbBackend::setupGrid)
  M43 modelToWorld;   // grid model -> world (voxel centres, COpenvdbBackend::setupGrid)
  M43 objModelToWorld;  // the object's own transform (hit normals, shaders.optix.cu:106)
  M43 worldToModel;   // mean-normal transform back to model space
  int nx, ny, nz;
  V3 voxelSize;       // (worldBB.max - worldBB.min) / numVoxels
  uint32_t spv, iters, clip, seed, lod;
  float sigma_t, alpha;
  uint32_t project;          // FP64 eigendecomposition + projection of S (r2_filter_params::sggx_projection)
  float floor;               // relative eigenvalue floor of the projection
  BvhView bvh;
  const float4* triN;        // 3 per BVH-order triangle: model-space vertex normals
  const uint32_t* triMat;    // per BVH-order triangle: material index
  const r2_material* mats;
  r2_voxel* out;
  float* wide;               // nullable
  uint16_t* fp16;            // nullable
  float* eig;                // nullable: 12 floats per voxel, eigenvalues and eigenvectors of the mean S
  uint32_t* work;            // candidate voxel ids
  uint32_t* counters;        // [0] candidates, [1] queue head
  unsigned long long* ops;   // nullable: counting build, [0] rays, [1] inner nodes visited, [2] triangles tested
  // texture maps (nullable): 3 texture coordinates per BVH-order triangle, the
  // texels, and per material its {albedo, glossy, normal, opacity} texture (-1: none)
  const float2* triUV;
  const float4* texels;
  const TexInfo* texInfo;
  const int4* matTex;
};

// Host launchers.  `classify` writes the empty payload for voxels whose
// bounding sphere overlaps no triangle box and appends the others to the
// work list; `sample` is the persistent warp-per-voxel kernel.
void launch_filter_classify(const FilterLaunch& L, cudaStream_t s);
void launch_filter_sample(const FilterLaunch& L, cudaStream_t s);

}  // namespace r2
