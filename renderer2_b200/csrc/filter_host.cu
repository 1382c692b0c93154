// Host side of the filter: grid setup (COpenvdbBackend::init/setupGrid,
// raytracer/src/filtering/openvdb_backend.cpp:26-106 of the reference), the
// device-resident filter scene, and the per-LOD launch (CFilter::runFiltering,
// raytracer/filter.cu:74-123).
#include <algorithm>
#include <vector>

#include "filter.cuh"
#include "filter_host.h"
#include "filter_math.h"
#include "host_math.h"

namespace r2 {

// ceil(extent / voxelSize - CEIL_EPS) with CEIL_EPS = 0.001 (openvdb_backend.cpp:11, 62-63).
static int num_voxels_axis(float extent, float vs) {
  float f = extent / vs;
  return (int)ceilf(f - 0.001f);
}

r2_filter_grid setup_grid(V3 minWorld, V3 maxWorld, const M43& worldToModel43, float voxelSize) {
  r2_filter_grid g;
  memset(&g, 0, sizeof(g));
  V3 ext = maxWorld - minWorld;
  int nv[3] = {num_voxels_axis(ext.x, voxelSize), num_voxels_axis(ext.y, voxelSize),
               num_voxels_axis(ext.z, voxelSize)};
  for (int k = 0; k < 3; ++k) g.num_voxels[k] = nv[k];
  M4 worldToModel = m43_to_m4(worldToModel43);
  V3 invN = v3(1.0f / (float)nv[0], 1.0f / (float)nv[1], 1.0f / (float)nv[2]);
  M4 indexToModel = m4_mul(m4_mul(m4_mul(worldToModel, m4_translate(minWorld)), m4_scale(ext)), m4_scale(invN));
  M4 modelToIndex = m4_inverse(indexToModel);
  M4 modelToWorld = m4_inverse(worldToModel);
  M4 indexToWorld = m4_mul(modelToWorld, indexToModel);
  V3 a = m4_point(indexToWorld, v3(0.0f));
  V3 b = m4_point(indexToWorld, v3((float)nv[0], (float)nv[1], (float)nv[2]));
  V3 lo = vmin(a, b), hi = vmax(a, b);
  m43_to_floats(m4_to_m43(indexToModel), g.index_to_model);
  m43_to_floats(m4_to_m43(modelToIndex), g.model_to_index);
  m43_to_floats(m4_to_m43(modelToWorld), g.model_to_world);
  m43_to_floats(worldToModel43, g.world_to_model);
  g.world_bb_min[0] = lo.x; g.world_bb_min[1] = lo.y; g.world_bb_min[2] = lo.z;
  g.world_bb_max[0] = hi.x; g.world_bb_max[1] = hi.y; g.world_bb_max[2] = hi.z;
  g.voxel_size = voxelSize;
  return g;
}

// World-space vertices of the filter scene (the filter traces in world space);
// the same single-precision products and sums as the host's xform_point.
__global__ void k_world_points(const float* model, uint32_t n, M43 m, float* world) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const V3 w = xform_point(m, v3(model[3 * v], model[3 * v + 1], model[3 * v + 2]));
    world[3 * v] = w.x;
    world[3 * v + 1] = w.y;
    world[3 * v + 2] = w.z;
  }
}

// Per BVH-order triangle: its model-space vertex normals and its material
// (triMat null: material 0).
__global__ void k_order_normals(const uint32_t* order, const uint32_t* idx, const float* nrm, const uint32_t* triMat,
                                uint32_t n, float4* triN, uint32_t* triMatOut) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = order[i];
    for (int k = 0; k < 3; ++k) {
      const uint32_t v = idx[3 * p + k];
      triN[3 * i + k] = make_float4(nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2], 0.0f);
    }
    triMatOut[i] = triMat ? triMat[p] : 0u;
  }
}

static int grid_for(uint32_t n) {
  return (int)std::max<uint32_t>(1u, std::min<uint32_t>((n + 255) / 256, (uint32_t)sm_count() * 16));
}

// SAABB::transform (include/intersect/aabb.hpp:9-13): only the min and max
// corners are transformed.
void world_aabb(V3 mlo, V3 mhi, const M43& modelToWorld, V3* wlo, V3* whi) {
  V3 a = xform_point(modelToWorld, mlo), b = xform_point(modelToWorld, mhi);
  *wlo = vmin(a, b);
  *whi = vmax(a, b);
}

FilterScene::FilterScene(const float* positions, uint32_t nverts, const uint32_t* indices,
                         uint32_t ntris, const float* normals, const r2_material* materials,
                         uint32_t nmaterials, const uint32_t* triMaterial, const float* modelToWorld,
                         const float* uvs, const r2_material_maps* maps) {
  R2_REQUIRE(positions && indices && normals && materials, R2_ERR_INVALID_ARGUMENT, "null mesh array");
  R2_REQUIRE(nverts > 0 && ntris > 0, R2_ERR_INVALID_ARGUMENT, "empty mesh");
  R2_CUDA(cudaGetDevice(&device_));
  R2_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  modelToWorld_ = m43_from_floats(modelToWorld);
  worldToModel_ = m4_to_m43(m4_inverse(m43_to_m4(modelToWorld_)));
  // model bounds and argument checks on the host; the world-space vertices
  // (the filter traces in world space) and the per-triangle gathers on the device
  V3 lo = v3(INFINITY), hi = v3(-INFINITY);
  for (uint32_t v = 0; v < nverts; ++v) {
    const V3 p = v3(positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]);
    lo = vmin(lo, p);
    hi = vmax(hi, p);
  }
  for (size_t i = 0; i < (size_t)3 * ntris; ++i)
    R2_REQUIRE(indices[i] < nverts, R2_ERR_INVALID_ARGUMENT, "triangle index out of range");
  if (triMaterial)
    for (uint32_t i = 0; i < ntris; ++i)
      R2_REQUIRE(triMaterial[i] < nmaterials, R2_ERR_INVALID_ARGUMENT, "material index out of range");
  R2_REQUIRE(nmaterials > 0, R2_ERR_INVALID_ARGUMENT, "material index out of range");
  modelLo_ = lo;
  modelHi_ = hi;
  world_aabb(lo, hi, modelToWorld_, &worldLo_, &worldHi_);
  ntris_ = ntris;
  DBuf<float> dmodel, dpos, dnrm;
  DBuf<uint32_t> didx, dmat;
  dmodel.upload(positions, (size_t)3 * nverts, stream_);
  dpos.alloc((size_t)3 * nverts);
  k_world_points<<<grid_for(nverts), 256, 0, stream_>>>(dmodel.get(), nverts, modelToWorld_, dpos.get());
  R2_CUDA(cudaGetLastError());
  didx.upload(indices, (size_t)3 * ntris, stream_);
  build_bvh(dpos.get(), didx.get(), ntris, &bvh_, stream_, true);
  dnrm.upload(normals, (size_t)3 * nverts, stream_);
  if (triMaterial) dmat.upload(triMaterial, ntris, stream_);
  triN_.alloc((size_t)3 * ntris);
  triMat_.alloc(ntris);
  k_order_normals<<<grid_for(ntris), 256, 0, stream_>>>(bvh_.order.get(), didx.get(), dnrm.get(),
                                                        triMaterial ? dmat.get() : nullptr, ntris, triN_.get(),
                                                        triMat_.get());
  R2_CUDA(cudaGetLastError());
  mats_.upload(materials, nmaterials, stream_);
  if (maps && uvs) {  // texture maps per material (CMaterial(aiMaterial*), material.cu:110-143)
    std::vector<uint32_t> order(ntris);
    bvh_.order.download(order.data(), ntris, stream_);
    R2_CUDA(cudaStreamSynchronize(stream_));
    std::vector<int4> mt(nmaterials);
    bool anyTex = false, anyAlpha = false;
    for (uint32_t m = 0; m < nmaterials; ++m) {
      int t[4];
      textures_.material_maps(materials[m], &maps[m], t);
      mt[m] = make_int4(t[0], t[1], t[2], t[3]);
      anyTex = anyTex || t[0] >= 0 || t[1] >= 0 || t[2] >= 0 || t[3] >= 0;
      anyAlpha = anyAlpha || t[3] >= 0;
    }
    if (anyTex) {
      std::vector<float2> triUV((size_t)3 * ntris);
      std::vector<int> triAlpha(ntris);
      for (uint32_t i = 0; i < ntris; ++i) {
        const uint32_t p = order[i];
        for (int k = 0; k < 3; ++k) {
          const uint32_t v = indices[3 * p + k];
          triUV[3 * i + k] = make_float2(uvs[2 * v], uvs[2 * v + 1]);
        }
        triAlpha[i] = mt[triMaterial ? triMaterial[p] : 0u].w;
      }
      triUV_.upload(triUV.data(), triUV.size(), stream_);
      matTex_.upload(mt.data(), mt.size(), stream_);
      textures_.upload(&texels_, &texInfo_, stream_);
      if (anyAlpha) triAlpha_.upload(triAlpha.data(), triAlpha.size(), stream_);
    }
  }
  counters_.alloc(2);
  R2_CUDA(cudaEventCreate(&ev0_));
  R2_CUDA(cudaEventCreate(&ev1_));
  R2_CUDA(cudaStreamSynchronize(stream_));
}

FilterScene::~FilterScene() {
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

r2_filter_grid FilterScene::grid(float voxelSize) const {
  R2_REQUIRE(voxelSize > 0.0f, R2_ERR_INVALID_ARGUMENT, "voxel size must be positive");
  return setup_grid(worldLo_, worldHi_, worldToModel_, voxelSize);
}

void FilterScene::run(const r2_filter_grid& g, const r2_filter_params& p, uint32_t lod, r2_voxel* d_out,
                      float* d_wide, uint16_t* d_fp16, cudaStream_t s, double* stats,
                      uint32_t* d_work, uint32_t* d_counters, unsigned long long* d_ops, float* d_eig) {
  R2_REQUIRE(d_out, R2_ERR_INVALID_ARGUMENT, "null output");
  R2_REQUIRE(p.sggx_projection <= 1u && p.sggx_floor >= 0.0f && p.sggx_floor < 1.0f, R2_ERR_INVALID_ARGUMENT,
             "sggx_projection must be 0 or 1 and sggx_floor in [0, 1)");
  R2_REQUIRE(p.samples_per_voxel >= 1 && p.samples_per_voxel <= kFilterMaxSpv, R2_ERR_UNSUPPORTED,
             "samples_per_voxel must be in [1, 1024]");
  R2_REQUIRE(p.sigma_t > 0.0f, R2_ERR_INVALID_ARGUMENT, "sigma_t must be positive");
  for (int k = 0; k < 3; ++k)
    R2_REQUIRE(g.num_voxels[k] > 0, R2_ERR_INVALID_ARGUMENT, "grid without voxels");
  const size_t nvox = (size_t)g.num_voxels[0] * g.num_voxels[1] * g.num_voxels[2];
  R2_REQUIRE(nvox < (1ull << 32), R2_ERR_UNSUPPORTED, "grid larger than 2^32 voxels");
  if (!s) s = stream_;
  FilterLaunch L;
  memset(&L, 0, sizeof(L));
  M43 indexToModel = m43_from_floats(g.index_to_model);
  M43 modelToWorld = m43_from_floats(g.model_to_world);
  L.indexToWorld = m4_to_m43(m4_mul(m43_to_m4(modelToWorld), m43_to_m4(indexToModel)));
  L.indexToModel = indexToModel;
  L.modelToWorld = modelToWorld;
  L.objModelToWorld = modelToWorld_;
  L.worldToModel = m43_from_floats(g.world_to_model);
  L.nx = g.num_voxels[0];
  L.ny = g.num_voxels[1];
  L.nz = g.num_voxels[2];
  V3 wlo = v3(g.world_bb_min[0], g.world_bb_min[1], g.world_bb_min[2]);
  V3 whi = v3(g.world_bb_max[0], g.world_bb_max[1], g.world_bb_max[2]);
  L.voxelSize = (whi - wlo) / v3((float)L.nx, (float)L.ny, (float)L.nz);
  L.spv = p.samples_per_voxel;
  L.iters = p.estimation_iterations;
  L.clip = p.clip_rays ? 1u : 0u;
  L.seed = p.seed;
  L.lod = lod;
  L.sigma_t = p.sigma_t;
  L.alpha = p.alpha;
  L.project = p.sggx_projection;
  L.floor = p.sggx_floor;
  L.eig = d_eig;
  L.bvh = bvh_.view();
  if (triUV_.get()) {
    L.triUV = triUV_.get();
    L.texels = texels_.get();
    L.texInfo = texInfo_.get();
    L.matTex = matTex_.get();
    if (triAlpha_.get()) {  // opacity cut-outs hide triangles from the filter rays too
      L.bvh.alpha.alphaTex = triAlpha_.get();
      L.bvh.alpha.uv = triUV_.get();
      L.bvh.alpha.texels = texels_.get();
      L.bvh.alpha.texInfo = texInfo_.get();
    }
  }
  L.triN = triN_.get();
  L.triMat = triMat_.get();
  L.mats = mats_.get();
  L.out = d_out;
  L.wide = d_wide;
  L.fp16 = d_fp16;
  if (d_work) {
    L.work = d_work;
  } else {
    work_.reserve(nvox);
    L.work = work_.get();
  }
  L.counters = d_counters ? d_counters : counters_.get();
  L.ops = d_ops;
  R2_CUDA(cudaMemsetAsync(L.counters, 0, 2 * sizeof(uint32_t), s));
  launch_filter_classify(L, s);
  R2_CUDA(cudaEventRecord(ev0_, s));
  launch_filter_sample(L, s);
  R2_CUDA(cudaEventRecord(ev1_, s));
  if (stats) {
    uint32_t cand = 0;
    R2_CUDA(cudaMemcpyAsync(&cand, L.counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    R2_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    R2_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    stats[0] = (double)nvox;
    stats[1] = (double)cand;
    stats[2] = (double)ms;
  }
}

}  // namespace r2
