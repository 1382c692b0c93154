// C ABI: status handling and the filter entry points.
#include <string.h>

#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bvh_build.cuh"
#include "capi_util.h"
#include "filter.cuh"
#include "filter_host.h"
#include "host_math.h"

namespace r2 {
static thread_local std::string g_lastError;
void set_last_error(const std::string& msg) { g_lastError = msg; }
const char* last_error() { return g_lastError.c_str(); }
}  // namespace r2

struct r2_filter_scene {
  std::unique_ptr<r2::FilterScene> impl;
};

extern "C" {

const char* r2_status_string(r2_status s) {
  switch (s) {
    case R2_OK: return "R2_OK";
    case R2_ERR_INVALID_ARGUMENT: return "R2_ERR_INVALID_ARGUMENT";
    case R2_ERR_INVALID_CONFIG: return "R2_ERR_INVALID_CONFIG";
    case R2_ERR_IO: return "R2_ERR_IO";
    case R2_ERR_OUT_OF_MEMORY: return "R2_ERR_OUT_OF_MEMORY";
    case R2_ERR_ADMISSION_REJECTED: return "R2_ERR_ADMISSION_REJECTED";
    case R2_ERR_DEVICE_TIMEOUT: return "R2_ERR_DEVICE_TIMEOUT";
    case R2_ERR_DEVICE: return "R2_ERR_DEVICE";
    case R2_ERR_UNSUPPORTED: return "R2_ERR_UNSUPPORTED";
    case R2_ERR_NO_DEVICE: return "R2_ERR_NO_DEVICE";
    case R2_ERR_PENDING: return "R2_ERR_PENDING";
  }
  return "R2_ERR_UNKNOWN";
}

const char* r2_last_error(void) { return r2::last_error(); }

int r2_version(void) { return 100; }

r2_status r2_set_bvh_method(int method) {
  R2_API_BEGIN
  R2_REQUIRE(method == R2_BVH_AUTO || method == R2_BVH_PLOC || method == R2_BVH_KARRAS, R2_ERR_INVALID_ARGUMENT,
             "unknown BVH method");
  r2::set_bvh_method(method == R2_BVH_KARRAS ? r2::kBvhKarras : (method == R2_BVH_PLOC ? r2::kBvhPloc : r2::kBvhAuto));
  R2_API_END
}

int r2_get_bvh_method(void) {
  const int m = r2::bvh_method();
  return m == r2::kBvhKarras ? R2_BVH_KARRAS : (m == r2::kBvhPloc ? R2_BVH_PLOC : R2_BVH_AUTO);
}

r2_status r2_filter_setup_grid(const float* model_bb_min, const float* model_bb_max, const float* model_to_world,
                               float voxel_size, r2_filter_grid* grid_out) {
  R2_API_BEGIN
  R2_REQUIRE(model_bb_min && model_bb_max && model_to_world && grid_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(voxel_size > 0.0f, R2_ERR_INVALID_ARGUMENT, "voxel size must be positive");
  r2::M43 m2w = r2::m43_from_floats(model_to_world);
  r2::V3 wlo, whi;
  r2::world_aabb(r2::v3(model_bb_min[0], model_bb_min[1], model_bb_min[2]),
                 r2::v3(model_bb_max[0], model_bb_max[1], model_bb_max[2]), m2w, &wlo, &whi);
  r2::M43 w2m = r2::m4_to_m43(r2::m4_inverse(r2::m43_to_m4(m2w)));
  *grid_out = r2::setup_grid(wlo, whi, w2m, voxel_size);
  R2_API_END
}

r2_status r2_filter_scene_create(const float* positions, uint32_t nverts, const uint32_t* indices, uint32_t ntris,
                                 const float* normals, const r2_material* material, const float* model_to_world,
                                 r2_filter_scene** out) {
  R2_API_BEGIN
  R2_REQUIRE(out && model_to_world, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  auto sc = new r2_filter_scene;
  try {
    sc->impl.reset(new r2::FilterScene(positions, nverts, indices, ntris, normals, material, 1, nullptr,
                                       model_to_world));
  } catch (...) {
    delete sc;
    throw;
  }
  *out = sc;
  R2_API_END
}

r2_status r2_filter_scene_create_textured(const float* positions, uint32_t nverts, const uint32_t* indices,
                                          uint32_t ntris, const float* normals, const float* uvs,
                                          const r2_material* material, const r2_material_maps* maps,
                                          const float* model_to_world, r2_filter_scene** out) {
  R2_API_BEGIN
  R2_REQUIRE(out && model_to_world && uvs && maps, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  auto sc = new r2_filter_scene;
  try {
    sc->impl.reset(new r2::FilterScene(positions, nverts, indices, ntris, normals, material, 1, nullptr,
                                       model_to_world, uvs, maps));
  } catch (...) {
    delete sc;
    throw;
  }
  *out = sc;
  R2_API_END
}

r2_status r2_filter_scene_destroy(r2_filter_scene* scene) {
  R2_API_BEGIN
  delete scene;
  R2_API_END
}

r2_status r2_filter_scene_grid(const r2_filter_scene* scene, float voxel_size, r2_filter_grid* grid_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && grid_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  *grid_out = scene->impl->grid(voxel_size);
  R2_API_END
}

r2_status r2_filter_scene_count(r2_filter_scene* scene, const r2_filter_grid* grid, const r2_filter_params* params,
                                r2_voxel* d_out, uint64_t* counts_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && grid && params && d_out && counts_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::DBuf<unsigned long long> ops(3);
  cudaStream_t s = scene->impl->stream();
  R2_CUDA(cudaMemsetAsync(ops.get(), 0, 3 * sizeof(unsigned long long), s));
  scene->impl->run(*grid, *params, 0, d_out, nullptr, nullptr, s, nullptr, nullptr, nullptr, ops.get());
  unsigned long long h[3] = {0, 0, 0};
  ops.download(h, 3, s);
  R2_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < 3; ++k) counts_out[k] = h[k];
  R2_API_END
}

r2_status r2_filter_scene_run(r2_filter_scene* scene, const r2_filter_grid* grid, const r2_filter_params* params,
                              r2_voxel* d_out, float* d_wide, uint16_t* d_fp16, void* stream, double* stats_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && grid && params && d_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->run(*grid, *params, 0, d_out, d_wide, d_fp16, (cudaStream_t)stream, stats_out);
  R2_API_END
}

r2_status r2_filter_scene_run_eig(r2_filter_scene* scene, const r2_filter_grid* grid, const r2_filter_params* params,
                                  r2_voxel* d_out, float* d_wide, uint16_t* d_fp16, float* d_eig, void* stream,
                                  double* stats_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && grid && params && d_out && d_eig, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->run(*grid, *params, 0, d_out, d_wide, d_fp16, (cudaStream_t)stream, stats_out, nullptr, nullptr,
                   nullptr, d_eig);
  R2_API_END
}

r2_status r2_filter_scene_bvh(const r2_filter_scene* scene, int32_t* nodes, size_t node_words, uint32_t* tri_order,
                              size_t ntris, uint32_t* nnodes_out, uint32_t* height_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null scene");
  const r2::DeviceBvh& b = scene->impl->bvh();
  if (nnodes_out) *nnodes_out = b.nnodes;
  if (height_out) *height_out = b.height;
  cudaStream_t s = scene->impl->stream();
  if (nodes) {
    R2_REQUIRE(node_words >= (size_t)b.nnodes * 16, R2_ERR_INVALID_ARGUMENT, "node buffer too small");
    R2_CUDA(cudaMemcpyAsync(nodes, b.nodes.get(), (size_t)b.nnodes * sizeof(r2::BvhNode), cudaMemcpyDeviceToHost, s));
  }
  if (tri_order) {
    R2_REQUIRE(ntris >= b.ntris, R2_ERR_INVALID_ARGUMENT, "order buffer too small");
    R2_CUDA(cudaMemcpyAsync(tri_order, b.order.get(), (size_t)b.ntris * 4, cudaMemcpyDeviceToHost, s));
  }
  R2_CUDA(cudaStreamSynchronize(s));
  R2_API_END
}

r2_status r2_filter_mesh(const float* positions, uint32_t nverts, const uint32_t* indices, uint32_t ntris,
                         const float* normals, const r2_material* material, const float* model_to_world,
                         const r2_filter_params* params, float voxel_size, r2_filter_grid* grid_out, r2_voxel* out,
                         float* wide_out, size_t out_capacity) {
  R2_API_BEGIN
  R2_REQUIRE(params && out && model_to_world, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  r2::FilterScene scene(positions, nverts, indices, ntris, normals, material, 1, nullptr, model_to_world);
  r2_filter_grid g = scene.grid(voxel_size);
  if (grid_out) *grid_out = g;
  size_t nvox = (size_t)g.num_voxels[0] * g.num_voxels[1] * g.num_voxels[2];
  R2_REQUIRE(out_capacity >= nvox, R2_ERR_INVALID_ARGUMENT,
             "output capacity " + std::to_string(out_capacity) + " < " + std::to_string(nvox) + " voxels");
  cudaStream_t s = scene.stream();
  r2::DBuf<r2_voxel> dout(nvox);
  r2::DBuf<float> dwide;
  if (wide_out) dwide.alloc(nvox * r2::kWideFloats);
  scene.run(g, *params, 0, dout.get(), wide_out ? dwide.get() : nullptr, nullptr, s, nullptr);
  dout.download(out, nvox, s);
  if (wide_out) dwide.download(wide_out, nvox * r2::kWideFloats, s);
  R2_CUDA(cudaStreamSynchronize(s));
  R2_API_END
}

}  // extern "C"

// Accessor for the allocation-free entry point (filter_static.cu).
r2::FilterScene* r2_filter_scene_impl(r2_filter_scene* scene) { return scene->impl.get(); }
