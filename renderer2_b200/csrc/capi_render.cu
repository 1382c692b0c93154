// C ABI: path tracer scene and frame entry points.
#include <algorithm>
#include <memory>

#include "capi_util.h"
#include "lod_select.h"
#include "render_host.h"

struct r2_scene {
  std::unique_ptr<r2::RenderScene> impl;
};

struct r2_render_batch {
  std::unique_ptr<r2::RenderBatch> impl;
};

r2::RenderScene* r2_scene_impl(r2_scene* scene) { return scene->impl.get(); }

extern "C" {

r2_status r2_scene_create(r2_scene** out) {
  R2_API_BEGIN
  R2_REQUIRE(out, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  auto sc = new r2_scene;
  try {
    sc->impl.reset(new r2::RenderScene());
  } catch (...) {
    delete sc;
    throw;
  }
  *out = sc;
  R2_API_END
}

r2_status r2_scene_destroy(r2_scene* scene) {
  R2_API_BEGIN
  delete scene;
  R2_API_END
}

r2_status r2_scene_add_mesh(r2_scene* scene, const float* positions, uint32_t nverts, const uint32_t* indices,
                            uint32_t ntris, const float* normals, const r2_material* material,
                            const float* model_to_world, uint32_t mask) {
  R2_API_BEGIN
  R2_REQUIRE(scene && material, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->add_mesh(positions, nverts, indices, ntris, normals, *material, model_to_world, mask);
  R2_API_END
}

r2_status r2_scene_add_mesh_asset(r2_scene* scene, const float* positions, uint32_t nverts, const uint32_t* indices,
                                  uint32_t ntris, const float* normals, const float* uvs, const r2_material* material,
                                  const r2_material_maps* maps, uint32_t* asset_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && material && asset_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  *asset_out = scene->impl->add_mesh_asset(positions, nverts, indices, ntris, normals, *material, uvs, maps);
  R2_API_END
}

r2_status r2_scene_add_mesh_instance(r2_scene* scene, uint32_t asset, const float* model_to_world, uint32_t mask) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->add_mesh_instance(asset, model_to_world, mask);
  R2_API_END
}

r2_status r2_scene_add_mesh_textured(r2_scene* scene, const float* positions, uint32_t nverts, const uint32_t* indices,
                                     uint32_t ntris, const float* normals, const float* uvs,
                                     const r2_material* material, const r2_material_maps* maps,
                                     const float* model_to_world, uint32_t mask) {
  R2_API_BEGIN
  R2_REQUIRE(scene && material && uvs, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->add_mesh(positions, nverts, indices, ntris, normals, *material, model_to_world, mask, uvs, maps);
  R2_API_END
}

r2_status r2_scene_add_shape(r2_scene* scene, int shape_type, const float* center, float radius, const float* normal,
                             const r2_material* material, uint32_t mask) {
  R2_API_BEGIN
  R2_REQUIRE(scene && material && center, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->add_shape(shape_type, center, radius, normal, *material, mask);
  R2_API_END
}

r2_status r2_scene_set_envmap(r2_scene* scene, const float* rgb, uint32_t width, uint32_t height) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->set_envmap(rgb, (int)width, (int)height);
  R2_API_END
}

r2_status r2_scene_add_medium(r2_scene* scene, const char* path, const float* sigma_a, const float* sigma_s,
                              const float* pos, const float* orientation, const float* scaling, uint32_t mask) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->add_medium(path, sigma_a, sigma_s, pos, orientation, scaling, mask);
  R2_API_END
}

r2_status r2_scene_add_medium_hg(r2_scene* scene, const char* path, const float* sigma_a, const float* sigma_s,
                                 float g, const float* pos, const float* orientation, const float* scaling,
                                 uint32_t mask) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->add_medium(path, sigma_a, sigma_s, pos, orientation, scaling, mask, true, g);
  R2_API_END
}

r2_status r2_scene_commit(r2_scene* scene) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->commit();
  R2_API_END
}

r2_status r2_scene_rebuild(r2_scene* scene, void* stream) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(scene->impl->committed(), R2_ERR_INVALID_ARGUMENT, "scene not committed");
  scene->impl->rebuild((cudaStream_t)stream);
  R2_API_END
}

r2_status r2_scene_bvh_info(r2_scene* scene, uint32_t* nodes, uint32_t* height, uint32_t* build_launches) {
  R2_API_BEGIN
  R2_REQUIRE(scene, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(scene->impl->committed(), R2_ERR_INVALID_ARGUMENT, "scene not committed");
  if (nodes) *nodes = scene->impl->bvh_nodes();
  if (height) *height = scene->impl->bvh_height();
  if (build_launches) *build_launches = (uint32_t)scene->impl->bvh_build_launches();
  R2_API_END
}

r2_status r2_scene_set_vertices(r2_scene* scene, const float* positions, const float* normals, uint32_t nverts,
                                void* stream) {
  R2_API_BEGIN
  R2_REQUIRE(scene && positions, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(scene->impl->committed(), R2_ERR_INVALID_ARGUMENT, "scene not committed");
  scene->impl->set_vertices(positions, normals, nverts, (cudaStream_t)stream);
  R2_API_END
}

r2_status r2_render_device(r2_scene* scene, const r2_camera* camera, const r2_render_params* params, float* d_rgb,
                           void* stream, double* stats_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && camera && params && d_rgb, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->render(*camera, *params, d_rgb, (cudaStream_t)stream, stats_out);
  if (stats_out) {
    const uint32_t b = scene->impl->bound_hits((cudaStream_t)stream);
    R2_REQUIRE(b == 0, R2_ERR_DEVICE_TIMEOUT, std::to_string(b) + " paths or shadow rays ended by a loop bound");
  }
  R2_API_END
}

r2_status r2_render_host(r2_scene* scene, const r2_camera* camera, const r2_render_params* params, float* rgb) {
  R2_API_BEGIN
  R2_REQUIRE(scene && camera && params && rgb, R2_ERR_INVALID_ARGUMENT, "null argument");
  size_t n = (size_t)camera->width * camera->height * 3;
  r2::DBuf<float>& d = scene->impl->host_frame();
  d.reserve(n);
  cudaStream_t s = scene->impl->stream();
  scene->impl->render(*camera, *params, d.get(), s, nullptr);
  d.download(rgb, n, s);
  R2_CUDA(cudaStreamSynchronize(s));
  const uint32_t b = scene->impl->bound_hits(s);
  R2_REQUIRE(b == 0, R2_ERR_DEVICE_TIMEOUT, std::to_string(b) + " paths or shadow rays ended by a loop bound");
  R2_API_END
}

r2_status r2_scene_set_tuning(r2_scene* scene, const r2_render_tuning* tuning) {
  R2_API_BEGIN
  R2_REQUIRE(scene && tuning, R2_ERR_INVALID_ARGUMENT, "null argument");
  scene->impl->set_tuning(*tuning);
  R2_API_END
}

r2_status r2_scene_get_tuning(r2_scene* scene, r2_render_tuning* tuning) {
  R2_API_BEGIN
  R2_REQUIRE(scene && tuning, R2_ERR_INVALID_ARGUMENT, "null argument");
  *tuning = scene->impl->tuning();
  R2_API_END
}

r2_status r2_scene_wave_samples(r2_scene* scene, const r2_camera* camera, const r2_render_params* params,
                                uint32_t* samples_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && camera && params && samples_out, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(params->spp > 0, R2_ERR_INVALID_ARGUMENT, "spp must be positive");
  *samples_out = scene->impl->wave_spp(camera->width * camera->height, params->spp);
  R2_API_END
}

r2_status r2_scene_autotune(r2_scene* scene, const r2_camera* camera, const r2_render_params* params,
                            r2_render_tuning* tuning_out) {
  R2_API_BEGIN
  R2_REQUIRE(scene && camera && params, R2_ERR_INVALID_ARGUMENT, "null argument");
  const r2_render_tuning t = scene->impl->autotune(*camera, *params);
  if (tuning_out) *tuning_out = t;
  R2_API_END
}

r2_status r2_render_batch_create(r2_scene* const* scenes, const r2_camera* cameras, const r2_render_params* params,
                                 float* const* d_rgb, uint32_t n, r2_render_batch** out) {
  R2_API_BEGIN
  R2_REQUIRE(scenes && cameras && params && d_rgb && out, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(n > 0, R2_ERR_INVALID_ARGUMENT, "empty batch");
  std::vector<r2::RenderScene*> sc(n);
  for (uint32_t i = 0; i < n; ++i) {
    R2_REQUIRE(scenes[i], R2_ERR_INVALID_ARGUMENT, "null scene in batch");
    sc[i] = scenes[i]->impl.get();
  }
  auto b = new r2_render_batch;
  try {
    b->impl.reset(new r2::RenderBatch(sc, std::vector<r2_camera>(cameras, cameras + n),
                                      std::vector<r2_render_params>(params, params + n),
                                      std::vector<float*>(d_rgb, d_rgb + n)));
  } catch (...) {
    delete b;
    throw;
  }
  *out = b;
  R2_API_END
}

r2_status r2_render_batch_destroy(r2_render_batch* batch) {
  R2_API_BEGIN
  delete batch;
  R2_API_END
}

r2_status r2_render_batch_run(r2_render_batch* batch, void* stream, double* ms_out) {
  R2_API_BEGIN
  R2_REQUIRE(batch, R2_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  const double ms = batch->impl->run(s, ms_out != nullptr);
  if (ms_out) {
    *ms_out = ms;
    const uint32_t b = batch->impl->bound_hits(s);
    R2_REQUIRE(b == 0, R2_ERR_DEVICE_TIMEOUT, std::to_string(b) + " paths or shadow rays ended by a loop bound");
  }
  R2_API_END
}

r2_status r2_select_lods(const r2_lod_camera* camera, const r2_lod_volume* lods, const uint32_t* model_first,
                         const uint32_t* model_count, uint32_t nmodels, const double* tree_pos,
                         const double* tree_scaling, const uint32_t* tree_model, uint32_t ntrees, double min_lod,
                         double covered_pixels, int32_t* lod_out) {
  R2_API_BEGIN
  R2_REQUIRE(camera && (nmodels == 0 || (lods && model_first && model_count)), R2_ERR_INVALID_ARGUMENT,
             "null argument");
  R2_REQUIRE(ntrees == 0 || (tree_pos && tree_scaling && tree_model && lod_out), R2_ERR_INVALID_ARGUMENT,
             "null argument");
  if (ntrees == 0) return R2_OK;
  r2::require_device();
  uint64_t nlods = 0;
  for (uint32_t m = 0; m < nmodels; ++m) nlods = std::max<uint64_t>(nlods, (uint64_t)model_first[m] + model_count[m]);
  R2_REQUIRE(nlods < (1ull << 31), R2_ERR_INVALID_ARGUMENT, "LOD table too large");
  r2::select_lods(*camera, lods, (uint32_t)nlods, model_first, model_count, nmodels, tree_pos, tree_scaling,
                  tree_model, ntrees, min_lod, covered_pixels, lod_out, nullptr);
  R2_API_END
}

}  // extern "C"
