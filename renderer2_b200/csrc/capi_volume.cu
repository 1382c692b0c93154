// C ABI: filter LOD loop with file outputs, NanoVDB / brick-grid queries.
#include <string.h>

#include <memory>

#include "capi_util.h"
#include "filter_run.h"
#include "host_math.h"
#include "volume.h"

struct r2_filter_scene;
r2::FilterScene* r2_filter_scene_impl(r2_filter_scene* scene);

extern "C" {

r2_status r2_filter_run_mesh(const float* positions, uint32_t nverts, const uint32_t* indices, uint32_t ntris,
                             const float* normals, const r2_material* material, const float* pos3,
                             const float* orientation3, const float* scaling3, const r2_filter_params* params,
                             const char* out_root, const char* model_name, double* stats_out) {
  R2_API_BEGIN
  R2_REQUIRE(params && pos3 && orientation3 && scaling3 && out_root && model_name, R2_ERR_INVALID_ARGUMENT,
             "null argument");
  r2::require_device();
  r2::V3 orient = r2::v3(orientation3[0], orientation3[1], orientation3[2]);
  r2::M4 m2w = r2::model_to_world_transform(r2::v3(pos3[0], pos3[1], pos3[2]), orient,
                                            r2::v3(scaling3[0], scaling3[1], scaling3[2]));
  float m43[12];
  r2::m43_to_floats(r2::m4_to_m43(m2w), m43);
  r2::FilterScene scene(positions, nverts, indices, ntris, normals, material, 1, nullptr, m43);
  r2::FilterRunResult r = r2::run_filter_lods(scene, *params, orient, out_root, model_name, nullptr);
  if (stats_out) {
    stats_out[0] = (double)r.paths.size();
    stats_out[1] = r.voxels;
    stats_out[2] = r.activeVoxels;
    stats_out[3] = r.kernelMs;
  }
  R2_API_END
}

r2_status r2_nvdb_info(const char* path, uint64_t* counts4, int32_t* index_bbox6, double* world_bbox6,
                       float* index_to_model12) {
  R2_API_BEGIN
  R2_REQUIRE(path, R2_ERR_INVALID_ARGUMENT, "null path");
  std::vector<uint8_t> g = r2::nvdb::read_file(path);
  const r2::nvdb::GridData* G = r2::nvdb::grid_data(g.data());
  const r2::nvdb::TreeData* T = r2::nvdb::tree_data(g.data());
  if (counts4) {
    counts4[0] = T->nodeCount[0];
    counts4[1] = T->nodeCount[1];
    counts4[2] = T->nodeCount[2];
    counts4[3] = T->voxelCount;
  }
  if (index_bbox6) r2::nvdb::index_bbox(g.data(), index_bbox6);
  if (world_bbox6) memcpy(world_bbox6, G->worldBBox, 6 * sizeof(double));
  if (index_to_model12) {
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) index_to_model12[3 * c + r] = G->map.matF[3 * r + c];
    for (int r = 0; r < 3; ++r) index_to_model12[9 + r] = G->map.vecF[r];
  }
  R2_API_END
}

r2_status r2_nvdb_lookup(const char* path, const int32_t* coords, uint32_t n, r2_voxel* out, uint8_t* active) {
  R2_API_BEGIN
  R2_REQUIRE(path && coords && out, R2_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<uint8_t> g = r2::nvdb::read_file(path);
  for (uint32_t i = 0; i < n; ++i) {
    bool a = false;
    out[i] = r2::nvdb::host_value(g.data(), coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], &a);
    if (active) active[i] = a ? 1 : 0;
  }
  R2_API_END
}

r2_status r2_brickgrid_info(const char* path, uint32_t* dims7, float* minmaj2, uint32_t* indirection,
                            uint32_t* range, size_t capacity) {
  R2_API_BEGIN
  R2_REQUIRE(path, R2_ERR_INVALID_ARGUMENT, "null path");
  r2::BrickGridHost b = r2::read_brick_grid(path);
  if (dims7) {
    for (int k = 0; k < 3; ++k) {
      dims7[k] = b.nBricks[k];
      dims7[3 + k] = b.atlasDim[k];
    }
    dims7[6] = b.brickCount;
  }
  if (minmaj2) {
    minmaj2[0] = b.minorant;
    minmaj2[1] = b.majorant;
  }
  if (indirection || range) {
    R2_REQUIRE(capacity >= b.range.size(), R2_ERR_INVALID_ARGUMENT, "brick buffer too small");
    if (indirection) memcpy(indirection, b.indirection.data(), b.indirection.size() * 4);
    if (range) memcpy(range, b.range.data(), b.range.size() * 4);
  }
  R2_API_END
}

}  // extern "C"
