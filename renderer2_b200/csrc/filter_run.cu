// The filter's LOD loop with its file outputs: CFilter::runFiltering
// (raytracer/filter.cu:74-123 of the reference): per LOD the voxel size
// doubles; each LOD is filtered on the device, its active leaves become a
// NanoVDB Vec4d grid (filtered_mesh_<vs>.nvdb), its density a brick grid
// (filtered_mesh_<vs>.brickgrid), and the LOD's model-space bounds an entry of
// ./filtering/volume_description.json.
#include <sys/stat.h>

#include <string>

#include "filter.cuh"
#include "filter_host.h"
#include "filter_run.h"
#include "host_math.h"
#include "json.h"
#include "volume.h"

namespace r2 {

static void make_dirs(const std::string& path) {
  std::string cur;
  for (size_t i = 0; i < path.size(); ++i) {
    cur += path[i];
    if (path[i] == '/' || i + 1 == path.size()) {
      if (!cur.empty() && cur != "/" && cur != "./") mkdir(cur.c_str(), 0755);
    }
  }
  struct stat st;
  R2_REQUIRE(stat(path.c_str(), &st) == 0 && S_ISDIR(st.st_mode), R2_ERR_IO, "cannot create directory " + path);
}

void store_volume_description(const std::string& path, const std::string& model, const std::string& key,
                              const VolumeDescription& d) {
  Json root = Json::object();
  struct stat st;
  if (stat(path.c_str(), &st) == 0) root = Json::parse(read_text_file(path));
  if (!root.is_object()) root = Json::object();
  // CVolumeDescriptionManager::getBoundingPoints (volume_description_manager.cpp:125-143)
  const float* mn = d.bbmin;
  const float* mx = d.bbmax;
  const float P[8][3] = {{mn[0], mn[1], mn[2]}, {mx[0], mn[1], mn[2]}, {mx[0], mn[1], mx[2]}, {mn[0], mn[1], mx[2]},
                         {mn[0], mx[1], mn[2]}, {mx[0], mx[1], mn[2]}, {mx[0], mx[1], mx[2]}, {mn[0], mx[1], mx[2]}};
  auto vec = [](const float* v) {
    Json a = Json::array();
    for (int k = 0; k < 3; ++k) a.push(Json::number((double)v[k]));
    return a;
  };
  Json e = Json::object();
  Json nv = Json::array();
  for (int k = 0; k < 3; ++k) nv.push(Json::number(d.numVoxels[k]));
  e.set("NumVoxels", nv);
  e.set("BBMin", vec(mn));
  e.set("BBMax", vec(mx));
  for (int p = 0; p < 8; ++p) e.set("P" + std::to_string(p), vec(P[p]));
  Json m = root[model].is_object() ? root[model] : Json::object();
  m.set(key, e);
  root.set(model, m);
  FILE* f = fopen(path.c_str(), "wb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot write " + path);
  std::string txt = root.dump(2);
  bool ok = fwrite(txt.data(), 1, txt.size(), f) == txt.size();
  ok = (fclose(f) == 0) && ok;
  R2_REQUIRE(ok, R2_ERR_IO, "short write to " + path);
}

FilterRunResult run_filter_lods(FilterScene& scene, const r2_filter_params& p, V3 orientation,
                                const std::string& outRoot, const std::string& model, cudaStream_t s) {
  R2_REQUIRE(p.lods >= 1 && p.lods <= 32, R2_ERR_INVALID_CONFIG, "LODs must be in [1, 32]");
  R2_REQUIRE(p.min_voxel_size > 0.0f, R2_ERR_INVALID_CONFIG, "MinVoxelSize must be positive");
  if (!s) s = scene.stream();
  FilterRunResult res;
  const std::string outDir = outRoot + "/" + model;
  make_dirs(outDir);
  float voxelSize = p.min_voxel_size;
  for (uint32_t lod = 0; lod < p.lods; ++lod, voxelSize *= 2.0f) {
    r2_filter_grid g = scene.grid(voxelSize);
    const size_t nvox = (size_t)g.num_voxels[0] * g.num_voxels[1] * g.num_voxels[2];
    DBuf<r2_voxel> dense(nvox);
    double stats[3];
    scene.run(g, p, lod, dense.get(), nullptr, nullptr, s, stats);
    std::vector<nvdb::LeafBlock> leaves;
    std::vector<r2_voxel> values;
    extract_leaves(dense.get(), g.num_voxels, s, &leaves, &values);
    std::vector<uint8_t> grid = nvdb::build_grid(leaves, values, g.index_to_model, g.model_to_index, "");
    BrickGridHost bricks;
    build_brick_grid(dense.get(), g.num_voxels, s, &bricks);
    const std::string base = outDir + "/filtered_mesh_" + float_key(voxelSize);
    nvdb::write_file(base + ".nvdb", grid);
    write_brick_grid(base + ".brickgrid", bricks);
    // model-space bounds: getRotation(orientation) * worldToModel applied to
    // the LOD's world box corners (filter.cu:109-114)
    M4 t = m4_mul(get_rotation(orientation), m43_to_m4(m43_from_floats(g.world_to_model)));
    V3 a = m4_point(t, v3(g.world_bb_min[0], g.world_bb_min[1], g.world_bb_min[2]));
    V3 b = m4_point(t, v3(g.world_bb_max[0], g.world_bb_max[1], g.world_bb_max[2]));
    VolumeDescription d;
    for (int k = 0; k < 3; ++k) d.numVoxels[k] = g.num_voxels[k];
    V3 lo = vmin(a, b), hi = vmax(a, b);
    d.bbmin[0] = lo.x; d.bbmin[1] = lo.y; d.bbmin[2] = lo.z;
    d.bbmax[0] = hi.x; d.bbmax[1] = hi.y; d.bbmax[2] = hi.z;
    store_volume_description(outRoot + "/volume_description.json", model, float_key(voxelSize), d);
    res.paths.push_back(base);
    res.voxels += (double)nvox;
    res.activeVoxels += (double)nvdb::tree_data(grid.data())->voxelCount;
    res.kernelMs += stats[2];
  }
  return res;
}

}  // namespace r2
