// C ABI of the pipeline: config loading (CConfigLoader::loadConfig), the
// filter run of the FILTER-masked mesh (CFilter, raytracer/filter.cu:20-123),
// frame rendering with the output stage (rt::Raytracer, raytracer.cu:129-210)
// and the asset files of the pipeline.
#include <string.h>

#include <map>
#include <memory>
#include <string>

#include "asset_io.h"
#include "capi_util.h"
#include "config.h"
#include "filter_run.h"
#include "host_math.h"
#include "render_host.h"
#include "tonemap.h"

struct r2_config {
  r2::PipelineConfig cfg;
  r2::RgbImage env;
  // per Mesh object (in scene order): its OBJ submeshes, each file read once
  // (CAssetManager::loadMesh caches by path, asset_manager.cu:86-112)
  std::vector<std::shared_ptr<const std::vector<r2::ObjSubmesh>>> meshes;
  std::unique_ptr<r2::RenderScene> scene;  // built at the first render, then resident
  r2::DBuf<float> frame;
  r2::DBuf<uint8_t> bytes;
  r2::DBuf<float> scratch;
};

namespace {

r2::M4 object_transform(const r2::SceneObjectDesc& o) {
  return r2::model_to_world_transform(r2::v3(o.pos[0], o.pos[1], o.pos[2]),
                                      r2::v3(o.orientation[0], o.orientation[1], o.orientation[2]),
                                      r2::v3(o.scaling[0], o.scaling[1], o.scaling[2]));
}

// Scene objects of type Mesh whose file is used by one object are flattened
// into world space; a file placed by several objects becomes one mesh asset
// per submesh with an instance per object (CAssetManager::loadMesh keeps one
// CMesh and GAS per file, asset_manager.cu, and every object is an instance).
void build_scene(r2_config* c) {
  auto sc = std::unique_ptr<r2::RenderScene>(new r2::RenderScene());
  std::map<const std::vector<r2::ObjSubmesh>*, int> uses;
  for (const auto& m : c->meshes) ++uses[m.get()];
  std::map<const r2::ObjSubmesh*, uint32_t> assetOf;
  size_t mi = 0;
  for (const r2::SceneObjectDesc& o : c->cfg.objects) {
    switch (o.kind) {
      case r2::SceneObjectDesc::kCircle:
      case r2::SceneObjectDesc::kSphere:
        sc->add_shape(o.kind == r2::SceneObjectDesc::kCircle ? r2::kShapeCircle : r2::kShapeSphere, o.pos, o.radius,
                      o.normal, o.material, o.mask);
        break;
      case r2::SceneObjectDesc::kMedium:
        sc->add_medium(o.path.c_str(), o.sigmaA, o.sigmaS, o.pos, o.orientation, o.scaling, o.mask, o.hasG, o.g);
        break;
      case r2::SceneObjectDesc::kMesh: {
        float m43[12];
        r2::m43_to_floats(r2::m4_to_m43(object_transform(o)), m43);
        const bool shared = uses[c->meshes[mi].get()] > 1;
        for (const r2::ObjSubmesh& s : *c->meshes[mi]) {
          const r2_material_maps maps = {s.texAlbedo.c_str(), s.texSpecular.c_str(), s.texNormal.c_str(),
                                         s.texAlpha.c_str()};
          const float* uv = s.uvs.empty() ? nullptr : s.uvs.data();
          if (!shared) {
            sc->add_mesh(s.positions.data(), (uint32_t)(s.positions.size() / 3), s.indices.data(),
                         (uint32_t)(s.indices.size() / 3), s.normals.data(), s.material, m43, o.mask, uv, &maps);
            continue;
          }
          auto it = assetOf.find(&s);
          if (it == assetOf.end())
            it = assetOf.emplace(&s, sc->add_mesh_asset(s.positions.data(), (uint32_t)(s.positions.size() / 3),
                                                        s.indices.data(), (uint32_t)(s.indices.size() / 3),
                                                        s.normals.data(), s.material, uv, &maps)).first;
          sc->add_mesh_instance(it->second, m43, o.mask);
        }
        ++mi;
        break;
      }
    }
  }
  sc->set_envmap(c->env.rgb.data(), (int)c->env.width, (int)c->env.height);
  sc->commit();
  c->scene = std::move(sc);
}

}  // namespace

extern "C" {

r2_status r2_config_load(const char* config_json_path, r2_config** out) {
  R2_API_BEGIN
  R2_REQUIRE(config_json_path && out, R2_ERR_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<r2_config> c(new r2_config());
  c->cfg = r2::load_config(config_json_path);
  c->env = r2::read_hdr(c->cfg.envmap);
  std::map<std::string, std::shared_ptr<const std::vector<r2::ObjSubmesh>>> loaded;
  for (const r2::SceneObjectDesc& o : c->cfg.objects) {
    if (o.kind != r2::SceneObjectDesc::kMesh) continue;
    auto& m = loaded[o.directory + "\n" + o.filename];
    if (!m) m = std::make_shared<const std::vector<r2::ObjSubmesh>>(r2::load_obj(o.directory, o.filename));
    c->meshes.push_back(m);
  }
  *out = c.release();
  R2_API_END
}

r2_status r2_config_free(r2_config* cfg) {
  R2_API_BEGIN
  delete cfg;
  R2_API_END
}

r2_status r2_config_info_get(const r2_config* cfg, r2_config_info* out) {
  R2_API_BEGIN
  R2_REQUIRE(cfg && out, R2_ERR_INVALID_ARGUMENT, "null argument");
  memset(out, 0, sizeof(*out));
  const r2::PipelineConfig& c = cfg->cfg;
  out->frame_width = c.frameWidth;
  out->frame_height = c.frameHeight;
  out->channels = c.channelsPerPixel;
  out->samples = c.samples;
  out->gamma = c.gamma;
  out->use_brick_grid = c.useBrickGrid ? 1u : 0u;
  out->filter_active = c.filterActive ? 1u : 0u;
  out->filter = c.filter;
  out->camera = c.camera;
  out->env_width = cfg->env.width;
  out->env_height = cfg->env.height;
  size_t mi = 0;
  for (const r2::SceneObjectDesc& o : c.objects) {
    if (o.kind == r2::SceneObjectDesc::kMedium) ++out->n_media;
    else if (o.kind == r2::SceneObjectDesc::kMesh) {
      for (const r2::ObjSubmesh& s : *cfg->meshes[mi]) {
        ++out->n_meshes;
        out->n_triangles += (uint32_t)(s.indices.size() / 3);
      }
      ++mi;
    } else {
      ++out->n_shapes;
    }
  }
  R2_API_END
}

r2_status r2_filter_run(r2_config* cfg, const char* out_root, double* stats_out) {
  R2_API_BEGIN
  R2_REQUIRE(cfg, R2_ERR_INVALID_ARGUMENT, "null argument");
  if (stats_out) memset(stats_out, 0, 4 * sizeof(double));
  // CHostScene::getObjectBBs(FILTER) (scene.cu:281-310): one mesh file, its
  // submeshes merged; the last FILTER object's transform
  std::string meshPath, name;
  std::vector<float> pos, nrm, uvs;
  std::vector<uint32_t> idx, triMat;
  std::vector<r2_material> mats;
  std::vector<r2_material_maps> maps;
  bool anyUV = false;
  const r2::SceneObjectDesc* last = nullptr;
  size_t mi = 0;
  for (const r2::SceneObjectDesc& o : cfg->cfg.objects) {
    const bool isMesh = o.kind == r2::SceneObjectDesc::kMesh;
    if (o.mask & R2_MASK_FILTER) {
      R2_REQUIRE(isMesh, R2_ERR_INVALID_CONFIG, "No mesh available: only meshes can be filtered");
      const std::string p = o.directory + "/" + o.filename;
      if (meshPath.empty()) meshPath = p;
      R2_REQUIRE(p == meshPath, R2_ERR_INVALID_CONFIG, "Filtering only available for single mesh");
      for (const r2::ObjSubmesh& s : *cfg->meshes[mi]) {
        const uint32_t base = (uint32_t)(pos.size() / 3);
        pos.insert(pos.end(), s.positions.begin(), s.positions.end());
        nrm.insert(nrm.end(), s.normals.begin(), s.normals.end());
        if (s.uvs.empty()) uvs.insert(uvs.end(), 2 * (s.positions.size() / 3), 0.0f);
        else uvs.insert(uvs.end(), s.uvs.begin(), s.uvs.end());
        anyUV = anyUV || !s.uvs.empty();
        maps.push_back({s.texAlbedo.c_str(), s.texSpecular.c_str(), s.texNormal.c_str(), s.texAlpha.c_str()});
        for (uint32_t i : s.indices) idx.push_back(base + i);
        for (size_t t = 0; t < s.indices.size() / 3; ++t) triMat.push_back((uint32_t)mats.size());
        mats.push_back(s.material);
      }
      last = &o;
    }
    if (isMesh) ++mi;
  }
  if (!last) return R2_OK;  // no bounding boxes: proceed without filtering (filter.cu:53-55)
  const std::string base = meshPath.substr(meshPath.find_last_of('/') + 1);
  name = base.substr(0, base.find_last_of('.'));
  float m43[12];
  r2::m43_to_floats(r2::m4_to_m43(object_transform(*last)), m43);
  r2::require_device();
  r2::FilterScene scene(pos.data(), (uint32_t)(pos.size() / 3), idx.data(), (uint32_t)(idx.size() / 3), nrm.data(),
                        mats.data(), (uint32_t)mats.size(), triMat.data(), m43, anyUV ? uvs.data() : nullptr,
                        maps.data());
  const r2::V3 orient = r2::v3(last->orientation[0], last->orientation[1], last->orientation[2]);
  r2::FilterRunResult r =
      r2::run_filter_lods(scene, cfg->cfg.filter, orient, out_root ? out_root : "./filtering", name, nullptr);
  if (stats_out) {
    stats_out[0] = (double)r.paths.size();
    stats_out[1] = r.voxels;
    stats_out[2] = r.activeVoxels;
    stats_out[3] = r.kernelMs;
  }
  R2_API_END
}

r2_status r2_render(r2_config* cfg, const r2_render_opts* opts, float* out_linear_rgb, uint8_t* out_bytes) {
  R2_API_BEGIN
  R2_REQUIRE(cfg, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  if (!cfg->scene) build_scene(cfg);
  r2_render_params p;
  p.spp = (opts && opts->spp) ? opts->spp : cfg->cfg.samples;
  p.max_depth = (opts && opts->max_depth) ? opts->max_depth : 50u;  // the reference's bounce cap
  p.seed = opts ? opts->seed : 0u;
  p.flags = cfg->cfg.useBrickGrid ? R2_RENDER_BRICK_GRID : 0u;
  const uint32_t W = cfg->cfg.frameWidth, H = cfg->cfg.frameHeight;
  const size_t n = (size_t)W * H * 3;
  cudaStream_t s = cfg->scene->stream();
  cfg->frame.reserve(n);
  cfg->scene->render(cfg->cfg.camera, p, cfg->frame.get(), s, nullptr);
  if (out_bytes) {
    cfg->bytes.reserve(n);
    cfg->scratch.reserve((size_t)W + 1);
    r2::tonemap_device(cfg->frame.get(), W, H, cfg->cfg.gamma, nullptr, cfg->bytes.get(), cfg->scratch.get(), s);
    cfg->bytes.download(out_bytes, n, s);
  }
  if (out_linear_rgb) cfg->frame.download(out_linear_rgb, n, s);
  R2_CUDA(cudaStreamSynchronize(s));
  const uint32_t b = cfg->scene->bound_hits(s);
  R2_REQUIRE(b == 0, R2_ERR_DEVICE_TIMEOUT, std::to_string(b) + " paths or shadow rays ended by a loop bound");
  R2_API_END
}

r2_status r2_tonemap(const float* linear_rgb, uint32_t width, uint32_t height, float gamma, float* out_rgb,
                     uint8_t* out_bytes) {
  R2_API_BEGIN
  R2_REQUIRE(linear_rgb && (out_rgb || out_bytes), R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::require_device();
  const size_t n = (size_t)width * height * 3;
  cudaStream_t s = nullptr;
  R2_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{s};
  r2::DBuf<float> in, out, scratch((size_t)width + 1);
  r2::DBuf<uint8_t> bytes;
  in.upload(linear_rgb, n, s);
  if (out_rgb) out.alloc(n);
  if (out_bytes) bytes.alloc(n);
  r2::tonemap_device(in.get(), width, height, gamma, out.get(), bytes.get(), scratch.get(), s);
  if (out_rgb) out.download(out_rgb, n, s);
  if (out_bytes) bytes.download(out_bytes, n, s);
  R2_CUDA(cudaStreamSynchronize(s));
  R2_API_END
}

r2_status r2_read_png(const char* path, uint8_t* rgba, size_t capacity, uint32_t* width, uint32_t* height,
                      int* channels_out) {
  R2_API_BEGIN
  R2_REQUIRE(path, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::RgbaImage8 img = r2::read_png(path);
  if (width) *width = img.width;
  if (height) *height = img.height;
  if (channels_out) *channels_out = img.channels;
  if (rgba) {
    R2_REQUIRE(capacity >= img.rgba.size(), R2_ERR_INVALID_ARGUMENT, "PNG larger than the output buffer");
    memcpy(rgba, img.rgba.data(), img.rgba.size());
  }
  R2_API_END
}

r2_status r2_write_jpg(const char* path, const uint8_t* rgb, uint32_t width, uint32_t height, int flip_vertical,
                       int quality) {
  R2_API_BEGIN
  R2_REQUIRE(path && rgb, R2_ERR_INVALID_ARGUMENT, "null argument");
  R2_REQUIRE(quality >= 1 && quality <= 100, R2_ERR_INVALID_ARGUMENT, "JPEG quality must be in [1, 100]");
  r2::write_jpg(path, rgb, width, height, flip_vertical != 0, quality);
  R2_API_END
}

r2_status r2_write_png(const char* path, const uint8_t* rgb, uint32_t width, uint32_t height, int flip_vertical) {
  R2_API_BEGIN
  R2_REQUIRE(path && rgb, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::write_png(path, rgb, width, height, flip_vertical != 0);
  R2_API_END
}

r2_status r2_read_hdr(const char* path, float* rgb, size_t capacity, uint32_t* width, uint32_t* height) {
  R2_API_BEGIN
  R2_REQUIRE(path, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::RgbImage img = r2::read_hdr(path);
  if (width) *width = img.width;
  if (height) *height = img.height;
  if (rgb) {
    R2_REQUIRE(capacity >= img.rgb.size(), R2_ERR_INVALID_ARGUMENT, "buffer too small");
    memcpy(rgb, img.rgb.data(), img.rgb.size() * sizeof(float));
  }
  R2_API_END
}

r2_status r2_write_hdr(const char* path, const float* rgb, uint32_t width, uint32_t height) {
  R2_API_BEGIN
  R2_REQUIRE(path && rgb && width > 0 && height > 0, R2_ERR_INVALID_ARGUMENT, "null argument");
  r2::write_hdr(path, rgb, width, height);
  R2_API_END
}

r2_status r2_obj_info(const char* directory, const char* filename, uint32_t* n_submeshes, uint32_t* n_vertices,
                      uint32_t* n_triangles, r2_material* first_material) {
  R2_API_BEGIN
  R2_REQUIRE(directory && filename, R2_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<r2::ObjSubmesh> subs = r2::load_obj(directory, filename);
  uint32_t nv = 0, nt = 0;
  for (const r2::ObjSubmesh& s : subs) {
    nv += (uint32_t)(s.positions.size() / 3);
    nt += (uint32_t)(s.indices.size() / 3);
  }
  if (n_submeshes) *n_submeshes = (uint32_t)subs.size();
  if (n_vertices) *n_vertices = nv;
  if (n_triangles) *n_triangles = nt;
  if (first_material) *first_material = subs[0].material;
  R2_API_END
}

}  // extern "C"
