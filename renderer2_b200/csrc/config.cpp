// config.json + scenedescription.json loading (see config.h).
#include "config.h"

#include <string.h>

#include "json.h"
#include "runtime.h"

namespace r2 {

namespace {

[[noreturn]] void invalid(const std::string& what) { throw Error{R2_ERR_INVALID_CONFIG, "could not parse config: " + what}; }

const Json& need(const Json& obj, const std::string& key, const std::string& where) {
  const Json& v = obj[key];
  if (v.is_null()) invalid(where + "." + key + " missing");
  return v;
}
float num(const Json& obj, const std::string& key, const std::string& where) {
  const Json& v = need(obj, key, where);
  if (!v.is_number()) invalid(where + "." + key + " is not a number");
  return (float)v.as_number();
}
uint32_t unum(const Json& obj, const std::string& key, const std::string& where) {
  const float v = num(obj, key, where);
  if (!(v >= 0.0f)) invalid(where + "." + key + " must be non-negative");
  return (uint32_t)obj[key].as_number();
}
bool flag(const Json& obj, const std::string& key, const std::string& where) {
  const Json& v = need(obj, key, where);
  if (!v.is_bool()) invalid(where + "." + key + " is not a boolean");
  return v.as_bool();
}
std::string str(const Json& obj, const std::string& key, const std::string& where) {
  const Json& v = need(obj, key, where);
  if (!v.is_string()) invalid(where + "." + key + " is not a string");
  return v.as_string();
}
// parseVec3: exactly three numbers
void vec3(const Json& obj, const std::string& key, const std::string& where, float* out) {
  const Json& v = need(obj, key, where);
  if (!v.is_array() || v.size() != 3) invalid(where + "." + key + " is not a 3-vector");
  for (size_t i = 0; i < 3; ++i) {
    if (!v[i].is_number()) invalid(where + "." + key + " is not a 3-vector");
    out[i] = (float)v[i].as_number();
  }
}
uint32_t mask_of(const Json& obj) {
  if (!obj.has("Mask")) return R2_MASK_RENDER;
  const Json& m = obj["Mask"];
  uint32_t r = 0;
  for (const Json& item : m.elements())
    if (item.is_string()) r |= mask_from_string(item.as_string());
  return r;
}

void shape_material(const Json& o, const std::string& where, r2_material* m) {
  memset(m, 0, sizeof(*m));
  vec3(o, "DiffuseReflection", where, m->diffuse);
  m->diffuse_roughness = num(o, "DiffuseRoughness", where);
  vec3(o, "SpecularReflection", where, m->specular);
  m->alpha_x = num(o, "AlphaX", where);
  m->alpha_y = num(o, "AlphaY", where);
  m->eta_i = num(o, "EtaI", where);
  m->eta_t = num(o, "EtaT", where);
}

}  // namespace

uint32_t mask_from_string(const std::string& s) {
  if (s == "NONE") return 0u;
  if (s == "FILTER") return R2_MASK_FILTER;
  if (s == "RENDER") return R2_MASK_RENDER;
  return R2_MASK_ALL;
}

PipelineConfig load_config(const std::string& configPath) {
  const Json root = Json::parse(read_text_file(configPath));
  PipelineConfig c;
  memset(&c.filter, 0, sizeof(c.filter));
  memset(&c.camera, 0, sizeof(c.camera));
  // General (fillGeneralInfo, config_loader.cu:44-76)
  const Json& g = need(root, "General", "config");
  c.frameWidth = unum(g, "FrameWidth", "General");
  c.frameHeight = unum(g, "FrameHeight", "General");
  c.channelsPerPixel = unum(g, "ChannelsPerPixel", "General");
  c.samples = unum(g, "Samples", "General");
  c.gamma = num(g, "Gamma", "General");
  c.useBrickGrid = flag(g, "UseBrickGrid", "General");
  c.debugMode = str(g, "DebugMode", "General");
  // Filtering (fillFilteringInfo, 78-104)
  const Json& f = need(root, "Filtering", "config");
  c.filterActive = flag(f, "Active", "Filtering");
  c.filter.samples_per_voxel = unum(f, "SamplesPerVoxel", "Filtering");
  c.filter.min_voxel_size = num(f, "MinVoxelSize", "Filtering");
  c.filter.lods = unum(f, "LODs", "Filtering");
  c.filterDebug = flag(f, "Debug", "Filtering");
  c.debugSamples = unum(f, "DebugSamples", "Filtering");
  c.filter.sigma_t = num(f, "SigmaT", "Filtering");
  c.filter.estimation_iterations = unum(f, "EstimationIterations", "Filtering");
  c.filter.alpha = num(f, "Alpha", "Filtering");
  c.filter.clip_rays = flag(f, "ClipRays", "Filtering") ? 1u : 0u;
  c.filter.seed = 0;
  // Camera (fillCameraInfo, 106-121)
  const Json& cam = need(root, "Camera", "config");
  c.camera.width = c.frameWidth;
  c.camera.height = c.frameHeight;
  c.camera.fov_deg = num(cam, "Fov", "Camera");
  vec3(cam, "Pos", "Camera", c.camera.pos);
  vec3(cam, "LookAt", "Camera", c.camera.look_at);
  vec3(cam, "Up", "Camera", c.camera.up);
  // Scene (fillSceneInfo, 306-338)
  const Json& sc = need(root, "Scene", "config");
  c.envmap = str(sc, "Envmap", "Scene");
  c.scenedescription = str(sc, "Scenedescription", "Scene");
  const Json objs = Json::parse(read_text_file(c.scenedescription));
  if (!objs.is_array()) invalid("scene description is not an array");
  for (size_t i = 0; i < objs.size(); ++i) {
    const Json& o = objs[i];
    const std::string where = "scene object " + std::to_string(i);
    const std::string type = str(o, "Type", where);
    SceneObjectDesc d;
    memset(&d.material, 0, sizeof(d.material));
    if (type == "Circle" || type == "Sphere") {
      d.kind = type == "Circle" ? SceneObjectDesc::kCircle : SceneObjectDesc::kSphere;
      vec3(o, "Pos", where, d.pos);
      d.radius = num(o, "Radius", where);
      vec3(o, "Normal", where, d.normal);
      shape_material(o, where, &d.material);
    } else if (type == "Medium") {
      d.kind = SceneObjectDesc::kMedium;
      d.path = str(o, "Path", where);
      vec3(o, "SigmaA", where, d.sigmaA);
      vec3(o, "SigmaS", where, d.sigmaS);
      if (o.has("G")) {
        d.hasG = true;
        d.g = num(o, "G", where);
      }
      vec3(o, "Pos", where, d.pos);
      vec3(o, "Orientation", where, d.orientation);
      vec3(o, "Scaling", where, d.scaling);
    } else if (type == "Mesh") {
      d.kind = SceneObjectDesc::kMesh;
      d.directory = str(o, "Directory", where);
      d.filename = str(o, "Filename", where);
      vec3(o, "Pos", where, d.pos);
      vec3(o, "Orientation", where, d.orientation);
      vec3(o, "Scaling", where, d.scaling);
    } else {
      continue;  // other types are ignored
    }
    d.mask = mask_of(o);
    c.objects.push_back(d);
  }
  return c;
}

}  // namespace r2
