// config.json + scenedescription.json: CConfigLoader::loadConfig
// (raytracer/src/backend/config_loader.cu:340-368) and the scene-object
// builders it calls (addCircle / addSphere / addMedium / addMesh, 123-305).
// Every key the reference requires is required here (a missing one makes the
// config invalid); relative paths resolve against the working directory, as
// in the reference.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/r2.h"

namespace r2 {

struct SceneObjectDesc {
  enum Kind { kCircle, kSphere, kMedium, kMesh } kind;
  float pos[3] = {0, 0, 0};
  float normal[3] = {0, 1, 0};       // Circle / Sphere "Normal"
  float orientation[3] = {0, 1, 0};  // Medium / Mesh "Orientation"
  float scaling[3] = {1, 1, 1};
  float radius = 0.0f;
  r2_material material;              // Circle / Sphere
  std::string path;                  // Medium (without extension)
  float sigmaA[3] = {0, 0, 0}, sigmaS[3] = {0, 0, 0};
  bool hasG = false;                 // Medium "G": Henyey-Greenstein phase function
  float g = 0.0f;
  std::string directory, filename;   // Mesh
  uint32_t mask = R2_MASK_RENDER;    // default when "Mask" is absent
};

struct PipelineConfig {
  // General
  uint32_t frameWidth = 0, frameHeight = 0, channelsPerPixel = 0, samples = 0;
  float gamma = 2.0f;
  bool useBrickGrid = false;
  std::string debugMode;
  // Filtering
  bool filterActive = false;
  r2_filter_params filter;
  bool filterDebug = false;
  uint32_t debugSamples = 0;
  // Camera
  r2_camera camera;
  // Scene
  std::string envmap, scenedescription;
  std::vector<SceneObjectDesc> objects;
};

// Throws Error(R2_ERR_INVALID_CONFIG) naming the first missing or malformed key.
PipelineConfig load_config(const std::string& configPath);

// "NONE" / "FILTER" / "RENDER" / anything else = ALL (sceneobject_mask.cpp:4-17).
uint32_t mask_from_string(const std::string& s);

}  // namespace r2
