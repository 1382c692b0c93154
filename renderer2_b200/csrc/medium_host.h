// Loading of a filtered medium for rendering: the NanoVDB grid (leaves copied
// to the device with a flat leaf index), the brick grid and the transforms of
// CNVDBMedium::init (raytracer/src/medium/nvdb_medium.cu:130-173,
// getIndexToModelTransformation / getMaxValue) and of the medium's scene
// object (raytracer/src/scene/sceneobject.cu:50-65, getFilterRenderRatio 108-114).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "media.cuh"
#include "runtime.h"
#include "volume.h"

namespace r2 {

// CNVDBMedium::getVoxelSizeFiltering (nvdb_medium.cu:180-188): the trailing
// "\d+\.\d+" of the path (without extension), as std::stof reads it.
float voxel_size_from_path(const std::string& path);

// One loaded medium (CNVDBMedium): grid, brick grid and the grid's
// transforms.  Instances placed in a scene share it; view holds the grid's
// fields (the instance fields are set per instance by place_medium).
struct MediumHost {
  MediumView view;  // device pointers are filled in by upload()
  V3 boxMin, boxMax;  // the grid's world box (model space of the medium)
  float voxelSizeFiltering;
  std::vector<uint8_t> leaves;
  std::vector<int32_t> leafIndex;
  BrickGridHost bricks;
  DBuf<uint8_t> dLeaves, dAtlas;
  DBuf<int32_t> dLeafIndex;
  DBuf<uint32_t> dIndirection, dRange, dMips[3];
  bool uploaded = false;
  void upload(cudaStream_t s);
  size_t device_bytes() const;
};

// Loads <path>.nvdb and <path>.brickgrid with the medium coefficients; hg
// selects the Henyey-Greenstein phase function with asymmetry g
// (CNVDBMedium(path, sigma_a, sigma_s, g), nvdb_medium.cu:27-43) instead of
// the SGGX one (45-61).
std::unique_ptr<MediumHost> load_medium(const std::string& path, const float sigmaA[3], const float sigmaS[3],
                                        bool hg = false, float g = 0.0f);

// The view of one instance of a loaded medium placed with
// T(pos) R(orientation) S(scaling) (the medium's scene object,
// sceneobject.cu:50-65, getFilterRenderRatio 108-114); device pointers are
// those of the last upload.
MediumView place_medium(const MediumHost& m, V3 pos, V3 orientation, V3 scaling);

}  // namespace r2
