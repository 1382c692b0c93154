// Filter output stage: active topology and leaf extraction for the NanoVDB
// grid (COpenvdbBackend::setValues, raytracer/src/filtering/openvdb_backend.cpp:108-132),
// the brick grid of density majorants (CHostBrickGrid,
// raytracer/src/grid_brick/host_grid_brick.cpp:61-152) and their files.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "nvdb.h"
#include "runtime.h"

namespace r2 {

// Brick grid constants (include/grid_brick/common.hpp:14-18).
constexpr uint32_t kBrickSize = 8;
constexpr uint32_t kBrickBitsPerAxis = 10;
constexpr uint32_t kMaxBricks = 1u << kBrickBitsPerAxis;
constexpr uint32_t kNumMipmaps = 3;

// Brick grid on the host (the .brickgrid contents, CHostBrickGrid's fields).
struct BrickGridHost {
  float transform[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};  // glm::mat4, identity when built
  uint32_t nBricks[3] = {0, 0, 0};   // per axis, multiple of 8
  uint32_t atlasDim[3] = {0, 0, 0};  // voxels
  uint32_t brickCount = 0;           // bricks with a non-constant range (atlas slots)
  float minorant = 0.0f, majorant = 0.0f;  // density min / max over the grid's voxels (getMinorantMajorant)
  std::vector<uint32_t> indirection;  // encode_ptr of the atlas slot, 0 for constant bricks
  std::vector<uint32_t> range;        // two IEEE halves (min, max) of the dilated brick
  std::vector<uint32_t> mips[kNumMipmaps];
  std::vector<uint8_t> atlas;         // atlasDim voxels, x fastest
};

// Extracts the active 8^3 leaves of a dense payload grid (active = density > 0
// or one of the 8 grid corners) with their masks and NanoVDB-ordered values.
void extract_leaves(const r2_voxel* d_dense, const int32_t numVoxels[3], cudaStream_t s,
                    std::vector<nvdb::LeafBlock>* leaves, std::vector<r2_voxel>* values);

// Builds the brick grid of the grid's density (inactive voxels read as 0).
void build_brick_grid(const r2_voxel* d_dense, const int32_t numVoxels[3], cudaStream_t s, BrickGridHost* out);

// The .brickgrid file in the reference's layout: a cereal PortableBinary
// archive of CHostBrickGrid (raytracer/src/grid_brick/serialization.cpp:37-40):
// a leading byte 1 (little-endian data), then transform (16 float, column
// major), n_bricks (3 uint32), min_maj (2 float), brick_counter (uint64), and
// the Buf3D fields indirection, range (uint32), atlas (uint8), each as its
// stride (3 uint32), element count (uint64) and elements, then range_mipmaps
// as a count (uint64) followed by that many uint32 Buf3Ds.
void write_brick_grid(const std::string& path, const BrickGridHost& g);
BrickGridHost read_brick_grid(const std::string& path);

// CHostBrickGrid encodings (common.hpp:23-53).
uint32_t encode_range(float lo, float hi);
void decode_range(uint32_t v, float* lo, float* hi);
uint32_t encode_ptr(uint32_t x, uint32_t y, uint32_t z);
void decode_ptr(uint32_t v, uint32_t* x, uint32_t* y, uint32_t* z);

// Volume description of one filtered LOD (CVolumeDescriptionManager,
// raytracer/src/filtering/volume_description_manager.cpp:50-144).
struct VolumeDescription {
  int32_t numVoxels[3];
  float bbmin[3], bbmax[3];
};
// Reads (if present) and rewrites ./filtering/volume_description.json with the
// entry descriptions[model][to_string(voxelSize)] added or replaced.
void store_volume_description(const std::string& path, const std::string& model, const std::string& voxelSizeKey,
                              const VolumeDescription& d);

// std::to_string(float) ("%f").
std::string float_key(float v);

}  // namespace r2
