// NanoVDB grid of SFilteredDataCompact payloads (the reference's
// Vec4d grid, tree 5-4-3: raytracer/include/filtering/openvdb_data.hpp:4-5,
// written by openToNanoVDB + io::writeGrid in openvdb_backend.cpp:134-157).
//
// The NanoVDB library is not available here; the byte layout below follows
// NanoVDB's published structure for version 32.3 (GridData 672 B, TreeData
// 64 B, RootData + 32-byte-aligned tiles, internal nodes with value/child
// masks and a tile/child-offset table, 8^3 leaves with a 512-bit value mask
// and 512 values stored z-fastest).  Statistics fields (min/max/average/
// standard deviation) are written as zero with the corresponding grid flags
// cleared, and the checksum is left empty.  Readers in this library rely only
// on the structure, not on those fields.
//
// For rendering, a loaded grid gets a flat leaf index (one int32 per 8^3
// block of the index box), so a voxel fetch is two dependent loads instead of
// a root/upper/lower walk; the leaf values are read in place from the NanoVDB
// buffer.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/r2.h"
#include "r2_core.h"

namespace r2 {
namespace nvdb {

constexpr uint64_t kMagic = 0x304244566f6e614eull;  // "NanoVDB0"
constexpr uint32_t kVersion = (32u << 21) | (3u << 10) | 3u;
constexpr uint32_t kGridTypeVec4d = 18;
constexpr uint32_t kGridClassUnknown = 0;
constexpr uint32_t kFlagHasBBox = 1u << 1;
constexpr uint32_t kFlagIsBreadthFirst = 1u << 5;

#pragma pack(push, 1)
struct Map {  // 264 B
  float matF[9], invMatF[9], vecF[3], taperF;
  double matD[9], invMatD[9], vecD[3], taperD;
};
#pragma pack(pop)
static_assert(sizeof(Map) == 264, "Map size");

struct alignas(32) GridData {  // 672 B
  uint64_t magic;
  uint64_t checksum;
  uint32_t version;
  uint32_t flags;
  uint32_t gridIndex;
  uint32_t gridCount;
  uint64_t gridSize;
  char gridName[256];
  Map map;
  double worldBBox[6];
  double voxelSize[3];
  uint32_t gridClass;
  uint32_t gridType;
  int64_t blindMetadataOffset;
  uint32_t blindMetadataCount;
};
static_assert(sizeof(GridData) == 672, "GridData size");

struct TreeData {  // 64 B
  uint64_t nodeOffset[4];  // leaf, lower, upper, root: byte offsets from the tree
  uint32_t nodeCount[3];   // leaf, lower, upper
  uint32_t tileCount[3];   // active tiles in lower, upper, root
  uint64_t voxelCount;
};
static_assert(sizeof(TreeData) == 64, "TreeData size");

struct alignas(32) RootData {  // 160 B, followed by tableSize tiles
  int32_t bbox[6];
  uint32_t tableSize;
  alignas(8) uint8_t background[32];
  uint8_t minimum[32];
  uint8_t maximum[32];
  double average;
  double stdDevi;
};
static_assert(sizeof(RootData) == 160, "RootData size");

struct alignas(32) RootTile {  // 64 B
  uint64_t key;
  int64_t child;  // byte offset from the root to the child (0: constant tile)
  uint32_t state;
  alignas(8) uint8_t value[32];
};
static_assert(sizeof(RootTile) == 64, "RootTile size");

// Internal node header; the table of (1 << 3*LOG2DIM) 32-byte entries follows
// at a 32-byte boundary.  Each entry is a tile value or an int64 byte offset
// from this node to its child.
template <int LOG2DIM>
struct alignas(32) InternalHeader {
  static constexpr int kWords = (1 << (3 * LOG2DIM)) / 64;
  int32_t bbox[6];
  uint64_t flags;
  uint64_t valueMask[kWords];
  uint64_t childMask[kWords];
  uint8_t minimum[32];
  uint8_t maximum[32];
  double average;
  double stdDevi;
};
static_assert(sizeof(InternalHeader<5>) == 8320, "upper header size");
static_assert(sizeof(InternalHeader<4>) == 1152, "lower header size");
constexpr size_t kUpperSize = sizeof(InternalHeader<5>) + 32768ull * 32;
constexpr size_t kLowerSize = sizeof(InternalHeader<4>) + 4096ull * 32;

struct alignas(32) LeafNode {  // 16544 B
  int32_t bboxMin[3];
  uint8_t bboxDif[3];
  uint8_t flags;
  uint64_t valueMask[8];
  uint8_t minimum[32];
  uint8_t maximum[32];
  double average;
  double stdDevi;
  r2_voxel values[512];  // index (x&7)<<6 | (y&7)<<3 | (z&7)
};
static_assert(sizeof(LeafNode) == 16544, "LeafNode size");

// One active 8^3 block produced on the device: origin (multiple of 8), value
// mask and the 512 payloads in NanoVDB order (inactive voxels = background).
struct LeafBlock {
  int32_t origin[3];
  uint64_t mask[8];
};

// Root key of a tile whose upper node starts at (x, y, z) (multiples of 4096).
inline uint64_t root_key(int32_t x, int32_t y, int32_t z) {
  return ((uint64_t)(uint32_t)z >> 12) | (((uint64_t)(uint32_t)y >> 12) << 21) |
         (((uint64_t)(uint32_t)x >> 12) << 42);
}

// Builds the breadth-first grid buffer.  index_to_model: the LOD's transform
// (12 floats, glm mat4x3); leaves: origins+masks; values: 512 payloads per
// leaf in the same order.
std::vector<uint8_t> build_grid(const std::vector<LeafBlock>& leaves, const std::vector<r2_voxel>& values,
                                const float* indexToModel, const float* modelToIndex, const char* name);

// NanoVDB file (io::writeGrid layout: 16-byte header, 176-byte grid
// metadata, name, grid buffer; codec NONE).
void write_file(const std::string& path, const std::vector<uint8_t>& grid);
std::vector<uint8_t> read_file(const std::string& path);

// Structure views of a grid buffer.
const GridData* grid_data(const uint8_t* buf);
const TreeData* tree_data(const uint8_t* buf);
// Host lookup (for tests and the loader): payload at index (x, y, z) and
// whether it is active.
r2_voxel host_value(const uint8_t* buf, int x, int y, int z, bool* active);
// Active index box [min, max] (inclusive) from the root node.
void index_bbox(const uint8_t* buf, int32_t out[6]);
// All leaves (byte offsets from the buffer start).
std::vector<size_t> leaf_offsets(const uint8_t* buf);

}  // namespace nvdb
}  // namespace r2
