// Host construction, file I/O and lookup of the NanoVDB grid (see nvdb.h).
#include "nvdb.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <map>
#include <stdexcept>
#include <tuple>

#include "runtime.h"

namespace r2 {
namespace nvdb {

namespace {

constexpr size_t kGridOff = 0;
constexpr size_t kTreeOff = sizeof(GridData);
constexpr size_t kRootOff = kTreeOff + sizeof(TreeData);

inline uint32_t lower_index_in_upper(int32_t x, int32_t y, int32_t z) {
  return ((uint32_t)((x & 4095) >> 7) << 10) | ((uint32_t)((y & 4095) >> 7) << 5) | (uint32_t)((z & 4095) >> 7);
}
inline uint32_t leaf_index_in_lower(int32_t x, int32_t y, int32_t z) {
  return ((uint32_t)((x & 127) >> 3) << 8) | ((uint32_t)((y & 127) >> 3) << 4) | (uint32_t)((z & 127) >> 3);
}

struct BBox {
  int32_t v[6] = {INT32_MAX, INT32_MAX, INT32_MAX, INT32_MIN, INT32_MIN, INT32_MIN};
  void add(const int32_t* o) {
    for (int k = 0; k < 3; ++k) {
      v[k] = std::min(v[k], o[k]);
      v[3 + k] = std::max(v[3 + k], o[3 + k]);
    }
  }
};

inline void set_bit(uint64_t* words, uint32_t i) { words[i >> 6] |= 1ull << (i & 63); }
inline bool get_bit(const uint64_t* words, uint32_t i) { return (words[i >> 6] >> (i & 63)) & 1ull; }

// Map from the glm mat4x3 index->model transform (row-major 3x3 + translation).
Map make_map(const float* i2m, const float* m2i) {
  Map m;
  memset(&m, 0, sizeof(m));
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) {
      m.matF[3 * r + c] = i2m[3 * c + r];
      m.invMatF[3 * r + c] = m2i[3 * c + r];
      m.matD[3 * r + c] = i2m[3 * c + r];
      m.invMatD[3 * r + c] = m2i[3 * c + r];
    }
    m.vecF[r] = i2m[9 + r];
    m.vecD[r] = i2m[9 + r];
  }
  m.taperF = 1.0f;
  m.taperD = 1.0;
  return m;
}

void apply_map(const Map& m, double x, double y, double z, double* o) {
  for (int r = 0; r < 3; ++r) o[r] = m.matD[3 * r] * x + m.matD[3 * r + 1] * y + m.matD[3 * r + 2] * z + m.vecD[r];
}

}  // namespace

std::vector<uint8_t> build_grid(const std::vector<LeafBlock>& leavesIn, const std::vector<r2_voxel>& valuesIn,
                                const float* indexToModel, const float* modelToIndex, const char* name) {
  R2_REQUIRE(valuesIn.size() == leavesIn.size() * 512, R2_ERR_INVALID_ARGUMENT, "leaf values size mismatch");
  // breadth-first order: upper tile key, lower index in upper, leaf index in lower
  std::vector<size_t> order(leavesIn.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  auto key = [&](size_t i) {
    const int32_t* o = leavesIn[i].origin;
    uint64_t k = root_key(o[0] & ~4095, o[1] & ~4095, o[2] & ~4095);
    return std::make_tuple(k, lower_index_in_upper(o[0], o[1], o[2]), leaf_index_in_lower(o[0], o[1], o[2]));
  };
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key(a) < key(b); });
  // distinct lower and upper nodes
  std::vector<std::array<int32_t, 3>> uppers, lowers;
  std::vector<uint32_t> leafLower(order.size()), lowerUpper;
  for (size_t k = 0; k < order.size(); ++k) {
    const int32_t* o = leavesIn[order[k]].origin;
    std::array<int32_t, 3> u = {o[0] & ~4095, o[1] & ~4095, o[2] & ~4095};
    std::array<int32_t, 3> l = {o[0] & ~127, o[1] & ~127, o[2] & ~127};
    if (uppers.empty() || uppers.back() != u) uppers.push_back(u);
    if (lowers.empty() || lowers.back() != l) {
      lowers.push_back(l);
      lowerUpper.push_back((uint32_t)uppers.size() - 1);
    }
    leafLower[k] = (uint32_t)lowers.size() - 1;
  }
  const size_t nLeaf = order.size(), nLower = lowers.size(), nUpper = uppers.size();
  const size_t upperOff = kRootOff + sizeof(RootData) + nUpper * sizeof(RootTile);
  const size_t lowerOff = upperOff + nUpper * kUpperSize;
  const size_t leafOff = lowerOff + nLower * kLowerSize;
  const size_t total = leafOff + nLeaf * sizeof(LeafNode);
  std::vector<uint8_t> buf(total, 0);
  uint8_t* B = buf.data();
  const r2_voxel bg = [] {
    r2_voxel v;
    memset(&v, 0, sizeof(v));
    v.ior = 0x3C00u;  // background: zeros with ior 1 (openvdb_backend.cpp:30-42)
    return v;
  }();

  // leaves
  std::vector<BBox> lowerBox(nLower), upperBox(nUpper);
  uint64_t voxelCount = 0;
  for (size_t k = 0; k < nLeaf; ++k) {
    const LeafBlock& lb = leavesIn[order[k]];
    LeafNode* L = reinterpret_cast<LeafNode*>(B + leafOff + k * sizeof(LeafNode));
    memcpy(L->valueMask, lb.mask, sizeof(lb.mask));
    memcpy(L->values, &valuesIn[order[k] * 512], 512 * sizeof(r2_voxel));
    int32_t mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (uint32_t i = 0; i < 512; ++i) {
      if (!get_bit(lb.mask, i)) continue;
      ++voxelCount;
      int32_t c[3] = {lb.origin[0] + (int32_t)(i >> 6), lb.origin[1] + (int32_t)((i >> 3) & 7),
                      lb.origin[2] + (int32_t)(i & 7)};
      for (int a = 0; a < 3; ++a) {
        mn[a] = std::min(mn[a], c[a]);
        mx[a] = std::max(mx[a], c[a]);
      }
    }
    for (int a = 0; a < 3; ++a) {
      L->bboxMin[a] = mn[a];
      L->bboxDif[a] = (uint8_t)(mx[a] - mn[a]);
    }
    L->flags = 0;
    int32_t bb[6] = {mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]};
    lowerBox[leafLower[k]].add(bb);
  }
  // lower nodes: child offsets to their leaves, tiles = background
  for (size_t l = 0; l < nLower; ++l) {
    uint8_t* N = B + lowerOff + l * kLowerSize;
    auto* H = reinterpret_cast<InternalHeader<4>*>(N);
    uint8_t* table = N + sizeof(InternalHeader<4>);
    for (uint32_t t = 0; t < 4096; ++t) memcpy(table + 32 * t, &bg, 32);
    memcpy(H->bbox, lowerBox[l].v, sizeof(H->bbox));
    upperBox[lowerUpper[l]].add(lowerBox[l].v);
  }
  for (size_t k = 0; k < nLeaf; ++k) {
    const int32_t* o = leavesIn[order[k]].origin;
    uint8_t* N = B + lowerOff + leafLower[k] * kLowerSize;
    auto* H = reinterpret_cast<InternalHeader<4>*>(N);
    uint32_t idx = leaf_index_in_lower(o[0], o[1], o[2]);
    set_bit(H->childMask, idx);
    int64_t off = (int64_t)(leafOff + k * sizeof(LeafNode)) - (int64_t)(lowerOff + leafLower[k] * kLowerSize);
    uint8_t* entry = N + sizeof(InternalHeader<4>) + 32 * idx;
    memset(entry, 0, 32);
    memcpy(entry, &off, 8);
  }
  // upper nodes
  for (size_t u = 0; u < nUpper; ++u) {
    uint8_t* N = B + upperOff + u * kUpperSize;
    auto* H = reinterpret_cast<InternalHeader<5>*>(N);
    uint8_t* table = N + sizeof(InternalHeader<5>);
    for (uint32_t t = 0; t < 32768; ++t) memcpy(table + 32 * t, &bg, 32);
    memcpy(H->bbox, upperBox[u].v, sizeof(H->bbox));
  }
  for (size_t l = 0; l < nLower; ++l) {
    const auto& lo = lowers[l];
    uint32_t u = lowerUpper[l];
    uint8_t* N = B + upperOff + u * kUpperSize;
    auto* H = reinterpret_cast<InternalHeader<5>*>(N);
    uint32_t idx = lower_index_in_upper(lo[0], lo[1], lo[2]);
    set_bit(H->childMask, idx);
    int64_t off = (int64_t)(lowerOff + l * kLowerSize) - (int64_t)(upperOff + u * kUpperSize);
    uint8_t* entry = N + sizeof(InternalHeader<5>) + 32 * idx;
    memset(entry, 0, 32);
    memcpy(entry, &off, 8);
  }
  // root
  RootData* R = reinterpret_cast<RootData*>(B + kRootOff);
  BBox rootBox;
  for (size_t u = 0; u < nUpper; ++u) rootBox.add(upperBox[u].v);
  if (nUpper == 0) memset(rootBox.v, 0, sizeof(rootBox.v));
  memcpy(R->bbox, rootBox.v, sizeof(R->bbox));
  R->tableSize = (uint32_t)nUpper;
  memcpy(R->background, &bg, 32);
  for (size_t u = 0; u < nUpper; ++u) {
    RootTile* T = reinterpret_cast<RootTile*>(B + kRootOff + sizeof(RootData) + u * sizeof(RootTile));
    T->key = root_key(uppers[u][0], uppers[u][1], uppers[u][2]);
    T->child = (int64_t)(upperOff + u * kUpperSize) - (int64_t)kRootOff;
    T->state = 0;
    memcpy(T->value, &bg, 32);
  }
  // tree
  TreeData* Tr = reinterpret_cast<TreeData*>(B + kTreeOff);
  Tr->nodeOffset[0] = leafOff - kTreeOff;
  Tr->nodeOffset[1] = lowerOff - kTreeOff;
  Tr->nodeOffset[2] = upperOff - kTreeOff;
  Tr->nodeOffset[3] = kRootOff - kTreeOff;
  Tr->nodeCount[0] = (uint32_t)nLeaf;
  Tr->nodeCount[1] = (uint32_t)nLower;
  Tr->nodeCount[2] = (uint32_t)nUpper;
  Tr->voxelCount = voxelCount;
  // grid
  GridData* G = reinterpret_cast<GridData*>(B + kGridOff);
  G->magic = kMagic;
  G->checksum = ~0ull;
  G->version = kVersion;
  G->flags = kFlagHasBBox | kFlagIsBreadthFirst;
  G->gridIndex = 0;
  G->gridCount = 1;
  G->gridSize = total;
  snprintf(G->gridName, sizeof(G->gridName), "%s", name ? name : "");
  G->map = make_map(indexToModel, modelToIndex);
  double a[3], b[3];
  apply_map(G->map, rootBox.v[0], rootBox.v[1], rootBox.v[2], a);
  apply_map(G->map, rootBox.v[3] + 1.0, rootBox.v[4] + 1.0, rootBox.v[5] + 1.0, b);
  for (int k = 0; k < 3; ++k) {
    G->worldBBox[k] = std::min(a[k], b[k]);
    G->worldBBox[3 + k] = std::max(a[k], b[k]);
    double c0 = G->map.matD[k], c1 = G->map.matD[3 + k], c2 = G->map.matD[6 + k];
    G->voxelSize[k] = sqrt(c0 * c0 + c1 * c1 + c2 * c2);  // length of column k
  }
  G->gridClass = kGridClassUnknown;
  G->gridType = kGridTypeVec4d;
  G->blindMetadataOffset = (int64_t)total;
  G->blindMetadataCount = 0;
  return buf;
}

#pragma pack(push, 1)
struct FileHeader {
  uint64_t magic;
  uint32_t version;
  uint16_t gridCount;
  uint16_t codec;
};
struct FileMeta {
  uint64_t gridSize, fileSize, nameKey, voxelCount;
  uint32_t gridType, gridClass;
  double worldBBox[6];
  int32_t indexBBox[6];
  double voxelSize[3];
  uint32_t nameSize;
  uint32_t nodeCount[4];
  uint32_t tileCount[3];
  uint16_t codec, padding;
  uint32_t version;
};
#pragma pack(pop)
static_assert(sizeof(FileHeader) == 16, "file header");
static_assert(sizeof(FileMeta) == 176, "file metadata");

void write_file(const std::string& path, const std::vector<uint8_t>& grid) {
  const GridData* G = grid_data(grid.data());
  const TreeData* T = tree_data(grid.data());
  FileHeader h = {kMagic, kVersion, 1, 0};
  FileMeta m;
  memset(&m, 0, sizeof(m));
  m.gridSize = grid.size();
  m.fileSize = grid.size();
  m.nameKey = 0;
  for (const unsigned char* s = (const unsigned char*)G->gridName; *s; ++s) m.nameKey = m.nameKey * 67 + *s;
  m.voxelCount = T->voxelCount;
  m.gridType = G->gridType;
  m.gridClass = G->gridClass;
  memcpy(m.worldBBox, G->worldBBox, sizeof(m.worldBBox));
  index_bbox(grid.data(), m.indexBBox);
  memcpy(m.voxelSize, G->voxelSize, sizeof(m.voxelSize));
  m.nameSize = (uint32_t)strlen(G->gridName) + 1;
  m.nodeCount[0] = T->nodeCount[0];
  m.nodeCount[1] = T->nodeCount[1];
  m.nodeCount[2] = T->nodeCount[2];
  m.nodeCount[3] = 1;
  m.version = kVersion;
  FILE* f = fopen(path.c_str(), "wb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path + " for writing");
  bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(&m, sizeof(m), 1, f) == 1 &&
            fwrite(G->gridName, 1, m.nameSize, f) == m.nameSize &&
            fwrite(grid.data(), 1, grid.size(), f) == grid.size();
  ok = (fclose(f) == 0) && ok;
  R2_REQUIRE(ok, R2_ERR_IO, "short write to " + path);
}

std::vector<uint8_t> read_file(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path);
  FileHeader h;
  FileMeta m;
  bool ok = fread(&h, sizeof(h), 1, f) == 1 && fread(&m, sizeof(m), 1, f) == 1;
  if (!ok || h.magic != kMagic || h.gridCount < 1 || h.codec != 0 || m.gridSize < kRootOff + sizeof(RootData) ||
      m.gridSize > (1ull << 40) || m.nameSize > (1u << 20)) {
    fclose(f);
    throw Error{R2_ERR_IO, "not an uncompressed NanoVDB file: " + path};
  }
  std::vector<char> name(m.nameSize);
  std::vector<uint8_t> grid(m.gridSize);
  ok = fread(name.data(), 1, m.nameSize, f) == m.nameSize && fread(grid.data(), 1, grid.size(), f) == grid.size();
  fclose(f);
  R2_REQUIRE(ok, R2_ERR_IO, "truncated NanoVDB file: " + path);
  const GridData* G = grid_data(grid.data());
  R2_REQUIRE(G->magic == kMagic && G->gridSize == grid.size(), R2_ERR_IO, "corrupt NanoVDB grid in " + path);
  R2_REQUIRE(G->gridType == kGridTypeVec4d, R2_ERR_UNSUPPORTED, "only Vec4d (SGGX payload) grids are supported");
  // structural checks so later lookups stay in bounds
  const TreeData* T = tree_data(grid.data());
  const size_t leafEnd = kTreeOff + T->nodeOffset[0] + (size_t)T->nodeCount[0] * sizeof(LeafNode);
  const size_t lowerEnd = kTreeOff + T->nodeOffset[1] + (size_t)T->nodeCount[1] * kLowerSize;
  const size_t upperEnd = kTreeOff + T->nodeOffset[2] + (size_t)T->nodeCount[2] * kUpperSize;
  R2_REQUIRE(leafEnd <= grid.size() && lowerEnd <= grid.size() && upperEnd <= grid.size(), R2_ERR_IO,
             "NanoVDB node tables exceed the grid size in " + path);
  const RootData* R = reinterpret_cast<const RootData*>(grid.data() + kRootOff);
  R2_REQUIRE(kRootOff + sizeof(RootData) + (size_t)R->tableSize * sizeof(RootTile) <= grid.size(), R2_ERR_IO,
             "NanoVDB root table exceeds the grid size in " + path);
  return grid;
}

const GridData* grid_data(const uint8_t* buf) { return reinterpret_cast<const GridData*>(buf + kGridOff); }
const TreeData* tree_data(const uint8_t* buf) { return reinterpret_cast<const TreeData*>(buf + kTreeOff); }

void index_bbox(const uint8_t* buf, int32_t out[6]) {
  const RootData* R = reinterpret_cast<const RootData*>(buf + kRootOff);
  memcpy(out, R->bbox, 6 * sizeof(int32_t));
}

r2_voxel host_value(const uint8_t* buf, int x, int y, int z, bool* active) {
  const RootData* R = reinterpret_cast<const RootData*>(buf + kRootOff);
  r2_voxel bg;
  memcpy(&bg, R->background, sizeof(bg));
  *active = false;
  uint64_t key = root_key(x & ~4095, y & ~4095, z & ~4095);
  const RootTile* tiles = reinterpret_cast<const RootTile*>(buf + kRootOff + sizeof(RootData));
  for (uint32_t i = 0; i < R->tableSize; ++i) {
    if (tiles[i].key != key) continue;
    if (tiles[i].child == 0) return bg;
    const uint8_t* U = buf + kRootOff + tiles[i].child;
    auto* UH = reinterpret_cast<const InternalHeader<5>*>(U);
    uint32_t ui = lower_index_in_upper(x, y, z);
    if (!get_bit(UH->childMask, ui)) return bg;
    int64_t off;
    memcpy(&off, U + sizeof(InternalHeader<5>) + 32 * ui, 8);
    const uint8_t* Lw = U + off;
    auto* LH = reinterpret_cast<const InternalHeader<4>*>(Lw);
    uint32_t li = leaf_index_in_lower(x, y, z);
    if (!get_bit(LH->childMask, li)) return bg;
    memcpy(&off, Lw + sizeof(InternalHeader<4>) + 32 * li, 8);
    const LeafNode* Lf = reinterpret_cast<const LeafNode*>(Lw + off);
    uint32_t vi = ((uint32_t)(x & 7) << 6) | ((uint32_t)(y & 7) << 3) | (uint32_t)(z & 7);
    *active = get_bit(Lf->valueMask, vi);
    return Lf->values[vi];
  }
  return bg;
}

std::vector<size_t> leaf_offsets(const uint8_t* buf) {
  const TreeData* T = tree_data(buf);
  std::vector<size_t> r(T->nodeCount[0]);
  for (size_t i = 0; i < r.size(); ++i) r[i] = kTreeOff + T->nodeOffset[0] + i * sizeof(LeafNode);
  return r;
}

}  // namespace nvdb
}  // namespace r2
