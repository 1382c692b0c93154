// Host side of medium loading (see medium_host.h).
#include <ctype.h>
#include <string.h>

#include <algorithm>

#include "host_math.h"
#include "medium_host.h"
#include "nvdb.h"

namespace r2 {

float voxel_size_from_path(const std::string& path) {
  // leftmost match of (\d+\.\d+)$: trailing digits, a dot, the maximal digit run before it
  size_t i = path.size();
  while (i > 0 && isdigit((unsigned char)path[i - 1])) --i;
  R2_REQUIRE(i < path.size() && i > 0 && path[i - 1] == '.', R2_ERR_INVALID_CONFIG,
             "medium path has no trailing voxel size (\\d+.\\d+): " + path);
  const size_t dot = i - 1;
  size_t k = dot;
  while (k > 0 && isdigit((unsigned char)path[k - 1])) --k;
  R2_REQUIRE(k < dot, R2_ERR_INVALID_CONFIG, "medium path has no trailing voxel size (\\d+.\\d+): " + path);
  return std::stof(path.substr(k));
}

// mat4 whose last row is exactly (0, 0, 0, 1), like glm::mat4(mat4x3).
static M4 affine(const M4& a) { return m43_to_m4(m4_to_m43(a)); }

std::unique_ptr<MediumHost> load_medium(const std::string& path, const float sigmaA[3], const float sigmaS[3],
                                        bool hg, float hgG) {
  std::unique_ptr<MediumHost> mh(new MediumHost());
  MediumView& v = mh->view;
  memset(&v, 0, sizeof(v));
  v.hg = hg ? 1 : 0;
  v.g = hgG;
  const std::vector<uint8_t> g = nvdb::read_file(path + ".nvdb");
  const nvdb::GridData* G = nvdb::grid_data(g.data());
  const nvdb::TreeData* T = nvdb::tree_data(g.data());
  // index box and size (nvdb_medium.cu:155-165)
  int32_t ibb[6];
  nvdb::index_bbox(g.data(), ibb);
  for (int k = 0; k < 3; ++k) {
    const int lo = T->voxelCount == 0 ? 0 : ibb[k];
    const int hi = T->voxelCount == 0 ? 0 : ibb[3 + k];
    R2_REQUIRE(hi >= lo, R2_ERR_IO, "empty index box in " + path + ".nvdb");
    v.ibbMin[k] = lo;
    v.size[k] = hi - lo + 1;
  }
  // getIndexToModelTransformation: NanoVDB map (row-major matF, vecF) times [0,1] -> index box
  M4 nano = m4_identity();
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) nano.m[c][r] = G->map.matF[3 * r + c];
  for (int r = 0; r < 3; ++r) nano.m[3][r] = G->map.vecF[r];
  M4 toNano = m4_identity();
  for (int k = 0; k < 3; ++k) {
    toNano.m[k][k] = (float)v.size[k];
    toNano.m[3][k] = (float)v.ibbMin[k];
  }
  const M4 i2m = affine(m4_mul(nano, toNano));
  const M4 m2i = affine(m4_inverse(i2m));
  const M4 s2i = affine(m4_inverse(toNano));  // scaledIndexToIndex
  v.indexToModel = m4_to_m43(i2m);
  v.modelToIndex = m4_to_m43(m2i);
  v.unitToScaled = m4_to_m43(m4_mul(toNano, m2i));
  v.scaledToModel = m4_to_m43(m4_mul(i2m, s2i));
  // coefficients (nvdb_medium.cu:45-61)
  v.sigmaS = v3(sigmaS[0], sigmaS[1], sigmaS[2]);
  v.sigmaT = fmaxf(sigmaA[0] + sigmaS[0], fmaxf(sigmaA[1] + sigmaS[1], sigmaA[2] + sigmaS[2]));
  R2_REQUIRE(v.sigmaT > 0.0f, R2_ERR_INVALID_CONFIG, "medium needs sigma_a + sigma_s > 0");
  // leaves: flat index over the 8^3 blocks they cover; global majorant
  const std::vector<size_t> offs = nvdb::leaf_offsets(g.data());
  float maxDensity = 0.0f;
  if (offs.empty()) {
    for (int k = 0; k < 3; ++k) v.L[k] = 1;
    mh->leafIndex.assign(1, -1);
  } else {
    // a leaf's bboxMin is the minimum of its active voxels; its origin is that & ~7
    int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (size_t off : offs) {
      const nvdb::LeafNode* lf = reinterpret_cast<const nvdb::LeafNode*>(g.data() + off);
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], lf->bboxMin[k] & ~7);
        hi[k] = std::max(hi[k], lf->bboxMin[k] & ~7);
      }
      for (int i = 0; i < 512; ++i) maxDensity = fmaxf(lf->values[i].density, maxDensity);
    }
    size_t blocks = 1;
    for (int k = 0; k < 3; ++k) {
      v.leafOrigin[k] = lo[k];
      const int64_t n = ((int64_t)hi[k] - lo[k]) / 8 + 1;
      R2_REQUIRE(n > 0 && n < (1 << 20), R2_ERR_UNSUPPORTED, "leaf extent too large in " + path + ".nvdb");
      v.L[k] = (int)n;
      blocks *= (size_t)n;
    }
    R2_REQUIRE(blocks <= (size_t(1) << 28), R2_ERR_UNSUPPORTED, "leaf index too large for " + path + ".nvdb");
    mh->leafIndex.assign(blocks, -1);
    for (size_t i = 0; i < offs.size(); ++i) {
      R2_REQUIRE(offs[i] == offs[0] + i * sizeof(nvdb::LeafNode), R2_ERR_IO, "leaves not contiguous");
      const nvdb::LeafNode* lf = reinterpret_cast<const nvdb::LeafNode*>(g.data() + offs[i]);
      const size_t b = (size_t)(((lf->bboxMin[0] & ~7) - lo[0]) / 8) +
                       (size_t)(((lf->bboxMin[1] & ~7) - lo[1]) / 8) * v.L[0] +
                       (size_t)(((lf->bboxMin[2] & ~7) - lo[2]) / 8) * v.L[0] * v.L[1];
      R2_REQUIRE(mh->leafIndex[b] < 0, R2_ERR_IO, "two leaves with one origin in " + path + ".nvdb");
      mh->leafIndex[b] = (int32_t)i;
    }
    mh->leaves.assign(g.begin() + (ptrdiff_t)offs[0],
                      g.begin() + (ptrdiff_t)(offs[0] + offs.size() * sizeof(nvdb::LeafNode)));
  }
  v.invMaxDensity = 1.0f / maxDensity;
  mh->boxMin = v3((float)G->worldBBox[0], (float)G->worldBBox[1], (float)G->worldBBox[2]);
  mh->boxMax = v3((float)G->worldBBox[3], (float)G->worldBBox[4], (float)G->worldBBox[5]);
  mh->voxelSizeFiltering = voxel_size_from_path(path);
  // brick grid
  mh->bricks = read_brick_grid(path + ".brickgrid");
  for (int k = 0; k < 3; ++k) {
    v.nb[k] = (int)mh->bricks.nBricks[k];
    v.ad[k] = (int)mh->bricks.atlasDim[k];
  }
  return mh;
}

MediumView place_medium(const MediumHost& mh, V3 pos, V3 orientation, V3 scaling) {
  MediumView v = mh.view;
  // T R S, world box from the model box's two corners (aabb.hpp:9-13)
  const M4 m2w = model_to_world_transform(pos, orientation, scaling);
  v.modelToWorld = m4_to_m43(m2w);
  v.worldToModel = m4_to_m43(m4_inverse(m2w));
  const V3 a = xform_point(v.modelToWorld, mh.boxMin), b = xform_point(v.modelToWorld, mh.boxMax);
  v.aabbMin = v3(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z);
  v.aabbMax = v3(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z);
  const float voxelSizeRendering = (v.aabbMax.x - v.aabbMin.x) / (float)v.size[0];
  v.filterRenderRatio = mh.voxelSizeFiltering / voxelSizeRendering;
  return v;
}

void MediumHost::upload(cudaStream_t s) {
  dLeaves.upload(leaves.data(), leaves.size(), s);
  dLeafIndex.upload(leafIndex.data(), leafIndex.size(), s);
  dIndirection.upload(bricks.indirection.data(), bricks.indirection.size(), s);
  dRange.upload(bricks.range.data(), bricks.range.size(), s);
  for (int i = 0; i < 3; ++i) dMips[i].upload(bricks.mips[i].data(), bricks.mips[i].size(), s);
  dAtlas.upload(bricks.atlas.data(), bricks.atlas.size(), s);
  view.leaves = dLeaves.get();
  view.leafIndex = dLeafIndex.get();
  view.indirection = dIndirection.get();
  view.range = dRange.get();
  for (int i = 0; i < 3; ++i) view.mips[i] = dMips[i].get();
  view.atlas = dAtlas.get();
  uploaded = true;
}

size_t MediumHost::device_bytes() const {
  size_t n = leaves.size() + leafIndex.size() * 4 + bricks.indirection.size() * 4 + bricks.range.size() * 4 +
             bricks.atlas.size();
  for (int i = 0; i < 3; ++i) n += bricks.mips[i].size() * 4;
  return n;
}

}  // namespace r2
