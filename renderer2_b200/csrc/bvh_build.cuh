// GPU LBVH builder (host interface).  See bvh_build.cu.
#pragma once
#include "bvh.h"
#include "radix_sort.cuh"
#include "runtime.h"

namespace r2 {

// SAH constants of the leaf-collapse pass: cost(leaf) = kSahTri * n,
// cost(inner) = kSahNode + (A_l cost_l + A_r cost_r) / A.
constexpr float kSahNode = 1.2f;
constexpr float kSahTri = 1.0f;
constexpr int kLeafMax = 8;
// Window of the PLOC nearest-neighbour search: positions i - r .. i + r.
constexpr int kPlocRadius = 16;

// Hierarchy over the Morton-sorted primitives: PLOC clustering or the Karras
// radix tree, both ending with the same SAH leaf collapse.  kBvhAuto (the
// default) takes PLOC for render scenes and the Karras tree for filter scenes,
// the faster choice of each (measured on the C2 scene and the C3 foliage).
enum BvhMethod { kBvhAuto = -1, kBvhPloc = 0, kBvhKarras = 1 };
// Process-wide choice for the BVHs built from now on.
int bvh_method();
void set_bvh_method(int method);
// The hierarchy a build uses: the process-wide choice, or under kBvhAuto the
// default of its purpose.
int resolve_bvh_method(bool filterScene);

// A triangle BVH resident in device memory.
struct DeviceBvh {
  DBuf<BvhNode> nodes;     // max(ntris-1, 1) nodes
  DBuf<float4> tris;       // 3 per triangle in BVH order
  DBuf<uint32_t> order;    // BVH position -> original triangle index
  uint32_t ntris = 0;
  uint32_t nnodes = 0;
  uint32_t height = 0;     // levels of inner nodes on the longest root-leaf path
  BvhView view() const {
    BvhView v;
    memset(&v, 0, sizeof(v));
    v.nodes = nodes.get();
    v.tris = tris.get();
    v.ntris = ntris;
    return v;
  }
};

// Builds BVHs with device scratch kept between builds (grown on demand), so
// that rebuilding a BVH of the same size allocates nothing and the output's
// buffers (and the pointers taken from them) stay in place.  The host waits
// for the build once, at its end, to check the tree height against the
// traversal stack.
class BvhBuilder {
 public:
  BvhBuilder() = default;
  BvhBuilder(const BvhBuilder&) = delete;
  BvhBuilder& operator=(const BvhBuilder&) = delete;
  ~BvhBuilder();
  void build(const float* d_pos, const uint32_t* d_idx, uint32_t ntris, DeviceBvh* out, cudaStream_t s);
  // leafMax: the most boxes a collapsed leaf may hold (1: no collapse, every
  // leaf one box).
  void build_boxes(const float4* d_lo, const float4* d_hi, uint32_t nboxes, DeviceBvh* out, cudaStream_t s,
                   int leafMax = kLeafMax);
  // Kernels the last build launched.
  int launches() const { return launches_; }
  // BVHs of filter scenes (their kBvhAuto default differs).
  void set_filter_scene(bool f) { filterScene_ = f; }

 private:
  void from_boxes(const float4* lo, const float4* hi, uint32_t n, const float* d_pos, const uint32_t* d_idx,
                  DeviceBvh* out, cudaStream_t s);
  int ploc(const float4* lo, const float4* hi, int n, DeviceBvh* out, cudaStream_t s);
  DBuf<float4> triLo_, triHi_, leafLo_, leafHi_, nodeLo_, nodeHi_;
  DBuf<float4> cLo_[2], cHi_[2];
  DBuf<uint64_t> keys_;
  DBuf<int> left_, right_, first_, last_, nodeParent_, leafParent_, nodeHeight_, collapse_, flags_;
  DBuf<int> cRef_[2], nn_, count_, leafPos_, state_;
  DBuf<int2> blockCounts_;
  DBuf<float> nodeCost_;
  DBuf<uint32_t> cb_, sorted_;
  RadixSortScratch sort_;
  void* hostState_ = nullptr;  // pinned copy of the PLOC iteration state
  int launches_ = 0;
  int leafMax_ = kLeafMax;
  bool filterScene_ = false;
};

// Builds the BVH over triangles (d_pos: 3 floats per vertex, d_idx: 3 per
// triangle, both device).  Deterministic: the result depends only on the input.
void build_bvh(const float* d_pos, const uint32_t* d_idx, uint32_t ntris, DeviceBvh* out,
               cudaStream_t stream, bool filterScene = false);

// The same hierarchy over boxes (d_lo/d_hi: one float4 per box, xyz used,
// device): leaves reference BVH positions, order[] maps them to box indices;
// no triangle array.
void build_box_bvh(const float4* d_lo, const float4* d_hi, uint32_t nboxes, DeviceBvh* out, cudaStream_t stream,
                   int leafMax = kLeafMax);

}  // namespace r2
