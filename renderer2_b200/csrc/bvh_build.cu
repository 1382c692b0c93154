// GPU LBVH builder for sm_100a.
//
// 1. triangle boxes and centroids (box midpoints);
// 2. centroid bounds (block reduction + ordered-integer atomics; min/max are exact);
// 3. 63-bit Morton codes (21 bits per axis);
// 4. stable radix sort of (code, triangle) pairs — ties keep triangle order
//    (radix_sort.cu);
// 5. the hierarchy over the sorted primitives: PLOC clustering (bvh_ploc.cu,
//    the default) or the Karras radix tree ("Maximizing Parallelism in the
//    Construction of BVHs, Octrees, and k-d Trees", HPG 2012);
// 6. boxes and the SAH cost of each node, collapsing a subtree into one leaf
//    when kSahTri*n <= kSahNode + (A_l c_l + A_r c_r)/A and n <= kLeafMax
//    (a bottom-up pass for the Karras tree; PLOC decides at each merge);
// 7. emission of the 64-byte nodes and the BVH-ordered triangle array.
// Every step is a pure function of the input, so the host oracle rebuilds the
// identical tree (same codes, same splits, same collapse decisions).
#include <atomic>

#include "bvh_build.cuh"

namespace r2 {
namespace {

__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t o) {
  uint32_t b = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
  return __uint_as_float(b);
}

// Block reduction of the threads' centroid bounds into cbounds (6 ordered
// words: min xyz, -max xyz), one atomicMin per word and block.
__device__ void reduce_centroid_bounds(V3 cmin, V3 cmax, uint32_t* __restrict__ cbounds) {
  float v[6] = {cmin.x, cmin.y, cmin.z, -cmax.x, -cmax.y, -cmax.z};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    for (int off = 16; off > 0; off >>= 1) v[k] = fminf(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], off));
  }
  __shared__ float sred[32][6];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) sred[warp][k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float x = lane < nw ? sred[lane][k] : INFINITY;
      for (int off = 16; off > 0; off >>= 1) x = fminf(x, __shfl_xor_sync(0xFFFFFFFFu, x, off));
      if (lane == 0) atomicMin(&cbounds[k], f2ord(x));
    }
  }
}

__global__ void k_tri_bounds(const float* __restrict__ pos, const uint32_t* __restrict__ idx,
                             uint32_t n, float4* __restrict__ lo, float4* __restrict__ hi,
                             uint32_t* __restrict__ cbounds /* 6 ordered words */) {
  V3 cmin = v3(INFINITY), cmax = v3(-INFINITY);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
    V3 a = v3(pos[3 * i0], pos[3 * i0 + 1], pos[3 * i0 + 2]);
    V3 b = v3(pos[3 * i1], pos[3 * i1 + 1], pos[3 * i1 + 2]);
    V3 c = v3(pos[3 * i2], pos[3 * i2 + 1], pos[3 * i2 + 2]);
    V3 l = vmin(vmin(a, b), c), h = vmax(vmax(a, b), c);
    lo[t] = make_float4(l.x, l.y, l.z, 0.0f);
    hi[t] = make_float4(h.x, h.y, h.z, 0.0f);
    V3 cen = (l + h) * 0.5f;
    cmin = vmin(cmin, cen);
    cmax = vmax(cmax, cen);
  }
  reduce_centroid_bounds(cmin, cmax, cbounds);
}

__global__ void k_box_bounds(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                             uint32_t* __restrict__ cbounds) {
  V3 cmin = v3(INFINITY), cmax = v3(-INFINITY);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const float4 l = lo[t], h = hi[t];
    const V3 cen = (v3(l.x, l.y, l.z) + v3(h.x, h.y, h.z)) * 0.5f;
    cmin = vmin(cmin, cen);
    cmax = vmax(cmax, cen);
  }
  reduce_centroid_bounds(cmin, cmax, cbounds);
}

__device__ __forceinline__ uint64_t expand21(uint32_t v) {
  uint64_t x = v & 0x1FFFFFu;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

__device__ __forceinline__ uint32_t quant21(float c, float cmin, float inv) {
  float q = (c - cmin) * inv * 2097152.0f;
  q = fminf(fmaxf(q, 0.0f), 2097151.0f);
  return (uint32_t)q;
}

__global__ void k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                         const uint32_t* __restrict__ cbounds, uint64_t* __restrict__ keys,
                         uint32_t* __restrict__ vals) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  V3 cmin = v3(ord2f(cbounds[0]), ord2f(cbounds[1]), ord2f(cbounds[2]));
  V3 cmax = v3(-ord2f(cbounds[3]), -ord2f(cbounds[4]), -ord2f(cbounds[5]));
  V3 ext = cmax - cmin;
  V3 inv = v3(ext.x > 0.0f ? 1.0f / ext.x : 0.0f, ext.y > 0.0f ? 1.0f / ext.y : 0.0f,
              ext.z > 0.0f ? 1.0f / ext.z : 0.0f);
  float4 l = lo[t], h = hi[t];
  V3 cen = (v3(l.x, l.y, l.z) + v3(h.x, h.y, h.z)) * 0.5f;
  uint32_t qx = quant21(cen.x, cmin.x, inv.x);
  uint32_t qy = quant21(cen.y, cmin.y, inv.y);
  uint32_t qz = quant21(cen.z, cmin.z, inv.z);
  keys[t] = (expand21(qx) << 2) | (expand21(qy) << 1) | expand21(qz);
  vals[t] = t;
}

__device__ __forceinline__ int kdelta(const uint64_t* __restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint64_t a = k[i], b = k[j];
  if (a == b) return 64 + __clz(i ^ j);
  return __clzll(a ^ b);
}

// Child encoding inside the builder: c >= 0 internal node, c < 0 leaf ~prim.
__global__ void k_karras(const uint64_t* __restrict__ keys, int n, int* __restrict__ left,
                         int* __restrict__ right, int* __restrict__ first, int* __restrict__ last,
                         int* __restrict__ nodeParent, int* __restrict__ leafParent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = kdelta(keys, n, i, i - d);
  int lmax = 2;
  while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2) {
    if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  }
  int j = i + l * d;
  int dnode = kdelta(keys, n, i, j);
  int s = 0;
  int div = 2;
  int t = (l + div - 1) / div;
  while (true) {
    if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
    div *= 2;
    t = (l + div - 1) / div;
  }
  int gamma = i + s * d + (d < 0 ? -1 : 0);
  int f = min(i, j), la = max(i, j);
  int lc = (f == gamma) ? ~gamma : gamma;
  int rc = (la == gamma + 1) ? ~(gamma + 1) : (gamma + 1);
  left[i] = lc;
  right[i] = rc;
  first[i] = f;
  last[i] = la;
  if (lc < 0) leafParent[~lc] = i; else nodeParent[lc] = i;
  if (rc < 0) leafParent[~rc] = i; else nodeParent[rc] = i;
  if (i == 0) nodeParent[0] = -1;
}

__device__ __forceinline__ float box_area(float4 l, float4 h) {
  float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
  return dx * dy + dy * dz + dz * dx;
}

struct ChildInfo {
  float4 lo, hi;
  float cost;
  int height;
};

__device__ __forceinline__ ChildInfo load_child(int c, const float4* leafLo, const float4* leafHi,
                                                const float4* nodeLo, const float4* nodeHi,
                                                const float* nodeCost, const int* nodeHeight) {
  ChildInfo ci;
  if (c < 0) {
    ci.lo = __ldcg(&leafLo[~c]);
    ci.hi = __ldcg(&leafHi[~c]);
    ci.cost = kSahTri;
    ci.height = 0;
  } else {
    ci.lo = __ldcg(&nodeLo[c]);
    ci.hi = __ldcg(&nodeHi[c]);
    ci.cost = __ldcg(&nodeCost[c]);
    ci.height = __ldcg(&nodeHeight[c]);
  }
  return ci;
}

__global__ void k_bottom_up(int n, const uint32_t* __restrict__ order, const float4* __restrict__ triLo,
                            const float4* __restrict__ triHi, const int* __restrict__ left,
                            const int* __restrict__ right, const int* __restrict__ first,
                            const int* __restrict__ last, const int* __restrict__ nodeParent,
                            const int* __restrict__ leafParent, float4* leafLo, float4* leafHi,
                            float4* nodeLo, float4* nodeHi, float* nodeCost, int* nodeHeight,
                            int* collapse, int* flags, int leafMax) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t prim = order[i];
  leafLo[i] = triLo[prim];
  leafHi[i] = triHi[prim];
  int p = leafParent[i];
  while (p >= 0 && p < n - 1) {
    __threadfence();
    if (atomicAdd(&flags[p], 1) == 0) return;  // sibling not finished yet
    __threadfence();
    ChildInfo a = load_child(left[p], leafLo, leafHi, nodeLo, nodeHi, nodeCost, nodeHeight);
    ChildInfo b = load_child(right[p], leafLo, leafHi, nodeLo, nodeHi, nodeCost, nodeHeight);
    float4 lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), 0.0f);
    float4 hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), 0.0f);
    float A = box_area(lo, hi);
    float Al = box_area(a.lo, a.hi), Ar = box_area(b.lo, b.hi);
    float inner = (A > 0.0f) ? kSahNode + (Al * a.cost + Ar * b.cost) / A : kSahNode + a.cost + b.cost;
    int count = last[p] - first[p] + 1;
    float leafc = kSahTri * (float)count;
    int col = (count <= leafMax && leafc <= inner) ? 1 : 0;
    nodeLo[p] = lo;
    nodeHi[p] = hi;
    nodeCost[p] = col ? leafc : inner;
    nodeHeight[p] = col ? 0 : 1 + max(a.height, b.height);
    collapse[p] = col;
    p = nodeParent[p];
  }
}

__device__ __forceinline__ int child_ref(int c, const int* collapse, const int* first, const int* last) {
  if (c < 0) return bvh_leaf_ref(~c, 1);
  if (collapse[c]) return bvh_leaf_ref(first[c], last[c] - first[c] + 1);
  return c;
}

__global__ void k_emit(int n, const int* __restrict__ left, const int* __restrict__ right,
                       const int* __restrict__ first, const int* __restrict__ last,
                       const int* __restrict__ nodeParent, const float4* __restrict__ leafLo,
                       const float4* __restrict__ leafHi, const float4* __restrict__ nodeLo,
                       const float4* __restrict__ nodeHi, const int* __restrict__ nodeHeight,
                       const int* __restrict__ collapse, BvhNode* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  BvhNode nd;
  if (i == 0 && collapse[0]) {
    float4 l = nodeLo[0], h = nodeHi[0];
    nd.b0 = make_float4(l.x, h.x, l.y, h.y);
    nd.b1 = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
    nd.bz = make_float4(l.z, h.z, INFINITY, -INFINITY);
    nd.ch = make_int4(bvh_leaf_ref(0, n), R2_BVH_NONE, -1, 0);
    out[0] = nd;
    return;
  }
  int lc = left[i], rc = right[i];
  float4 ll = lc < 0 ? leafLo[~lc] : nodeLo[lc];
  float4 lh = lc < 0 ? leafHi[~lc] : nodeHi[lc];
  float4 rl = rc < 0 ? leafLo[~rc] : nodeLo[rc];
  float4 rh = rc < 0 ? leafHi[~rc] : nodeHi[rc];
  nd.b0 = make_float4(ll.x, lh.x, ll.y, lh.y);
  nd.b1 = make_float4(rl.x, rh.x, rl.y, rh.y);
  nd.bz = make_float4(ll.z, lh.z, rl.z, rh.z);
  nd.ch = make_int4(child_ref(lc, collapse, first, last), child_ref(rc, collapse, first, last),
                    nodeParent[i], nodeHeight[i]);
  out[i] = nd;
}

__global__ void k_single_leaf(const float4* lo, const float4* hi, BvhNode* out) {
  float4 l = lo[0], h = hi[0];
  BvhNode nd;
  nd.b0 = make_float4(l.x, h.x, l.y, h.y);
  nd.b1 = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
  nd.bz = make_float4(l.z, h.z, INFINITY, -INFINITY);
  nd.ch = make_int4(bvh_leaf_ref(0, 1), R2_BVH_NONE, -1, 0);
  out[0] = nd;
}

__global__ void k_gather_tris(const float* __restrict__ pos, const uint32_t* __restrict__ idx,
                              const uint32_t* __restrict__ order, uint32_t n,
                              float4* __restrict__ tris) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t p = order[i];
  uint32_t i0 = idx[3 * p], i1 = idx[3 * p + 1], i2 = idx[3 * p + 2];
  tris[3 * i + 0] = make_float4(pos[3 * i0], pos[3 * i0 + 1], pos[3 * i0 + 2], __uint_as_float(p));
  tris[3 * i + 1] = make_float4(pos[3 * i1], pos[3 * i1 + 1], pos[3 * i1 + 2], 0.0f);
  tris[3 * i + 2] = make_float4(pos[3 * i2], pos[3 * i2 + 1], pos[3 * i2 + 2], 0.0f);
}

__global__ void k_init_bounds(uint32_t* cb) {
  if (threadIdx.x < 6) cb[threadIdx.x] = 0xFFFFFFFFu;
}

}  // namespace

static std::atomic<int> g_bvhMethod{kBvhAuto};
int bvh_method() { return g_bvhMethod.load(); }
void set_bvh_method(int method) {
  g_bvhMethod.store(method == kBvhKarras ? kBvhKarras : (method == kBvhPloc ? kBvhPloc : kBvhAuto));
}
int resolve_bvh_method(bool filterScene) {
  const int m = bvh_method();
  if (m != kBvhAuto) return m;
  return filterScene ? kBvhKarras : kBvhPloc;
}

// Steps 3-7 over primitive boxes whose centroid bounds are in cb_; with
// d_pos/d_idx the BVH-ordered triangle array is gathered too.
void BvhBuilder::from_boxes(const float4* triLo, const float4* triHi, uint32_t ntris, const float* d_pos,
                            const uint32_t* d_idx, DeviceBvh* out, cudaStream_t s) {
  const int n = (int)ntris;
  keys_.reserve(n);
  out->order.reserve(n);
  const bool usePloc = n > 1 && resolve_bvh_method(filterScene_) == kBvhPloc;
  if (usePloc) sorted_.reserve(n);
  uint32_t* sorted = usePloc ? sorted_.get() : out->order.get();
  k_morton<<<(n + 255) / 256, 256, 0, s>>>(triLo, triHi, ntris, cb_.get(), keys_.get(), sorted);
  const int sortLaunches = radix_sort_pairs(keys_.get(), sorted, ntris, 63, &sort_, s);
  launches_ += 1 + sortLaunches;
  out->ntris = ntris;
  auto gather = [&]() {
    if (!d_pos) return;
    out->tris.reserve((size_t)3 * n);
    k_gather_tris<<<(n + 255) / 256, 256, 0, s>>>(d_pos, d_idx, out->order.get(), ntris, out->tris.get());
    ++launches_;
  };
  if (usePloc) {
    const int h = ploc(triLo, triHi, n, out, s);  // waits for the device
    gather();
    R2_CUDA(cudaGetLastError());
    out->height = h ? (uint32_t)h : 1u;
    R2_REQUIRE(out->height <= R2_BVH_STACK, R2_ERR_UNSUPPORTED,
               "BVH deeper than the traversal stack (" + std::to_string(out->height) + " levels)");
    return;
  }
  gather();
  if (n == 1) {
    out->nodes.reserve(1);
    out->nnodes = 1;
    out->height = 1;
    k_single_leaf<<<1, 1, 0, s>>>(triLo, triHi, out->nodes.get());
    ++launches_;
    R2_CUDA(cudaGetLastError());
    R2_CUDA(cudaStreamSynchronize(s));
    return;
  }
  const int ni = n - 1;
  left_.reserve(ni); right_.reserve(ni); first_.reserve(ni); last_.reserve(ni);
  nodeParent_.reserve(ni); leafParent_.reserve(n);
  leafLo_.reserve(n); leafHi_.reserve(n); nodeLo_.reserve(ni); nodeHi_.reserve(ni);
  nodeCost_.reserve(ni); nodeHeight_.reserve(ni); collapse_.reserve(ni); flags_.reserve(ni);
  // parents default to -1 so a malformed hierarchy ends the bottom-up walk
  R2_CUDA(cudaMemsetAsync(nodeParent_.get(), 0xFF, sizeof(int) * ni, s));
  R2_CUDA(cudaMemsetAsync(leafParent_.get(), 0xFF, sizeof(int) * n, s));
  k_karras<<<(ni + 255) / 256, 256, 0, s>>>(keys_.get(), n, left_.get(), right_.get(), first_.get(), last_.get(),
                                            nodeParent_.get(), leafParent_.get());
  R2_CUDA(cudaMemsetAsync(flags_.get(), 0, sizeof(int) * ni, s));
  k_bottom_up<<<(n + 255) / 256, 256, 0, s>>>(n, out->order.get(), triLo, triHi, left_.get(), right_.get(),
                                              first_.get(), last_.get(), nodeParent_.get(), leafParent_.get(),
                                              leafLo_.get(), leafHi_.get(), nodeLo_.get(), nodeHi_.get(),
                                              nodeCost_.get(), nodeHeight_.get(), collapse_.get(), flags_.get(),
                                              leafMax_);
  out->nodes.reserve(ni);
  out->nnodes = ni;
  k_emit<<<(ni + 255) / 256, 256, 0, s>>>(n, left_.get(), right_.get(), first_.get(), last_.get(),
                                          nodeParent_.get(), leafLo_.get(), leafHi_.get(), nodeLo_.get(),
                                          nodeHi_.get(), nodeHeight_.get(), collapse_.get(), out->nodes.get());
  launches_ += 3;  // karras, bottom-up, emit
  R2_CUDA(cudaGetLastError());
  int root[2] = {0, 0};
  R2_CUDA(cudaMemcpyAsync(&root[0], nodeHeight_.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaMemcpyAsync(&root[1], collapse_.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaStreamSynchronize(s));
  out->height = root[1] ? 1 : (uint32_t)root[0];
  R2_REQUIRE(out->height <= R2_BVH_STACK, R2_ERR_UNSUPPORTED,
             "BVH deeper than the traversal stack (" + std::to_string(out->height) + " levels)");
}

void BvhBuilder::build(const float* d_pos, const uint32_t* d_idx, uint32_t ntris, DeviceBvh* out, cudaStream_t s) {
  R2_REQUIRE(ntris > 0, R2_ERR_INVALID_ARGUMENT, "BVH over zero triangles");
  R2_REQUIRE(ntris < (1u << 26), R2_ERR_UNSUPPORTED, "BVH supports fewer than 2^26 triangles");
  leafMax_ = kLeafMax;
  triLo_.reserve(ntris);
  triHi_.reserve(ntris);
  cb_.reserve(6);
  k_init_bounds<<<1, 32, 0, s>>>(cb_.get());
  int nb = (int)std::min<uint32_t>((ntris + 255) / 256, (uint32_t)sm_count() * 8);
  k_tri_bounds<<<nb, 256, 0, s>>>(d_pos, d_idx, ntris, triLo_.get(), triHi_.get(), cb_.get());
  launches_ = 2;
  from_boxes(triLo_.get(), triHi_.get(), ntris, d_pos, d_idx, out, s);
}

void BvhBuilder::build_boxes(const float4* d_lo, const float4* d_hi, uint32_t nboxes, DeviceBvh* out,
                             cudaStream_t s, int leafMax) {
  R2_REQUIRE(nboxes > 0, R2_ERR_INVALID_ARGUMENT, "BVH over zero boxes");
  R2_REQUIRE(leafMax >= 1 && leafMax <= kLeafMax, R2_ERR_INVALID_ARGUMENT, "leaf size out of range");
  leafMax_ = leafMax;
  R2_REQUIRE(nboxes < (1u << 26), R2_ERR_UNSUPPORTED, "BVH supports fewer than 2^26 boxes");
  cb_.reserve(6);
  k_init_bounds<<<1, 32, 0, s>>>(cb_.get());
  int nb = (int)std::min<uint32_t>((nboxes + 255) / 256, (uint32_t)sm_count() * 8);
  k_box_bounds<<<nb, 256, 0, s>>>(d_lo, d_hi, nboxes, cb_.get());
  launches_ = 2;
  from_boxes(d_lo, d_hi, nboxes, nullptr, nullptr, out, s);
}

void build_bvh(const float* d_pos, const uint32_t* d_idx, uint32_t ntris, DeviceBvh* out, cudaStream_t s,
               bool filterScene) {
  BvhBuilder b;
  b.set_filter_scene(filterScene);
  b.build(d_pos, d_idx, ntris, out, s);
}

void build_box_bvh(const float4* d_lo, const float4* d_hi, uint32_t nboxes, DeviceBvh* out, cudaStream_t s,
                   int leafMax) {
  BvhBuilder b;
  b.build_boxes(d_lo, d_hi, nboxes, out, s, leafMax);
}

}  // namespace r2
