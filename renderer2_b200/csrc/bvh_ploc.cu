// PLOC hierarchy for the BVH builder: parallel locally-ordered clustering
// (Meister & Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
// Hierarchy Construction", IEEE TVCG 2018) over the Morton-sorted primitives.
//
// Each iteration works on the ordered list of clusters (initially the sorted
// primitives):
//   1. every cluster i finds its nearest neighbour j among the clusters at
//      most kPlocRadius positions away, by the surface area of the box
//      enclosing both; equal areas go to the closer position, then to the
//      pair whose lower position is even, then to the lower position (so that
//      a run of identical boxes pairs up neighbour by neighbour and halves,
//      instead of chaining into a list);
//   2. mutual nearest neighbours (nn[nn[i]] == i) merge into a new inner node
//      that takes the smaller position; the other position is dropped and the
//      list is compacted in order.
// The order above is a total order on unordered pairs, so the pair that comes
// first overall is chosen by both of its clusters: every iteration merges at
// least once.  Inner nodes are numbered
// downwards from n-2 in merge order (within an iteration by position), so
// the last merge, the root, is node 0 and every parent has a smaller index
// than its children.  Boxes, SAH costs, primitive counts and leaf-collapse
// decisions are made when a node is created, from its finished children,
// with the same formulas as the Karras path.  Primitives are finally placed
// in depth-first (left-first) order so that every subtree, collapsed leaves
// included, covers a contiguous range of the BVH-ordered triangle array.
//
// Large lists iterate with four launches per step (neighbours, block counts,
// a scan of the counts, compaction), a few steps between host reads of the
// cluster count; from kPlocTail clusters on one block finishes the hierarchy
// alone.  All
// choices are pure functions of the input, so the host oracle rebuilds the
// identical tree.
#include <algorithm>

#include "bvh_build.cuh"

namespace r2 {
namespace {

constexpr int kPlocBlock = 256;
constexpr int kPlocTail = 4096;
constexpr int kPlocTailThreads = 1024;
constexpr int kPlocScanThreads = 1024;

struct PlocState {
  int m[2];    // clusters in cluster buffer 0 / 1 (the current list's buffer alternates)
  int k;       // merges of the last iteration
  int cursor;  // lowest inner-node index handed out so far
  int error;   // the single-block finish ran out of iterations
};

__device__ __forceinline__ float area_of(float4 l, float4 h) {
  const float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
  return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ float union_area(float4 al, float4 ah, float4 bl, float4 bh) {
  const float dx = fmaxf(ah.x, bh.x) - fminf(al.x, bl.x);
  const float dy = fmaxf(ah.y, bh.y) - fminf(al.y, bl.y);
  const float dz = fmaxf(ah.z, bh.z) - fminf(al.z, bl.z);
  return dx * dy + dy * dz + dz * dx;
}

// Nearest-neighbour key of the pair (i, j): the area's bits (monotonic for
// areas >= 0), then |i - j| (1..kPlocRadius), the parity of min(i, j) and
// min(i, j) itself (< 2^26).  Symmetric in i and j and distinct per pair.
__device__ __forceinline__ uint64_t nn_key(float a, int i, int j) {
  const uint32_t d = (uint32_t)abs(i - j), lo = (uint32_t)min(i, j);
  return ((uint64_t)__float_as_uint(a) << 32) | ((uint64_t)d << 27) | ((uint64_t)(lo & 1u) << 26) | lo;
}
// The partner of i that a key names.
__device__ __forceinline__ int nn_partner(uint64_t key, int i) {
  const int lo = (int)(key & 0x03FFFFFFu), d = (int)((key >> 27) & 31u);
  return lo < i ? lo : i + d;
}

// The node arrays a merge writes and reads.
struct PlocNodes {
  int* left;
  int* right;
  int* parent;      // of inner nodes (-1: root)
  int* leafParent;  // of sorted primitives
  int* count;
  int* height;
  int* collapse;
  float* cost;
  float4* lo;
  float4* hi;
  int leafMax;
};

// Creates inner node nd over clusters (a, boxes al/ah) and (b, bl/bh); returns
// nothing, the caller stores the merged cluster (nd, union box).
__device__ void make_node(const PlocNodes& N, int nd, int a, float4 al, float4 ah, int b, float4 bl, float4 bh) {
  const float ca = a < 0 ? kSahTri : N.cost[a], cb = b < 0 ? kSahTri : N.cost[b];
  const int na = a < 0 ? 1 : N.count[a], nb = b < 0 ? 1 : N.count[b];
  const int ha = a < 0 ? 0 : N.height[a], hb = b < 0 ? 0 : N.height[b];
  const float4 lo = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
  const float4 hi = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
  const float A = area_of(lo, hi);
  const float Al = area_of(al, ah), Ar = area_of(bl, bh);
  const float inner = (A > 0.0f) ? kSahNode + (Al * ca + Ar * cb) / A : kSahNode + ca + cb;
  const int count = na + nb;
  const float leafc = kSahTri * (float)count;
  const int col = (count <= N.leafMax && leafc <= inner) ? 1 : 0;
  N.left[nd] = a;
  N.right[nd] = b;
  N.lo[nd] = lo;
  N.hi[nd] = hi;
  N.cost[nd] = col ? leafc : inner;
  N.count[nd] = count;
  N.height[nd] = col ? 0 : 1 + max(ha, hb);
  N.collapse[nd] = col;
  if (a < 0) N.leafParent[~a] = nd; else N.parent[a] = nd;
  if (b < 0) N.leafParent[~b] = nd; else N.parent[b] = nd;
}

__global__ void k_ploc_init(const float4* __restrict__ triLo, const float4* __restrict__ triHi,
                            const uint32_t* __restrict__ sorted, int n, float4* __restrict__ leafLo,
                            float4* __restrict__ leafHi, int* __restrict__ cRef, float4* __restrict__ cLo,
                            float4* __restrict__ cHi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = sorted[i];
  const float4 l = triLo[p], h = triHi[p];
  leafLo[i] = l;
  leafHi[i] = h;
  cRef[i] = ~i;
  cLo[i] = l;
  cHi[i] = h;
}

// Step 1 for a tile of kPlocBlock clusters, their boxes and the window on
// either side staged in shared memory.
__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                        const int* __restrict__ mPtr, int* __restrict__ nn) {
  __shared__ float4 sl[kPlocBlock + 2 * kPlocRadius], sh[kPlocBlock + 2 * kPlocRadius];
  const int m = *mPtr;
  const int b0 = blockIdx.x * kPlocBlock;
  if (m < 2 || b0 >= m) return;  // the whole block: the grid is sized for an upper bound of m
  for (int k = threadIdx.x; k < kPlocBlock + 2 * kPlocRadius; k += blockDim.x) {
    const int g = b0 - kPlocRadius + k;
    if (g >= 0 && g < m) {
      sl[k] = lo[g];
      sh[k] = hi[g];
    }
  }
  __syncthreads();
  const int i = b0 + threadIdx.x;
  if (i >= m) return;
  const float4 il = sl[threadIdx.x + kPlocRadius], ih = sh[threadIdx.x + kPlocRadius];
  uint64_t best = ~0ull;
  const int j0 = max(0, i - kPlocRadius), j1 = min(m - 1, i + kPlocRadius);
  for (int j = j0; j <= j1; ++j) {
    if (j == i) continue;
    const int k = j - b0 + kPlocRadius;
    best = min(best, nn_key(union_area(il, ih, sl[k], sh[k]), i, j));
  }
  nn[i] = nn_partner(best, i);
}

// Merge (i takes the pair) and keep (i stays in the list) flags of position i.
__device__ __forceinline__ void ploc_flags(const int* nn, int i, int m, bool* merge, bool* keep) {
  *merge = false;
  *keep = i < m;
  if (i >= m || m < 2) return;
  const int j = nn[i];
  const bool mutual = nn[j] == i;
  *merge = mutual && i < j;
  *keep = !(mutual && j < i);
}

__global__ void __launch_bounds__(kPlocBlock) k_ploc_count(const int* __restrict__ nn, const int* __restrict__ mPtr,
                                                           int2* __restrict__ blockCounts) {
  const int m = *mPtr;
  const int i = blockIdx.x * kPlocBlock + threadIdx.x;
  bool merge, keep;
  ploc_flags(nn, i, m, &merge, &keep);
  const int nm = __syncthreads_count(merge);
  const int nk = __syncthreads_count(keep);
  if (threadIdx.x == 0) blockCounts[blockIdx.x] = make_int2(nm, nk);
}

// Block-wide exclusive scan of (merges, kept) pairs; returns the block totals.
template <int kThreads>
__device__ int2 block_scan2(int2 v, int2* total) {
  __shared__ int2 warpSum[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int2 x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ax = __shfl_up_sync(0xFFFFFFFFu, x.x, o), ay = __shfl_up_sync(0xFFFFFFFFu, x.y, o);
    if (lane >= o) {
      x.x += ax;
      x.y += ay;
    }
  }
  if (lane == 31) warpSum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int2 w = lane < kThreads / 32 ? warpSum[lane] : make_int2(0, 0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ax = __shfl_up_sync(0xFFFFFFFFu, w.x, o), ay = __shfl_up_sync(0xFFFFFFFFu, w.y, o);
      if (lane >= o) {
        w.x += ax;
        w.y += ay;
      }
    }
    if (lane < kThreads / 32) warpSum[lane] = w;  // inclusive per warp
  }
  __syncthreads();
  const int2 before = warp ? warpSum[warp - 1] : make_int2(0, 0);
  *total = warpSum[kThreads / 32 - 1];
  __syncthreads();  // warpSum is reused by the next call
  return make_int2(before.x + x.x - v.x, before.y + x.y - v.y);
}

// Exclusive scan of the block counts (one block), the iteration's totals and
// the new node cursor.
__global__ void __launch_bounds__(kPlocScanThreads) k_ploc_scan(int2* __restrict__ blockCounts, int nb,
                                                                PlocState* __restrict__ st, int cur) {
  int2 carry = make_int2(0, 0);
  for (int b0 = 0; b0 < nb; b0 += kPlocScanThreads) {
    const int b = b0 + threadIdx.x;
    const int2 v = b < nb ? blockCounts[b] : make_int2(0, 0);
    int2 tot;
    const int2 ex = block_scan2<kPlocScanThreads>(v, &tot);
    if (b < nb) blockCounts[b] = make_int2(carry.x + ex.x, carry.y + ex.y);
    carry.x += tot.x;
    carry.y += tot.y;
  }
  if (threadIdx.x == 0) {
    st->k = carry.x;
    st->m[cur ^ 1] = carry.y;
    st->cursor -= carry.x;
  }
}

__global__ void __launch_bounds__(kPlocBlock) k_ploc_compact(const int* __restrict__ nn, const int* mPtr,
                                                             const int2* __restrict__ blockOffsets,
                                                             const PlocState* __restrict__ st,
                                                             const int* __restrict__ cRef,
                                                             const float4* __restrict__ cLo,
                                                             const float4* __restrict__ cHi, int* __restrict__ oRef,
                                                             float4* __restrict__ oLo, float4* __restrict__ oHi,
                                                             PlocNodes N) {
  const int m = *mPtr;
  const int i = blockIdx.x * kPlocBlock + threadIdx.x;
  bool merge, keep;
  ploc_flags(nn, i, m, &merge, &keep);
  int2 tot;
  const int2 r = block_scan2<kPlocBlock>(make_int2(merge ? 1 : 0, keep ? 1 : 0), &tot);
  if (!keep) return;
  const int2 off = blockOffsets[blockIdx.x];
  const int pos = off.y + r.y;
  if (merge) {
    const int j = nn[i];
    const int nd = st->cursor + off.x + r.x;
    const float4 al = cLo[i], ah = cHi[i], bl = cLo[j], bh = cHi[j];
    make_node(N, nd, cRef[i], al, ah, cRef[j], bl, bh);
    oRef[pos] = nd;
    oLo[pos] = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
    oHi[pos] = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
  } else {
    oRef[pos] = cRef[i];
    oLo[pos] = cLo[i];
    oHi[pos] = cHi[i];
  }
}

// The remaining iterations in one block (m <= kPlocTail), ping-ponging between
// the two cluster buffers in global memory; the same steps, ranks and node
// numbers as the multi-block iterations.  Bounded by kPlocTail iterations
// (each merges at least once); running out sets st->error.
__global__ void __launch_bounds__(kPlocTailThreads) k_ploc_tail(int* refA, float4* loA, float4* hiA, int* refB,
                                                                float4* loB, float4* hiB, int* nn, PlocState* st,
                                                                int cur0, PlocNodes N) {
  int m = st->m[cur0];
  int cursor = st->cursor;
  int* cRef = refA;
  float4 *cLo = loA, *cHi = hiA;
  int* oRef = refB;
  float4 *oLo = loB, *oHi = hiB;
  __shared__ int2 sCarry;
  int it = 0;
  for (; m > 1 && it < kPlocTail; ++it) {
    for (int i = threadIdx.x; i < m; i += kPlocTailThreads) {
      const float4 il = cLo[i], ih = cHi[i];
      uint64_t best = ~0ull;
      const int j0 = max(0, i - kPlocRadius), j1 = min(m - 1, i + kPlocRadius);
      for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        best = min(best, nn_key(union_area(il, ih, cLo[j], cHi[j]), i, j));
      }
      nn[i] = nn_partner(best, i);
    }
    __syncthreads();
    // merges of the whole list first: node numbers start at cursor - k
    int km = 0;
    for (int c0 = 0; c0 < m; c0 += kPlocTailThreads) {
      bool merge, keep;
      ploc_flags(nn, c0 + threadIdx.x, m, &merge, &keep);
      km += __syncthreads_count(merge);
    }
    const int base = cursor - km;
    if (threadIdx.x == 0) sCarry = make_int2(0, 0);
    __syncthreads();
    for (int c0 = 0; c0 < m; c0 += kPlocTailThreads) {
      const int i = c0 + threadIdx.x;
      bool merge, keep;
      ploc_flags(nn, i, m, &merge, &keep);
      int2 tot;
      const int2 r = block_scan2<kPlocTailThreads>(make_int2(merge ? 1 : 0, keep ? 1 : 0), &tot);
      const int2 carry = sCarry;
      if (keep) {
        const int pos = carry.y + r.y;
        if (merge) {
          const int j = nn[i];
          const int nd = base + carry.x + r.x;
          const float4 al = cLo[i], ah = cHi[i], bl = cLo[j], bh = cHi[j];
          make_node(N, nd, cRef[i], al, ah, cRef[j], bl, bh);
          oRef[pos] = nd;
          oLo[pos] = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
          oHi[pos] = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
        } else {
          oRef[pos] = cRef[i];
          oLo[pos] = cLo[i];
          oHi[pos] = cHi[i];
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) sCarry = make_int2(carry.x + tot.x, carry.y + tot.y);
      __syncthreads();
    }
    m = sCarry.y;
    cursor = base;
    int* tr = cRef; cRef = oRef; oRef = tr;
    float4* tl = cLo; cLo = oLo; oLo = tl;
    float4* th = cHi; cHi = oHi; oHi = th;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st->m[cur0] = m;
    st->cursor = cursor;
    st->error = m > 1 ? 1 : 0;
  }
}

__device__ __forceinline__ int subtree_count(const int* count, int ref) { return ref < 0 ? 1 : count[ref]; }

// Depth-first position of every sorted primitive (left subtrees first): the
// sum of the left siblings' primitive counts on its path to the root; then the
// first position of every node whose leftmost primitive it is.  The walks are
// bounded by the traversal stack depth the tree was checked against.
__global__ void k_ploc_positions(int n, const int* __restrict__ left, const int* __restrict__ right,
                                 const int* __restrict__ parent, const int* __restrict__ leafParent,
                                 const int* __restrict__ count, const uint32_t* __restrict__ sorted,
                                 int* __restrict__ leafPos, int* __restrict__ nodeFirst, uint32_t* __restrict__ order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int cur = ~i, p = leafParent[i], pos = 0;
  for (int s = 0; p >= 0 && s <= R2_BVH_STACK + 1; ++s) {
    if (right[p] == cur) pos += subtree_count(count, left[p]);
    cur = p;
    p = parent[p];
  }
  leafPos[i] = pos;
  order[pos] = sorted[i];
  cur = ~i;
  p = leafParent[i];
  for (int s = 0; p >= 0 && s <= R2_BVH_STACK + 1 && left[p] == cur; ++s) {
    nodeFirst[p] = pos;
    cur = p;
    p = parent[p];
  }
}

__device__ __forceinline__ int ploc_child_ref(int c, const int* leafPos, const int* nodeFirst, const int* count,
                                              const int* collapse) {
  if (c < 0) return bvh_leaf_ref(leafPos[~c], 1);
  if (collapse[c]) return bvh_leaf_ref(nodeFirst[c], count[c]);
  return c;
}

__global__ void k_ploc_emit(int n, const int* __restrict__ left, const int* __restrict__ right,
                            const int* __restrict__ parent, const int* __restrict__ count,
                            const int* __restrict__ height, const int* __restrict__ collapse,
                            const int* __restrict__ leafPos, const int* __restrict__ nodeFirst,
                            const float4* __restrict__ leafLo, const float4* __restrict__ leafHi,
                            const float4* __restrict__ nodeLo, const float4* __restrict__ nodeHi,
                            BvhNode* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  BvhNode nd;
  if (i == 0 && collapse[0]) {
    const float4 l = nodeLo[0], h = nodeHi[0];
    nd.b0 = make_float4(l.x, h.x, l.y, h.y);
    nd.b1 = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
    nd.bz = make_float4(l.z, h.z, INFINITY, -INFINITY);
    nd.ch = make_int4(bvh_leaf_ref(0, n), R2_BVH_NONE, -1, 0);
    out[0] = nd;
    return;
  }
  const int lc = left[i], rc = right[i];
  const float4 ll = lc < 0 ? leafLo[~lc] : nodeLo[lc];
  const float4 lh = lc < 0 ? leafHi[~lc] : nodeHi[lc];
  const float4 rl = rc < 0 ? leafLo[~rc] : nodeLo[rc];
  const float4 rh = rc < 0 ? leafHi[~rc] : nodeHi[rc];
  nd.b0 = make_float4(ll.x, lh.x, ll.y, lh.y);
  nd.b1 = make_float4(rl.x, rh.x, rl.y, rh.y);
  nd.bz = make_float4(ll.z, lh.z, rl.z, rh.z);
  nd.ch = make_int4(ploc_child_ref(lc, leafPos, nodeFirst, count, collapse),
                    ploc_child_ref(rc, leafPos, nodeFirst, count, collapse), parent[i], height[i]);
  out[i] = nd;
}

}  // namespace

BvhBuilder::~BvhBuilder() {
  if (hostState_) cudaFreeHost(hostState_);
}

// Steps 5-7 of the PLOC method: sorted_ holds the Morton-sorted primitive
// indices; writes out->order (BVH positions) and out->nodes, returns the
// root's height (0: the root is one collapsed leaf).
int BvhBuilder::ploc(const float4* triLo, const float4* triHi, int n, DeviceBvh* out, cudaStream_t s) {
  const int ni = n - 1;
  if (!hostState_) R2_CUDA(cudaMallocHost((void**)&hostState_, sizeof(PlocState)));
  leafLo_.reserve(n); leafHi_.reserve(n);
  cRef_[0].reserve(n); cRef_[1].reserve(n);
  cLo_[0].reserve(n); cLo_[1].reserve(n); cHi_[0].reserve(n); cHi_[1].reserve(n);
  nn_.reserve(n);
  left_.reserve(ni); right_.reserve(ni); nodeParent_.reserve(ni); leafParent_.reserve(n);
  nodeLo_.reserve(ni); nodeHi_.reserve(ni); nodeCost_.reserve(ni); nodeHeight_.reserve(ni);
  collapse_.reserve(ni); count_.reserve(ni); first_.reserve(ni); leafPos_.reserve(n);
  const int nbMax = (n + kPlocBlock - 1) / kPlocBlock;
  blockCounts_.reserve(nbMax);
  state_.reserve((sizeof(PlocState) + sizeof(int) - 1) / sizeof(int));
  R2_CUDA(cudaMemsetAsync(nodeParent_.get(), 0xFF, sizeof(int) * ni, s));
  R2_CUDA(cudaMemsetAsync(leafParent_.get(), 0xFF, sizeof(int) * n, s));
  k_ploc_init<<<(n + 255) / 256, 256, 0, s>>>(triLo, triHi, sorted_.get(), n, leafLo_.get(), leafHi_.get(),
                                              cRef_[0].get(), cLo_[0].get(), cHi_[0].get());
  PlocState init{{n, 0}, 0, ni, 0};
  *static_cast<PlocState*>(hostState_) = init;
  R2_CUDA(cudaMemcpyAsync(state_.get(), hostState_, sizeof(PlocState), cudaMemcpyHostToDevice, s));
  PlocNodes N{left_.get(), right_.get(), nodeParent_.get(), leafParent_.get(), count_.get(), nodeHeight_.get(),
              collapse_.get(), nodeCost_.get(), nodeLo_.get(), nodeHi_.get(), leafMax_};
  PlocState* st = reinterpret_cast<PlocState*>(state_.get());
  launches_ += 3;  // init, positions, emit
  // Multi-block iterations in batches of kPlocBatch between reads of the
  // cluster count: each kernel reads the current count from the device and
  // the grids are sized for the count read last (an upper bound).
  constexpr int kPlocBatch = 6;
  int cur = 0, m = n;
  for (int it = 0; m > kPlocTail && it < n;) {
    const int nb = (m + kPlocBlock - 1) / kPlocBlock;
    for (int b = 0; b < kPlocBatch; ++b, ++it) {
      k_ploc_nn<<<nb, kPlocBlock, 0, s>>>(cLo_[cur].get(), cHi_[cur].get(), &st->m[cur], nn_.get());
      k_ploc_count<<<nb, kPlocBlock, 0, s>>>(nn_.get(), &st->m[cur], blockCounts_.get());
      k_ploc_scan<<<1, kPlocScanThreads, 0, s>>>(blockCounts_.get(), nb, st, cur);
      k_ploc_compact<<<nb, kPlocBlock, 0, s>>>(nn_.get(), &st->m[cur], blockCounts_.get(), st, cRef_[cur].get(),
                                               cLo_[cur].get(), cHi_[cur].get(), cRef_[cur ^ 1].get(),
                                               cLo_[cur ^ 1].get(), cHi_[cur ^ 1].get(), N);
      launches_ += 4;
      cur ^= 1;
    }
    R2_CUDA(cudaMemcpyAsync(hostState_, st, sizeof(PlocState), cudaMemcpyDeviceToHost, s));
    R2_CUDA(cudaStreamSynchronize(s));
    const int m2 = static_cast<PlocState*>(hostState_)->m[cur];
    R2_REQUIRE(m2 < m && m2 >= 1, R2_ERR_DEVICE, "PLOC iterations merged no clusters");
    m = m2;
  }
  if (m > 1) {
    k_ploc_tail<<<1, kPlocTailThreads, 0, s>>>(cRef_[cur].get(), cLo_[cur].get(), cHi_[cur].get(),
                                               cRef_[cur ^ 1].get(), cLo_[cur ^ 1].get(), cHi_[cur ^ 1].get(),
                                               nn_.get(), st, cur, N);
    ++launches_;
  }
  k_ploc_positions<<<(n + 255) / 256, 256, 0, s>>>(n, left_.get(), right_.get(), nodeParent_.get(),
                                                   leafParent_.get(), count_.get(), sorted_.get(), leafPos_.get(),
                                                   first_.get(), out->order.get());
  out->nodes.reserve(ni);
  out->nnodes = ni;
  k_ploc_emit<<<(ni + 255) / 256, 256, 0, s>>>(n, left_.get(), right_.get(), nodeParent_.get(), count_.get(),
                                               nodeHeight_.get(), collapse_.get(), leafPos_.get(), first_.get(),
                                               leafLo_.get(), leafHi_.get(), nodeLo_.get(), nodeHi_.get(),
                                               out->nodes.get());
  R2_CUDA(cudaGetLastError());
  R2_CUDA(cudaMemcpyAsync(hostState_, st, sizeof(PlocState), cudaMemcpyDeviceToHost, s));
  int root[2] = {0, 0};
  R2_CUDA(cudaMemcpyAsync(&root[0], nodeHeight_.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaMemcpyAsync(&root[1], collapse_.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  R2_CUDA(cudaStreamSynchronize(s));
  const PlocState* hs = static_cast<const PlocState*>(hostState_);
  R2_REQUIRE(hs->error == 0 && hs->m[cur] == 1 && hs->cursor == 0, R2_ERR_DEVICE,
             "PLOC clustering did not end in one root");
  return root[1] ? 0 : root[0];
}

}  // namespace r2
