// SGGX mesh-to-volume filter kernels for sm_100a.
//
// Reference path: __raygen__filtering (raytracer/src/backend/shaders.optix.cu:258-284)
// launches one OptiX thread per voxel running CMeshFilter::run
// (raytracer/include/filtering/mesh_filter.hpp:51-122) and estimateDensity (182-204).
//
// B200 design:
//  * k_filter_classify: one thread per voxel tests the voxel's bounding sphere
//    (radius 1.1 * |voxelSize| / 2, inflated by 0.1%) against the BVH boxes.
//    Every filter ray starts inside the voxel and ends inside that sphere, so a
//    voxel whose sphere touches no triangle box has zero hits for certain: it
//    gets the empty payload here.  The others are appended to a work list with
//    warp-aggregated atomics (ballot + popc).
//  * k_filter_sample: a persistent kernel; each warp pops one voxel at a time
//    from the work list and its 32 lanes trace the voxel's samples (lane l owns
//    samples l, l+32, ...), so a warp's rays share one BVH neighbourhood.  The
//    warp first collects the triangles whose boxes overlap the box that holds
//    all of the voxel's rays (at most kCandMax, in shared memory); every ray
//    then tests exactly those, the lanes in step, instead of walking the BVH
//    on its own.  Voxels with more candidates trace through the BVH from the
//    deepest node that holds them.  Hit ray lengths live in shared memory (no
//    4 KB per-thread local array).  Sums are compensated per lane and across
//    the warp (TwoSum butterfly).  The density fit runs its iterations as warp
//    reductions.
#include "filter.cuh"
#include "filter_math.h"
#include "texture_shade.cuh"

namespace r2 {
namespace {

constexpr int kSampleWarps = 4;  // warps per block of the sampling kernel
constexpr int kCandMax = 512;    // candidate triangles of a voxel tested without the BVH
constexpr int kCandStage = 32;   // candidates whose vertices a warp copies into shared memory
static_assert(kCandStage <= 32, "the staging copies one candidate per lane");

// Dynamic shared memory of a sampling block, per warp: the staged candidate
// vertices (kCandStage x 3 float4), the candidate list (kCandMax ints), the
// samples' hit lengths (spv floats).
__host__ __device__ constexpr size_t sample_smem_per_warp(uint32_t spv) {
  return (size_t)kCandStage * 3 * sizeof(float4) + (size_t)kCandMax * sizeof(int) + (size_t)spv * sizeof(float);
}

__device__ __forceinline__ V3 voxel_center(const FilterLaunch& L, int x, int y, int z) {
  V3 pm = xform_point(L.indexToModel, v3((float)x + 0.5f, (float)y + 0.5f, (float)z + 0.5f));
  return xform_point(L.modelToWorld, pm);
}

__device__ __forceinline__ bool box_overlap(float lox, float hix, float loy, float hiy, float loz,
                                            float hiz, V3 qlo, V3 qhi) {
  return !(lox > qhi.x || hix < qlo.x || loy > qhi.y || hiy < qlo.y || loz > qhi.z || hiz < qlo.z);
}

// Does any triangle box overlap the query box?
__device__ bool bvh_any_box(const BvhView& bvh, V3 qlo, V3 qhi) {
  int stack[R2_BVH_STACK];
  int sp = 0;
  int cur = 0;
  while (true) {
    if (cur >= 0) {
      const BvhNode* nd = &bvh.nodes[cur];
      float4 b0 = __ldg(&nd->b0), b1 = __ldg(&nd->b1), bz = __ldg(&nd->bz);
      int4 ch = __ldg(&nd->ch);
      bool h0 = box_overlap(b0.x, b0.y, b0.z, b0.w, bz.x, bz.y, qlo, qhi);
      bool h1 = ch.y != R2_BVH_NONE && box_overlap(b1.x, b1.y, b1.z, b1.w, bz.z, bz.w, qlo, qhi);
      if (h0 && h1) {
        stack[sp++] = ch.y;
        cur = ch.x;
        continue;
      } else if (h0) {
        cur = ch.x;
        continue;
      } else if (h1) {
        cur = ch.y;
        continue;
      }
    } else {
      int first = bvh_leaf_first(cur), count = bvh_leaf_count(cur);
      for (int i = 0; i < count; ++i) {
        int t = first + i;
        float4 a = __ldg(&bvh.tris[3 * t]), b = __ldg(&bvh.tris[3 * t + 1]), c = __ldg(&bvh.tris[3 * t + 2]);
        float lx = fminf(fminf(a.x, b.x), c.x), hx = fmaxf(fmaxf(a.x, b.x), c.x);
        float ly = fminf(fminf(a.y, b.y), c.y), hy = fmaxf(fmaxf(a.y, b.y), c.y);
        float lz = fminf(fminf(a.z, b.z), c.z), hz = fmaxf(fmaxf(a.z, b.z), c.z);
        if (box_overlap(lx, hx, ly, hy, lz, hz, qlo, qhi)) return true;
      }
    }
    if (sp == 0) return false;
    cur = stack[--sp];
  }
}

// The deepest node whose subtree holds every leaf whose box overlaps the
// query box: descend while exactly one child's box overlaps it.  A leaf that
// a ray confined to the query box can hit overlaps it, and so does every box
// above that leaf, so a traversal started here finds the same closest hit as
// one started at the root.
__device__ int bvh_local_root(const BvhView& bvh, V3 qlo, V3 qhi) {
  int cur = 0;
  for (int depth = 0; depth < R2_BVH_STACK && cur >= 0; ++depth) {
    const BvhNode* nd = &bvh.nodes[cur];
    const float4 b0 = __ldg(&nd->b0), b1 = __ldg(&nd->b1), bz = __ldg(&nd->bz);
    const int4 ch = __ldg(&nd->ch);
    const bool h0 = box_overlap(b0.x, b0.y, b0.z, b0.w, bz.x, bz.y, qlo, qhi);
    const bool h1 = ch.y != R2_BVH_NONE && box_overlap(b1.x, b1.y, b1.z, b1.w, bz.z, bz.w, qlo, qhi);
    if (h0 == h1) return cur;  // both children (or neither): start here
    cur = h0 ? ch.x : ch.y;
  }
  return cur;
}

// The candidate triangles of a voxel: every triangle whose box overlaps the
// query box [qlo, qhi], which holds every sample ray of the voxel, so these
// are all the triangles its rays can hit.  A depth-first walk from root that
// every lane of the warp takes in step (same nodes, same branches); the
// triangles of a leaf are tested one per lane and appended in order to list.
// Returns their number, or -1 as soon as there are more than kCandMax (the
// caller then traces the voxel's rays through the BVH).  nodes: inner nodes
// visited (the counting build; lane 0 counts).
__device__ int gather_candidates(const BvhView& bvh, int root, V3 qlo, V3 qhi, int* list, int lane,
                                 uint32_t* nodes) {
  int stack[R2_BVH_STACK];
  int sp = 0;
  int cur = root;
  int n = 0;
  while (true) {
    if (cur >= 0) {
      if (lane == 0) ++*nodes;
      const BvhNode* nd = &bvh.nodes[cur];
      const float4 b0 = __ldg(&nd->b0), b1 = __ldg(&nd->b1), bz = __ldg(&nd->bz);
      const int4 ch = __ldg(&nd->ch);
      const bool h0 = box_overlap(b0.x, b0.y, b0.z, b0.w, bz.x, bz.y, qlo, qhi);
      const bool h1 = ch.y != R2_BVH_NONE && box_overlap(b1.x, b1.y, b1.z, b1.w, bz.z, bz.w, qlo, qhi);
      if (h0 && h1) {
        stack[sp++] = ch.y;
        cur = ch.x;
        continue;
      }
      if (h0 || h1) {
        cur = h0 ? ch.x : ch.y;
        continue;
      }
    } else {
      const int first = bvh_leaf_first(cur), count = bvh_leaf_count(cur);  // count <= 31 < 32 lanes
      bool ov = false;
      if (lane < count) {
        const int t = first + lane;
        const float4 a = __ldg(&bvh.tris[3 * t]), b = __ldg(&bvh.tris[3 * t + 1]), c = __ldg(&bvh.tris[3 * t + 2]);
        ov = box_overlap(fminf(fminf(a.x, b.x), c.x), fmaxf(fmaxf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y),
                         fmaxf(fmaxf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z), fmaxf(fmaxf(a.z, b.z), c.z), qlo,
                         qhi);
      }
      const unsigned m = __ballot_sync(0xFFFFFFFFu, ov);
      const int k = __popc(m);
      if (n + k > kCandMax) return -1;
      if (ov) list[n + __popc(m & ((1u << lane) - 1u))] = first + lane;
      n += k;
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
  return n;
}

// The closest hit of one ray among the candidate triangles list[0 .. n-1],
// with the test and the (t, triangle) order of the BVH traversal: the same hit
// as bvh_trace over the whole scene.  Every lane walks the same list; the
// vertices of the first nStaged candidates come from the warp's shared copy
// `staged`, the others from the BVH's triangle array.
template <bool kAlpha>
__device__ Hit trace_candidates(const BvhView& bvh, const int* list, int n, const float4* staged, int nStaged, V3 o,
                                V3 d, float tmax) {
  const RayPre r = make_ray_pre(o, d);
  Hit best;
  best.t = tmax;
  best.b1 = best.b2 = 0.0f;
  best.tri = 0x7FFFFFFF;
  bool found = false;
  for (int c = 0; c < n; ++c) {
    const int tri = list[c];
    float4 a, b, e;
    if (c < nStaged) {
      a = staged[3 * c];
      b = staged[3 * c + 1];
      e = staged[3 * c + 2];
    } else {
      a = __ldg(&bvh.tris[3 * tri]);
      b = __ldg(&bvh.tris[3 * tri + 1]);
      e = __ldg(&bvh.tris[3 * tri + 2]);
    }
    if (tri_test<kAlpha>(r, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(e.x, e.y, e.z), tri, tri, &best, &bvh.alpha))
      found = true;
  }
  if (!found) best.tri = -1;
  return best;
}

__device__ __forceinline__ void write_voxel(r2_voxel* out, size_t vid, const r2_voxel& v) {
  const uint4* src = reinterpret_cast<const uint4*>(&v);
  uint4* dst = reinterpret_cast<uint4*>(out + vid);
  dst[0] = src[0];
  dst[1] = src[1];
}

__device__ __forceinline__ void write_empty(const FilterLaunch& L, size_t vid) {
  write_voxel(L.out, vid, empty_voxel());
  if (L.wide) {
    float* w = L.wide + vid * kWideFloats;
    for (int k = 0; k < kWideFloats; ++k) w[k] = 0.0f;
    w[16] = 1.0f;
  }
  if (L.fp16) {
    uint4* f = reinterpret_cast<uint4*>(L.fp16 + vid * 8);
    *f = make_uint4(0, 0, 0, 0);
  }
  if (L.eig) {
    float4* e = reinterpret_cast<float4*>(L.eig + vid * 12);
    e[0] = e[1] = e[2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

// FP64 eigendecomposition of the voxel's mean SGGX matrix (compensated FP32
// sums promoted to double), written to L.eig (lanes 0..11, one float each),
// and, with the projection on, the projected matrix in wv[1..6].  Every lane
// computes the same values.  Out of line: only this tail uses double registers.
__device__ __noinline__ void sggx_eig_tail(const FilterLaunch& L, uint32_t vid, int lane, const CSum* S,
                                           uint32_t hits, float* wv) {
  double m[6], w[3], V[3][3];
  const double inv = 1.0 / (double)hits;
  for (int k = 0; k < 6; ++k) m[k] = ((double)S[k].s + (double)S[k].c) * inv;
  sym3_eig_jacobi(m, w, V);
  if (L.eig && lane < 12) {
    const double v = lane < 3 ? w[lane] : V[(lane - 3) % 3][(lane - 3) / 3];
    L.eig[(size_t)vid * 12 + lane] = (float)v;
  }
  if (L.project) {
    double P[6];
    sym3_project(w, V, (double)L.floor, P);
    for (int k = 0; k < 6; ++k) wv[1 + k] = (float)P[k];
  }
}

__global__ void __launch_bounds__(256) k_filter_classify(FilterLaunch L) {
  const size_t nvox = (size_t)L.nx * L.ny * L.nz;
  // Reach of a filter ray from the voxel centre: with ClipRays the ray ends on
  // the bounding sphere; otherwise it starts anywhere in the voxel and runs
  // voxelSize.x (mesh_filter.hpp:72-82).
  const float radius = L.clip ? 1.1f * length(L.voxelSize) / 2.0f : length(L.voxelSize) / 2.0f + L.voxelSize.x;
  const float rq = radius * 1.001f + 1e-6f;
  const int lane = threadIdx.x & 31;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t base = (size_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < nvox; base += stride) {
    size_t vid = base + lane;
    bool valid = vid < nvox;
    bool cand = false;
    if (valid) {
      int x = (int)(vid % L.nx), y = (int)((vid / L.nx) % L.ny), z = (int)(vid / ((size_t)L.nx * L.ny));
      V3 c = voxel_center(L, x, y, z);
      cand = bvh_any_box(L.bvh, c - v3(rq), c + v3(rq));
      if (!cand) write_empty(L, vid);
    }
    unsigned m = __ballot_sync(0xFFFFFFFFu, cand);
    if (m) {
      uint32_t slot = 0;
      int leader = __ffs(m) - 1;
      if (lane == leader) slot = atomicAdd(&L.counters[0], (uint32_t)__popc(m));
      slot = __shfl_sync(0xFFFFFFFFu, slot, leader);
      if (cand) L.work[slot + __popc(m & ((1u << lane) - 1u))] = (uint32_t)vid;
    }
  }
}

__device__ __forceinline__ CSum warp_csum(CSum v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    CSum o;
    o.s = __shfl_xor_sync(0xFFFFFFFFu, v.s, off);
    o.c = __shfl_xor_sync(0xFFFFFFFFu, v.c, off);
    v = ccombine(v, o);
  }
  return v;
}

// 8 resident blocks per SM (64 registers a thread): traversal is issue and
// latency bound, and the extra warps hide more than the few spilled values of
// the shading tail cost (measured on the 256^3 filter: 96 registers and 5
// blocks 18.6 M voxels/s, 64 and 8 blocks 21.6 M).
// kEig: the build with the FP64 eigendecomposition tail (eigen output or
// projection requested); the default build carries none of its code.
template <bool kCount, bool kEig>
__global__ void __launch_bounds__(kSampleWarps * 32, 8) k_filter_sample(FilterLaunch L) {
  extern __shared__ float4 sSample[];  // sample_smem_per_warp(L.spv) bytes per warp
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* myV = sSample + warp * kCandStage * 3;
  int* myCand = reinterpret_cast<int*>(sSample + kSampleWarps * kCandStage * 3) + warp * kCandMax;
  float* myTs = reinterpret_cast<float*>(reinterpret_cast<int*>(sSample + kSampleWarps * kCandStage * 3) +
                                         kSampleWarps * kCandMax) + (size_t)warp * L.spv;
  const uint32_t ncand = *(volatile uint32_t*)&L.counters[0];
  const float radius = 1.1f * length(L.voxelSize) / 2.0f;
  const float tMaxFixed = L.voxelSize.x;
  uint32_t cRays = 0, cNodes = 0, cTris = 0;  // counting build only
  while (true) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(&L.counters[1], 1u);
    w = __shfl_sync(0xFFFFFFFFu, w, 0);
    if (w >= ncand) break;
    const uint32_t vid = L.work[w];
    const int x = (int)(vid % (uint32_t)L.nx);
    const int y = (int)((vid / (uint32_t)L.nx) % (uint32_t)L.ny);
    const int z = (int)(vid / ((uint32_t)L.nx * (uint32_t)L.ny));
    const V3 center = voxel_center(L, x, y, z);
    const V3 cv = v3((float)x, (float)y, (float)z);
    // every sample ray stays within `reach` of the centre (the classification's
    // radius), padded for rounding: its traversal starts at the local root
    const float reach = L.clip ? radius : length(L.voxelSize) / 2.0f + tMaxFixed;
    const float pad = reach * 1.01f + 1e-5f * (fabsf(center.x) + fabsf(center.y) + fabsf(center.z) + 1.0f);
    const V3 qlo = center - v3(pad), qhi = center + v3(pad);
    const int root = bvh_local_root(L.bvh, qlo, qhi);
    // few candidate triangles (the usual case): every ray tests them all, the
    // warp's lanes in step; otherwise the rays traverse the BVH from root
    const int ncand = gather_candidates(L.bvh, root, qlo, qhi, myCand, lane, &cNodes);
    __syncwarp();
    const int nStaged = ncand < 0 ? 0 : min(ncand, kCandStage);
    if (lane < nStaged) {
      const int t = myCand[lane];
      myV[3 * lane] = __ldg(&L.bvh.tris[3 * t]);
      myV[3 * lane + 1] = __ldg(&L.bvh.tris[3 * t + 1]);
      myV[3 * lane + 2] = __ldg(&L.bvh.tris[3 * t + 2]);
    }
    __syncwarp();

    CSum S[6], nrm[3], dist;
    float dif[3] = {0.f, 0.f, 0.f}, spe[3] = {0.f, 0.f, 0.f}, rough = 0.f, ior = 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) S[k] = csum0();
#pragma unroll
    for (int k = 0; k < 3; ++k) nrm[k] = csum0();
    dist = csum0();
    uint32_t hits = 0;

    for (uint32_t s = lane; s < L.spv; s += 32) {
      const U4 r0 = philox4x32_10(u4(s, 0u, L.lod, 0u), vid, L.seed);
      const U4 r1 = philox4x32_10(u4(s, 1u, L.lod, 0u), vid, L.seed);
      const V3 oi = cv + v3(u01(r0.x), u01(r0.y), u01(r0.z));
      const V3 o = xform_point(L.indexToWorld, oi);
      const V3 d = uniform_sample_sphere(u01(r0.w), u01(r1.x));
      const float tmax = L.clip ? sphere_exit(o, d, center, radius) : tMaxFixed;
      Hit h;
      if (ncand >= 0) {
        h = L.bvh.alpha.alphaTex ? trace_candidates<true>(L.bvh, myCand, ncand, myV, nStaged, o, d, tmax)
                                 : trace_candidates<false>(L.bvh, myCand, ncand, myV, nStaged, o, d, tmax);
        if (kCount) cTris += (uint32_t)ncand;
      } else {
        h = bvh_trace<false, kCount>(L.bvh, o, d, tmax, &cNodes, &cTris, root);
      }
      if (kCount) ++cRays;
      float tsv = -1.0f;
      if (h.tri >= 0) {
        const float4 n0 = __ldg(&L.triN[3 * h.tri]);
        const float4 n1 = __ldg(&L.triN[3 * h.tri + 1]);
        const float4 n2 = __ldg(&L.triN[3 * h.tri + 2]);
        const float b0 = (1.0f - h.b1) - h.b2;
        V3 gn = v3(n0.x, n0.y, n0.z) * b0 + v3(n1.x, n1.y, n1.z) * h.b1 + v3(n2.x, n2.y, n2.z) * h.b2;
        gn = normalize(gn);
        V3 n = normalize(xform_vector(L.objModelToWorld, gn));
        const uint32_t mi = __ldg(&L.triMat[h.tri]);
        const r2_material& m = L.mats[mi];
        V3 kd = v3(m.diffuse[0], m.diffuse[1], m.diffuse[2]), ks = v3(m.specular[0], m.specular[1], m.specular[2]);
        if (L.triUV) {  // diffuse(tc), glossy(tc) and the normal-mapped normal (mesh_filter.hpp:300-371)
          const int4 mt = L.matTex[mi];
          if (mt.x >= 0 || mt.y >= 0 || mt.z >= 0) {
            const TexView tv = {L.triUV, L.texels, L.texInfo, L.bvh.tris};
            const TexShade ts = textured_surface(tv, mt.x, mt.y, mt.z, h.tri, h.b1, h.b2, n, kd, ks);
            n = ts.n;
            kd = ts.diffuse;
            ks = ts.specular;
          }
        }
        float bs[6];
        build_s(n, m.alpha_x, bs);
#pragma unroll
        for (int k = 0; k < 6; ++k) cadd(S[k], bs[k]);
        cadd(nrm[0], n.x);
        cadd(nrm[1], n.y);
        cadd(nrm[2], n.z);
        cadd(dist, tmax);
        dif[0] += kd.x;
        dif[1] += kd.y;
        dif[2] += kd.z;
        spe[0] += ks.x;
        spe[1] += ks.y;
        spe[2] += ks.z;
        rough += m.alpha_x;
        ior += m.eta_t;
        ++hits;
        tsv = tmax;
      }
      myTs[s] = tsv;
    }

    // warp reductions (butterfly: every lane ends with the same totals)
#pragma unroll
    for (int k = 0; k < 6; ++k) S[k] = warp_csum(S[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) nrm[k] = warp_csum(nrm[k]);
    dist = warp_csum(dist);
    CSum cd[3], cs[3], cr, ci;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      cd[k].s = dif[k]; cd[k].c = 0.f; cd[k] = warp_csum(cd[k]);
      cs[k].s = spe[k]; cs[k].c = 0.f; cs[k] = warp_csum(cs[k]);
    }
    cr.s = rough; cr.c = 0.f; cr = warp_csum(cr);
    ci.s = ior; ci.c = 0.f; ci = warp_csum(ci);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) hits += __shfl_xor_sync(0xFFFFFFFFu, hits, off);

    // the hit samples' lengths packed into myTs[0 .. hits-1] in sample order, so
    // that every iteration of the density fit visits the hits only
    if (L.clip) {
      uint32_t packed = 0;
      for (uint32_t base = 0; base < L.spv; base += 32) {
        const uint32_t s = base + lane;
        const float t = s < L.spv ? myTs[s] : -1.0f;
        const unsigned m = __ballot_sync(0xFFFFFFFFu, t >= 0.0f);
        __syncwarp();  // every lane has read its entry before any is overwritten
        if (t >= 0.0f) myTs[packed + __popc(m & ((1u << lane) - 1u))] = t;
        packed += (uint32_t)__popc(m);
      }
      __syncwarp();
    }

    float wv[kWideFloats];
#pragma unroll
    for (int k = 0; k < kWideFloats; ++k) wv[k] = 0.0f;
    if (hits > 0) {
      // estimateDensity (mesh_filter.hpp:182-204)
      const float avgDist = cvalue(dist) / (float)hits;
      const float pMesh = (float)hits / (float)L.spv;
      float density = -logf(1.0f - pMesh) / (avgDist * L.sigma_t);
      const float nAlpha = L.alpha / L.sigma_t;
      for (uint32_t it = 0; it < L.iters; ++it) {
        float pVol;
        if (L.clip) {
          CSum p = csum0();
          for (uint32_t s = lane; s < hits; s += 32) cadd(p, expf(-density * L.sigma_t * myTs[s]));
          p = warp_csum(p);
          pVol = 1.0f - cvalue(p) / (float)hits;
        } else {
          pVol = 1.0f - expf(-density * L.sigma_t * tMaxFixed);
        }
        density = density - nAlpha * (pVol - pMesh);
      }
      const float inv = 1.0f / (float)hits;
      wv[0] = density;
#pragma unroll
      for (int k = 0; k < 6; ++k) wv[1 + k] = cvalue(S[k]) * inv;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        wv[7 + k] = cvalue(cd[k]) * inv;
        wv[10 + k] = cvalue(cs[k]) * inv;
      }
      const V3 nm = normalize(xform_vector(L.worldToModel, v3(cvalue(nrm[0]), cvalue(nrm[1]), cvalue(nrm[2])) * inv));
      wv[13] = nm.x;
      wv[14] = nm.y;
      wv[15] = nm.z;
      wv[16] = cvalue(ci) * inv;
      wv[17] = (float)hits;
      wv[18] = avgDist;
      wv[19] = cvalue(cr) * inv;
      if (kEig) sggx_eig_tail(L, vid, lane, S, hits, wv);
    } else {
      wv[16] = 1.0f;
      if (kEig && L.eig && lane < 12) L.eig[(size_t)vid * 12 + lane] = 0.0f;
    }
    if (lane == 0) {
      write_voxel(L.out, vid, hits > 0 ? encode_voxel(wv) : empty_voxel());
      if (L.fp16) {
        uint16_t h[8];
#pragma unroll
        for (int k = 0; k < 7; ++k) h[k] = f32_to_f16_bits(wv[k]);
        h[7] = 0;
        *reinterpret_cast<uint4*>(L.fp16 + (size_t)vid * 8) = *reinterpret_cast<const uint4*>(h);
      }
    }
    if (L.wide && lane < kWideFloats) {
      float val = wv[0];
#pragma unroll
      for (int k = 1; k < kWideFloats; ++k) if (lane == k) val = wv[k];
      L.wide[(size_t)vid * kWideFloats + lane] = val;
    }
    __syncwarp();
  }
  if (kCount) {
    unsigned long long r = cRays, n = cNodes, t = cTris;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      r += __shfl_xor_sync(0xFFFFFFFFu, r, off);
      n += __shfl_xor_sync(0xFFFFFFFFu, n, off);
      t += __shfl_xor_sync(0xFFFFFFFFu, t, off);
    }
    if (lane == 0) {
      atomicAdd(&L.ops[0], r);
      atomicAdd(&L.ops[1], n);
      atomicAdd(&L.ops[2], t);
    }
  }
}

}  // namespace

void launch_filter_classify(const FilterLaunch& L, cudaStream_t s) {
  const size_t nvox = (size_t)L.nx * L.ny * L.nz;
  int blocks = (int)std::min<size_t>((nvox + 255) / 256, (size_t)sm_count() * 16);
  if (blocks < 1) blocks = 1;
  k_filter_classify<<<blocks, 256, 0, s>>>(L);
  R2_CUDA(cudaGetLastError());
}

template <bool kCount, bool kEig>
static void launch_sample(const FilterLaunch& L, cudaStream_t s) {
  const size_t smem = kSampleWarps * sample_smem_per_warp(L.spv);  // <= 4 x 30 KB at spv 1024
  int n = 0;
  R2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_filter_sample<kCount, kEig>, kSampleWarps * 32, smem));
  k_filter_sample<kCount, kEig><<<sm_count() * std::max(n, 1), kSampleWarps * 32, smem, s>>>(L);
}

void launch_filter_sample(const FilterLaunch& L, cudaStream_t s) {
  const bool eig = L.eig || L.project;
  if (L.ops) {
    if (eig) launch_sample<true, true>(L, s);
    else launch_sample<true, false>(L, s);
  } else {
    if (eig) launch_sample<false, true>(L, s);
    else launch_sample<false, false>(L, s);
  }
  R2_CUDA(cudaGetLastError());
}

}  // namespace r2
