// Screen-space LOD selection of many-instance scenes on the GPU: the forest
// generator's selectLOD (raytracer/src/filtering/generate_random_forest.py:179-225)
// for every tree at once, one thread per tree, in double precision.
//
// The generator evaluates this per tree in numpy and scipy; the arithmetic
// here follows its expressions step by step (elementwise numpy operations are
// single IEEE operations, so products and sums are kept separate — the
// library is built with -fmad=false — and the 3-vector norms accumulate with
// fused multiply-adds in index order as numpy's dot does on this image).
// The convex hull area (scipy ConvexHull(...).volume) is the shoelace area
// of Andrew's monotone-chain hull of the 8 projected corners.
#include "lod_select.h"

#include <vector>

#include "runtime.h"

namespace r2 {
namespace {

struct D3 {
  double x, y, z;
};

__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return d3(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)); }
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return d3(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)); }
__device__ __forceinline__ D3 dscale(double s, D3 a) { return d3(__dmul_rn(s, a.x), __dmul_rn(s, a.y), __dmul_rn(s, a.z)); }
__device__ __forceinline__ D3 ddivs(D3 a, double s) { return d3(__ddiv_rn(a.x, s), __ddiv_rn(a.y, s), __ddiv_rn(a.z, s)); }
__device__ __forceinline__ D3 ddiv(D3 a, D3 b) { return d3(__ddiv_rn(a.x, b.x), __ddiv_rn(a.y, b.y), __ddiv_rn(a.z, b.z)); }
__device__ __forceinline__ double dcomp(D3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// np.linalg.norm of a 3-vector: sqrt(x.dot(x)).
__device__ __forceinline__ double dnorm(D3 a) {
  double s = __dmul_rn(a.x, a.x);
  s = __fma_rn(a.y, a.y, s);
  s = __fma_rn(a.z, a.z, s);
  return __dsqrt_rn(s);
}

// np.cross(a, b).
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
  return d3(__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
            __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// scaling * p + pos (numpy elementwise).
__device__ __forceinline__ D3 place(const double* p, double scaling, D3 pos) {
  return dadd(dscale(scaling, d3(p[0], p[1], p[2])), pos);
}

// project(np.dot(WorldToView, vec4(p, 1)), camera): 2D sensor position and
// the sign marker -copysign(d, z) (> 0: behind the camera).
__device__ void project(const r2_lod_camera& c, D3 p, double* x, double* y, double* w) {
  double v[3];
  for (int r = 0; r < 3; ++r) {
    const double* m = c.world_to_view + 4 * r;
    double s = __dmul_rn(m[0], p.x);
    s = __fma_rn(m[1], p.y, s);
    s = __fma_rn(m[2], p.z, s);
    s = __fma_rn(m[3], 1.0, s);
    v[r] = s;
  }
  const double d = c.near_plane_distance;
  const double z = -v[2];
  const double q = __ddiv_rn(d, z);
  *x = __dmul_rn(q, v[0]);
  *y = __dmul_rn(q, v[1]);
  *w = -copysign(d, z);
}

__device__ __forceinline__ bool outside_frustum(const r2_lod_camera& c, double x, double y, double w) {
  const double ps = c.pixel_size;
  return w > 0.0 || fabs(x) > __dmul_rn(__dmul_rn(c.sensor_width, 0.5), ps) ||
         fabs(y) > __dmul_rn(__dmul_rn(c.sensor_height, 0.5), ps);
}

__device__ __forceinline__ double turn(double ox, double oy, double ax, double ay, double bx, double by) {
  return __dsub_rn(__dmul_rn(__dsub_rn(ax, ox), __dsub_rn(by, oy)), __dmul_rn(__dsub_rn(ay, oy), __dsub_rn(bx, ox)));
}

// Area of the convex hull of 8 points (0 when they are collinear).
__device__ double hull_area(double* px, double* py) {
  // insertion sort by (x, y)
  for (int i = 1; i < 8; ++i) {
    const double kx = px[i], ky = py[i];
    int j = i - 1;
    while (j >= 0 && (px[j] > kx || (px[j] == kx && py[j] > ky))) {
      px[j + 1] = px[j];
      py[j + 1] = py[j];
      --j;
    }
    px[j + 1] = kx;
    py[j + 1] = ky;
  }
  double hx[17], hy[17];
  int k = 0;
  for (int i = 0; i < 8; ++i) {  // lower hull
    while (k >= 2 && turn(hx[k - 2], hy[k - 2], hx[k - 1], hy[k - 1], px[i], py[i]) <= 0.0) --k;
    hx[k] = px[i];
    hy[k] = py[i];
    ++k;
  }
  for (int i = 6, t = k + 1; i >= 0; --i) {  // upper hull
    while (k >= t && turn(hx[k - 2], hy[k - 2], hx[k - 1], hy[k - 1], px[i], py[i]) <= 0.0) --k;
    hx[k] = px[i];
    hy[k] = py[i];
    ++k;
  }
  if (k < 4) return 0.0;  // fewer than 3 distinct hull points
  double a = 0.0;
  for (int i = 0; i + 1 < k; ++i) a = __dadd_rn(a, __dsub_rn(__dmul_rn(hx[i], hy[i + 1]), __dmul_rn(hx[i + 1], hy[i])));
  return __dmul_rn(fabs(a), 0.5);
}

// intersectBB: the smallest far-plane distance (scaled by far_scale) of the
// ray from the box centre; its point.
__device__ D3 intersect_bb(D3 o, D3 dir, D3 lo, D3 hi, double farScale) {
  double t1 = 3.4028234663852886e38;  // np.finfo(np.float32).max
  for (int i = 0; i < 3; ++i) {
    const double inv = __ddiv_rn(1.0, dcomp(dir, i));
    double tn = __dmul_rn(__dsub_rn(dcomp(lo, i), dcomp(o, i)), inv);
    double tf = __dmul_rn(__dsub_rn(dcomp(hi, i), dcomp(o, i)), inv);
    if (tn > tf) tf = tn;
    tf = __dmul_rn(tf, farScale);
    t1 = tf < t1 ? tf : t1;
  }
  return dadd(o, dscale(t1, dir));
}

// approximateNumVoxels2: visible voxels of a LOD as the product of the voxel
// counts along two axes of the box's cross-section facing the camera.
__device__ double approx_voxels(const r2_lod_camera& c, const r2_lod_volume& v, D3 pos, double scaling) {
  const D3 start = place(v.bb_min, scaling, pos);
  const D3 end = place(v.bb_max, scaling, pos);
  const D3 origin = dscale(0.5, dadd(start, end));
  D3 n = dsub(d3(c.pos[0], c.pos[1], c.pos[2]), origin);
  n = ddivs(n, dnorm(n));
  D3 xz = dcross(n, d3(0.0, 1.0, 0.0));
  xz = ddivs(xz, dnorm(xz));
  const D3 b1 = intersect_bb(origin, xz, start, end, c.far_scale);
  D3 perp = dcross(xz, n);
  perp = ddivs(perp, dnorm(perp));
  const D3 b2 = intersect_bb(origin, perp, start, end, c.far_scale);
  const D3 vs = ddiv(dsub(end, start), d3(v.num_voxels[0], v.num_voxels[1], v.num_voxels[2]));
  const D3 n1 = ddiv(dscale(2.0, dsub(origin, b1)), vs);
  const D3 n2 = ddiv(dscale(2.0, dsub(origin, b2)), vs);
  return ceil(__dmul_rn(dnorm(n1), dnorm(n2)));
}

__global__ void k_select_lods(r2_lod_camera cam, const r2_lod_volume* __restrict__ lods,
                              const uint32_t* __restrict__ first, const uint32_t* __restrict__ count,
                              const double* __restrict__ treePos, const double* __restrict__ treeScaling,
                              const uint32_t* __restrict__ treeModel, uint32_t ntrees, double minLod,
                              double coveredPixels, int32_t* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntrees) return;
  const uint32_t m = treeModel[t];
  const uint32_t f = first[m], n = count[m];
  const D3 pos = d3(treePos[3 * t], treePos[3 * t + 1], treePos[3 * t + 2]);
  const double scaling = treeScaling[t];
  // the coarsest LOD: the largest voxel size, the first of equal ones
  int coarsest = -1;
  double maxSize = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    if (lods[f + i].voxel_size > maxSize) {
      maxSize = lods[f + i].voxel_size;
      coarsest = (int)(f + i);
    }
  }
  if (coarsest < 0) {  // no LOD with a positive voxel size: the mesh
    out[t] = -1;
    return;
  }
  double px[8], py[8];
  int outside = 0;
  for (int k = 0; k < 8; ++k) {
    double w;
    project(cam, place(lods[coarsest].corners[k], scaling, pos), &px[k], &py[k], &w);
    outside += outside_frustum(cam, px[k], py[k], w) ? 1 : 0;
  }
  if (outside == 8) {
    out[t] = coarsest;
    return;
  }
  const double covered = ceil(__ddiv_rn(hull_area(px, py), cam.pixel_area));
  int best = -1;
  for (uint32_t i = 0; i < n; ++i) {
    const r2_lod_volume& v = lods[f + i];
    if (v.voxel_size >= minLod) {
      const double a = approx_voxels(cam, v, pos, scaling);
      if (__dmul_rn(a, coveredPixels) > covered) {
        best = (int)(f + i);
      } else {
        break;
      }
    }
  }
  out[t] = best;
}

}  // namespace

void select_lods(const r2_lod_camera& cam, const r2_lod_volume* lods, uint32_t nlods, const uint32_t* modelFirst,
                 const uint32_t* modelCount, uint32_t nmodels, const double* treePos, const double* treeScaling,
                 const uint32_t* treeModel, uint32_t ntrees, double minLod, double coveredPixels, int32_t* out,
                 cudaStream_t s) {
  for (uint32_t m = 0; m < nmodels; ++m)
    R2_REQUIRE((uint64_t)modelFirst[m] + modelCount[m] <= nlods, R2_ERR_INVALID_ARGUMENT,
               "model " + std::to_string(m) + " names LODs beyond the table");
  for (uint32_t t = 0; t < ntrees; ++t)
    R2_REQUIRE(treeModel[t] < nmodels, R2_ERR_INVALID_ARGUMENT,
               "tree " + std::to_string(t) + " names model " + std::to_string(treeModel[t]));
  if (ntrees == 0) return;
  DBuf<r2_lod_volume> dLods;
  DBuf<uint32_t> dFirst, dCount, dModel;
  DBuf<double> dPos, dScaling;
  DBuf<int32_t> dOut(ntrees);
  dLods.upload(lods, nlods, s);
  dFirst.upload(modelFirst, nmodels, s);
  dCount.upload(modelCount, nmodels, s);
  dPos.upload(treePos, (size_t)3 * ntrees, s);
  dScaling.upload(treeScaling, ntrees, s);
  dModel.upload(treeModel, ntrees, s);
  k_select_lods<<<(ntrees + 127) / 128, 128, 0, s>>>(cam, dLods.get(), dFirst.get(), dCount.get(), dPos.get(),
                                                     dScaling.get(), dModel.get(), ntrees, minLod, coveredPixels,
                                                     dOut.get());
  R2_CUDA(cudaGetLastError());
  dOut.download(out, ntrees, s);
  R2_CUDA(cudaStreamSynchronize(s));
}

}  // namespace r2
