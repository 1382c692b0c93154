/*
 * Screen-space LOD selection — TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Restates selectLOD of the reference's forest generator
 * (raytracer/src/filtering/generate_random_forest.py:179-225) and the helpers
 * it calls: project (73-80), projectLOD (82-101), outsideFrustum (103-105),
 * gamma (132-133, applied by the host as far_scale), intersectBB (135-151),
 * approximateNumVoxels2 (153-177).  Double precision with numpy's operation
 * order: elementwise products and sums are single IEEE operations, 3-vector
 * norms accumulate x0*x0 then fused multiply-adds (numpy's dot on this image),
 * the 4x4 matrix-vector product accumulates by fused multiply-adds in column
 * order.  scipy's ConvexHull(...).volume of the 8 projected corners is
 * restated as the shoelace area of the monotone-chain hull (Andrew 1979);
 * qhull sums the same area in another order, so the two can differ in the
 * last bits, never by a pixel in the decisions checked by the golden vectors.
 */
#include <math.h>
#include <stdint.h>

#include "oracle.h"

typedef struct { double x, y, z; } v3d;

static v3d V(double x, double y, double z) { v3d r = {x, y, z}; return r; }
static v3d vadd(v3d a, v3d b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3d vsub(v3d a, v3d b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3d vscale(double s, v3d a) { return V(s * a.x, s * a.y, s * a.z); }
static v3d vdivs(v3d a, double s) { return V(a.x / s, a.y / s, a.z / s); }
static v3d vdiv(v3d a, v3d b) { return V(a.x / b.x, a.y / b.y, a.z / b.z); }
static double vc(v3d a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static double vnorm(v3d a) { return sqrt(fma(a.z, a.z, fma(a.y, a.y, a.x * a.x))); }
static v3d vcross(v3d a, v3d b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static v3d place(const double* p, double s, v3d pos) { return vadd(vscale(s, V(p[0], p[1], p[2])), pos); }

static void project(const orc_lod_camera* c, v3d p, double* x, double* y, double* w) {
  double v[3];
  for (int r = 0; r < 3; ++r) {
    const double* m = c->world_to_view + 4 * r;
    v[r] = fma(m[3], 1.0, fma(m[2], p.z, fma(m[1], p.y, m[0] * p.x)));
  }
  const double d = c->near_plane_distance, z = -v[2];
  *x = d / z * v[0];
  *y = d / z * v[1];
  *w = -copysign(d, z);
}

static int outside(const orc_lod_camera* c, double x, double y, double w) {
  return w > 0.0 || fabs(x) > c->sensor_width * 0.5 * c->pixel_size || fabs(y) > c->sensor_height * 0.5 * c->pixel_size;
}

static double turn(double ox, double oy, double ax, double ay, double bx, double by) {
  return (ax - ox) * (by - oy) - (ay - oy) * (bx - ox);
}

static double hull_area(double* px, double* py) {
  for (int i = 1; i < 8; ++i) {
    double kx = px[i], ky = py[i];
    int j = i - 1;
    while (j >= 0 && (px[j] > kx || (px[j] == kx && py[j] > ky))) { px[j + 1] = px[j]; py[j + 1] = py[j]; --j; }
    px[j + 1] = kx;
    py[j + 1] = ky;
  }
  double hx[17], hy[17];
  int k = 0;
  for (int i = 0; i < 8; ++i) {
    while (k >= 2 && turn(hx[k - 2], hy[k - 2], hx[k - 1], hy[k - 1], px[i], py[i]) <= 0.0) --k;
    hx[k] = px[i]; hy[k] = py[i]; ++k;
  }
  for (int i = 6, t = k + 1; i >= 0; --i) {
    while (k >= t && turn(hx[k - 2], hy[k - 2], hx[k - 1], hy[k - 1], px[i], py[i]) <= 0.0) --k;
    hx[k] = px[i]; hy[k] = py[i]; ++k;
  }
  if (k < 4) return 0.0;
  double a = 0.0;
  for (int i = 0; i + 1 < k; ++i) a += hx[i] * hy[i + 1] - hx[i + 1] * hy[i];
  return fabs(a) * 0.5;
}

static v3d intersect_bb(v3d o, v3d dir, v3d lo, v3d hi, double far_scale) {
  double t1 = 3.4028234663852886e38;
  for (int i = 0; i < 3; ++i) {
    const double inv = 1.0 / vc(dir, i);
    const double tn = (vc(lo, i) - vc(o, i)) * inv;
    double tf = (vc(hi, i) - vc(o, i)) * inv;
    if (tn > tf) tf = tn;
    tf *= far_scale;
    t1 = tf < t1 ? tf : t1;
  }
  return vadd(o, vscale(t1, dir));
}

static double approx_voxels(const orc_lod_camera* c, const orc_lod_volume* v, v3d pos, double s) {
  const v3d start = place(v->bb_min, s, pos), end = place(v->bb_max, s, pos);
  const v3d origin = vscale(0.5, vadd(start, end));
  v3d n = vsub(V(c->pos[0], c->pos[1], c->pos[2]), origin);
  n = vdivs(n, vnorm(n));
  v3d xz = vcross(n, V(0.0, 1.0, 0.0));
  xz = vdivs(xz, vnorm(xz));
  const v3d b1 = intersect_bb(origin, xz, start, end, c->far_scale);
  v3d perp = vcross(xz, n);
  perp = vdivs(perp, vnorm(perp));
  const v3d b2 = intersect_bb(origin, perp, start, end, c->far_scale);
  const v3d vs = vdiv(vsub(end, start), V(v->num_voxels[0], v->num_voxels[1], v->num_voxels[2]));
  const v3d n1 = vdiv(vscale(2.0, vsub(origin, b1)), vs);
  const v3d n2 = vdiv(vscale(2.0, vsub(origin, b2)), vs);
  return ceil(vnorm(n1) * vnorm(n2));
}

int orc_select_lods(const orc_lod_camera* cam, const orc_lod_volume* lods, const uint32_t* model_first,
                    const uint32_t* model_count, uint32_t nmodels, const double* tree_pos, const double* tree_scaling,
                    const uint32_t* tree_model, uint32_t ntrees, double min_lod, double covered_pixels,
                    int32_t* lod_out, double* diag) {
  for (uint32_t t = 0; t < ntrees; ++t) {
    const uint32_t m = tree_model[t];
    if (m >= nmodels) return -1;
    const uint32_t f = model_first[m], n = model_count[m];
    const v3d pos = V(tree_pos[3 * t], tree_pos[3 * t + 1], tree_pos[3 * t + 2]);
    const double s = tree_scaling[t];
    int coarsest = -1;
    double max_size = 0.0;
    for (uint32_t i = 0; i < n; ++i)
      if (lods[f + i].voxel_size > max_size) { max_size = lods[f + i].voxel_size; coarsest = (int)(f + i); }
    if (diag) { diag[3 * t] = -1.0; diag[3 * t + 1] = 0.0; diag[3 * t + 2] = 0.0; }
    if (coarsest < 0) { lod_out[t] = -1; continue; }
    double px[8], py[8];
    int nout = 0;
    for (int k = 0; k < 8; ++k) {
      double w;
      project(cam, place(lods[coarsest].corners[k], s, pos), &px[k], &py[k], &w);
      nout += outside(cam, px[k], py[k], w);
    }
    if (nout == 8) { lod_out[t] = coarsest; continue; }
    const double area = hull_area(px, py);
    const double covered = ceil(area / cam->pixel_area);
    if (diag) { diag[3 * t] = covered; diag[3 * t + 1] = area; }
    int best = -1;
    for (uint32_t i = 0; i < n; ++i) {
      const orc_lod_volume* v = &lods[f + i];
      if (v->voxel_size >= min_lod) {
        if (approx_voxels(cam, v, pos, s) * covered_pixels > covered) best = (int)(f + i);
        else break;
      }
    }
    lod_out[t] = best;
  }
  return 0;
}
