// Per-voxel filter math shared by the sampling kernel and the host runtime:
// SGGX construction, bounding-sphere clipping, the 32-byte payload encoding and
// compensated (error-free TwoSum) accumulation.
#pragma once
#include "r2_core.h"
#include "../../include/r2.h"

namespace r2 {

// CSGGXMicroflakeDistribution::buildS (include/medium/sggx_phase_function.hpp:95-105):
// S = n n^T + sigma (I - n n^T), returned as (xx, yy, zz, xy, xz, yz).
R2_HD void build_s(V3 n, float sigma, float S[6]) {
  float xx = n.x * n.x, xy = n.x * n.y, xz = n.x * n.z;
  float yy = n.y * n.y, yz = n.y * n.z, zz = n.z * n.z;
  S[0] = xx + sigma * (yy + zz);
  S[1] = yy + sigma * (xx + zz);
  S[2] = zz + sigma * (xx + yy);
  S[3] = xy + sigma * (-xy);
  S[4] = xz + sigma * (-xz);
  S[5] = yz + sigma * (-yz);
}

// Sphere::intersect (include/shapes/sphere.hpp:33-90) for a ray whose origin
// lies inside the voxel's bounding sphere: returns the far root (exit distance).
// The sphere frame is a pure translation here (the reference's CShape adds an
// axis permutation from getRotation((1,0,0)), which only reorders the sums).
R2_HD float sphere_exit(V3 o, V3 d, V3 center, float radius) {
  V3 oc = o - center;
  float a = dot(d, d);
  float b = 2.0f * dot(d, oc);
  float c = dot(oc, oc) - radius * radius;
  float disc = b * b - 4.0f * a * c;
  if (disc == 0.0f) {
    float t = (-b + sqrtf(disc)) / (2.0f * a);
    return t > 0.0f ? t : 0.0f;
  }
  if (disc > 0.0f) {
    float sq = sqrtf(disc);
    float den = 1.0f / (2.0f * a);
    float t1 = (-b + sq) * den;
    float t2 = (-b - sq) * den;
    float mn = fminf(t1, t2), mx = fmaxf(t1, t2);
    if (mx > 0.0f) return mn > 0.0f ? mn : mx;
  }
  return 0.0f;
}

// Error-free transformation a + b = s + e (Knuth's TwoSum).
R2_HD void two_sum(float a, float b, float* s, float* e) {
  float sum = a + b;
  float bb = sum - a;
  *e = (a - (sum - bb)) + (b - bb);
  *s = sum;
}

// Compensated sum: value = s + c.
struct CSum {
  float s, c;
};
R2_HD CSum csum0() { CSum r; r.s = 0.0f; r.c = 0.0f; return r; }
R2_HD void cadd(CSum& x, float v) {
  float s, e;
  two_sum(x.s, v, &s, &e);
  x.s = s;
  x.c += e;
}
R2_HD CSum ccombine(CSum a, CSum b) {
  float s, e;
  two_sum(a.s, b.s, &s, &e);
  CSum r;
  r.s = s;
  r.c = (a.c + b.c) + e;
  return r;
}
R2_HD float cvalue(CSum x) { return x.s + x.c; }

// float -> uint16 as the reference's implicit conversion after glm::clamp
// (truncation toward zero); NaN (0/0 of an empty S) maps to 0.
R2_HD uint16_t to_u16(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 65535.0f) return 65535;
  return (uint16_t)v;
}
R2_HD uint8_t to_u8(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 255.0f) return 255;
  return (uint8_t)v;
}

// SFilteredDataCompact(const SFilteredData&) (filtered_data.hpp:91-107) from
// the wide record: [0] density, [1..6] Sxx Syy Szz Sxy Sxz Syz, [7..9] diffuse,
// [10..12] specular, [13..15] normal, [16] ior.
R2_HD r2_voxel encode_voxel(const float* w) {
  const float M16 = 65535.0f, M8 = 255.0f;
  r2_voxel v;
  v.density = w[0];
  float sxx = w[1], syy = w[2], szz = w[3], sxy = w[4], sxz = w[5], syz = w[6];
  v.sigma_x = to_u16(clampf(M16 * sqrtf(sxx), 0.0f, M16));
  v.sigma_y = to_u16(clampf(M16 * sqrtf(syy), 0.0f, M16));
  v.sigma_z = to_u16(clampf(M16 * sqrtf(szz), 0.0f, M16));
  v.r_xy = to_u16(clampf(M16 * 0.5f * (sxy / sqrtf(sxx * syy) + 1.0f), 0.0f, M16));
  v.r_xz = to_u16(clampf(M16 * 0.5f * (sxz / sqrtf(sxx * szz) + 1.0f), 0.0f, M16));
  v.r_yz = to_u16(clampf(M16 * 0.5f * (syz / sqrtf(syy * szz) + 1.0f), 0.0f, M16));
  for (int k = 0; k < 3; ++k) {
    v.diffuse[k] = to_u8(clampf(M8 * w[7 + k], 0.0f, M8));
    v.specular[k] = to_u8(clampf(M8 * w[10 + k], 0.0f, M8));
  }
  V3 n = normalize(v3(w[13], w[14], w[15]));  // SFilteredData::n()
  v.normal[0] = to_u16(clampf(M16 * 0.5f * (n.x + 1.0f), 0.0f, M16));
  v.normal[1] = to_u16(clampf(M16 * 0.5f * (n.y + 1.0f), 0.0f, M16));
  v.normal[2] = to_u16(clampf(M16 * 0.5f * (n.z + 1.0f), 0.0f, M16));
  v.ior = f32_to_f16_bits(w[16]);
  v.pad = 0;
  return v;
}

// Eigendecomposition of the symmetric 3x3 matrix S (xx yy zz xy xz yz) in
// double precision by cyclic Jacobi rotations (Jacobi 1846; Golub and Van
// Loan, Matrix Computations, 4th ed., section 8.5): S = V diag(w) V^T with
// w[0] >= w[1] >= w[2] and V's columns (V[row][col]) orthonormal
// eigenvectors, each with its largest-magnitude entry non-negative.  A
// rotation in the plane (p, q) zeroes the entry a_pq; sweeps repeat until the
// off-diagonal mass is below double rounding of the diagonal (four sweeps at
// most for a 3x3 in practice; eight are allowed).  Near-planar SGGX matrices
// (one eigenvalue near 1, two near 0) are resolved to full double accuracy
// because rotations, not a characteristic polynomial, find the eigenvalues.
R2_HD void sym3_eig_jacobi(const double S[6], double w[3], double V[3][3]) {
  double a[3][3] = {{S[0], S[3], S[4]}, {S[3], S[1], S[5]}, {S[4], S[5], S[2]}};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) V[r][c] = r == c ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 8; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (!(off > 4.93e-32 * diag)) break;
    for (int r = 0; r < 3; ++r) {
      const int p = r == 2 ? 1 : 0, q = r == 0 ? 1 : 2;  // (0,1), (0,2), (1,2)
      const double apq = a[p][q];
      if (apq == 0.0) continue;
      const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
      for (int k = 0; k < 3; ++k) {  // A J
        const double akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - sn * akq;
        a[k][q] = sn * akp + c * akq;
      }
      for (int k = 0; k < 3; ++k) {  // J^T (A J)
        const double apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - sn * aqk;
        a[q][k] = sn * apk + c * aqk;
      }
      for (int k = 0; k < 3; ++k) {  // V J
        const double vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c * vkp - sn * vkq;
        V[k][q] = sn * vkp + c * vkq;
      }
    }
  }
  for (int k = 0; k < 3; ++k) w[k] = a[k][k];
  for (int i = 0; i < 2; ++i)  // descending order, columns follow
    for (int j = 0; j < 2 - i; ++j)
      if (w[j] < w[j + 1]) {
        const double tw = w[j];
        w[j] = w[j + 1];
        w[j + 1] = tw;
        for (int k = 0; k < 3; ++k) {
          const double tv = V[k][j];
          V[k][j] = V[k][j + 1];
          V[k][j + 1] = tv;
        }
      }
  for (int c = 0; c < 3; ++c) {
    int m = 0;
    for (int k = 1; k < 3; ++k)
      if (fabs(V[k][c]) > fabs(V[m][c])) m = k;
    if (V[m][c] < 0.0)
      for (int k = 0; k < 3; ++k) V[k][c] = -V[k][c];
  }
}

// Projection of S onto the SGGX matrices with every eigenvalue at least
// floor * (largest eigenvalue), floor >= 0: V diag(max(w, floor w0)) V^T.
// With floor 0 it is the projection onto the positive semidefinite cone; with
// floor > 0 it regularises near-planar voxels so that det(S) > 0 and the
// phase function's inverse(S) stays finite.
R2_HD void sym3_project(const double w[3], const double V[3][3], double floor, double S[6]) {
  double l[3];
  const double lo = floor * (w[0] > 0.0 ? w[0] : 0.0);
  for (int k = 0; k < 3; ++k) l[k] = w[k] > lo ? w[k] : lo;
  const int rr[6] = {0, 1, 2, 0, 0, 1}, cc[6] = {0, 1, 2, 1, 2, 2};
  for (int e = 0; e < 6; ++e) {
    double acc = 0.0;
    for (int k = 0; k < 3; ++k) acc += l[k] * V[rr[e]][k] * V[cc[e]][k];
    S[e] = acc;
  }
}

// Payload of a voxel without hits (mesh_filter.hpp:112-119): zeros, ior = 1.
R2_HD r2_voxel empty_voxel() {
  r2_voxel v;
  memset(&v, 0, sizeof(v));
  v.ior = 0x3C00u;
  return v;
}

}  // namespace r2
