// Host-side 4x4 matrix helpers with glm's column-major conventions, used for
// grid setup and scene transforms.  Products accumulate in glm's order
// (result column j = A0*B[j][0] + A1*B[j][1] + A2*B[j][2] + A3*B[j][3]) so the
// structured matrices of the filter grid round exactly as glm would.
#pragma once
#include <math.h>
#include <string.h>

#include "r2_core.h"

namespace r2 {

struct M4 {
  float m[4][4];  // m[col][row]
};

inline M4 m4_identity() {
  M4 r;
  memset(&r, 0, sizeof(r));
  for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
  return r;
}

inline M4 m4_mul(const M4& a, const M4& b) {
  M4 r;
  for (int j = 0; j < 4; ++j) {
    for (int i = 0; i < 4; ++i) {
      float v = a.m[0][i] * b.m[j][0];
      v = v + a.m[1][i] * b.m[j][1];
      v = v + a.m[2][i] * b.m[j][2];
      v = v + a.m[3][i] * b.m[j][3];
      r.m[j][i] = v;
    }
  }
  return r;
}

inline M4 m4_translate(V3 t) {
  M4 r = m4_identity();
  r.m[3][0] = t.x;
  r.m[3][1] = t.y;
  r.m[3][2] = t.z;
  return r;
}

inline M4 m4_scale(V3 s) {
  M4 r = m4_identity();
  r.m[0][0] = s.x;
  r.m[1][1] = s.y;
  r.m[2][2] = s.z;
  return r;
}

// Inverse computed in double by Gauss-Jordan elimination with partial pivoting,
// rounded to float.  (glm::inverse uses float cofactors; both agree to rounding.)
inline M4 m4_inverse(const M4& a) {
  double A[4][8];
  for (int r = 0; r < 4; ++r) {
    for (int c = 0; c < 4; ++c) A[r][c] = a.m[c][r];
    for (int c = 0; c < 4; ++c) A[r][4 + c] = (r == c) ? 1.0 : 0.0;
  }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 8; ++k) { double t = A[c][k]; A[c][k] = A[piv][k]; A[piv][k] = t; }
    double p = A[c][c];
    if (p == 0.0) return m4_identity();
    for (int k = 0; k < 8; ++k) A[c][k] /= p;
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      double f = A[r][c];
      if (f == 0.0) continue;
      for (int k = 0; k < 8; ++k) A[r][k] -= f * A[c][k];
    }
  }
  M4 r;
  for (int row = 0; row < 4; ++row)
    for (int c = 0; c < 4; ++c) r.m[c][row] = (float)A[row][4 + c];
  return r;
}

inline M43 m4_to_m43(const M4& a) {
  M43 r;
  for (int c = 0; c < 4; ++c) r.c[c] = v3(a.m[c][0], a.m[c][1], a.m[c][2]);
  return r;
}

inline M4 m43_to_m4(const M43& a) {
  M4 r;
  for (int c = 0; c < 4; ++c) {
    r.m[c][0] = a.c[c].x;
    r.m[c][1] = a.c[c].y;
    r.m[c][2] = a.c[c].z;
    r.m[c][3] = (c == 3) ? 1.0f : 0.0f;
  }
  return r;
}

inline M43 m43_from_floats(const float* f) {
  M43 r;
  for (int c = 0; c < 4; ++c) r.c[c] = v3(f[3 * c], f[3 * c + 1], f[3 * c + 2]);
  return r;
}

inline void m43_to_floats(const M43& m, float* f) {
  for (int c = 0; c < 4; ++c) {
    f[3 * c] = m.c[c].x;
    f[3 * c + 1] = m.c[c].y;
    f[3 * c + 2] = m.c[c].z;
  }
}

// mat4 * vec4(p, 1) with glm's accumulation order.
inline V3 m4_point(const M4& a, V3 p) { return xform_point(m4_to_m43(a), p); }

// getRotation (include/utility/functions.hpp:128-142): rotation taking the
// object's +Y axis to `normal`, entries rounded to the nearest integer.
inline M4 get_rotation(V3 normal) {
  float c = dot(normal, v3(0.0f, 1.0f, 0.0f));
  if (c == 1.0f) return m4_identity();
  if (c == -1.0f) {
    M4 r = m4_identity();
    for (int i = 0; i < 3; ++i) r.m[i][i] = -1.0f;
    return r;
  }
  float angle = acosf(c);
  V3 axis = normalize(cross(normal, v3(0.0f, 1.0f, 0.0f)));
  // glm::rotate(mat4(1), angle, axis)
  float cs = cosf(angle), sn = sinf(angle);
  V3 temp = axis * (1.0f - cs);
  M4 r = m4_identity();
  r.m[0][0] = cs + temp.x * axis.x;
  r.m[0][1] = temp.x * axis.y + sn * axis.z;
  r.m[0][2] = temp.x * axis.z - sn * axis.y;
  r.m[1][0] = temp.y * axis.x - sn * axis.z;
  r.m[1][1] = cs + temp.y * axis.y;
  r.m[1][2] = temp.y * axis.z + sn * axis.x;
  r.m[2][0] = temp.z * axis.x + sn * axis.y;
  r.m[2][1] = temp.z * axis.y - sn * axis.x;
  r.m[2][2] = cs + temp.z * axis.z;
  for (int c2 = 0; c2 < 4; ++c2)
    for (int i = 0; i < 4; ++i) r.m[c2][i] = roundf(r.m[c2][i]);
  return r;
}

// CHostSceneobject::getModelToWorldTransform (src/scene/sceneobject.cu:375-377).
inline M4 model_to_world_transform(V3 pos, V3 orientation, V3 scaling) {
  return m4_mul(m4_mul(m4_translate(pos), get_rotation(orientation)), m4_scale(scaling));
}

}  // namespace r2
