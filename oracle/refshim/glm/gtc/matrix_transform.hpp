// glm/gtc/matrix_transform.hpp subset (test infrastructure): translate,
// scale, rotate (Rodrigues' formula about a normalised axis), lookAt (right
// handed view matrix with rows s, u, -f).
#ifndef R2_REFSHIM_GLM_GTC_MATRIX_TRANSFORM_HPP
#define R2_REFSHIM_GLM_GTC_MATRIX_TRANSFORM_HPP
#include "../glm.hpp"

namespace glm {
inline mat4 translate(const mat4& m, const vec3& v) {
  mat4 r = m;
  r[3] = m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3];
  return r;
}
inline mat4 scale(const mat4& m, const vec3& v) {
  mat4 r;
  r[0] = m[0] * v.x;
  r[1] = m[1] * v.y;
  r[2] = m[2] * v.z;
  r[3] = m[3];
  return r;
}
inline mat4 rotate(const mat4& m, float angle, const vec3& v) {
  const float c = std::cos(angle), s = std::sin(angle);
  vec3 axis = normalize(v);
  vec3 temp = axis * (1.0f - c);
  float R[3][3];
  R[0][0] = c + temp.x * axis.x;
  R[0][1] = temp.x * axis.y + s * axis.z;
  R[0][2] = temp.x * axis.z - s * axis.y;
  R[1][0] = temp.y * axis.x - s * axis.z;
  R[1][1] = c + temp.y * axis.y;
  R[1][2] = temp.y * axis.z + s * axis.x;
  R[2][0] = temp.z * axis.x + s * axis.y;
  R[2][1] = temp.z * axis.y - s * axis.x;
  R[2][2] = c + temp.z * axis.z;
  mat4 r;
  for (int j = 0; j < 3; ++j) r[j] = m[0] * R[j][0] + m[1] * R[j][1] + m[2] * R[j][2];
  r[3] = m[3];
  return r;
}
inline mat4 lookAt(const vec3& eye, const vec3& center, const vec3& up) {
  const vec3 f = normalize(center - eye);
  const vec3 s = normalize(cross(f, up));
  const vec3 u = cross(s, f);
  mat4 r(1.0f);
  r[0][0] = s.x; r[1][0] = s.y; r[2][0] = s.z;
  r[0][1] = u.x; r[1][1] = u.y; r[2][1] = u.z;
  r[0][2] = -f.x; r[1][2] = -f.y; r[2][2] = -f.z;
  r[3][0] = -dot(s, eye);
  r[3][1] = -dot(u, eye);
  r[3][2] = dot(f, eye);
  return r;
}
}  // namespace glm
#endif
