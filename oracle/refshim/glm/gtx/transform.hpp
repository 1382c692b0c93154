// glm/gtx/transform.hpp subset for host compilation of the reference headers
// (test infrastructure): translate/scale/rotate building 4x4 matrices.
#ifndef R2_REFSHIM_GLM_GTX_TRANSFORM_HPP
#define R2_REFSHIM_GLM_GTX_TRANSFORM_HPP
#include "../glm.hpp"
#include "../gtc/matrix_transform.hpp"

namespace glm {
inline mat4 translate(const vec3& v) { return translate(mat4(1.0f), v); }
inline mat4 scale(const vec3& v) { return scale(mat4(1.0f), v); }
inline mat4 rotate(float angle, const vec3& axis) { return rotate(mat4(1.0f), angle, axis); }
}  // namespace glm
#endif
