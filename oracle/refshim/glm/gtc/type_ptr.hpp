// glm/gtc/type_ptr.hpp subset (test infrastructure).
#ifndef R2_REFSHIM_GLM_GTC_TYPE_PTR_HPP
#define R2_REFSHIM_GLM_GTC_TYPE_PTR_HPP
#include "../glm.hpp"
namespace glm {
template <length_t C, length_t R, typename T, qualifier Q> const T* value_ptr(const mat<C, R, T, Q>& m) { return &m[0][0]; }
template <length_t L, typename T, qualifier Q> const T* value_ptr(const vec<L, T, Q>& v) { return &v[0]; }
}  // namespace glm
#endif
