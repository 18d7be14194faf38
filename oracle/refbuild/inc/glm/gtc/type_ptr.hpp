// glm/gtc/type_ptr.hpp - pointers to the components of vectors and matrices.  Test
// infrastructure; see glm/glm.hpp in this directory.
#pragma once
#include "../glm.hpp"

namespace glm {
template <length_t L, typename T, qualifier Q> GLMS_FN T* value_ptr(vec<L, T, Q>& v) { return &v[0]; }
template <length_t L, typename T, qualifier Q> GLMS_FN T const* value_ptr(vec<L, T, Q> const& v) { return &v[0]; }
template <length_t C, length_t R, typename T, qualifier Q> GLMS_FN T* value_ptr(mat<C, R, T, Q>& m) { return &m[0][0]; }
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN T const* value_ptr(mat<C, R, T, Q> const& m) { return &m[0][0]; }
}  // namespace glm
