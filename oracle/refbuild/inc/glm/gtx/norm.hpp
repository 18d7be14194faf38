// glm/gtx/norm.hpp - squared length and distance (dot(v, v), as glm).  Test infrastructure;
// see glm/glm.hpp in this directory.
#pragma once
#include "../glm.hpp"

namespace glm {
template <length_t L, typename T, qualifier Q> GLMS_FN T length2(vec<L, T, Q> const& v) { return dot(v, v); }
template <typename T> GLMS_FN typename std::enable_if<std::is_arithmetic<T>::value, T>::type length2(T x) { return x * x; }
template <length_t L, typename T, qualifier Q> GLMS_FN T distance2(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    return length2(b - a);
}
}  // namespace glm
