// glm/gtx/compatibility.hpp - isfinite, lerp, saturate and atan2 (HLSL-style names).  Test
// infrastructure; see glm/glm.hpp in this directory.
#pragma once
#include "../glm.hpp"

namespace glm {
template <typename T> GLMS_FN bool isfinite(T x) {
#if defined(__CUDA_ARCH__)
    return ::isfinite(x);
#else
    return std::isfinite(x);
#endif
}
template <length_t L, typename T, qualifier Q> GLMS_FN vec<L, bool, Q> isfinite(vec<L, T, Q> const& v) {
    vec<L, bool, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = isfinite(v[i]);
    return r;
}
template <typename T> GLMS_FN T lerp(T x, T y, T a) { return mix(x, y, a); }
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> lerp(vec<L, T, Q> const& x, vec<L, T, Q> const& y, T a) { return mix(x, y, a); }
template <typename T> GLMS_FN T saturate(T x) { return clamp(x, T(0), T(1)); }
template <typename T> GLMS_FN T atan2(T y, T x) { return atan(y, x); }
}  // namespace glm
