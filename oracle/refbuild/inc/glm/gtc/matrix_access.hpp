// glm/gtc/matrix_access.hpp - row and column access.  Test infrastructure; see glm/glm.hpp.
#pragma once
#include "../glm.hpp"

namespace glm {
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN vec<R, T, Q> column(mat<C, R, T, Q> const& m, length_t i) { return m[i]; }
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN vec<C, T, Q> row(mat<C, R, T, Q> const& m, length_t i) {
    vec<C, T, Q> r;
    for (length_t c = 0; c < C; c++) r[c] = m[c][i];
    return r;
}
}  // namespace glm
