// glm/gtc/matrix_transform.hpp - translate / rotate / scale of a 4x4 matrix (glm 1.0.1
// semantics: the transform is applied on the right, m * T).  Test infrastructure; see
// glm/glm.hpp in this directory.
#pragma once
#include "../glm.hpp"

namespace glm {
template <typename T, qualifier Q>
GLMS_FN mat<4, 4, T, Q> translate(mat<4, 4, T, Q> const& m, vec<3, T, Q> const& v) {
    mat<4, 4, T, Q> r(m);
    r[3] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2] + m[3];
    return r;
}
template <typename T, qualifier Q>
GLMS_FN mat<4, 4, T, Q> scale(mat<4, 4, T, Q> const& m, vec<3, T, Q> const& v) {
    mat<4, 4, T, Q> r;
    r[0] = m[0] * v[0];
    r[1] = m[1] * v[1];
    r[2] = m[2] * v[2];
    r[3] = m[3];
    return r;
}
template <typename T, qualifier Q>
GLMS_FN mat<4, 4, T, Q> rotate(mat<4, 4, T, Q> const& m, T angle, vec<3, T, Q> const& v) {
    const T c = cos(angle), s = sin(angle);
    const vec<3, T, Q> axis(normalize(v));
    const vec<3, T, Q> temp((T(1) - c) * axis);
    mat<4, 4, T, Q> rot;
    rot[0][0] = c + temp[0] * axis[0];
    rot[0][1] = temp[0] * axis[1] + s * axis[2];
    rot[0][2] = temp[0] * axis[2] - s * axis[1];
    rot[1][0] = temp[1] * axis[0] - s * axis[2];
    rot[1][1] = c + temp[1] * axis[1];
    rot[1][2] = temp[1] * axis[2] + s * axis[0];
    rot[2][0] = temp[2] * axis[0] + s * axis[1];
    rot[2][1] = temp[2] * axis[1] - s * axis[0];
    rot[2][2] = c + temp[2] * axis[2];
    mat<4, 4, T, Q> r;
    r[0] = m[0] * rot[0][0] + m[1] * rot[0][1] + m[2] * rot[0][2];
    r[1] = m[0] * rot[1][0] + m[1] * rot[1][1] + m[2] * rot[1][2];
    r[2] = m[0] * rot[2][0] + m[1] * rot[2][1] + m[2] * rot[2][2];
    r[3] = m[3];
    return r;
}
}  // namespace glm
