// glm/glm.hpp - minimal restatement of the subset of OpenGL Mathematics (glm 1.0.1, MIT
// licence, https://github.com/g-truc/glm) that the reference's simulator headers use.
//
// Test infrastructure only: the reference (KittenEngine/YarnBall) includes glm, which is not
// vendored in the reference and not installed here, so the recipe in oracle/refbuild compiles
// the reference's own sources against this header instead.  It is written from glm's
// documented semantics; where the order of floating-point operations decides the rounded
// result it follows glm's published implementation:
//   dot(vec3)  (a.x*b.x + a.y*b.y) + a.z*b.z     dot(vec4)  ((x + y) + z) + w of the products
//                                                (glm's MSVC branch; the reference builds with MSVC)
//   length     sqrt(dot(v, v))                   normalize  v * (1 / sqrt(dot(v, v)))
//   cross      (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
//   mix        x * (1 - a) + y * a               clamp      min(max(x, lo), hi)
//   min        (y < x) ? y : x                   max        (x < y) ? y : x
//   mat * vec  sum over columns in column order  inverse    adjugate times 1 / determinant
//                                                           (determinant by the first column)
// Conversions between vector sizes and component types are implicit, as in glm without
// GLM_FORCE_EXPLICIT_CTOR; default constructors leave components uninitialised, as in glm
// without GLM_FORCE_CTOR_INIT.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <type_traits>

#if defined(__CUDACC__)
#define GLMS_FN __host__ __device__ inline
#else
#define GLMS_FN inline
#endif

namespace glm {

typedef int length_t;
enum qualifier { packed_highp, packed_mediump, packed_lowp, highp = packed_highp, mediump = packed_mediump,
                 lowp = packed_lowp, aligned_highp = packed_highp, defaultp = packed_highp };

typedef std::int8_t i8;
typedef std::int16_t i16;
typedef std::int32_t i32;
typedef std::int64_t i64;
typedef std::uint8_t u8;
typedef std::uint16_t u16;
typedef std::uint32_t u32;
typedef std::uint64_t u64;
typedef unsigned int uint;

template <length_t L, typename T, qualifier Q = defaultp> struct vec;
template <length_t C, length_t R, typename T, qualifier Q = defaultp> struct mat;

namespace detail {
template <typename... A> struct all_arith;
template <> struct all_arith<> { static constexpr bool value = true; };
template <typename H, typename... A> struct all_arith<H, A...> {
    static constexpr bool value = std::is_arithmetic<typename std::decay<H>::type>::value && all_arith<A...>::value;
};
}  // namespace detail

// ---------------------------------------------------------------------------- vectors
template <typename T, qualifier Q>
struct vec<1, T, Q> {
    typedef T value_type;
    T x;
    vec() = default;
    GLMS_FN explicit vec(T s) : x(s) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<1, U, P> const& v) : x(static_cast<T>(v.x)) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<2, U, P> const& v) : x(static_cast<T>(v.x)) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<3, U, P> const& v) : x(static_cast<T>(v.x)) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<4, U, P> const& v) : x(static_cast<T>(v.x)) {}
    static constexpr length_t length() { return 1; }
    GLMS_FN T& operator[](length_t i) { return (&x)[i]; }
    GLMS_FN T const& operator[](length_t i) const { return (&x)[i]; }
};

template <typename T, qualifier Q>
struct vec<2, T, Q> {
    typedef T value_type;
    T x, y;
    vec() = default;
    GLMS_FN explicit vec(T s) : x(s), y(s) {}
    template <typename A, typename B> GLMS_FN vec(A a, B b) : x(static_cast<T>(a)), y(static_cast<T>(b)) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<2, U, P> const& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<3, U, P> const& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)) {}
    template <typename U, qualifier P> GLMS_FN vec(vec<4, U, P> const& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)) {}
    static constexpr length_t length() { return 2; }
    GLMS_FN T& operator[](length_t i) { return (&x)[i]; }
    GLMS_FN T const& operator[](length_t i) const { return (&x)[i]; }
};

template <typename T, qualifier Q>
struct vec<3, T, Q> {
    typedef T value_type;
    T x, y, z;
    vec() = default;
    GLMS_FN explicit vec(T s) : x(s), y(s), z(s) {}
    template <typename A, typename B, typename C>
    GLMS_FN vec(A a, B b, C c) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)) {}
    template <typename A, typename B, qualifier P>
    GLMS_FN vec(vec<2, A, P> const& a, B b) : x(static_cast<T>(a.x)), y(static_cast<T>(a.y)), z(static_cast<T>(b)) {}
    template <typename A, typename B, qualifier P>
    GLMS_FN vec(A a, vec<2, B, P> const& b) : x(static_cast<T>(a)), y(static_cast<T>(b.x)), z(static_cast<T>(b.y)) {}
    template <typename U, qualifier P>
    GLMS_FN vec(vec<3, U, P> const& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)) {}
    template <typename U, qualifier P>
    GLMS_FN vec(vec<4, U, P> const& v) : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)) {}
    static constexpr length_t length() { return 3; }
    GLMS_FN T& operator[](length_t i) { return (&x)[i]; }
    GLMS_FN T const& operator[](length_t i) const { return (&x)[i]; }
};

template <typename T, qualifier Q>
struct vec<4, T, Q> {
    typedef T value_type;
    T x, y, z, w;
    vec() = default;
    GLMS_FN explicit vec(T s) : x(s), y(s), z(s), w(s) {}
    template <typename A, typename B, typename C, typename D>
    GLMS_FN vec(A a, B b, C c, D d) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)), w(static_cast<T>(d)) {}
    template <typename A, typename B, qualifier P>
    GLMS_FN vec(vec<3, A, P> const& a, B b)
        : x(static_cast<T>(a.x)), y(static_cast<T>(a.y)), z(static_cast<T>(a.z)), w(static_cast<T>(b)) {}
    template <typename A, typename B, qualifier P>
    GLMS_FN vec(A a, vec<3, B, P> const& b)
        : x(static_cast<T>(a)), y(static_cast<T>(b.x)), z(static_cast<T>(b.y)), w(static_cast<T>(b.z)) {}
    template <typename A, typename B, qualifier P1, qualifier P2>
    GLMS_FN vec(vec<2, A, P1> const& a, vec<2, B, P2> const& b)
        : x(static_cast<T>(a.x)), y(static_cast<T>(a.y)), z(static_cast<T>(b.x)), w(static_cast<T>(b.y)) {}
    template <typename A, typename B, typename C, qualifier P>
    GLMS_FN vec(vec<2, A, P> const& a, B b, C c)
        : x(static_cast<T>(a.x)), y(static_cast<T>(a.y)), z(static_cast<T>(b)), w(static_cast<T>(c)) {}
    template <typename U, qualifier P>
    GLMS_FN vec(vec<4, U, P> const& v)
        : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)), w(static_cast<T>(v.w)) {}
    static constexpr length_t length() { return 4; }
    GLMS_FN T& operator[](length_t i) { return (&x)[i]; }
    GLMS_FN T const& operator[](length_t i) const { return (&x)[i]; }
};

#define GLMS_VV(OP)                                                                        \
    template <length_t L, typename T, qualifier Q>                                         \
    GLMS_FN vec<L, T, Q> operator OP(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {       \
        vec<L, T, Q> r;                                                                    \
        for (length_t i = 0; i < L; i++) r[i] = a[i] OP b[i];                              \
        return r;                                                                          \
    }                                                                                      \
    template <length_t L, typename T, qualifier Q>                                         \
    GLMS_FN vec<L, T, Q> operator OP(vec<L, T, Q> const& a, T b) {                         \
        vec<L, T, Q> r;                                                                    \
        for (length_t i = 0; i < L; i++) r[i] = a[i] OP b;                                 \
        return r;                                                                          \
    }                                                                                      \
    template <length_t L, typename T, qualifier Q>                                         \
    GLMS_FN vec<L, T, Q> operator OP(T a, vec<L, T, Q> const& b) {                         \
        vec<L, T, Q> r;                                                                    \
        for (length_t i = 0; i < L; i++) r[i] = a OP b[i];                                 \
        return r;                                                                          \
    }                                                                                      \
    template <length_t L, typename T, qualifier Q, typename U>                             \
    GLMS_FN vec<L, T, Q>& operator OP##=(vec<L, T, Q>& a, vec<L, U, Q> const& b) {         \
        for (length_t i = 0; i < L; i++) a[i] = a[i] OP static_cast<T>(b[i]);              \
        return a;                                                                          \
    }                                                                                      \
    template <length_t L, typename T, qualifier Q, typename U,                             \
              typename std::enable_if<std::is_arithmetic<U>::value, int>::type = 0>        \
    GLMS_FN vec<L, T, Q>& operator OP##=(vec<L, T, Q>& a, U b) {                           \
        for (length_t i = 0; i < L; i++) a[i] = a[i] OP static_cast<T>(b);                 \
        return a;                                                                          \
    }
GLMS_VV(+)
GLMS_VV(-)
GLMS_VV(*)
GLMS_VV(/)
#undef GLMS_VV

template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> operator-(vec<L, T, Q> const& a) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = -a[i];
    return r;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> operator+(vec<L, T, Q> const& a) { return a; }
template <length_t L, typename T, qualifier Q>
GLMS_FN bool operator==(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    for (length_t i = 0; i < L; i++)
        if (!(a[i] == b[i])) return false;
    return true;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN bool operator!=(vec<L, T, Q> const& a, vec<L, T, Q> const& b) { return !(a == b); }
template <length_t L, typename T, qualifier Q, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
GLMS_FN vec<L, T, Q> operator%(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = a[i] % b[i];
    return r;
}

// ---------------------------------------------------------------------------- scalar functions
template <typename T> GLMS_FN T min(T x, T y) { return (y < x) ? y : x; }
template <typename T> GLMS_FN T max(T x, T y) { return (x < y) ? y : x; }
template <typename T> GLMS_FN T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
template <typename T> GLMS_FN T abs(T x) { return x >= T(0) ? x : -x; }
template <typename T> GLMS_FN T sign(T x) { return T(T(0) < x) - T(x < T(0)); }
template <typename T> GLMS_FN T mix(T x, T y, T a) { return x * (T(1) - a) + y * a; }
template <typename T> GLMS_FN T floor(T x) { using std::floor; return floor(x); }
template <typename T> GLMS_FN T ceil(T x) { using std::ceil; return ceil(x); }
template <typename T> GLMS_FN T fract(T x) { return x - floor(x); }
template <typename T> GLMS_FN T sqrt(T x) { using std::sqrt; return sqrt(x); }
template <typename T> GLMS_FN T inversesqrt(T x) { return static_cast<T>(1) / sqrt(x); }
template <typename T> GLMS_FN T exp(T x) { using std::exp; return exp(x); }
template <typename T> GLMS_FN T log(T x) { using std::log; return log(x); }
template <typename T> GLMS_FN T pow(T x, T y) { using std::pow; return pow(x, y); }
template <typename T> GLMS_FN T sin(T x) { using std::sin; return sin(x); }
template <typename T> GLMS_FN T cos(T x) { using std::cos; return cos(x); }
template <typename T> GLMS_FN T tan(T x) { using std::tan; return tan(x); }
template <typename T> GLMS_FN T asin(T x) { using std::asin; return asin(x); }
template <typename T> GLMS_FN T acos(T x) { using std::acos; return acos(x); }
template <typename T> GLMS_FN T atan(T y, T x) { using std::atan2; return atan2(y, x); }
template <typename T> GLMS_FN T atan(T x) { using std::atan; return atan(x); }
template <typename T> GLMS_FN T radians(T d) { return d * static_cast<T>(0.01745329251994329576923690768489); }
template <typename T> GLMS_FN T degrees(T r) { return r * static_cast<T>(57.295779513082320876798154814105); }
template <typename T> GLMS_FN bool isnan(T x) {
#if defined(__CUDA_ARCH__)
    return ::isnan(x);
#else
    return std::isnan(x);
#endif
}
template <typename T> GLMS_FN bool isinf(T x) {
#if defined(__CUDA_ARCH__)
    return ::isinf(x);
#else
    return std::isinf(x);
#endif
}

// ---------------------------------------------------------------------------- vector functions
#define GLMS_MAP1(NAME)                                                                    \
    template <length_t L, typename T, qualifier Q>                                         \
    GLMS_FN vec<L, T, Q> NAME(vec<L, T, Q> const& a) {                                     \
        vec<L, T, Q> r;                                                                    \
        for (length_t i = 0; i < L; i++) r[i] = NAME(a[i]);                                \
        return r;                                                                          \
    }
GLMS_MAP1(abs)
GLMS_MAP1(sign)
GLMS_MAP1(floor)
GLMS_MAP1(ceil)
GLMS_MAP1(fract)
GLMS_MAP1(sqrt)
GLMS_MAP1(inversesqrt)
GLMS_MAP1(exp)
GLMS_MAP1(log)
GLMS_MAP1(sin)
GLMS_MAP1(cos)
GLMS_MAP1(tan)
GLMS_MAP1(asin)
GLMS_MAP1(acos)
GLMS_MAP1(radians)
GLMS_MAP1(degrees)
#undef GLMS_MAP1

template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> min(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = min(a[i], b[i]);
    return r;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> min(vec<L, T, Q> const& a, T b) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = min(a[i], b);
    return r;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> max(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = max(a[i], b[i]);
    return r;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> max(vec<L, T, Q> const& a, T b) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = max(a[i], b);
    return r;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> clamp(vec<L, T, Q> const& x, T lo, T hi) {
    return min(max(x, lo), hi);
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> clamp(vec<L, T, Q> const& x, vec<L, T, Q> const& lo, vec<L, T, Q> const& hi) {
    return min(max(x, lo), hi);
}
template <length_t L, typename T, qualifier Q, typename U>
GLMS_FN vec<L, T, Q> mix(vec<L, T, Q> const& x, vec<L, T, Q> const& y, U a) {
    return vec<L, T, Q>(vec<L, U, Q>(x) * (static_cast<U>(1) - a) + vec<L, U, Q>(y) * a);
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> mix(vec<L, T, Q> const& x, vec<L, T, Q> const& y, vec<L, T, Q> const& a) {
    return x * (static_cast<T>(1) - a) + y * a;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> pow(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = pow(a[i], b[i]);
    return r;
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> atan(vec<L, T, Q> const& y, vec<L, T, Q> const& x) {
    vec<L, T, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = atan(y[i], x[i]);
    return r;
}

template <typename T, qualifier Q> GLMS_FN T dot(vec<1, T, Q> const& a, vec<1, T, Q> const& b) { return a.x * b.x; }
template <typename T, qualifier Q> GLMS_FN T dot(vec<2, T, Q> const& a, vec<2, T, Q> const& b) {
    vec<2, T, Q> t(a * b);
    return t.x + t.y;
}
template <typename T, qualifier Q> GLMS_FN T dot(vec<3, T, Q> const& a, vec<3, T, Q> const& b) {
    vec<3, T, Q> t(a * b);
    return t.x + t.y + t.z;
}
// glm 1.0.1 sums a vec4 dot product left to right when compiled by MSVC (the reference's
// toolchain, YarnBall.vcxproj; other compilers pair the terms): ((x + y) + z) + w.
template <typename T, qualifier Q> GLMS_FN T dot(vec<4, T, Q> const& a, vec<4, T, Q> const& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
template <typename T> GLMS_FN typename std::enable_if<std::is_arithmetic<T>::value, T>::type dot(T a, T b) { return a * b; }
template <typename T, qualifier Q>
GLMS_FN vec<3, T, Q> cross(vec<3, T, Q> const& x, vec<3, T, Q> const& y) {
    return vec<3, T, Q>(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
template <length_t L, typename T, qualifier Q> GLMS_FN T length(vec<L, T, Q> const& v) { return sqrt(dot(v, v)); }
template <typename T> GLMS_FN typename std::enable_if<std::is_arithmetic<T>::value, T>::type length(T x) { return abs(x); }
template <length_t L, typename T, qualifier Q> GLMS_FN T distance(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {
    return length(b - a);
}
template <length_t L, typename T, qualifier Q> GLMS_FN vec<L, T, Q> normalize(vec<L, T, Q> const& v) {
    return v * inversesqrt(dot(v, v));
}
template <length_t L, typename T, qualifier Q>
GLMS_FN vec<L, T, Q> reflect(vec<L, T, Q> const& I, vec<L, T, Q> const& N) {
    return I - N * dot(N, I) * static_cast<T>(2);
}

#define GLMS_CMP(NAME, OP)                                                                 \
    template <length_t L, typename T, qualifier Q>                                         \
    GLMS_FN vec<L, bool, Q> NAME(vec<L, T, Q> const& a, vec<L, T, Q> const& b) {           \
        vec<L, bool, Q> r;                                                                 \
        for (length_t i = 0; i < L; i++) r[i] = a[i] OP b[i];                              \
        return r;                                                                          \
    }
GLMS_CMP(lessThan, <)
GLMS_CMP(lessThanEqual, <=)
GLMS_CMP(greaterThan, >)
GLMS_CMP(greaterThanEqual, >=)
GLMS_CMP(equal, ==)
GLMS_CMP(notEqual, !=)
#undef GLMS_CMP
template <length_t L, qualifier Q> GLMS_FN bool all(vec<L, bool, Q> const& v) {
    bool r = true;
    for (length_t i = 0; i < L; i++) r = r && v[i];
    return r;
}
template <length_t L, qualifier Q> GLMS_FN bool any(vec<L, bool, Q> const& v) {
    bool r = false;
    for (length_t i = 0; i < L; i++) r = r || v[i];
    return r;
}
template <length_t L, qualifier Q> GLMS_FN vec<L, bool, Q> not_(vec<L, bool, Q> const& v) {
    vec<L, bool, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = !v[i];
    return r;
}
template <length_t L, typename T, qualifier Q> GLMS_FN vec<L, bool, Q> isnan(vec<L, T, Q> const& v) {
    vec<L, bool, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = isnan(v[i]);
    return r;
}
template <length_t L, typename T, qualifier Q> GLMS_FN vec<L, bool, Q> isinf(vec<L, T, Q> const& v) {
    vec<L, bool, Q> r;
    for (length_t i = 0; i < L; i++) r[i] = isinf(v[i]);
    return r;
}

// ---------------------------------------------------------------------------- matrices
template <length_t C, length_t R, typename T, qualifier Q>
struct mat {
    typedef vec<R, T, Q> col_type;
    typedef vec<C, T, Q> row_type;
    typedef T value_type;
    col_type value[C];

    mat() = default;
    GLMS_FN explicit mat(T s) {
        for (length_t c = 0; c < C; c++)
            for (length_t r = 0; r < R; r++) value[c][r] = c == r ? s : T(0);
    }
    template <typename... A,
              typename std::enable_if<(sizeof...(A) == C * R) && (C * R > 1) && detail::all_arith<A...>::value,
                                      int>::type = 0>
    GLMS_FN mat(A... a) {
        const T tmp[C * R] = {static_cast<T>(a)...};
        for (length_t i = 0; i < C * R; i++) value[i / R][i % R] = tmp[i];
    }
    template <typename... A,
              typename std::enable_if<(sizeof...(A) == C) && (C > 1) && !detail::all_arith<A...>::value, int>::type = 0>
    GLMS_FN mat(A const&... a) {
        const col_type tmp[C] = {col_type(a)...};
        for (length_t i = 0; i < C; i++) value[i] = tmp[i];
    }
    // conversions: the overlapping block is copied, the rest is the identity's
    template <length_t C2, length_t R2, typename U, qualifier P>
    GLMS_FN mat(mat<C2, R2, U, P> const& m) {
        for (length_t c = 0; c < C; c++)
            for (length_t r = 0; r < R; r++)
                value[c][r] = (c < C2 && r < R2) ? static_cast<T>(m[c][r]) : (c == r ? T(1) : T(0));
    }
    static constexpr length_t length() { return C; }
    GLMS_FN col_type& operator[](length_t i) { return value[i]; }
    GLMS_FN col_type const& operator[](length_t i) const { return value[i]; }

    GLMS_FN mat& operator+=(mat const& m) {
        for (length_t c = 0; c < C; c++) value[c] += m[c];
        return *this;
    }
    GLMS_FN mat& operator-=(mat const& m) {
        for (length_t c = 0; c < C; c++) value[c] -= m[c];
        return *this;
    }
    template <typename U, typename std::enable_if<std::is_arithmetic<U>::value, int>::type = 0>
    GLMS_FN mat& operator*=(U s) {
        for (length_t c = 0; c < C; c++) value[c] *= static_cast<T>(s);
        return *this;
    }
    template <typename U, typename std::enable_if<std::is_arithmetic<U>::value, int>::type = 0>
    GLMS_FN mat& operator/=(U s) {
        for (length_t c = 0; c < C; c++) value[c] /= static_cast<T>(s);
        return *this;
    }
};

template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator+(mat<C, R, T, Q> const& a, mat<C, R, T, Q> const& b) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = a[c] + b[c];
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator-(mat<C, R, T, Q> const& a, mat<C, R, T, Q> const& b) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = a[c] - b[c];
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator-(mat<C, R, T, Q> const& a) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = -a[c];
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator*(mat<C, R, T, Q> const& a, T s) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = a[c] * s;
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator*(T s, mat<C, R, T, Q> const& a) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = s * a[c];
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator/(mat<C, R, T, Q> const& a, T s) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = a[c] / s;
    return m;
}
template <typename M> struct mat_traits;
template <length_t C, length_t R, typename T, qualifier Q> struct mat_traits<mat<C, R, T, Q>> {
    typedef vec<C, T, Q> row_type;
    typedef vec<R, T, Q> col_type;
};
// m * v: sum over columns in column order (the row vector argument converts implicitly)
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN vec<R, T, Q> operator*(mat<C, R, T, Q> const& m, typename mat_traits<mat<C, R, T, Q>>::row_type const& v) {
    vec<R, T, Q> out;
    for (length_t r = 0; r < R; r++) {
        T acc = m[0][r] * v[0];
        for (length_t c = 1; c < C; c++) acc = acc + m[c][r] * v[c];
        out[r] = acc;
    }
    return out;
}
// v * m: each column dotted with v, terms in row order
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN vec<C, T, Q> operator*(typename mat_traits<mat<C, R, T, Q>>::col_type const& v, mat<C, R, T, Q> const& m) {
    vec<C, T, Q> out;
    for (length_t c = 0; c < C; c++) {
        T acc = m[c][0] * v[0];
        for (length_t r = 1; r < R; r++) acc = acc + m[c][r] * v[r];
        out[c] = acc;
    }
    return out;
}
template <length_t K, length_t R, length_t C, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> operator*(mat<K, R, T, Q> const& a, mat<C, K, T, Q> const& b) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = a * b[c];
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN bool operator==(mat<C, R, T, Q> const& a, mat<C, R, T, Q> const& b) {
    for (length_t c = 0; c < C; c++)
        if (!(a[c] == b[c])) return false;
    return true;
}

template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<R, C, T, Q> transpose(mat<C, R, T, Q> const& m) {
    mat<R, C, T, Q> t;
    for (length_t c = 0; c < C; c++)
        for (length_t r = 0; r < R; r++) t[r][c] = m[c][r];
    return t;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> outerProduct(vec<R, T, Q> const& c, vec<C, T, Q> const& r) {
    mat<C, R, T, Q> m;
    for (length_t i = 0; i < C; i++) m[i] = c * r[i];
    return m;
}
template <length_t C, length_t R, typename T, qualifier Q>
GLMS_FN mat<C, R, T, Q> matrixCompMult(mat<C, R, T, Q> const& a, mat<C, R, T, Q> const& b) {
    mat<C, R, T, Q> m;
    for (length_t c = 0; c < C; c++) m[c] = a[c] * b[c];
    return m;
}
template <typename T, qualifier Q> GLMS_FN T determinant(mat<2, 2, T, Q> const& m) {
    return m[0][0] * m[1][1] - m[1][0] * m[0][1];
}
template <typename T, qualifier Q> GLMS_FN T determinant(mat<3, 3, T, Q> const& m) {
    return +m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
           m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}
template <typename T, qualifier Q> GLMS_FN mat<2, 2, T, Q> inverse(mat<2, 2, T, Q> const& m) {
    const T ood = static_cast<T>(1) / (+m[0][0] * m[1][1] - m[1][0] * m[0][1]);
    return mat<2, 2, T, Q>(+m[1][1] * ood, -m[0][1] * ood, -m[1][0] * ood, +m[0][0] * ood);
}
template <typename T, qualifier Q> GLMS_FN mat<3, 3, T, Q> inverse(mat<3, 3, T, Q> const& m) {
    const T ood = static_cast<T>(1) / (+m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                                       m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
                                       m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]));
    mat<3, 3, T, Q> r;
    r[0][0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * ood;
    r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * ood;
    r[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * ood;
    r[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * ood;
    r[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * ood;
    r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * ood;
    r[0][2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * ood;
    r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * ood;
    r[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * ood;
    return r;
}
// 4x4 inverse by Gauss-Jordan elimination with partial pivoting (not used on the simulation
// path; present so that the reference's matrix helpers compile).
template <typename T, qualifier Q> GLMS_FN mat<4, 4, T, Q> inverse(mat<4, 4, T, Q> const& m) {
    T a[4][8];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) {
            a[r][c] = m[c][r];
            a[r][4 + c] = r == c ? T(1) : T(0);
        }
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (abs(a[r][c]) > abs(a[p][c])) p = r;
        for (int k = 0; k < 8; k++) {
            const T t = a[c][k];
            a[c][k] = a[p][k];
            a[p][k] = t;
        }
        const T ip = T(1) / a[c][c];
        for (int k = 0; k < 8; k++) a[c][k] *= ip;
        for (int r = 0; r < 4; r++)
            if (r != c) {
                const T f = a[r][c];
                for (int k = 0; k < 8; k++) a[r][k] -= f * a[c][k];
            }
    }
    mat<4, 4, T, Q> out;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) out[c][r] = a[r][4 + c];
    return out;
}

// ---------------------------------------------------------------------------- type names
typedef vec<1, float> vec1;
typedef vec<2, float> vec2;
typedef vec<3, float> vec3;
typedef vec<4, float> vec4;
typedef vec<2, double> dvec2;
typedef vec<3, double> dvec3;
typedef vec<4, double> dvec4;
typedef vec<2, int> ivec2;
typedef vec<3, int> ivec3;
typedef vec<4, int> ivec4;
typedef vec<2, unsigned> uvec2;
typedef vec<3, unsigned> uvec3;
typedef vec<4, unsigned> uvec4;
typedef vec<2, bool> bvec2;
typedef vec<3, bool> bvec3;
typedef vec<4, bool> bvec4;
typedef vec<2, i64> i64vec2;
typedef vec<3, i64> i64vec3;
typedef vec<4, i64> i64vec4;
typedef mat<2, 2, float> mat2;
typedef mat<3, 3, float> mat3;
typedef mat<4, 4, float> mat4;
typedef mat<2, 2, float> mat2x2;
typedef mat<2, 3, float> mat2x3;
typedef mat<2, 4, float> mat2x4;
typedef mat<3, 2, float> mat3x2;
typedef mat<3, 3, float> mat3x3;
typedef mat<3, 4, float> mat3x4;
typedef mat<4, 2, float> mat4x2;
typedef mat<4, 3, float> mat4x3;
typedef mat<4, 4, float> mat4x4;
typedef mat<2, 2, double> dmat2;
typedef mat<3, 3, double> dmat3;
typedef mat<4, 4, double> dmat4;
typedef mat<2, 2, double> dmat2x2;
typedef mat<2, 3, double> dmat2x3;
typedef mat<3, 2, double> dmat3x2;
typedef mat<3, 3, double> dmat3x3;
typedef mat<4, 3, double> dmat4x3;
typedef mat<4, 4, double> dmat4x4;

}  // namespace glm
