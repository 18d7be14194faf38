// ybmath.cuh - host+device vector, rotor and 3x3 algebra for the Cosserat rod substep.
//
// Everything is templated on the working precision R (float for the production build,
// double for the FP64 build of the same kernels).  Two flavours of the segment-segment
// predicates exist:
//   * the "exact" flavour (Ex<R>) issues every multiply/add/divide/sqrt as a separately
//     rounded IEEE operation (no FMA contraction on the device, and the host side is compiled
//     with -ffp-contract=off).  Detection (AABB padding, the narrow-phase distance filter and
//     the step-size limit) uses it, so its decisions are reproducible bit for bit by a CPU
//     restatement that evaluates the same expressions in the same order.
//   * the ordinary flavour lets the compiler contract to FMA; the Newton iteration uses it.
//
// Semantics follow the reference math helpers:
//   segmentClosestPoints  KittenEngine/KittenEngine/includes/modules/Common.h:318-336
//   hess3                 KittenEngine/KittenEngine/includes/modules/SymMat.h:8-107
//   Rotor (x,y,z bivector, w scalar), product, inverse, rotate, fromTo
//                         KittenEngine/KittenEngine/includes/modules/Rotor.h:57-105,185-188,230-232
//   orthoBasisX           KittenEngine/KittenEngine/includes/modules/Common.h:235-251
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define YB_HD __host__ __device__ __forceinline__
#else
#define YB_HD inline
#endif

namespace yb {

// ---------------------------------------------------------------------------------------
// Storage vector (16 B for float, 32 B for double) - one coalesced vector load per element.
template <typename R>
struct alignas(sizeof(R) * 4) V4 {
    R x, y, z, w;
};

template <typename R>
struct V3 {
    R x, y, z;
    YB_HD V3() {}
    YB_HD V3(R a, R b, R c) : x(a), y(b), z(c) {}
    YB_HD explicit V3(R s) : x(s), y(s), z(s) {}
    YB_HD R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <typename R> YB_HD V3<R> xyz(const V4<R>& v) { return V3<R>(v.x, v.y, v.z); }
template <typename R> YB_HD V4<R> v4(const V3<R>& v, R w) { V4<R> r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = w; return r; }

template <typename R> YB_HD V3<R> operator+(V3<R> a, V3<R> b) { return V3<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename R> YB_HD V3<R> operator-(V3<R> a, V3<R> b) { return V3<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename R> YB_HD V3<R> operator-(V3<R> a) { return V3<R>(-a.x, -a.y, -a.z); }
template <typename R> YB_HD V3<R> operator*(R s, V3<R> a) { return V3<R>(s * a.x, s * a.y, s * a.z); }
template <typename R> YB_HD V3<R> operator*(V3<R> a, R s) { return V3<R>(a.x * s, a.y * s, a.z * s); }
template <typename R> YB_HD V3<R>& operator+=(V3<R>& a, V3<R> b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
template <typename R> YB_HD V3<R>& operator-=(V3<R>& a, V3<R> b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
template <typename R> YB_HD V3<R>& operator*=(V3<R>& a, R s) { a.x *= s; a.y *= s; a.z *= s; return a; }
template <typename R> YB_HD R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> YB_HD R len2(V3<R> a) { return dot(a, a); }
template <typename R> YB_HD V3<R> cross(V3<R> a, V3<R> b) {
    return V3<R>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
// glm-style mix: x * (1 - t) + y * t
template <typename R> YB_HD V3<R> mix(V3<R> a, V3<R> b, R t) { return a * (R(1) - t) + b * t; }

template <typename R> YB_HD R ysqrt(R x);
template <> YB_HD float ysqrt<float>(float x) { return sqrtf(x); }
template <> YB_HD double ysqrt<double>(double x) { return sqrt(x); }
template <typename R> YB_HD R ylog(R x);
template <> YB_HD float ylog<float>(float x) { return logf(x); }
template <> YB_HD double ylog<double>(double x) { return log(x); }
template <typename R> YB_HD R ymin(R a, R b) { return b < a ? b : a; }
template <typename R> YB_HD R ymax(R a, R b) { return a < b ? b : a; }
template <typename R> YB_HD R yclamp(R v, R lo, R hi) { return ymin(ymax(v, lo), hi); }
template <typename R> YB_HD R len(V3<R> a) { return ysqrt(len2(a)); }
template <typename R> YB_HD bool yfinite(R v) { return isfinite(v); }

template <typename R> YB_HD R yinf() { return (R)INFINITY; }

// ---------------------------------------------------------------------------------------
// Separately rounded IEEE operations.  On the device the _rn intrinsics are never fused;
// on the host the translation unit is compiled with -ffp-contract=off.
template <typename R> struct Ex;
template <> struct Ex<float> {
#if defined(__CUDA_ARCH__)
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
#else
    static inline float mul(float a, float b) { return a * b; }
    static inline float add(float a, float b) { return a + b; }
    static inline float sub(float a, float b) { return a - b; }
    static inline float div(float a, float b) { return a / b; }
    static inline float sqrt(float a) { return ::sqrtf(a); }
#endif
};
template <> struct Ex<double> {
#if defined(__CUDA_ARCH__)
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
#else
    static inline double mul(double a, double b) { return a * b; }
    static inline double add(double a, double b) { return a + b; }
    static inline double sub(double a, double b) { return a - b; }
    static inline double div(double a, double b) { return a / b; }
    static inline double sqrt(double a) { return ::sqrt(a); }
#endif
};

template <typename R> YB_HD V3<R> xadd(V3<R> a, V3<R> b) { return V3<R>(Ex<R>::add(a.x, b.x), Ex<R>::add(a.y, b.y), Ex<R>::add(a.z, b.z)); }
template <typename R> YB_HD V3<R> xsub(V3<R> a, V3<R> b) { return V3<R>(Ex<R>::sub(a.x, b.x), Ex<R>::sub(a.y, b.y), Ex<R>::sub(a.z, b.z)); }
template <typename R> YB_HD V3<R> xscale(R s, V3<R> a) { return V3<R>(Ex<R>::mul(s, a.x), Ex<R>::mul(s, a.y), Ex<R>::mul(s, a.z)); }
template <typename R> YB_HD R xdot(V3<R> a, V3<R> b) {
    return Ex<R>::add(Ex<R>::add(Ex<R>::mul(a.x, b.x), Ex<R>::mul(a.y, b.y)), Ex<R>::mul(a.z, b.z));
}
template <typename R> YB_HD R xlen2(V3<R> a) { return xdot(a, a); }
template <typename R> YB_HD V3<R> xmix(V3<R> a, V3<R> b, R t) {
    R omt = Ex<R>::sub(R(1), t);
    return xadd(xscale(omt, a), xscale(t, b));
}

// ---------------------------------------------------------------------------------------
// Closest points between segment A = [0, a1] and segment B = [b0, b1] (A's first endpoint
// is the origin), returned as (u, v) with points mix(0, a1, u) and mix(b0, b1, v).
// Steps (Common.h:318-336): unconstrained v from the 2x2 normal equations, 0.5 when that is
// not finite, clamp, re-project u onto A, clamp, re-project v onto B, clamp.
//
// Near-parallel pairs: the denominator a*c - b*b cancels catastrophically.  When it falls
// below PARALLEL_EPS * a * c, the unconstrained v is recomputed in FP64 from the same
// FP32 inputs (the only FP64 on this path).  Both flavours make the same decision, so the
// host restatement can repeat it exactly.
constexpr float PARALLEL_EPS = 1e-3f;

struct UV { float u, v; };
template <typename R> struct UVT { R u, v; };

template <typename R>
YB_HD UVT<R> closest_uv_exact(V3<R> a1, V3<R> b0, V3<R> b1) {
    typedef Ex<R> E;
    V3<R> A1 = xsub(b1, b0);
    R a = xlen2(a1);
    R b = xdot(a1, A1);
    R c = xlen2(A1);
    R da = xdot(a1, b0);
    R db = xdot(A1, b0);
    R num = E::sub(E::mul(b, da), E::mul(a, db));
    R ac = E::mul(a, c);
    R den = E::sub(ac, E::mul(b, b));
    R v;
    if (sizeof(R) == 4 && den < E::mul(R(PARALLEL_EPS), ac)) {
        typedef Ex<double> D;
        double ax = a1.x, ay = a1.y, az = a1.z;
        double ex = (double)A1.x, ey = (double)A1.y, ez = (double)A1.z;
        double bx = b0.x, by = b0.y, bz = b0.z;
        double aa = D::add(D::add(D::mul(ax, ax), D::mul(ay, ay)), D::mul(az, az));
        double ab = D::add(D::add(D::mul(ax, ex), D::mul(ay, ey)), D::mul(az, ez));
        double cc = D::add(D::add(D::mul(ex, ex), D::mul(ey, ey)), D::mul(ez, ez));
        double dda = D::add(D::add(D::mul(ax, bx), D::mul(ay, by)), D::mul(az, bz));
        double ddb = D::add(D::add(D::mul(ex, bx), D::mul(ey, by)), D::mul(ez, bz));
        double vn = D::sub(D::mul(ab, dda), D::mul(aa, ddb));
        double vd = D::sub(D::mul(aa, cc), D::mul(ab, ab));
        v = (R)D::div(vn, vd);
    } else {
        v = E::div(num, den);
    }
    if (!yfinite(v)) v = R(0.5);
    v = yclamp(v, R(0), R(1));
    R u = yclamp(E::div(xdot(xmix(b0, b1, v), a1), a), R(0), R(1));
    v = yclamp(E::div(xdot(xsub(xscale(u, a1), b0), A1), c), R(0), R(1));
    UVT<R> r; r.u = u; r.v = v;
    return r;
}

// Same computation with FMA contraction allowed (used inside the Newton iteration).
template <typename R>
YB_HD UVT<R> closest_uv(V3<R> a1, V3<R> b0, V3<R> b1) {
    V3<R> A1 = b1 - b0;
    R a = len2(a1);
    R b = dot(a1, A1);
    R c = len2(A1);
    R da = dot(a1, b0);
    R db = dot(A1, b0);
    R ac = a * c;
    R den = ac - b * b;
    R v;
    if (sizeof(R) == 4 && den < R(PARALLEL_EPS) * ac) {
        double ax = a1.x, ay = a1.y, az = a1.z;
        double ex = A1.x, ey = A1.y, ez = A1.z;
        double bx = b0.x, by = b0.y, bz = b0.z;
        double aa = ax * ax + ay * ay + az * az;
        double ab = ax * ex + ay * ey + az * ez;
        double cc = ex * ex + ey * ey + ez * ez;
        double dda = ax * bx + ay * by + az * bz;
        double ddb = ex * bx + ey * by + ez * bz;
        v = (R)((ab * dda - aa * ddb) / (aa * cc - ab * ab));
    } else {
        v = (b * da - a * db) / den;
    }
    if (!yfinite(v)) v = R(0.5);
    v = yclamp(v, R(0), R(1));
    R u = yclamp(dot(mix(b0, b1, v), a1) / a, R(0), R(1));
    v = yclamp(dot(u * a1 - b0, A1) / c, R(0), R(1));
    UVT<R> r; r.u = u; r.v = v;
    return r;
}

// ---------------------------------------------------------------------------------------
// Symmetric 3x3 (diag xx,yy,zz then xy,xz,yz) - the layout of hess3.
template <typename R>
struct H3 {
    R d[6];
    YB_HD void zero() {
#pragma unroll
        for (int i = 0; i < 6; i++) d[i] = R(0);
    }
    YB_HD void diag(R s) { d[0] = s; d[1] = s; d[2] = s; d[3] = R(0); d[4] = R(0); d[5] = R(0); }
    YB_HD void add_diag(R s) { d[0] += s; d[1] += s; d[2] += s; }
    YB_HD void add(const H3& o) {
#pragma unroll
        for (int i = 0; i < 6; i++) d[i] += o.d[i];
    }
    // += s * n n^T
    YB_HD void add_outer(V3<R> n, R s) {
        d[0] += s * (n.x * n.x); d[1] += s * (n.y * n.y); d[2] += s * (n.z * n.z);
        d[3] += s * (n.x * n.y); d[4] += s * (n.x * n.z); d[5] += s * (n.y * n.z);
    }
};

// x = H^{-1} f through the adjugate (H symmetric).
template <typename R>
YB_HD V3<R> solve3(const H3<R>& H, V3<R> f) {
    const R a = H.d[0], b = H.d[1], c = H.d[2], xy = H.d[3], xz = H.d[4], yz = H.d[5];
    const R c00 = b * c - yz * yz;
    const R c01 = xz * yz - xy * c;
    const R c02 = xy * yz - xz * b;
    const R c11 = a * c - xz * xz;
    const R c12 = xy * xz - a * yz;
    const R c22 = a * b - xy * xy;
    const R det = a * c00 + xy * c01 + xz * c02;
    const R inv = R(1) / det;
    return V3<R>((c00 * f.x + c01 * f.y + c02 * f.z) * inv,
                 (c01 * f.x + c11 * f.y + c12 * f.z) * inv,
                 (c02 * f.x + c12 * f.y + c22 * f.z) * inv);
}

// ---------------------------------------------------------------------------------------
// Rotor (quaternion) with (x, y, z) the bivector part and w the scalar.
template <typename R>
struct Q {
    R x, y, z, w;
};
template <typename R> YB_HD Q<R> qmk(V3<R> v, R w) { Q<R> q; q.x = v.x; q.y = v.y; q.z = v.z; q.w = w; return q; }
template <typename R> YB_HD Q<R> qmk(R x, R y, R z, R w) { Q<R> q; q.x = x; q.y = y; q.z = z; q.w = w; return q; }
template <typename R> YB_HD Q<R> qof(const V4<R>& v) { return qmk(v.x, v.y, v.z, v.w); }
template <typename R> YB_HD V4<R> v4of(const Q<R>& q) { V4<R> v; v.x = q.x; v.y = q.y; v.z = q.z; v.w = q.w; return v; }
template <typename R> YB_HD V3<R> qv(const Q<R>& q) { return V3<R>(q.x, q.y, q.z); }
template <typename R> YB_HD Q<R> qinv(const Q<R>& q) { return qmk(-q.x, -q.y, -q.z, q.w); }
template <typename R> YB_HD Q<R> qmul(const Q<R>& l, const Q<R>& r) {
    V3<R> lq = qv(l), rq = qv(r);
    V3<R> v = l.w * rq + r.w * lq + cross(lq, rq);
    return qmk(v, l.w * r.w - dot(lq, rq));
}
template <typename R> YB_HD R qdot(const Q<R>& a, const Q<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <typename R> YB_HD R qlen(const Q<R>& a) { return ysqrt(qdot(a, a)); }
template <typename R> YB_HD Q<R> qscale(R s, const Q<R>& a) { return qmk(s * a.x, s * a.y, s * a.z, s * a.w); }
template <typename R> YB_HD Q<R> qadd(const Q<R>& a, const Q<R>& b) { return qmk(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
template <typename R> YB_HD Q<R> qnormalize(const Q<R>& a) { return qscale(R(1) / qlen(a), a); }
// q * v * q^-1 (Rotor.h:96-105)
template <typename R> YB_HD V3<R> qrotate(const Q<R>& q, V3<R> v) {
    V3<R> qq = qv(q);
    V3<R> a = q.w * v + cross(qq, v);
    R c = dot(v, qq);
    return q.w * a + cross(qq, a) + c * qq;
}

// ---------------------------------------------------------------------------------------
// 10-bit -> 30-bit Morton spread (bit i of v moves to bit 3i).
YB_HD uint32_t morton_spread10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

}  // namespace yb
