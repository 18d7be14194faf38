// ref_device.cu - device-only build of the reference's simulator kernels (test infrastructure).
//
// The recipe (oracle/refbuild/build.py) compiles this file with `nvcc -fatbin` for sm_100a,
// with the reference project (KittenEngine/) and oracle/refbuild/inc on the include path.  It
// includes the reference's own sources unchanged:
//   YarnBall/sim/iteration.cu   initItr, endItr
//   YarnBall/sim/collision.cu   buildAABBs, buildCollisionList, recomputeStepLimitKernel
//   YarnBall/sim/cosserat.cu    cosseratItr, quaternionLambdaItr
//   YarnBall/YarnBall.cu        copyTempData (the upload's per-vertex copy)
// and, through them, KittenEngine/includes/modules/{Common,Rotor,SymMat,Bound}.h.  Only device
// code is generated: the reference's host code needs MSVC (members with constructors inside
// anonymous structs, SymMat.h:9-14 and Rotor.h:13-19, which GCC rejects), so the host side of
// the schedule is restated in ref_host.cpp and the kernels are launched from there.
//
// Added here, in this repository's code: kernels that evaluate the reference's math helpers on
// arrays (for bit-for-bit comparison with the oracle's restatement), a brute-force
// overlapping-box pair query that stands in for the reference's absent LBVH, and the layout
// of the reference's types for the host harness to check.
#include <cstddef>

#include "YarnBall/YarnBall.h"
#include "YarnBall/sim/iteration.cu"
#include "YarnBall/sim/collision.cu"
#include "YarnBall/sim/cosserat.cu"
#include "YarnBall/YarnBall.cu"

namespace YarnBall {
// The kernel instances the reference's host code launches (collision.cu:96-117, 161-171).
template __global__ void buildAABBs<true>(MetaData*, int*);
template __global__ void buildAABBs<false>(MetaData*, int*);
template __global__ void buildCollisionList<true>(MetaData*, int, int*);
template __global__ void buildCollisionList<false>(MetaData*, int, int*);
template __global__ void recomputeStepLimitKernel<true, true>(MetaData*);
template __global__ void recomputeStepLimitKernel<true, false>(MetaData*);
template __global__ void recomputeStepLimitKernel<false, true>(MetaData*);
template __global__ void recomputeStepLimitKernel<false, false>(MetaData*);
}  // namespace YarnBall

// Layout of the reference's types as this compilation sees them.
extern "C" __device__ unsigned long long refk_layout[10] = {
    sizeof(YarnBall::MetaData),
    offsetof(YarnBall::MetaData, gravity),
    sizeof(YarnBall::Vertex),
    sizeof(Kitten::LBVH::aabb),
    sizeof(Kitten::Rotor),
    sizeof(glm::vec3),
    sizeof(glm::ivec2),
    offsetof(YarnBall::MetaData, d_boundColList),
    offsetof(YarnBall::MetaData, useVelocityRadius),
    (unsigned long long)YarnBall::MAX_COLLISIONS_PER_SEGMENT,
};

namespace {
__device__ inline glm::vec3 ld3(const float* p) { return glm::vec3(p[0], p[1], p[2]); }
__device__ inline Kitten::Rotor ld4(const float* p) { return Kitten::Rotor(p[0], p[1], p[2], p[3]); }
__device__ inline void st3(float* p, const glm::vec3& v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
__device__ inline void st4(float* p, const Kitten::Rotor& r) { p[0] = r.x; p[1] = r.y; p[2] = r.z; p[3] = r.w; }
}  // namespace

// Kitten::segmentClosestPoints (Common.h:318-336); in: n x {a0, a1, b0, b1}, out: n x uv.
extern "C" __global__ void refk_closest(const float* in, float* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 12 * (size_t)i;
    const glm::vec2 uv = Kitten::segmentClosestPoints(ld3(p), ld3(p + 3), ld3(p + 6), ld3(p + 9));
    out[2 * i] = uv.x;
    out[2 * i + 1] = uv.y;
}

// Rotor product (Rotor.h:185-188), rotation (:96-105), fromTo (:57-64); 4 floats per rotor.
extern "C" __global__ void refk_rotor_mul(const float* l, const float* r, float* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st4(out + 4 * (size_t)i, ld4(l + 4 * (size_t)i) * ld4(r + 4 * (size_t)i));
}
extern "C" __global__ void refk_rotor_rotate(const float* q, const float* v, float* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st3(out + 3 * (size_t)i, ld4(q + 4 * (size_t)i).rotate(ld3(v + 3 * (size_t)i)));
}
extern "C" __global__ void refk_rotor_from_to(const float* from, const float* to, float* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st4(out + 4 * (size_t)i, Kitten::Rotor::fromTo(ld3(from + 3 * (size_t)i), ld3(to + 3 * (size_t)i)));
}
// glm::normalize of a vec4 (cosserat.cu:249, YarnBall.cu:143).
extern "C" __global__ void refk_normalize4(const float* v, float* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = v + 4 * (size_t)i;
    const glm::vec4 r = glm::normalize(glm::vec4(p[0], p[1], p[2], p[3]));
    out[4 * i] = r.x; out[4 * i + 1] = r.y; out[4 * i + 2] = r.z; out[4 * i + 3] = r.w;
}
// hess3 (SymMat.h:8-107): H += outer(nrm) * s, then the local solve inverse((mat3)H) * f of
// cosserat.cu:197.  h: n x {xx, yy, zz, xy, xz, yz}; hOut receives the updated H.
extern "C" __global__ void refk_hess3(const float* h, const float* nrm, const float* s, const float* f, float* hOut,
                                      float* solve, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Kitten::hess3 H;
    for (int k = 0; k < 6; k++) H[k] = h[6 * (size_t)i + k];
    H += Kitten::hess3::outer(ld3(nrm + 3 * (size_t)i)) * s[i];
    for (int k = 0; k < 6; k++) hOut[6 * (size_t)i + k] = H[k];
    st3(solve + 3 * (size_t)i, glm::inverse((glm::mat3)H) * ld3(f + 3 * (size_t)i));
}

// Stand-in for the absent LBVH query (collision.cu:111): every pair i < j of boxes that
// overlap (closed intervals on all axes) is appended as (i, j) while fewer than cap pairs have
// been written; *count receives the number of overlapping pairs found (which exceeds cap when
// the output was truncated).  Empty boxes (min > max, Bound.h:11-14) overlap nothing.  One
// thread per box i scans the boxes j > i from shared-memory tiles.
extern "C" __global__ void refk_pairs(const Kitten::LBVH::aabb* boxes, int n, int* out, unsigned long long cap,
                                      unsigned long long* count) {
    constexpr int TILE = 256;
    __shared__ float smn[3][TILE], smx[3][TILE];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    glm::vec3 amn(0.f), amx(-1.f);
    if (i < n) {
        amn = boxes[i].min;
        amx = boxes[i].max;
    }
    const bool live = i < n && amn.x <= amx.x && amn.y <= amx.y && amn.z <= amx.z;
    for (int base = blockIdx.x * blockDim.x; base < n; base += TILE) {
        __syncthreads();
        const int j = base + threadIdx.x;
        if (j < n) {
            const glm::vec3 mn = boxes[j].min, mx = boxes[j].max;
            smn[0][threadIdx.x] = mn.x; smn[1][threadIdx.x] = mn.y; smn[2][threadIdx.x] = mn.z;
            smx[0][threadIdx.x] = mx.x; smx[1][threadIdx.x] = mx.y; smx[2][threadIdx.x] = mx.z;
        }
        __syncthreads();
        if (!live) continue;
        const int lim = min(TILE, n - base);
        for (int t = 0; t < lim; t++) {
            const int jj = base + t;
            if (jj <= i) continue;
            if (smn[0][t] <= amx.x && amn.x <= smx[0][t] && smn[1][t] <= amx.y && amn.y <= smx[1][t] &&
                smn[2][t] <= amx.z && amn.z <= smx[2][t] && smn[0][t] <= smx[0][t] && smn[1][t] <= smx[1][t] &&
                smn[2][t] <= smx[2][t]) {
                const unsigned long long slot = atomicAdd(count, 1ull);
                if (slot < cap) {
                    out[2 * slot] = i;
                    out[2 * slot + 1] = jj;
                }
            }
        }
    }
}
