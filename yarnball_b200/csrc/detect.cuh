// detect.cuh - separately rounded detection predicates shared by the BVH and step kernels.
//
//   segment AABB        collision.cu:10-37   (buildAABBs, velocity radius included)
//   narrow-phase keep   collision.cu:39-92   (buildCollisionList: glue/neighbour exemptions,
//                                             closest points, d^2 < r^2)
//   step-size limit     collision.cu:121-159 (recomputeStepLimitKernel)
//
// The pair test is always evaluated with the lower segment index as segment A, so both
// segments of a pair reach the same decision and every contact list is symmetric.
#pragma once
#include "engine.cuh"

namespace yb {

template <typename R>
struct Box {
    R mn[3], mx[3];
};

// Padded AABB of segment k (k has hasNext).
template <typename R>
__device__ __forceinline__ Box<R> segment_box(const Dev<R>& d, int k, const SceneParams<R>& sp) {
    typedef Ex<R> E;
    const V4<R> p0 = d.pos[k];
    const V4<R> p1 = d.pos[k + 1];
    R pad = sp.sdr;
    if (sp.useVelRadius) {
        const D2<R> dk = d.dx[0][k];
        const R l0 = xlen2(xyz(dk.a));
        const R l1 = xlen2(xyz(dk.b));
        pad = E::add(pad, E::sqrt(ymax(l0, l1)));
    }
    Box<R> b;
    b.mn[0] = E::sub(ymin(p0.x, p1.x), pad);
    b.mn[1] = E::sub(ymin(p0.y, p1.y), pad);
    b.mn[2] = E::sub(ymin(p0.z, p1.z), pad);
    b.mx[0] = E::add(ymax(p0.x, p1.x), pad);
    b.mx[1] = E::add(ymax(p0.y, p1.y), pad);
    b.mx[2] = E::add(ymax(p0.z, p1.z), pad);
    return b;
}

// Closed-interval overlap of a query box with a stored box.
template <typename R>
__device__ __forceinline__ bool box_overlap(const Box<R>& q, const R* mn, const R* mx) {
    return q.mn[0] <= mx[0] && mn[0] <= q.mx[0] && q.mn[1] <= mx[1] && mn[1] <= q.mx[1] && q.mn[2] <= mx[2] &&
           mn[2] <= q.mx[2];
}

// Narrow-phase decision for segments x < y (both with hasNext, same scene).
template <typename R>
__device__ __forceinline__ bool pair_keep(const Dev<R>& d, int x, int y, const SceneParams<R>& sp) {
    typedef Ex<R> E;
    const int c0 = d.vp[x].cid;
    const int c1 = d.vp[x + 1].cid;
    if (c0 == y || c1 == y || c0 == y + 1 || c1 == y + 1) return false;
    if (y - x <= 2) return false;
    const V3<R> a0 = xyz(d.pos[x]);
    const V3<R> a1 = xsub(xyz(d.pos[x + 1]), a0);
    const V3<R> b0 = xsub(xyz(d.pos[y]), a0);
    const V3<R> b1 = xsub(xyz(d.pos[y + 1]), a0);
    const UVT<R> uv = closest_uv_exact(a1, b0, b1);
    const V3<R> nrm = xsub(xscale(uv.u, a1), xmix(b0, b1, uv.v));
    const R d2 = xlen2(nrm);
    R r = E::mul(R(2), sp.sdr);
    if (sp.useVelRadius) {
        const D2<R> dxx = d.dx[0][x], dxy = d.dx[0][y];
        r = E::add(r, E::sqrt(ymax(xlen2(xyz(dxx.a)), xlen2(xyz(dxx.b)))));
        r = E::add(r, E::sqrt(ymax(xlen2(xyz(dxy.a)), xlen2(xyz(dxy.b)))));
    }
    return d2 < E::mul(r, r);
}

// Step-size limit (collision.cu:121-159), split so that contacts can be spread over threads:
// step_limit_base is the per-segment start value, contact_step_limit one contact's bound
// 0.45 x centre-line distance.  A contact also stages the partner's endpoints relative to p0
// in slot `stage` of relA/relB (read by every Newton iteration of the substep; NO_STAGE: not
// staged), reports an interpenetration (distance at or below 2 radius, each unordered pair
// once, o > k) and returns the centre-line distance in dist.
constexpr size_t NO_STAGE = ~(size_t)0;

template <typename R>
__device__ __forceinline__ R step_limit_base(const Dev<R>& d, int k, const SceneParams<R>& sp) {
    typedef Ex<R> E;
    R m = sp.stepBase;
    if (sp.useVelRadius) m = E::add(m, E::sqrt(xlen2(xyz(d.dx[0][k].a))));
    return m;
}

template <typename R>
__device__ __forceinline__ R contact_step_limit(const Dev<R>& d, int k, size_t stage, int o, const V3<R>& a0,
                                                const V3<R>& a1, const SceneParams<R>& sp, bool& pen, R& dist) {
    typedef Ex<R> E;
    const V3<R> b0 = xsub(xyz(d.pos[o]), a0);
    const V3<R> b1 = xsub(xyz(d.pos[o + 1]), a0);
    if (stage != NO_STAGE) {
        d.relA[stage] = v4(b0, b1.x);
        R2<R> rb;
        rb.x = b1.y;
        rb.y = b1.z;
        d.relB[stage] = rb;
    }
    const UVT<R> uv = closest_uv_exact(a1, b0, b1);
    const V3<R> nrm = xsub(xscale(uv.u, a1), xmix(b0, b1, uv.v));
    const R l = E::sqrt(xlen2(nrm));
    pen = o > k && l <= sp.twoR;
    dist = l;
    const R safe = E::mul(E::sub(R(1), R(0.1f)), R(0.5f));
    return E::mul(safe, l);
}

}  // namespace yb
