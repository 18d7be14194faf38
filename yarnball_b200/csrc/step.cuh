// step.cuh - device functions of the substep shared by the iteration kernels (k_step.cu) and
// the one-block small-scene kernel (k_small.cu), so that both evaluate every expression alike.
//
//   predict               initItr, KittenEngine/YarnBall/sim/iteration.cu:7-41
//   barrier_terms,
//   contact_term          cosseratItr's contact loop, sim/cosserat.cu:92-148
//   add_own_terms         cosseratItr's inertia, glue and stretch terms, sim/cosserat.cu:40-81
//   orientation_update    quaternionLambdaItr, sim/cosserat.cu:209-253
#pragma once
#include "detect.cuh"

namespace yb {

template <typename R>
__device__ __forceinline__ const SceneParams<R>& scene_params(const Dev<R>& d, uint32_t flags) {
    return d.sp[scene_of(flags)];
}

// ---------------------------------------------------------------------------------------
// Predictor (iteration.cu:7-41).  Every operation separately rounded: dx0 feeds the
// bit-exact collision filter through the velocity radius.  Reads only; the reference's
// `lastVels = vel` store happens in k_end instead, so that thread i can also predict vertex
// i+1 for the iterate pair without racing with thread i+1.
template <typename R>
__device__ __forceinline__ V3<R> predict(const Dev<R>& d, int i) {
    typedef Ex<R> E;
    const SceneParams<R>& sp = d.sp[scene_of(d.vp[i].flags)];
    const V4<R> vel4 = d.vel[i];
    const V4<R> lv4 = d.lastVel[i];
    const R h = sp.h;
    const V3<R> v = xyz(vel4);
    V3<R> dx = xscale(h, v);
    if (d.pos[i].w != R(0)) {
        const R g2 = sp.g2;
        if (g2 > R(0)) {
            const V3<R> g(sp.gx, sp.gy, sp.gz);
            const V3<R> a(E::div(E::sub(v.x, lv4.x), sp.lastH), E::div(E::sub(v.y, lv4.y), sp.lastH),
                          E::div(E::sub(v.z, lv4.z), sp.lastH));
            const R s = yclamp(E::div(xdot(a, g), g2), R(0), R(1));
            dx = xadd(dx, xscale(E::mul(E::mul(h, h), s), g));
        }
    }
    return dx;
}

// ---------------------------------------------------------------------------------------
// IPC log barrier E(d) = -kCollision (d-1)^2 ln d on the normalised gap d, clamped to 1e-3:
// returns dH = E''(d) / b^2 and the force magnitude ff (cosserat.cu:114-125).  Below d=1e-2
// the log and the reciprocals are evaluated in FP64.

template <typename R>
__device__ __forceinline__ void barrier_terms(R d, R kCol, R invb, R& dH, R& ff) {
    if (sizeof(R) == 4 && d < R(1e-2)) {
        const double dd = d;
        const double invd = 1.0 / dd;
        const double logd = log(dd);
        dH = (R)((-3.0 + (2.0 + invd) * invd - 2.0 * logd) * (double)kCol * (double)invb);
        ff = (R)(-(1.0 - dd) * (dd - 1.0 + 2.0 * dd * logd) * invd * (double)kCol);
    } else {
        const R invd = R(1) / d;
        const R logd = ylog(d);
        dH = (R(-3) + (R(2) + invd) * invd - R(2) * logd) * kCol * invb;
        ff = -(R(1) - d) * (d - R(1) + R(2) * d * logd) * invd * kCol;
    }
}

// Contact of segment (p0,p1) with segment (b0,b1) on the current iterate (cosserat.cu:92-148),
// in coordinates relative to p0: e = p1 - p0, r0 = b0 - p0, r1 = b1 - p0 (the closest points
// and the gap only depend on differences).  Accumulates into the forces/Hessians of the
// segment's two endpoints.
template <typename R>
__device__ __forceinline__ void contact_term(V3<R> e, V3<R> dx0, V3<R> dx1, V3<R> r0, V3<R> r1, V3<R> db0, V3<R> db1,
                                             const SceneParams<R>& sp, V3<R>& fa, H3<R>& Ha, V3<R>& fb, H3<R>& Hb) {
    const UVT<R> uv = closest_uv(e + (dx1 - dx0), r0 + (db0 - dx0), r1 + (db1 - dx0));
    const V3<R> dpos = uv.u * e - mix(r0, r1, uv.v);
    const V3<R> ddpos = mix(dx0, dx1, uv.u) - mix(db0, db1, uv.v);
    V3<R> nrm = dpos + ddpos;
    const R dist = len(nrm);
    nrm *= R(1) / dist;
    const R wb = uv.u;
    const R wa = R(1) - uv.u;
    R gap = (dist - sp.twoR) * sp.invb;
    if (gap > R(1)) return;
    gap = ymax(gap, R(1e-3f));
    R dH, ff;
    barrier_terms(gap, sp.kCol, sp.invb, dH, ff);
    const R D = sp.D;
    fa += (ff * wa - D * dH * wa * wa * dot(nrm, dx0)) * nrm;
    fb += (ff * wb - D * dH * wb * wb * dot(nrm, dx1)) * nrm;
    dH *= R(1) + D;
    Ha.add_outer(nrm, dH * wa * wa);
    Hb.add_outer(nrm, dH * wb * wb);
    // Friction on the current iterate: tangential relative displacement.
    const V3<R> u = ddpos - dot(nrm, ddpos) * nrm;
    const R ul = len(u);
    if (ul > R(0)) {
        const R f1 = ymin(sp.fricK, sp.fricMu * ff / ul);
        fa -= (f1 * wa) * u;
        fb -= (f1 * wb) * u;
        const R sa = wa * wa * f1, sb = wb * wb * f1;
        Ha.add_diag(sa); Ha.add_outer(nrm, -sa);
        Hb.add_diag(sb); Hb.add_outer(nrm, -sb);
    }
}

// Packed contacts of segment k (written by the list pass of this substep): first slot in off,
// count returned.  A range the packed arrays cannot hold (the list pass reports it) reads as
// empty.
template <typename R>
__device__ __forceinline__ int contact_range(const Dev<R>& d, int k, unsigned& off) {
    off = d.csrOff[k];
    const unsigned end = d.csrOff[k + 1];
    if (end < off || end - off > (unsigned)MAX_COLS || end > d.csrCap) return 0;
    return (int)(end - off);
}

// Whether j can be a contact partner (a segment start: j and j + 1 are vertices).
template <typename R>
__device__ __forceinline__ bool partner_ok(const Dev<R>& d, int j) {
    return (unsigned)j < (unsigned)(d.n - 1);
}

// Endpoints of partner segment j relative to p0: staged by the list pass in packed slot g, or
// gathered when g is past the staging capacity (the same differences either way).
template <typename R>
__device__ __forceinline__ void partner_rel(const Dev<R>& d, unsigned g, int j, const V3<R>& p0, V3<R>& r0, V3<R>& r1) {
    if (g < d.relCap) {
        const V4<R> A = d.relA[g];
        const R2<R> Bq = d.relB[g];
        r0 = V3<R>(A.x, A.y, A.z);
        r1 = V3<R>(A.w, Bq.x, Bq.y);
    } else {
        r0 = xyz(d.pos[j]) - p0;
        r1 = xyz(d.pos[j + 1]) - p0;
    }
}

// Predicted iterate pair of vertex i (dx[i], dx[i+1]) into dx[0] (the k_init pass).
template <typename R>
__device__ __forceinline__ void init_vertex(const Dev<R>& d, int i) {
    D2<R> o;
    o.a = v4(predict(d, i), R(0));
    o.b = v4(i + 1 < d.n ? predict(d, i + 1) : V3<R>(R(0)), R(0));
    d.dx[0][i] = o;
}

// Advection of vertex i from the final iterate in dx[fb] (endItr, iteration.cu:48-61), with
// Kahan-compensated positions when kahan is set; stores the substep's starting velocity as
// lastVel (iteration.cu:19-20) and copies the final rotor into q[0] when it is in q[1].
template <typename R>
__device__ __forceinline__ void end_vertex(const Dev<R>& d, int i, int fb, int copyQ, int kahan) {
    typedef Ex<R> E;
    const uint32_t flags = d.vp[i].flags;
    const SceneParams<R>& sp = scene_params(d, flags);
    const V4<R> dx = d.dx[fb][i].a;
    V4<R> p = d.pos[i];
    d.lastVel[i] = d.vel[i];
    if (p.w != R(0)) {
        V4<R> v;
        v.x = dx.x * sp.invH * sp.dragFactor;
        v.y = dx.y * sp.invH * sp.dragFactor;
        v.z = dx.z * sp.invH * sp.dragFactor;
        v.w = R(0);
        d.vel[i] = v;
    }
    if (kahan) {
        V4<R> c = d.posC[i];
        R yx = E::sub(dx.x, c.x), yy = E::sub(dx.y, c.y), yz = E::sub(dx.z, c.z);
        R tx = E::add(p.x, yx), ty = E::add(p.y, yy), tz = E::add(p.z, yz);
        c.x = E::sub(E::sub(tx, p.x), yx);
        c.y = E::sub(E::sub(ty, p.y), yy);
        c.z = E::sub(E::sub(tz, p.z), yz);
        p.x = tx; p.y = ty; p.z = tz;
        d.posC[i] = c;
    } else {
        p.x += dx.x; p.y += dx.y; p.z += dx.z;
    }
    d.pos[i] = p;
    if (copyQ) d.q[0][i] = d.q[1][i];
}

// ---------------------------------------------------------------------------------------
// The vertex's own terms (cosserat.cu:40-81) added to force and Hessian sums that already hold
// its contacts: inertia (H = m/h^2, f = m/h^2 (y - dx), y = h v + h^2 g formed here), the glue
// spring to a connected vertex, and the stretch-shear coupling of segment k to its orientation
// (its other endpoint's share in fb, Hb).  Also returns the vertex's flags, mass, segment
// constants, step limit and orientation.
template <typename R>
__device__ __forceinline__ void add_own_terms(const Dev<R>& d, int k, const D2<R>* __restrict__ DX,
                                              const V4<R>* __restrict__ QO, const SceneParams<R>& sp, const V3<R>& p0,
                                              const V3<R>& e, const V3<R>& dx, const V3<R>& dx1, V3<R>& fa, H3<R>& Ha,
                                              V3<R>& fb, H3<R>& Hb, uint32_t& flags, R& invMass, R& lRest, R& kStretch,
                                              R& sl, Q<R>& q0) {
    const VP<R> vp = d.vp[k];
    flags = vp.flags;
    lRest = vp.lRest;
    kStretch = vp.kStretch;
    invMass = d.pos[k].w;
    q0 = qof(QO[k]);
    const R D = sp.D;
    if (invMass != R(0)) {
        const V4<R> v = d.vel[k];
        const R hh = sp.hh;
        const V3<R> y(sp.h * v.x + hh * sp.gx, sp.h * v.y + hh * sp.gy, sp.h * v.z + hh * sp.gz);
        Ha.add_diag(R(1) / (invMass * hh));
        fa += (R(1) / (hh * invMass)) * (y - dx);
    }
    if (vp.cid >= 0) {
        const R stiff = R(40);
        const V3<R> pc = xyz(d.pos[vp.cid]);
        const V3<R> dc = xyz(DX[vp.cid].a);
        fa -= stiff * ((p0 - pc) + (dx - dc) + D * dx);
        Ha.add_diag(stiff * (R(1) + D));
    }
    if (flags & F_HAS_NEXT) {
        sl = d.stepLim[k];
        const R invl = R(1) / lRest;
        const V3<R> c = (e + (dx1 - dx)) * invl - qrotate(q0, V3<R>(R(1), R(0), R(0)));
        const R ks = kStretch * invl;
        R dd = ks * invl;
        fa += ks * c - (D * dd) * dx;
        fb += -ks * c - (D * dd) * dx1;
        dd *= R(1) + D;
        Ha.add_diag(dd);
        Hb.add_diag(dd);
    }
}

// Closed-form orientation update of segment k (quaternionLambdaItr, cosserat.cu:209-253) from
// the new iterates of its endpoints (dxn, dxb) and the previous iteration's rotors.  A
// single-segment yarn has no bending neighbours (b = 0): the closed form is 0/0 there (the
// reference produces NaN); its orientation is kept.
template <typename R>
__device__ __forceinline__ Q<R> orientation_update(const Dev<R>& d, int k, const V4<R>* __restrict__ QO,
                                                   uint32_t flags, const V3<R>& e, const V3<R>& dxn, const V3<R>& dxb,
                                                   R lRest, R kStretch, const Q<R>& q0) {
    Q<R> qn = q0;
    if (!(flags & F_FIX_ORI) && (flags & F_HAS_NEXT)) {
        V3<R> v = (e + (dxb - dxn)) * (R(1) / lRest);
        v *= R(-2) * kStretch;
        Q<R> b = qmk(R(0), R(0), R(0), R(0));
        if (flags & F_HAS_PREV) {
            const Q<R> qr = qof(d.qRest[k - 1]);
            const Q<R> qq = qof(QO[k - 1]);
            const R s = qdot(qmul(qinv(qq), q0), qr) > R(0) ? R(1) : R(-1);
            b = qadd(b, qscale(s, qmul(qq, qr)));
        }
        if (flags & F_HAS_NEXT_ORI) {
            const Q<R> qr = qof(d.qRest[k]);
            const Q<R> qq = qof(QO[k + 1]);
            const R s = qdot(qmul(qinv(q0), qq), qr) > R(0) ? R(1) : R(-1);
            b = qadd(b, qscale(s, qmul(qq, qinv(qr))));
        }
        const R bl = qlen(b);
        if (bl > R(0)) {
            const R lambda = len(v) + bl;
            const Q<R> vb1 = qmul(qmul(qmk(v, R(0)), b), qmk(R(1), R(0), R(0), R(0)));
            qn = qnormalize(qadd(vb1, qscale(lambda, b)));
        }
    }
    return qn;
}

}  // namespace yb
