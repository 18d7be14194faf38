// k_step.cu - predictor, fused block-Jacobi Newton + orientation iteration, advection.
//
// Reference semantics (file:line in the reference project):
//   initItr               KittenEngine/YarnBall/sim/iteration.cu:7-41
//   cosseratItr           KittenEngine/YarnBall/sim/cosserat.cu:20-207
//   quaternionLambdaItr   KittenEngine/YarnBall/sim/cosserat.cu:209-253
//   endItr                KittenEngine/YarnBall/sim/iteration.cu:48-61
//
// Deliberate differences from the reference, all in the direction of determinism:
//   * strict Jacobi: iteration k reads only iteration k-1's dx and q (double buffers); the
//     reference updates both in place while neighbouring threads read them.
//   * one kernel per iteration does the position solve and the orientation update: a block
//     owns B-2 vertices and recomputes one halo segment on each side, so the orientation of
//     segment i sees the new dx of vertices i and i+1 without a second launch.
//   * contact lists are sorted by partner id, so force sums have a fixed order.
#include "step.cuh"

namespace yb {

template <typename R>
__global__ void __launch_bounds__(256) k_init(Dev<R> d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    init_vertex(d, i);
}

// ---------------------------------------------------------------------------------------
// Advection (iteration.cu:48-61) with Kahan-compensated position accumulation (FP32 build);
// also stores the start-of-substep velocity as lastVel (iteration.cu:19-20).
template <typename R>
__global__ void __launch_bounds__(256) k_end(Dev<R> d, int fb, int copyQ, int kahan) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    end_vertex(d, i, fb, copyQ, kahan);
}

// ---------------------------------------------------------------------------------------
// One block-Jacobi iteration: position solve (cosseratItr) then orientation update
// (quaternionLambdaItr), strict Jacobi.  A block has B vertex slots of T lanes each
// (NT = B*T threads): slot t handles vertex/segment k = b*(B-2)-1+t, writes it when
// t in [1, B-2] and only recomputes the halo slots t=0 and t=B-1.  The T lanes of a slot
// split the segment's contact loop (contacts s, s+T, ...) and combine their partial sums
// with an xor-shuffle butterfly, so every lane of the slot holds the identical total; the
// vertex solve and the orientation update are then evaluated by all T lanes and stored by
// lane 0.
template <typename R, int T>
__device__ __forceinline__ R slot_sum(R v) {
#pragma unroll
    for (int o = 1; o < T; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R, int NT, int T, int MINB, bool PIPE>
__global__ void __launch_bounds__(NT, MINB) k_iter(Dev<R> d, int src) {
    constexpr int B = NT / T;
    constexpr int CORE = B - 2;
    const int t = threadIdx.x / T;
    const int lane = threadIdx.x % T;
    const int k = blockIdx.x * CORE - 1 + t;
    const int n = d.n;
    const bool valid = (k >= 0) && (k < n);
    const D2<R>* __restrict__ DX = d.dx[src];
    const V4<R>* __restrict__ QO = d.q[src];

    __shared__ R sFb[3][B];
    __shared__ R sHb[6][B];
    __shared__ R sSL[B];
    __shared__ R sDX[3][B];

    V3<R> fa(R(0)), fb(R(0));
    H3<R> Ha, Hb;
    Ha.zero(); Hb.zero();
    R sl = yinf<R>();
    uint32_t flags = 0;
    R invMass = R(0), lRest = R(1), kStretch = R(0);
    V3<R> p0(R(0)), p1(R(0)), dx(R(0)), dx1(R(0));
    Q<R> q0 = qmk(R(0), R(0), R(0), R(1));
    const SceneParams<R>* spp = d.sp;

    if (valid) {
        const VP<R> vp = d.vp[k];
        flags = vp.flags;
        lRest = vp.lRest;
        kStretch = vp.kStretch;
        spp = &d.sp[scene_of(flags)];
        const SceneParams<R>& sp = *spp;
        const V4<R> P = d.pos[k];
        p0 = xyz(P);
        invMass = P.w;
        const D2<R> own = DX[k];
        dx = xyz(own.a);
        dx1 = xyz(own.b);
        q0 = qof(QO[k]);
        const R D = sp.D;
        if (lane == 0) {
            if (invMass != R(0)) {
                // Inertia: H = m/h^2, f = m/h^2 (y - dx), y = h v + h^2 g (iteration.cu:26, cosserat.cu:40-45)
                const V4<R> v = d.vel[k];
                const R hh = sp.hh;
                const V3<R> y(sp.h * v.x + hh * sp.gx, sp.h * v.y + hh * sp.gy, sp.h * v.z + hh * sp.gz);
                Ha.diag(R(1) / (invMass * hh));
                fa = (R(1) / (hh * invMass)) * (y - dx);
            }
            if (vp.cid >= 0) {
                // Glue spring to the connected vertex (cosserat.cu:46-53)
                const R stiff = R(40);
                const V3<R> pc = xyz(d.pos[vp.cid]);
                const V3<R> dc = xyz(DX[vp.cid].a);
                fa -= stiff * ((p0 - pc) + (dx - dc) + D * dx);
                Ha.add_diag(stiff * (R(1) + D));
            }
        }
        if (flags & F_HAS_NEXT) {
            p1 = xyz(d.pos[k + 1]);
            sl = d.stepLim[k];
            if (lane == 0) {
                // Stretch-shear coupling to the segment orientation (cosserat.cu:63-81)
                const R invl = R(1) / lRest;
                const V3<R> c = ((p1 - p0) + (dx1 - dx)) * invl - qrotate(q0, V3<R>(R(1), R(0), R(0)));
                const R ks = kStretch * invl;
                R dd = ks * invl;
                fa += ks * c - (D * dd) * dx;
                fb += -ks * c - (D * dd) * dx1;
                dd *= R(1) + D;
                Ha.add_diag(dd);
                Hb.add_diag(dd);
            }
            // Barrier + friction over this lane's share of the contact list (packed slots).
            // Partner positions relative to p0 are staged per substep in the slots below
            // relCap; the partner's iterate pair is one 32-byte gather.
            // With PIPE the loads of the lane's next contact are issued before the current
            // contact's arithmetic, so the dependent partner gather overlaps it (more
            // registers); without it each contact loads then computes.
            unsigned off;
            const int nc = contact_range(d, k, off);
            const int* __restrict__ cl = d.csrCols + off;
            const V3<R> e = p1 - p0;
            if constexpr (!PIPE) {
                for (int c2 = lane; c2 < nc; c2 += T) {
                    const int j = __ldg(cl + c2);
                    if (!partner_ok(d, j)) continue;
                    V3<R> r0, r1;
                    partner_rel(d, off + c2, j, p0, r0, r1);
                    const D2<R> pd = DX[j];
                    contact_term(e, dx, dx1, r0, r1, xyz(pd.a), xyz(pd.b), sp, fa, Ha, fb, Hb);
                }
            } else {
            int c2 = lane;
            V3<R> r0n(R(0)), r1n(R(0));
            D2<R> pdn;
            bool okn = false;
            if (c2 < nc) {
                const int j = __ldg(cl + c2);
                okn = partner_ok(d, j);
                if (okn) {
                    partner_rel(d, off + c2, j, p0, r0n, r1n);
                    pdn = DX[j];
                }
            }
            while (c2 < nc) {
                const V3<R> r0 = r0n, r1 = r1n;
                const D2<R> pd = pdn;
                const bool ok = okn;
                c2 += T;
                if (c2 < nc) {
                    const int j = __ldg(cl + c2);
                    okn = partner_ok(d, j);
                    if (okn) {
                        partner_rel(d, off + c2, j, p0, r0n, r1n);
                        pdn = DX[j];
                    }
                }
                if (ok) contact_term(e, dx, dx1, r0, r1, xyz(pd.a), xyz(pd.b), sp, fa, Ha, fb, Hb);
            }
            }
        }
    }
    if (T > 1) {
        fa.x = slot_sum<R, T>(fa.x); fa.y = slot_sum<R, T>(fa.y); fa.z = slot_sum<R, T>(fa.z);
        fb.x = slot_sum<R, T>(fb.x); fb.y = slot_sum<R, T>(fb.y); fb.z = slot_sum<R, T>(fb.z);
#pragma unroll
        for (int e = 0; e < 6; e++) {
            Ha.d[e] = slot_sum<R, T>(Ha.d[e]);
            Hb.d[e] = slot_sum<R, T>(Hb.d[e]);
        }
    }
    if (lane == 0) {
        sFb[0][t] = fb.x; sFb[1][t] = fb.y; sFb[2][t] = fb.z;
#pragma unroll
        for (int e = 0; e < 6; e++) sHb[e][t] = Hb.d[e];
        sSL[t] = sl;
    }
    __syncthreads();

    // Vertex solve: own segment + previous segment's endpoint share (cosserat.cu:175-205)
    V3<R> dxn = dx;
    if (valid && t > 0) {
        if (flags & F_HAS_PREV) {
            fa += V3<R>(sFb[0][t - 1], sFb[1][t - 1], sFb[2][t - 1]);
            H3<R> hp;
#pragma unroll
            for (int e = 0; e < 6; e++) hp.d[e] = sHb[e][t - 1];
            Ha.add(hp);
            sl = ymin(sl, sSL[t - 1]);
        }
        if (invMass != R(0)) {
            dxn = dx + spp->accel * solve3(Ha, fa);
            const R l = len(dxn);
            if (l > sl && l > R(0)) dxn *= sl / l;
        }
    }
    if (lane == 0) { sDX[0][t] = dxn.x; sDX[1][t] = dxn.y; sDX[2][t] = dxn.z; }
    const bool core = valid && t >= 1 && t <= CORE;
    __syncthreads();

    // New iterate pair and orientation update of segment k (cosserat.cu:209-253)
    if (core && lane == 0) {
        const V3<R> dxb(sDX[0][t + 1], sDX[1][t + 1], sDX[2][t + 1]);
        D2<R> o;
        o.a = v4(dxn, R(0));
        o.b = v4(k + 1 < n ? dxb : V3<R>(R(0)), R(0));
        d.dx[src ^ 1][k] = o;
        Q<R> qn = q0;
        if (!(flags & F_FIX_ORI) && (flags & F_HAS_NEXT)) {
            V3<R> v = ((p1 - p0) + (dxb - dxn)) * (R(1) / lRest);
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
            // A single-segment yarn has no bending neighbours (b = 0): the closed form is
            // 0/0 there (the reference produces NaN); keep the orientation instead.
            const R bl = qlen(b);
            if (bl > R(0)) {
                const R lambda = len(v) + bl;
                const Q<R> vb1 = qmul(qmul(qmk(v, R(0)), b), qmk(R(1), R(0), R(0), R(0)));
                qn = qnormalize(qadd(vb1, qscale(lambda, b)));
            }
        }
        d.q[src ^ 1][k] = v4of(qn);
    }
}

// ---------------------------------------------------------------------------------------
// Load-balanced variant of k_iter (one lane per vertex).  The contact lists of the block's
// B segments are consecutive in the packed layout (slots base + f, f = 0 .. total - 1); every
// thread takes contacts f = tid, tid + B, ... of that range, so a warp never waits for its
// longest list, the partner ids and staged positions are read coalesced, and the partner
// gathers of the whole block are in flight together.  Each thread writes its
// contact's 18-value contribution to shared memory (four 16-byte and one 8-byte store); the
// owning segment then adds its contacts in list order, so the result is deterministic.  The
// rest (own terms, vertex solve, orientation update) is k_iter's.
template <typename R, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_iter_bal(Dev<R> d, int src) {
    constexpr int B = NT;
    constexpr int CORE = B - 2;
    constexpr int NW = NT / 32;
    const int t = threadIdx.x;
    const int k = blockIdx.x * CORE - 1 + t;
    const int n = d.n;
    const bool valid = (k >= 0) && (k < n);
    const D2<R>* __restrict__ DX = d.dx[src];
    const V4<R>* __restrict__ QO = d.q[src];

    __shared__ R sSeg[12][B];  // p0, e = p1 - p0, dx, dx1 of each slot's segment
    // contributions of one chunk of contacts, double buffered, in 16-byte groups:
    // (fa, fb.x) (fb.yz, Ha0-1) (Ha2-5) (Hb0-3), then (Hb4-5)
    __shared__ V4<R> sCon4[2][4][B];
    __shared__ R2<R> sCon2[2][B];
    __shared__ int sOwn[2][B];     // owning slot of each contact of a chunk (double buffered)
    __shared__ int sOff[B + 1];
    __shared__ int sScene[B];
    __shared__ int sWarp[NW];
    __shared__ unsigned sBase;

    // The contact loop runs first and accumulates from zero; the vertex's own terms (inertia,
    // glue, stretch) are loaded and added after it, so their inputs are not live (in
    // registers) across the loop.
    V3<R> fa(R(0)), fb(R(0));
    H3<R> Ha, Hb;
    Ha.zero(); Hb.zero();
    int nc = 0, sc = 0;
    if (t == 0) sBase = d.csrOff[k < 0 ? 0 : k];  // the block's first packed slot (k < n here)
    {
        V3<R> p0(R(0)), e(R(0)), dx(R(0)), dx1(R(0));
        if (valid) {
            // inputs of the vertex's own terms, used after the contact loop
            prefetch_l1(d.vel + k);
            prefetch_l1(QO + k);
            prefetch_l1(d.qRest + k);
            prefetch_l1(d.stepLim + k);
            const uint32_t fl = d.vp[k].flags;
            sc = scene_of(fl);
            const D2<R> own = DX[k];
            dx = xyz(own.a);
            dx1 = xyz(own.b);
            p0 = xyz(d.pos[k]);
            if (fl & F_HAS_NEXT) {
                e = xyz(d.pos[k + 1]) - p0;
                unsigned off;
                nc = contact_range(d, k, off);
            }
        }
        sSeg[0][t] = p0.x; sSeg[1][t] = p0.y; sSeg[2][t] = p0.z;
        sSeg[3][t] = e.x; sSeg[4][t] = e.y; sSeg[5][t] = e.z;
        sSeg[6][t] = dx.x; sSeg[7][t] = dx.y; sSeg[8][t] = dx.z;
        sSeg[9][t] = dx1.x; sSeg[10][t] = dx1.y; sSeg[11][t] = dx1.z;
        sScene[t] = sc;
    }
    // block exclusive scan of the contact counts (the block's packed slots are base + offset)
    {
        const int lane = t & 31, w = t >> 5;
        int x = nc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sWarp[w] = x;
        __syncthreads();
        int wo = 0;
        for (int i = 0; i < w; i++) wo += sWarp[i];
        sOff[t] = wo + x - nc;
        if (t == B - 1) sOff[B] = wo + x;
        __syncthreads();
    }
    int total = sOff[B];
    int myOff = sOff[t];
    const unsigned base = sBase;
    if (base > d.csrCap || d.csrCap - base < (unsigned)total) {  // only a packing the list pass reported as failed
        total = 0;
        myOff = 0;
        nc = 0;
    }
    // Chunks of NT contacts, one per thread.  Each thread writes its own slot index over its
    // contacts of the next chunk before the current chunk's barrier, which publishes it, and
    // the contributions are double buffered: a buffer is written again only after the next
    // chunk's barrier, which every thread reaches after summing it, so each chunk needs one
    // barrier.
    for (int g = myOff; g < min(myOff + nc, NT); g++) sOwn[0][g] = t;
    __syncthreads();
    int buf = 0;
    // The partner id of this thread's contact is loaded one chunk ahead (after the previous
    // chunk's barrier, before its summation), so a chunk starts with the partner gather.
    int jn = 0;
    if (t < total) jn = __ldg(d.csrCols + (base + t));
    for (int b0 = 0; b0 < total; b0 += NT, buf ^= 1) {
        const int f = b0 + t;
        {
            const int nb = b0 + NT;
            const int g1 = min(myOff + nc, nb + NT);
            for (int g = max(myOff, nb); g < g1; g++) sOwn[buf ^ 1][g - nb] = t;
        }
        V3<R> cfa(R(0)), cfb(R(0));
        H3<R> cHa, cHb;
        cHa.zero(); cHb.zero();
        if (f < total && partner_ok(d, jn)) {
            const int s = sOwn[buf][t];
            const int j = jn;
            const V3<R> sp0(sSeg[0][s], sSeg[1][s], sSeg[2][s]);
            V3<R> r0, r1;
            partner_rel(d, base + f, j, sp0, r0, r1);
            const D2<R> pd = DX[j];
            const V3<R> se(sSeg[3][s], sSeg[4][s], sSeg[5][s]);
            const V3<R> sdx(sSeg[6][s], sSeg[7][s], sSeg[8][s]);
            const V3<R> sdx1(sSeg[9][s], sSeg[10][s], sSeg[11][s]);
            contact_term(se, sdx, sdx1, r0, r1, xyz(pd.a), xyz(pd.b), d.sp[sScene[s]], cfa, cHa, cfb, cHb);
        }
        {
            V4<R> w;
            w.x = cfa.x; w.y = cfa.y; w.z = cfa.z; w.w = cfb.x; sCon4[buf][0][t] = w;
            w.x = cfb.y; w.y = cfb.z; w.z = cHa.d[0]; w.w = cHa.d[1]; sCon4[buf][1][t] = w;
            w.x = cHa.d[2]; w.y = cHa.d[3]; w.z = cHa.d[4]; w.w = cHa.d[5]; sCon4[buf][2][t] = w;
            w.x = cHb.d[0]; w.y = cHb.d[1]; w.z = cHb.d[2]; w.w = cHb.d[3]; sCon4[buf][3][t] = w;
            R2<R> w2;
            w2.x = cHb.d[4]; w2.y = cHb.d[5];
            sCon2[buf][t] = w2;
        }
        __syncthreads();
        {
            // next chunk: partner id, and the staged partner positions into L1
            const int fn = b0 + NT + t;
            if (fn < total) {
                const unsigned g = base + fn;
                jn = __ldg(d.csrCols + g);
                if (g < d.relCap) {
                    prefetch_l1(d.relA + g);
                    prefetch_l1(d.relB + g);
                }
            }
        }
        const int f0 = max(myOff, b0), f1 = min(myOff + nc, b0 + NT);
        for (int g = f0; g < f1; g++) {
            const int i = g - b0;
            const V4<R> w0 = sCon4[buf][0][i], w1 = sCon4[buf][1][i], w2 = sCon4[buf][2][i], w3 = sCon4[buf][3][i];
            const R2<R> w4 = sCon2[buf][i];
            fa += V3<R>(w0.x, w0.y, w0.z);
            fb += V3<R>(w0.w, w1.x, w1.y);
            Ha.d[0] += w1.z; Ha.d[1] += w1.w;
            Ha.d[2] += w2.x; Ha.d[3] += w2.y; Ha.d[4] += w2.z; Ha.d[5] += w2.w;
            Hb.d[0] += w3.x; Hb.d[1] += w3.y; Hb.d[2] += w3.z; Hb.d[3] += w3.w;
            Hb.d[4] += w4.x; Hb.d[5] += w4.y;
        }
    }

    // The halo exchange after the loop uses the contribution buffer the last chunk did not
    // use (buf), viewed as 16 rows of B values: every thread finished reading it before the
    // last chunk's barrier.
    R (*rows)[B] = reinterpret_cast<R (*)[B]>(&sCon4[buf][0][0]);
    R (*sFb)[B] = rows;       // rows 0-2
    R (*sHb)[B] = rows + 3;   // rows 3-8
    R* sSL = rows[9];
    R (*sDX)[B] = rows + 10;  // rows 10-12

    // the vertex's own terms (cosserat.cu:40-81)
    R sl = yinf<R>();
    uint32_t flags = 0;
    R invMass = R(0), lRest = R(1), kStretch = R(0);
    const V3<R> p0(sSeg[0][t], sSeg[1][t], sSeg[2][t]);
    const V3<R> e(sSeg[3][t], sSeg[4][t], sSeg[5][t]);
    const V3<R> dx(sSeg[6][t], sSeg[7][t], sSeg[8][t]);
    Q<R> q0 = qmk(R(0), R(0), R(0), R(1));
    const SceneParams<R>* spp = d.sp;
    if (valid) {
        spp = &d.sp[sc];
        add_own_terms(d, k, DX, QO, *spp, p0, e, dx, V3<R>(sSeg[9][t], sSeg[10][t], sSeg[11][t]), fa, Ha, fb, Hb,
                      flags, invMass, lRest, kStretch, sl, q0);
    }

    sFb[0][t] = fb.x; sFb[1][t] = fb.y; sFb[2][t] = fb.z;
#pragma unroll
    for (int q = 0; q < 6; q++) sHb[q][t] = Hb.d[q];
    sSL[t] = sl;
    __syncthreads();

    V3<R> dxn = dx;
    if (valid && t > 0) {
        if (flags & F_HAS_PREV) {
            fa += V3<R>(sFb[0][t - 1], sFb[1][t - 1], sFb[2][t - 1]);
            H3<R> hp;
#pragma unroll
            for (int q = 0; q < 6; q++) hp.d[q] = sHb[q][t - 1];
            Ha.add(hp);
            sl = ymin(sl, sSL[t - 1]);
        }
        if (invMass != R(0)) {
            dxn = dx + spp->accel * solve3(Ha, fa);
            const R l = len(dxn);
            if (l > sl && l > R(0)) dxn *= sl / l;
        }
    }
    sDX[0][t] = dxn.x; sDX[1][t] = dxn.y; sDX[2][t] = dxn.z;
    const bool core = valid && t >= 1 && t <= CORE;
    __syncthreads();

    if (core) {
        const V3<R> dxb(sDX[0][t + 1], sDX[1][t + 1], sDX[2][t + 1]);
        D2<R> o;
        o.a = v4(dxn, R(0));
        o.b = v4(k + 1 < n ? dxb : V3<R>(R(0)), R(0));
        d.dx[src ^ 1][k] = o;
        d.q[src ^ 1][k] = v4of(orientation_update(d, k, QO, flags, e, dxn, dxb, lRest, kStretch, q0));
    }
}

// Warp-balanced variant of k_iter_bal: each warp flattens the contact lists of its own 32
// vertices (warp scan) and processes them 32 at a time, so the contact loop needs no block
// barrier and warps of one block proceed independently; per vertex the contributions are still
// summed in list order.
template <typename R, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_iter_wbal(Dev<R> d, int src) {
    constexpr int B = NT;
    constexpr int CORE = B - 2;
    constexpr int NW = NT / 32;
    const int t = threadIdx.x;
    const int k = blockIdx.x * CORE - 1 + t;
    const int n = d.n;
    const bool valid = (k >= 0) && (k < n);
    const D2<R>* __restrict__ DX = d.dx[src];
    const V4<R>* __restrict__ QO = d.q[src];

    __shared__ R sFb[3][B];
    __shared__ R sHb[6][B];
    __shared__ R sSL[B];
    __shared__ R sDX[3][B];
    __shared__ R sSeg[12][B];  // p0, e = p1 - p0, dx, dx1 of each slot's segment
    __shared__ R sCon[18][B];  // contributions of one chunk of contacts
    __shared__ int sOffW[NW][33];
    __shared__ int sScene[B];
    __shared__ unsigned sKOff[B];  // first packed slot of each slot's contacts

    // The contact loop runs first and accumulates from zero; the vertex's own terms are
    // loaded and added after it (their inputs are not live across the loop).
    V3<R> fa(R(0)), fb(R(0));
    H3<R> Ha, Hb;
    Ha.zero(); Hb.zero();
    int nc = 0, sc = 0;
    unsigned kOff = 0;
    {
        V3<R> p0(R(0)), e(R(0)), dx(R(0)), dx1(R(0));
        if (valid) {
            const uint32_t fl = d.vp[k].flags;
            sc = scene_of(fl);
            const D2<R> own = DX[k];
            dx = xyz(own.a);
            dx1 = xyz(own.b);
            p0 = xyz(d.pos[k]);
            if (fl & F_HAS_NEXT) {
                e = xyz(d.pos[k + 1]) - p0;
                nc = contact_range(d, k, kOff);
            }
        }
        sSeg[0][t] = p0.x; sSeg[1][t] = p0.y; sSeg[2][t] = p0.z;
        sSeg[3][t] = e.x; sSeg[4][t] = e.y; sSeg[5][t] = e.z;
        sSeg[6][t] = dx.x; sSeg[7][t] = dx.y; sSeg[8][t] = dx.z;
        sSeg[9][t] = dx1.x; sSeg[10][t] = dx1.y; sSeg[11][t] = dx1.z;
        sScene[t] = sc;
        sKOff[t] = kOff;
    }
    // warp exclusive scan of the contact counts: each warp flattens its own 32 vertices
    const int lane = t & 31, wp = t >> 5, w0 = wp << 5;
    int incl = nc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    sOffW[wp][lane] = incl - nc;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 31) sOffW[wp][32] = total;
    __syncwarp();
    const int myOff = incl - nc;
    for (int base = 0; base < total; base += 32) {
        const int f = base + lane;
        V3<R> cfa(R(0)), cfb(R(0));
        H3<R> cHa, cHb;
        cHa.zero(); cHb.zero();
        if (f < total) {
            int lo = 0, hi = 31;  // owner: the last lane of the warp whose offset is <= f
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sOffW[wp][mid] <= f) lo = mid; else hi = mid - 1;
            }
            const int s = w0 + lo, c = f - sOffW[wp][lo];
            const unsigned g = sKOff[s] + c;
            const int j = __ldg(d.csrCols + g);
            if (partner_ok(d, j)) {
                const V3<R> sp0(sSeg[0][s], sSeg[1][s], sSeg[2][s]);
                V3<R> r0, r1;
                partner_rel(d, g, j, sp0, r0, r1);
                const D2<R> pd = DX[j];
                const V3<R> se(sSeg[3][s], sSeg[4][s], sSeg[5][s]);
                const V3<R> sdx(sSeg[6][s], sSeg[7][s], sSeg[8][s]);
                const V3<R> sdx1(sSeg[9][s], sSeg[10][s], sSeg[11][s]);
                contact_term(se, sdx, sdx1, r0, r1, xyz(pd.a), xyz(pd.b), d.sp[sScene[s]], cfa, cHa, cfb, cHb);
            }
        }
        sCon[0][t] = cfa.x; sCon[1][t] = cfa.y; sCon[2][t] = cfa.z;
        sCon[3][t] = cfb.x; sCon[4][t] = cfb.y; sCon[5][t] = cfb.z;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            sCon[6 + q][t] = cHa.d[q];
            sCon[12 + q][t] = cHb.d[q];
        }
        __syncwarp();
        const int f0 = max(myOff, base), f1 = min(myOff + nc, base + 32);
        for (int g = f0; g < f1; g++) {
            const int i = w0 + g - base;
            fa += V3<R>(sCon[0][i], sCon[1][i], sCon[2][i]);
            fb += V3<R>(sCon[3][i], sCon[4][i], sCon[5][i]);
#pragma unroll
            for (int q = 0; q < 6; q++) {
                Ha.d[q] += sCon[6 + q][i];
                Hb.d[q] += sCon[12 + q][i];
            }
        }
        __syncwarp();
    }

    // the vertex's own terms (cosserat.cu:40-81)
    R sl = yinf<R>();
    uint32_t flags = 0;
    R invMass = R(0), lRest = R(1), kStretch = R(0);
    const V3<R> p0(sSeg[0][t], sSeg[1][t], sSeg[2][t]);
    const V3<R> e(sSeg[3][t], sSeg[4][t], sSeg[5][t]);
    const V3<R> dx(sSeg[6][t], sSeg[7][t], sSeg[8][t]);
    Q<R> q0 = qmk(R(0), R(0), R(0), R(1));
    const SceneParams<R>* spp = d.sp;
    if (valid) {
        spp = &d.sp[sc];
        add_own_terms(d, k, DX, QO, *spp, p0, e, dx, V3<R>(sSeg[9][t], sSeg[10][t], sSeg[11][t]), fa, Ha, fb, Hb,
                      flags, invMass, lRest, kStretch, sl, q0);
    }

    sFb[0][t] = fb.x; sFb[1][t] = fb.y; sFb[2][t] = fb.z;
#pragma unroll
    for (int q = 0; q < 6; q++) sHb[q][t] = Hb.d[q];
    sSL[t] = sl;
    __syncthreads();

    V3<R> dxn = dx;
    if (valid && t > 0) {
        if (flags & F_HAS_PREV) {
            fa += V3<R>(sFb[0][t - 1], sFb[1][t - 1], sFb[2][t - 1]);
            H3<R> hp;
#pragma unroll
            for (int q = 0; q < 6; q++) hp.d[q] = sHb[q][t - 1];
            Ha.add(hp);
            sl = ymin(sl, sSL[t - 1]);
        }
        if (invMass != R(0)) {
            dxn = dx + spp->accel * solve3(Ha, fa);
            const R l = len(dxn);
            if (l > sl && l > R(0)) dxn *= sl / l;
        }
    }
    sDX[0][t] = dxn.x; sDX[1][t] = dxn.y; sDX[2][t] = dxn.z;
    const bool core = valid && t >= 1 && t <= CORE;
    __syncthreads();

    if (core) {
        const V3<R> dxb(sDX[0][t + 1], sDX[1][t + 1], sDX[2][t + 1]);
        D2<R> o;
        o.a = v4(dxn, R(0));
        o.b = v4(k + 1 < n ? dxb : V3<R>(R(0)), R(0));
        d.dx[src ^ 1][k] = o;
        d.q[src ^ 1][k] = v4of(orientation_update(d, k, QO, flags, e, dxn, dxb, lRest, kStretch, q0));
    }
}

// ---------------------------------------------------------------------------------------
template <typename R>
void launch_init(const Dev<R>& d, cudaStream_t s) {
    if (d.n <= 0) return;
    k_init<R><<<(d.n + 255) / 256, 256, 0, s>>>(d);
}

template <typename R>
void launch_end(const Dev<R>& d, int finalBuf, bool copyQ, bool kahan, cudaStream_t s) {
    if (d.n <= 0) return;
    k_end<R><<<(d.n + 255) / 256, 256, 0, s>>>(d, finalBuf, copyQ ? 1 : 0, kahan ? 1 : 0);
}

// Newton iteration launch shapes: NT threads per block, T lanes per vertex, pipelined or not;
// lanes = 0 selects a load-balanced kernel (one lane per vertex, flattened contact lists):
// per block (pipe = 0) or per warp (pipe = 1).
template <typename R>
void launch_iter(const Dev<R>& d, int srcBuf, int threads, int lanes, int pipe, cudaStream_t s) {
    if (d.n <= 0) return;
#define YB_ITER(NT, T, MINB, P) \
    k_iter<R, NT, T, MINB, P><<<(d.n + (NT / T) - 3) / ((NT / T) - 2), NT, 0, s>>>(d, srcBuf)
    if (lanes == 0 && pipe) {  // warp-balanced contact loop
        if constexpr (sizeof(R) == 4)
            k_iter_wbal<R, 128, 6><<<(d.n + 125) / 126, 128, 0, s>>>(d, srcBuf);
        else
            k_iter_wbal<R, 64, 4><<<(d.n + 61) / 62, 64, 0, s>>>(d, srcBuf);
    } else if (lanes == 0) {  // block-balanced contact loop (shared memory bounds the block size)
        if constexpr (sizeof(R) == 4)
            k_iter_bal<R, 128, 7><<<(d.n + 125) / 126, 128, 0, s>>>(d, srcBuf);
        else
            k_iter_bal<R, 64, 4><<<(d.n + 61) / 62, 64, 0, s>>>(d, srcBuf);
    } else if (pipe) {
        if (lanes == 4) YB_ITER(256, 4, 2, true);
        else if (threads == 128) YB_ITER(128, 1, 4, true);
        else YB_ITER(256, 1, 2, true);
    } else if (lanes == 2) {
        YB_ITER(256, 2, 3, false);
    } else if (lanes == 4) {
        if (threads == 512) YB_ITER(512, 4, 2, false); else YB_ITER(256, 4, 3, false);
    } else if (lanes == 8) {
        if (threads == 512) YB_ITER(512, 8, 2, false); else YB_ITER(256, 8, 3, false);
    } else {
        if (threads == 128) YB_ITER(128, 1, 6, false); else YB_ITER(256, 1, 2, false);
    }
#undef YB_ITER
}

template void launch_init<float>(const Dev<float>&, cudaStream_t);
template void launch_init<double>(const Dev<double>&, cudaStream_t);
template void launch_end<float>(const Dev<float>&, int, bool, bool, cudaStream_t);
template void launch_end<double>(const Dev<double>&, int, bool, bool, cudaStream_t);
template void launch_iter<float>(const Dev<float>&, int, int, int, int, cudaStream_t);
template void launch_iter<double>(const Dev<double>&, int, int, int, int, cudaStream_t);

}  // namespace yb
