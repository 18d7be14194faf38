// k_small.cu - one thread block advances a small simulation through every substep of an
// advance() in a single launch.
//
// A scene of a few hundred vertices keeps a B200 busy for microseconds per kernel, so the
// per-substep kernel sequence (predictor, BVH refit and traversal, list pass, numItr Newton
// launches, advection) is bound by launch latency: the README two-yarn scene (64 vertices)
// takes ~64 us per substep that way.  Here one block of SMALL_THREADS threads, one vertex per
// thread, runs all substeps with block barriers between the phases: the same device functions
// as the multi-block kernels (step.cuh, detect.cuh) in the same order and with the
// load-balanced Newton kernel's summation order, and the same contact set (every pair of
// segments goes through the narrow-phase filter; a pair the filter keeps has overlapping padded
// boxes, which is all the BVH query contributes).  The compiler may contract multiplies and
// adds into fused operations differently in this one kernel than in the separate kernels, so
// the two paths agree to rounding rather than bit for bit.
//
// Reference semantics: Sim::advance (sim/step.cpp:36-55) with initItr / endItr
// (sim/iteration.cu), detectCollisions + buildCollisionList (sim/collision.cu:39-119),
// recomputeStepLimitKernel (collision.cu:121-159), cosseratItr + quaternionLambdaItr
// (sim/cosserat.cu).
#include "step.cuh"

namespace yb {

constexpr int SMALL_THREADS = 256;  // largest simulation this path runs (vertices)

template <typename R>
__device__ __forceinline__ void small_append(const Dev<R>& d, int x, int y) {
    const int at = atomicAdd(&d.numCols[x], 1);
    if (at < MAX_COLS) d.cols[col_at(x, at)] = y;
}

template <typename R>
__global__ void __launch_bounds__(SMALL_THREADS) k_small(Dev<R> d, int steps, int numItr, unsigned long long step0,
                                                         int detectionPeriod, int kahan) {
    __shared__ R sFb[3][SMALL_THREADS];
    __shared__ R sHb[6][SMALL_THREADS];
    __shared__ R sSL[SMALL_THREADS];
    __shared__ R sDX[3][SMALL_THREADS];
    typedef Ex<R> E;
    const int k = threadIdx.x;
    const int n = d.n;
    const bool valid = k < n;
    const uint32_t fl0 = valid ? d.vp[k].flags : 0u;
    const bool seg = valid && (fl0 & F_HAS_NEXT);
    const int sc = scene_of(fl0);
    for (int s = 0; s < steps; s++) {
        // predictor (k_init)
        if (valid) init_vertex(d, k);
        __syncthreads();
        const bool detect = detectionPeriod > 0 && (step0 + (unsigned long long)s) % (unsigned long long)detectionPeriod == 0;
        if (detect) {
            if (valid) d.numCols[k] = 0;
            __syncthreads();
            // narrow phase over every pair of segments of the scene, lower index first (k_traverse)
            if (seg) {
                const SceneParams<R>& sp = d.sp[sc];
                for (int y = k + 3; y < n; y++) {
                    const uint32_t fy = d.vp[y].flags;
                    if (!(fy & F_HAS_NEXT) || scene_of(fy) != sc) continue;
                    if (pair_keep(d, k, y, sp)) {
                        small_append(d, k, y);
                        small_append(d, y, k);
                    }
                }
            }
            __syncthreads();
            // list clamp, overflow error and sort by partner id (k_lists)
            if (seg) {
                int nc = d.numCols[k];
                if (nc) atomicMax(&d.err[EW_MAX_COLS], nc);
                if (nc > MAX_COLS) d.err[EW_ERROR] = 1;
                nc = min(nc, MAX_COLS);
                d.numCols[k] = nc;
                int* row = d.cols + col_at(k, 0);
                for (int i = 1; i < nc; i++) {
                    const int v = row[i];
                    int j = i - 1;
                    while (j >= 0 && row[j] > v) {
                        row[j + 1] = row[j];
                        j--;
                    }
                    row[j + 1] = v;
                }
            }
        }
        // step limit, staged partner positions, interpenetration statistics (k_lists)
        if (seg) {
            const SceneParams<R>& sp = d.sp[sc];
            const int nc = d.numCols[k];
            const V3<R> a0 = xyz(d.pos[k]);
            const V3<R> a1 = xsub(xyz(d.pos[k + 1]), a0);
            R m = step_limit_base(d, k, sp);
            int pens = 0;
            float dmin = INFINITY;
            for (int c = 0; c < nc; c++) {
                const int o = d.cols[col_at(k, c)];
                bool pen;
                R dist;
                const R lim =
                    contact_step_limit(d, k, c < RELCAP ? rel_at(k, c) : NO_STAGE, o, a0, a1, sp, pen, dist);
                pens += pen;
                dmin = fminf(dmin, (float)dist);
                m = ymin(m, lim);
            }
            if (pens) {
                atomicAdd(&d.err[EW_PENETRATIONS], pens);
                d.err[EW_WARNING] = 2;
            }
            if (dmin < INFINITY) atomicMin(&d.err[EW_MIN_DIST], __float_as_int(dmin));
            d.stepLim[k] = sp.useStepLimit ? m : yinf<R>();
        }
        __syncthreads();
        // Newton + orientation iterations (k_iter_bal's arithmetic and summation order)
        for (int it = 0; it < numItr; it++) {
            const int src = it & 1;
            const D2<R>* __restrict__ DX = d.dx[src];
            const V4<R>* __restrict__ QO = d.q[src];
            V3<R> p0(R(0)), e(R(0)), dx(R(0)), dx1(R(0));
            int nc = 0;
            if (valid) {
                const D2<R> own = DX[k];
                dx = xyz(own.a);
                dx1 = xyz(own.b);
                p0 = xyz(d.pos[k]);
                if (seg) {
                    e = xyz(d.pos[k + 1]) - p0;
                    nc = d.numCols[k];
                }
            }
            V3<R> fa(R(0)), fb(R(0));
            H3<R> Ha, Hb;
            Ha.zero();
            Hb.zero();
            if (nc) {
                const SceneParams<R>& sp = d.sp[sc];
                for (int c = 0; c < nc; c++) {
                    const int j = d.cols[col_at(k, c)];
                    V3<R> r0, r1;
                    if (c < RELCAP) {
                        const size_t at = rel_at(k, c);
                        const V4<R> A = d.relA[at];
                        const R2<R> Bq = d.relB[at];
                        r0 = V3<R>(A.x, A.y, A.z);
                        r1 = V3<R>(A.w, Bq.x, Bq.y);
                    } else {
                        r0 = xyz(d.pos[j]) - p0;
                        r1 = xyz(d.pos[j + 1]) - p0;
                    }
                    const D2<R> pd = DX[j];
                    V3<R> cfa(R(0)), cfb(R(0));
                    H3<R> cHa, cHb;
                    cHa.zero();
                    cHb.zero();
                    contact_term(e, dx, dx1, r0, r1, xyz(pd.a), xyz(pd.b), sp, cfa, cHa, cfb, cHb);
                    // Separately rounded sums: k_iter_bal adds each contribution after a trip
                    // through shared memory, so the compiler cannot fuse the contribution's last
                    // multiply into the sum there; it must not here either.
                    fa = V3<R>(E::add(fa.x, cfa.x), E::add(fa.y, cfa.y), E::add(fa.z, cfa.z));
                    fb = V3<R>(E::add(fb.x, cfb.x), E::add(fb.y, cfb.y), E::add(fb.z, cfb.z));
#pragma unroll
                    for (int q = 0; q < 6; q++) {
                        Ha.d[q] = E::add(Ha.d[q], cHa.d[q]);
                        Hb.d[q] = E::add(Hb.d[q], cHb.d[q]);
                    }
                }
            }
            R sl = yinf<R>();
            uint32_t flags = 0;
            R invMass = R(0), lRest = R(1), kStretch = R(0);
            Q<R> q0 = qmk(R(0), R(0), R(0), R(1));
            if (valid)
                add_own_terms(d, k, DX, QO, d.sp[sc], p0, e, dx, dx1, fa, Ha, fb, Hb, flags, invMass, lRest, kStretch,
                              sl, q0);
            sFb[0][k] = fb.x; sFb[1][k] = fb.y; sFb[2][k] = fb.z;
#pragma unroll
            for (int q = 0; q < 6; q++) sHb[q][k] = Hb.d[q];
            sSL[k] = sl;
            __syncthreads();
            V3<R> dxn = dx;
            if (valid) {
                if (flags & F_HAS_PREV) {
                    fa += V3<R>(sFb[0][k - 1], sFb[1][k - 1], sFb[2][k - 1]);
                    H3<R> hp;
#pragma unroll
                    for (int q = 0; q < 6; q++) hp.d[q] = sHb[q][k - 1];
                    Ha.add(hp);
                    sl = ymin(sl, sSL[k - 1]);
                }
                if (invMass != R(0)) {
                    dxn = dx + d.sp[sc].accel * solve3(Ha, fa);
                    const R l = len(dxn);
                    if (l > sl && l > R(0)) dxn *= sl / l;
                }
            }
            sDX[0][k] = dxn.x; sDX[1][k] = dxn.y; sDX[2][k] = dxn.z;
            __syncthreads();
            if (valid) {
                const V3<R> dxb = k + 1 < n ? V3<R>(sDX[0][k + 1], sDX[1][k + 1], sDX[2][k + 1]) : V3<R>(R(0));
                D2<R> o;
                o.a = v4(dxn, R(0));
                o.b = v4(dxb, R(0));
                d.dx[src ^ 1][k] = o;
                d.q[src ^ 1][k] = v4of(orientation_update(d, k, QO, flags, e, dxn, dxb, lRest, kStretch, q0));
            }
            __syncthreads();
        }
        // advection (k_end)
        if (valid) end_vertex(d, k, numItr & 1, (numItr & 1) != 0, kahan);
        __syncthreads();
    }
}

template <typename R>
bool small_path_fits(const Dev<R>& d) {
    return d.n > 0 && d.n <= SMALL_THREADS;
}

template <typename R>
void launch_small(const Dev<R>& d, int steps, int numItr, unsigned long long step0, int detectionPeriod, bool kahan,
                  cudaStream_t s) {
    if (d.n <= 0 || steps <= 0) return;
    k_small<R><<<1, SMALL_THREADS, 0, s>>>(d, steps, numItr, step0, detectionPeriod, kahan ? 1 : 0);
}

template bool small_path_fits<float>(const Dev<float>&);
template bool small_path_fits<double>(const Dev<double>&);
template void launch_small<float>(const Dev<float>&, int, int, unsigned long long, int, bool, cudaStream_t);
template void launch_small<double>(const Dev<double>&, int, int, unsigned long long, int, bool, cudaStream_t);

}  // namespace yb
