// k_io.cu - host<->device layout conversion (AoS host arrays <-> SoA device state),
// velocity reset, BVH root boxes and the FP64 diagnostic reductions.
//
//   upload/copyTempData  KittenEngine/YarnBall/YarnBall.cu:239-254
//   download             KittenEngine/YarnBall/YarnBall.cu:256-261
//   zeroVels             KittenEngine/YarnBall/YarnBall.cu:263-274
//   bounds               KittenEngine/YarnBall/YarnBall.cu:87-89
#include "detect.cuh"
#include "io.cuh"

namespace yb {

struct HostVertex {  // yb_vertex
    float pos[3];
    float invMass, lRest, kStretch;
    int cid;
    uint32_t flags;
};

template <typename R>
__global__ void k_convert_in(Dev<R> d, const HostVertex* __restrict__ hv, const float* __restrict__ hvel,
                             const float* __restrict__ hq, const float* __restrict__ hqr,
                             const int* __restrict__ sceneOf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const HostVertex v = hv[i];
    V4<R> p; p.x = v.pos[0]; p.y = v.pos[1]; p.z = v.pos[2]; p.w = v.invMass;
    d.pos[i] = p;
    V4<R> z; z.x = R(0); z.y = R(0); z.z = R(0); z.w = R(0);
    d.posC[i] = z;
    VP<R> vp; vp.lRest = v.lRest; vp.kStretch = v.kStretch; vp.cid = v.cid;
    uint32_t fl = v.flags & F_USER_MASK;
    // The last vertex of a scene never starts a segment (its successor is another scene).
    if (i == d.n - 1 || sceneOf[i + 1] != sceneOf[i]) fl &= ~(uint32_t)(F_HAS_NEXT | F_HAS_NEXT_ORI);
    // ... and the first vertex of a scene has no predecessor.
    if (i == 0 || sceneOf[i - 1] != sceneOf[i]) fl &= ~(uint32_t)F_HAS_PREV;
    vp.flags = fl | ((uint32_t)sceneOf[i] << 8);
    d.vp[i] = vp;
    V4<R> vel; vel.x = hvel[3 * i]; vel.y = hvel[3 * i + 1]; vel.z = hvel[3 * i + 2]; vel.w = R(0);
    d.vel[i] = vel;
    V4<R> q; q.x = hq[4 * i]; q.y = hq[4 * i + 1]; q.z = hq[4 * i + 2]; q.w = hq[4 * i + 3];
    d.q[0][i] = q;
    V4<R> qr; qr.x = hqr[4 * i]; qr.y = hqr[4 * i + 1]; qr.z = hqr[4 * i + 2]; qr.w = hqr[4 * i + 3];
    d.qRest[i] = qr;
}

template <typename R>
__global__ void k_convert_out(Dev<R> d, HostVertex* __restrict__ hv, float* __restrict__ hvel, float* __restrict__ hq,
                              int first, int count) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= count) return;
    const int i = first + ii;
    const V4<R> p = d.pos[i];
    const VP<R> vp = d.vp[i];
    HostVertex v;
    v.pos[0] = (float)p.x; v.pos[1] = (float)p.y; v.pos[2] = (float)p.z;
    v.invMass = (float)p.w; v.lRest = (float)vp.lRest; v.kStretch = (float)vp.kStretch;
    v.cid = vp.cid; v.flags = vp.flags & F_USER_MASK;
    hv[i] = v;
    const V4<R> vel = d.vel[i];
    hvel[3 * i] = (float)vel.x; hvel[3 * i + 1] = (float)vel.y; hvel[3 * i + 2] = (float)vel.z;
    const V4<R> q = d.q[0][i];
    hq[4 * i] = (float)q.x; hq[4 * i + 1] = (float)q.y; hq[4 * i + 2] = (float)q.z; hq[4 * i + 3] = (float)q.w;
}

// After scenes were copied into a new layout: scene ids in the flags, scene-boundary flags,
// and connection indices shifted by each scene's offset change.
template <typename R>
__global__ void k_relayout(Dev<R> d, const int* __restrict__ sceneOf, const int* __restrict__ delta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    VP<R> vp = d.vp[i];
    const int sc = sceneOf[i];
    uint32_t fl = vp.flags & F_USER_MASK;
    if (i == d.n - 1 || sceneOf[i + 1] != sc) fl &= ~(uint32_t)(F_HAS_NEXT | F_HAS_NEXT_ORI);
    if (i == 0 || sceneOf[i - 1] != sc) fl &= ~(uint32_t)F_HAS_PREV;
    vp.flags = fl | ((uint32_t)sc << 8);
    if (vp.cid >= 0) vp.cid += delta[sc];
    d.vp[i] = vp;
}

// Kinematic driver (the per-frame twist/pull of KittenEngine/main.cpp:54-121, on the device):
// x(t) = c + Rot(a, omega s(t)) (x0 - c) + v s(t), s(t) = clamp(t - t0, 0, t1 - t0).
__device__ inline void pin_place(const PinMotion& m, const double x0[3], double t, double out[3]) {
    const double s = fmin(fmax(t - m.t0, 0.0), m.t1 - m.t0);
    const double th = m.omega * s;
    const double ct = cos(th), st = sin(th);
    const double r[3] = {x0[0] - m.c[0], x0[1] - m.c[1], x0[2] - m.c[2]};
    const double kd = m.a[0] * r[0] + m.a[1] * r[1] + m.a[2] * r[2];
    const double kx[3] = {m.a[1] * r[2] - m.a[2] * r[1], m.a[2] * r[0] - m.a[0] * r[2], m.a[0] * r[1] - m.a[1] * r[0]};
    for (int i = 0; i < 3; i++)
        out[i] = m.c[i] + r[i] * ct + kx[i] * st + m.a[i] * kd * (1.0 - ct) + m.v[i] * s;
}

template <typename R>
__global__ void k_pin_drive(Dev<R> d, const float4* __restrict__ init, const unsigned char* __restrict__ group,
                            const PinMotion* __restrict__ motions, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int g = group[i];
    if (g == 0) return;
    const PinMotion& m = motions[g - 1];
    const double t = d.sp[scene_of(d.vp[i].flags)].time;
    const float4 x0f = init[i];
    const double x0[3] = {x0f.x, x0f.y, x0f.z};
    double a[3], b[3];
    pin_place(m, x0, t, a);
    pin_place(m, x0, t + dt, b);
    V4<R> p = d.pos[i];
    p.x = (R)a[0]; p.y = (R)a[1]; p.z = (R)a[2];
    d.pos[i] = p;
    V4<R> z; z.x = R(0); z.y = R(0); z.z = R(0); z.w = R(0);
    d.posC[i] = z;
    V4<R> v;
    v.x = (R)((b[0] - a[0]) / dt); v.y = (R)((b[1] - a[1]) / dt); v.z = (R)((b[2] - a[2]) / dt); v.w = R(0);
    d.vel[i] = v;
}

template <typename R>
__global__ void k_zero_vel(Dev<R> d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    V4<R> z; z.x = R(0); z.y = R(0); z.z = R(0); z.w = R(0);
    d.vel[i] = z;
    d.lastVel[i] = z;
}

template <typename R>
__global__ void k_state_f64(Dev<R> d, int buf, double* pos, double* vel, double* q, double* dx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    if (pos) { const V4<R> p = d.pos[i]; pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z; }
    if (vel) { const V4<R> v = d.vel[i]; vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z; }
    if (q) { const V4<R> a = d.q[buf][i]; q[4 * i] = a.x; q[4 * i + 1] = a.y; q[4 * i + 2] = a.z; q[4 * i + 3] = a.w; }
    if (dx) { const V4<R> a = d.dx[buf][i].a; dx[4 * i] = a.x; dx[4 * i + 1] = a.y; dx[4 * i + 2] = a.z; dx[4 * i + 3] = a.w; }
}

// Root box of each scene's subtree (refit must have run).
template <typename R>
__global__ void k_scene_root_box(Dev<R> d, float* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.numScenes) return;
    const int r = d.sceneRoot[s];
    float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    if (r >= 0) {
        const BNode<R>& nd = d.nodes[r];
        for (int a = 0; a < 3; a++) {
            b[a] = (float)ymin(nd.lmin[a], nd.rmin[a]);
            b[3 + a] = (float)ymax(nd.lmax[a], nd.rmax[a]);
        }
    } else if (r != INT_MIN) {
        const int k = -r - 1;
        const Box<R> bx = segment_box(d, k, d.sp[s]);
        for (int a = 0; a < 3; a++) { b[a] = (float)bx.mn[a]; b[3 + a] = (float)bx.mx[a]; }
    }
    for (int a = 0; a < 6; a++) out[6 * s + a] = b[a];
}

// ---------------------------------------------------------------------------------------
// FP64 diagnostics.  Definitions (per scene parameters; sums over all scenes):
//   kinetic   sum_i 1/2 m_i |v_i|^2                 over unpinned vertices (m = 1/invMass)
//   gravity   - sum_i m_i g . x_i                    over unpinned vertices
//   stretch   sum_seg 1/2 kStretch |(x_{i+1}-x_i)/l - q_i e1|^2   (kStretch already holds
//             k * l, so this is the energy whose gradient is the stretch force of
//             cosserat.cu:63-81)
//   bend      sum_bonds |r_i| - |<q_i r_i, q_{i+1}>|  (r_i = qRest_i; the orientation update
//             of cosserat.cu:209-253 maximises <q_i, b_i>, b_i being the gradient of the
//             bond terms, so this is the bending/twisting energy it decreases)
//   barrier   sum_pairs -kCollision (d-1)^2 ln d,  d = (dist - 2 radius)/barrierThickness
//             clamped to 1e-3, pairs with d < 1 (each unordered pair once)
//   max |v|, min normalised gap d over listed contacts, number of listed contact pairs.
// Per-block partials are written to a buffer and summed in a fixed order on the host, so
// repeated calls give identical results.
template <typename R>
__global__ void __launch_bounds__(256) k_diag(Dev<R> d, double* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e[8] = {0, 0, 0, 0, 0, 0, 1e300, 0};
    if (i < d.n) {
        const VP<R> vp = d.vp[i];
        const SceneParams<R>& sp = d.sp[scene_of(vp.flags)];
        const V4<R> P = d.pos[i];
        const V4<R> V = d.vel[i];
        const double vx = V.x, vy = V.y, vz = V.z;
        if (P.w != R(0)) {
            const double m = 1.0 / (double)P.w;
            e[0] = 0.5 * m * (vx * vx + vy * vy + vz * vz);
            e[1] = -m * ((double)sp.gx * P.x + (double)sp.gy * P.y + (double)sp.gz * P.z);
        }
        e[5] = sqrt(vx * vx + vy * vy + vz * vz);
        if (vp.flags & F_HAS_NEXT) {
            const V4<R> P1 = d.pos[i + 1];
            const Q<double> q = qmk((double)d.q[0][i].x, (double)d.q[0][i].y, (double)d.q[0][i].z, (double)d.q[0][i].w);
            const V3<double> t = qrotate(q, V3<double>(1.0, 0.0, 0.0));
            const double il = 1.0 / (double)vp.lRest;
            const V3<double> c((P1.x - (double)P.x) * il - t.x, (P1.y - (double)P.y) * il - t.y,
                               (P1.z - (double)P.z) * il - t.z);
            e[2] = 0.5 * (double)vp.kStretch * len2(c);
            if (vp.flags & F_HAS_NEXT_ORI) {
                const V4<R> rr = d.qRest[i];
                const Q<double> r = qmk((double)rr.x, (double)rr.y, (double)rr.z, (double)rr.w);
                const V4<R> qn = d.q[0][i + 1];
                const Q<double> q1 = qmk((double)qn.x, (double)qn.y, (double)qn.z, (double)qn.w);
                e[3] = qlen(r) - fabs(qdot(qmul(q, r), q1));
            }
            const int nc = d.numCols[i];
            const double twoR = (double)sp.twoR, invb = (double)sp.invb;
            for (int c2 = 0; c2 < nc; c2++) {
                const int j = d.cols[col_at(i, c2)];
                if (j < i) continue;
                const V3<double> a0(P.x, P.y, P.z), a1(P1.x, P1.y, P1.z);
                const V4<R> B0 = d.pos[j], B1 = d.pos[j + 1];
                const V3<double> b0(B0.x, B0.y, B0.z), b1(B1.x, B1.y, B1.z);
                const UVT<double> uv = closest_uv(a1 - a0, b0 - a0, b1 - a0);
                const double dist = len(mix(a0, a1, uv.u) - mix(b0, b1, uv.v));
                double g = (dist - twoR) * invb;
                e[6] = fmin(e[6], g);
                e[7] += 1.0;
                if (g < 1.0) {
                    g = fmax(g, 1e-3);
                    e[4] += -(double)sp.kCol / invb * (g - 1.0) * (g - 1.0) * log(g);
                }
            }
        }
    }
    __shared__ double sh[8][256];
    for (int a = 0; a < 8; a++) sh[a][threadIdx.x] = e[a];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            for (int a = 0; a < 8; a++) {
                const double o = sh[a][threadIdx.x + s];
                if (a == 5) sh[a][threadIdx.x] = fmax(sh[a][threadIdx.x], o);
                else if (a == 6) sh[a][threadIdx.x] = fmin(sh[a][threadIdx.x], o);
                else sh[a][threadIdx.x] += o;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 8) part[(size_t)blockIdx.x * 8 + threadIdx.x] = sh[threadIdx.x][0];
}

template <typename R>
void launch_convert_in(const Dev<R>& d, const void* hv, const float* hvel, const float* hq, const float* hqr,
                       const int* sceneOf, cudaStream_t s) {
    if (d.n <= 0) return;
    k_convert_in<R><<<(d.n + 255) / 256, 256, 0, s>>>(d, (const HostVertex*)hv, hvel, hq, hqr, sceneOf);
}
template <typename R>
void launch_convert_out(const Dev<R>& d, void* hv, float* hvel, float* hq, int first, int count, cudaStream_t s) {
    if (count <= 0) return;
    k_convert_out<R><<<(count + 255) / 256, 256, 0, s>>>(d, (HostVertex*)hv, hvel, hq, first, count);
}
template <typename R>
void launch_pin_drive(const Dev<R>& d, const float4* init, const unsigned char* group, const PinMotion* m, double dt,
                      cudaStream_t s) {
    if (d.n <= 0) return;
    k_pin_drive<R><<<(d.n + 255) / 256, 256, 0, s>>>(d, init, group, m, dt);
}
template <typename R>
void launch_relayout(const Dev<R>& d, const int* sceneOf, const int* delta, cudaStream_t s) {
    if (d.n <= 0) return;
    k_relayout<R><<<(d.n + 255) / 256, 256, 0, s>>>(d, sceneOf, delta);
}
template <typename R>
void launch_zero_vel(const Dev<R>& d, cudaStream_t s) {
    if (d.n <= 0) return;
    k_zero_vel<R><<<(d.n + 255) / 256, 256, 0, s>>>(d);
}
template <typename R>
void launch_state_f64(const Dev<R>& d, int buf, double* pos, double* vel, double* q, double* dx, cudaStream_t s) {
    if (d.n <= 0) return;
    k_state_f64<R><<<(d.n + 255) / 256, 256, 0, s>>>(d, buf, pos, vel, q, dx);
}
template <typename R>
void launch_scene_root_box(const Dev<R>& d, float* out, cudaStream_t s) {
    k_scene_root_box<R><<<(d.numScenes + 127) / 128, 128, 0, s>>>(d, out);
}
template <typename R>
int launch_diag(const Dev<R>& d, double* part, cudaStream_t s) {
    const int nb = (d.n + 255) / 256;
    if (nb > 0) k_diag<R><<<nb, 256, 0, s>>>(d, part);
    return nb;
}

template <typename R>
__global__ void __launch_bounds__(256) k_iter_delta(Dev<R> d, int src, unsigned long long* slot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < d.n) {
        const V4<R> a = d.dx[src][i].a, b = d.dx[src ^ 1][i].a;
        const double x = (double)b.x - (double)a.x, y = (double)b.y - (double)a.y, z = (double)b.z - (double)a.z;
        v = sqrt(x * x + y * y + z * z);
    }
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

template <typename R>
void launch_iter_delta(const Dev<R>& d, int src, unsigned long long* slot, cudaStream_t s) {
    if (d.n <= 0) return;
    k_iter_delta<R><<<(d.n + 255) / 256, 256, 0, s>>>(d, src, slot);
}

#define YB_INST(R)                                                                                          \
    template void launch_convert_in<R>(const Dev<R>&, const void*, const float*, const float*, const float*, \
                                       const int*, cudaStream_t);                                            \
    template void launch_convert_out<R>(const Dev<R>&, void*, float*, float*, int, int, cudaStream_t);       \
    template void launch_relayout<R>(const Dev<R>&, const int*, const int*, cudaStream_t);                   \
    template void launch_pin_drive<R>(const Dev<R>&, const float4*, const unsigned char*, const PinMotion*, double, \
                                      cudaStream_t);                                                         \
    template void launch_zero_vel<R>(const Dev<R>&, cudaStream_t);                                           \
    template void launch_state_f64<R>(const Dev<R>&, int, double*, double*, double*, double*, cudaStream_t); \
    template void launch_scene_root_box<R>(const Dev<R>&, float*, cudaStream_t);                             \
    template void launch_iter_delta<R>(const Dev<R>&, int, unsigned long long*, cudaStream_t);               \
    template int launch_diag<R>(const Dev<R>&, double*, cudaStream_t);
YB_INST(float)
YB_INST(double)

}  // namespace yb
