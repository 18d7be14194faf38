// yb_oracle.cpp - CPU oracle (test infrastructure): plain C++/OpenMP restatement of the
// reference's substep.  See yb_oracle.h for scope and the "parity unpinned" note.
//
// Reference functions restated here (paths inside the reference project):
//   Sim::Sim defaults          KittenEngine/YarnBall/YarnBall.cu:11-51
//   Sim::configure             KittenEngine/YarnBall/YarnBall.cu:91-157
//   setKStretch / setKBend     KittenEngine/YarnBall/YarnBall.cu:202-224
//   uploadMeta                 KittenEngine/YarnBall/YarnBall.cu:226-234
//   initItr / endItr           KittenEngine/YarnBall/sim/iteration.cu:7-61
//   buildAABBs                 KittenEngine/YarnBall/sim/collision.cu:10-37
//   buildCollisionList         KittenEngine/YarnBall/sim/collision.cu:39-92
//   recomputeStepLimitKernel   KittenEngine/YarnBall/sim/collision.cu:121-159
//   cosseratItr                KittenEngine/YarnBall/sim/cosserat.cu:20-207
//   quaternionLambdaItr        KittenEngine/YarnBall/sim/cosserat.cu:209-253
//   Sim::advance               KittenEngine/YarnBall/sim/step.cpp:36-55
//   segmentClosestPoints       KittenEngine/KittenEngine/includes/modules/Common.h:318-336
//   Rotor ops                  KittenEngine/KittenEngine/includes/modules/Rotor.h:57-105,185-188
//   hess3                      KittenEngine/KittenEngine/includes/modules/SymMat.h:8-107
// Compiled with -ffp-contract=off: every FP32 expression is rounded operation by operation
// in source order, which is what makes the detection predicates reproducible bit for bit.
#include "yb_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr int MAXC = 128;  // MAX_COLLISIONS_PER_SEGMENT, YarnBall.h:20
enum : uint32_t { HAS_PREV = 1, HAS_NEXT = 2, HAS_NEXT_ORI = 4, FIX_ORI = 8 };

template <typename T>
struct v3 {
    T x, y, z;
};
template <typename T> inline v3<T> mk(T x, T y, T z) { return v3<T>{x, y, z}; }
template <typename T> inline v3<T> operator+(v3<T> a, v3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> inline v3<T> operator-(v3<T> a, v3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> inline v3<T> operator*(T s, v3<T> a) { return mk(s * a.x, s * a.y, s * a.z); }
template <typename T> inline v3<T> operator*(v3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <typename T> inline T dot(v3<T> a, v3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <typename T> inline T len2(v3<T> a) { return dot(a, a); }
template <typename T> inline T len(v3<T> a) { return std::sqrt(len2(a)); }
template <typename T> inline v3<T> cross(v3<T> a, v3<T> b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
// glm::mix(x, y, a) = x * (1 - a) + y * a
template <typename T> inline v3<T> mixv(v3<T> a, v3<T> b, T t) {
    const T o = T(1) - t;
    return mk(o * a.x + t * b.x, o * a.y + t * b.y, o * a.z + t * b.z);
}
template <typename T> inline T clampT(T v, T lo, T hi) { return std::min(std::max(v, lo), hi); }

// Rotor: x,y,z bivector part, w scalar (Rotor.h:11-20)
template <typename T>
struct rot {
    T x, y, z, w;
};
template <typename T> inline rot<T> rmul(rot<T> l, rot<T> r) {
    // Rotor.h:185-188: (l.w r.q + r.w l.q + l.q x r.q, l.w r.w - l.q . r.q)
    const v3<T> lq = mk(l.x, l.y, l.z), rq = mk(r.x, r.y, r.z);
    const v3<T> c = cross(lq, rq);
    return rot<T>{l.w * rq.x + r.w * lq.x + c.x, l.w * rq.y + r.w * lq.y + c.y, l.w * rq.z + r.w * lq.z + c.z,
                  l.w * r.w - dot(lq, rq)};
}
template <typename T> inline rot<T> rinv(rot<T> q) { return rot<T>{-q.x, -q.y, -q.z, q.w}; }
template <typename T> inline T rdot(rot<T> a, rot<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <typename T> inline T rlen(rot<T> a) { return std::sqrt(rdot(a, a)); }
template <typename T> inline rot<T> rscale(T s, rot<T> a) { return rot<T>{s * a.x, s * a.y, s * a.z, s * a.w}; }
template <typename T> inline rot<T> radd(rot<T> a, rot<T> b) { return rot<T>{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <typename T> inline v3<T> rrotate(rot<T> q, v3<T> v) {
    // Rotor.h:96-105
    const v3<T> qq = mk(q.x, q.y, q.z);
    const v3<T> a = q.w * v + cross(qq, v);
    const T c = dot(v, qq);
    return q.w * a + cross(qq, a) + c * qq;
}

// ---------------------------------------------------------------------------------------
// segmentClosestPoints(0, a1, b0, b1), Common.h:318-336, with the engine's optional FP64
// recomputation of the unconstrained parameter for near-parallel FP32 pairs.
template <typename T>
inline void closest(v3<T> a1, v3<T> b0, v3<T> b1, bool islands, T& u, T& v) {
    const v3<T> A1 = b1 - b0;
    const T a = len2(a1);
    const T b = dot(a1, A1);
    const T c = len2(A1);
    const T da = dot(a1, b0);
    const T db = dot(A1, b0);
    const T num = b * da - a * db;
    const T ac = a * c;
    const T den = ac - b * b;
    if (sizeof(T) == 4 && islands && den < T(1e-3f) * ac) {
        const v3<double> A = mk<double>(a1.x, a1.y, a1.z), E = mk<double>(A1.x, A1.y, A1.z),
                         B = mk<double>(b0.x, b0.y, b0.z);
        const double aa = len2(A), ab = dot(A, E), cc = len2(E), dda = dot(A, B), ddb = dot(E, B);
        v = (T)((ab * dda - aa * ddb) / (aa * cc - ab * ab));
    } else {
        v = num / den;
    }
    if (!std::isfinite(v)) v = T(0.5);
    v = clampT(v, T(0), T(1));
    u = clampT(dot(mixv(b0, b1, v), a1) / a, T(0), T(1));
    v = clampT(dot(u * a1 - b0, A1) / c, T(0), T(1));
}

template <typename T>
struct hs3 {  // hess3: diag xx,yy,zz then xy,xz,yz
    T d[6];
};
template <typename T> inline void hzero(hs3<T>& h) { for (auto& e : h.d) e = T(0); }
template <typename T> inline void hdiag(hs3<T>& h, T s) { h.d[0] += s; h.d[1] += s; h.d[2] += s; }
template <typename T> inline void houter(hs3<T>& h, v3<T> n, T s) {
    h.d[0] += (n.x * n.x) * s; h.d[1] += (n.y * n.y) * s; h.d[2] += (n.z * n.z) * s;
    h.d[3] += (n.x * n.y) * s; h.d[4] += (n.x * n.z) * s; h.d[5] += (n.y * n.z) * s;
}
// inverse(mat3(H)) * f as an explicit inverse (cofactors / determinant).
template <typename T> inline v3<T> hsolve(const hs3<T>& H, v3<T> f) {
    const T m00 = H.d[0], m11 = H.d[1], m22 = H.d[2], m01 = H.d[3], m02 = H.d[4], m12 = H.d[5];
    const T c00 = m11 * m22 - m12 * m12, c01 = m02 * m12 - m01 * m22, c02 = m01 * m12 - m11 * m02;
    const T c11 = m00 * m22 - m02 * m02, c12 = m01 * m02 - m00 * m12, c22 = m00 * m11 - m01 * m01;
    const T idet = T(1) / (m00 * c00 + m01 * c01 + m02 * c02);
    return mk((c00 * idet) * f.x + (c01 * idet) * f.y + (c02 * idet) * f.z,
              (c01 * idet) * f.x + (c11 * idet) * f.y + (c12 * idet) * f.z,
              (c02 * idet) * f.x + (c12 * idet) * f.y + (c22 * idet) * f.z);
}

template <typename T>
struct Par {  // per-scene parameters in working precision (same derivations as the engine)
    T h, lastH, invH, hh, gx, gy, gz, g2, dragFactor, D, accel, twoR, invb, kCol, fricK, fricMu, sdr, stepBase;
    bool useStepLimit, useVelRadius;
};

template <typename T>
Par<T> params_of(const orc_meta& m) {
    Par<T> p;
    p.h = (T)m.h;
    p.lastH = (T)m.lastH;
    p.invH = T(1) / p.h;
    p.hh = p.h * p.h;
    p.gx = (T)m.gravity[0]; p.gy = (T)m.gravity[1]; p.gz = (T)m.gravity[2];
    p.g2 = (p.gx * p.gx + p.gy * p.gy) + p.gz * p.gz;
    p.dragFactor = T(1) - (T)m.drag * p.h;
    p.D = (T)m.damping / p.h;
    p.accel = (T)m.accelerationRatio;
    p.twoR = T(2) * (T)m.radius;
    p.invb = T(1) / (T)m.barrierThickness;
    p.kCol = (T)m.kCollision * p.invb;
    p.fricK = (T)m.kFriction;
    p.fricMu = (T)m.frictionCoeff;
    const T dr = (T)m.radius + T(0.5f) * (T)m.barrierThickness;
    p.sdr = dr * (T)m.detectionScaler;
    p.stepBase = dr * ((T)m.detectionScaler - T(1));
    p.useStepLimit = m.useStepSizeLimit != 0;
    p.useVelRadius = m.useVelocityRadius != 0;
    return p;
}

struct SimBase {
    virtual ~SimBase() {}
    virtual void set_state(const orc_vertex*, const float*, const float*, const float*, const int32_t*, int,
                           const orc_meta*) = 0;
    virtual void set_meta(int, const orc_meta*) = 0;
    virtual void set_last_vel(const double*) = 0;
    virtual int advance(float dt, float maxH) = 0;
    virtual int phases(int mask, float h) = 0;
    virtual void get_state(double*, double*, double*, double*, double*) = 0;
    virtual void get_contacts(int32_t*, int32_t*, double*) = 0;
    virtual void diagnostics(double*) = 0;
    uint64_t stepCounter = 0;
    int64_t penetrations = 0;
};

template <typename T>
struct Sim : SimBase {
    int n;
    bool islands, kahan;
    std::vector<v3<T>> pos, posC, vel, lastVel, y, dx, dxn;
    std::vector<rot<T>> q, qn, qRest;
    std::vector<T> invMass, lRest, kStretch, stepLim;
    std::vector<int> cid, scene;
    std::vector<uint32_t> flags;
    std::vector<orc_meta> meta;
    std::vector<Par<T>> par;
    std::vector<std::vector<int>> cols;
    // per-segment contributions of one iteration
    std::vector<v3<T>> fA, fB;
    std::vector<hs3<T>> HA, HB;

    Sim(int n_, bool isl, bool kah) : n(n_), islands(isl), kahan(kah) {
        pos.resize(n); posC.assign(n, mk(T(0), T(0), T(0))); vel.resize(n); lastVel.assign(n, mk(T(0), T(0), T(0)));
        y.resize(n); dx.resize(n); dxn.resize(n); q.resize(n); qn.resize(n); qRest.resize(n);
        invMass.resize(n); lRest.resize(n); kStretch.resize(n); stepLim.assign(n, T(INFINITY));
        cid.resize(n); scene.assign(n, 0); flags.resize(n); cols.assign(n, {});
        fA.resize(n); fB.resize(n); HA.resize(n); HB.resize(n);
    }

    bool seg(int i) const { return (flags[i] & HAS_NEXT) != 0; }

    void set_state(const orc_vertex* V, const float* vels, const float* qs, const float* qr, const int32_t* sceneOf,
                   int numScenes, const orc_meta* m) override {
        for (int i = 0; i < n; i++) {
            pos[i] = mk<T>(V[i].pos[0], V[i].pos[1], V[i].pos[2]);
            posC[i] = mk(T(0), T(0), T(0));
            invMass[i] = V[i].invMass;
            lRest[i] = V[i].lRest;
            kStretch[i] = V[i].kStretch;
            cid[i] = V[i].connectionIndex;
            flags[i] = V[i].flags & 0xFFu;
            vel[i] = mk<T>(vels[3 * i], vels[3 * i + 1], vels[3 * i + 2]);
            q[i] = rot<T>{(T)qs[4 * i], (T)qs[4 * i + 1], (T)qs[4 * i + 2], (T)qs[4 * i + 3]};
            qRest[i] = rot<T>{(T)qr[4 * i], (T)qr[4 * i + 1], (T)qr[4 * i + 2], (T)qr[4 * i + 3]};
            scene[i] = sceneOf ? sceneOf[i] : 0;
        }
        // the last vertex of a scene never starts a segment
        for (int i = 0; i < n; i++)
            if (i == n - 1 || scene[i + 1] != scene[i]) flags[i] &= ~(HAS_NEXT | HAS_NEXT_ORI);
        meta.assign(m, m + numScenes);
        par.resize(numScenes);
        for (int s = 0; s < numScenes; s++) par[s] = params_of<T>(meta[s]);
    }

    void set_meta(int s, const orc_meta* m) override {
        meta[s] = *m;
        par[s] = params_of<T>(meta[s]);
    }

    void set_last_vel(const double* lv) override {
        for (int i = 0; i < n; i++) lastVel[i] = mk<T>((T)lv[3 * i], (T)lv[3 * i + 1], (T)lv[3 * i + 2]);
    }

    // initItr, iteration.cu:7-41
    void init_itr() {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            const Par<T>& p = par[scene[i]];
            const T h = p.h;
            const v3<T> v = vel[i];
            v3<T> d = h * v;
            const v3<T> lv = lastVel[i];
            lastVel[i] = v;
            const v3<T> g = mk(p.gx, p.gy, p.gz);
            y[i] = d + p.hh * g;
            if (invMass[i] != T(0)) {
                const T g2 = p.g2;
                if (g2 > T(0)) {
                    const v3<T> a = mk((v.x - lv.x) / p.lastH, (v.y - lv.y) / p.lastH, (v.z - lv.z) / p.lastH);
                    const T s = clampT(dot(a, g) / g2, T(0), T(1));
                    d = d + ((h * h) * s) * g;
                }
            }
            dx[i] = d;
        }
    }

    // buildAABBs, collision.cu:10-37
    void box(int k, T* mn, T* mx) const {
        const Par<T>& p = par[scene[k]];
        const v3<T> p0 = pos[k], p1 = pos[k + 1];
        T pad = p.sdr;
        if (p.useVelRadius) pad = pad + std::sqrt(std::max(len2(dx[k]), len2(dx[k + 1])));
        mn[0] = std::min(p0.x, p1.x) - pad; mn[1] = std::min(p0.y, p1.y) - pad; mn[2] = std::min(p0.z, p1.z) - pad;
        mx[0] = std::max(p0.x, p1.x) + pad; mx[1] = std::max(p0.y, p1.y) + pad; mx[2] = std::max(p0.z, p1.z) + pad;
    }

    // buildCollisionList's decision for x < y, collision.cu:45-77
    bool keep(int x, int yy) const {
        const int c0 = cid[x], c1 = cid[x + 1];
        if (c0 == yy || c1 == yy || c0 == yy + 1 || c1 == yy + 1) return false;
        if (std::abs(yy - x) <= 2) return false;
        const Par<T>& p = par[scene[x]];
        const v3<T> a0 = pos[x];
        const v3<T> a1 = pos[x + 1] - a0;
        const v3<T> b0 = pos[yy] - a0;
        const v3<T> b1 = pos[yy + 1] - a0;
        T u, v;
        closest(a1, b0, b1, islands, u, v);
        const v3<T> nrm = u * a1 - mixv(b0, b1, v);
        const T d2 = len2(nrm);
        T r = T(2) * p.sdr;
        if (p.useVelRadius) {
            r = r + std::sqrt(std::max(len2(dx[x]), len2(dx[x + 1])));
            r = r + std::sqrt(std::max(len2(dx[yy]), len2(dx[yy + 1])));
        }
        return d2 < r * r;
    }

    // Broadphase: uniform grid over the padded boxes, then the narrow-phase filter.
    int detect() {
        std::vector<int> segs;
        for (int i = 0; i < n; i++)
            if (seg(i)) segs.push_back(i);
        const int m = (int)segs.size();
        std::vector<T> bmn(3 * (size_t)m), bmx(3 * (size_t)m);
        double ext = 0, lo[3] = {INFINITY, INFINITY, INFINITY};
        for (int s = 0; s < m; s++) {
            box(segs[s], &bmn[3 * s], &bmx[3 * s]);
            for (int a = 0; a < 3; a++) {
                ext = std::max(ext, (double)bmx[3 * s + a] - (double)bmn[3 * s + a]);
                lo[a] = std::min(lo[a], (double)bmn[3 * s + a]);
            }
        }
        const double cs = ext * 1.01 + 1e-30;
        auto cellOf = [&](int s, int a) { return (int64_t)std::floor(((double)bmn[3 * s + a] - lo[a]) / cs); };
        auto key = [](int64_t x, int64_t y, int64_t z, int sc) {
            return ((uint64_t)(sc & 0x3FF) << 54) | ((uint64_t)(x & 0x3FFFF) << 36) | ((uint64_t)(y & 0x3FFFF) << 18) |
                   (uint64_t)(z & 0x3FFFF);
        };
        std::vector<std::pair<uint64_t, int>> cells(m);
        for (int s = 0; s < m; s++)
            cells[s] = {key(cellOf(s, 0), cellOf(s, 1), cellOf(s, 2), scene[segs[s]]), s};
        std::sort(cells.begin(), cells.end());
        std::vector<std::vector<int>> found(m);
        int overflow = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : overflow)
        for (int s = 0; s < m; s++) {
            const int k = segs[s];
            const int64_t cx = cellOf(s, 0), cy = cellOf(s, 1), cz = cellOf(s, 2);
            std::vector<int>& out = found[s];
            for (int dxc = -1; dxc <= 1; dxc++)
                for (int dyc = -1; dyc <= 1; dyc++)
                    for (int dzc = -1; dzc <= 1; dzc++) {
                        const uint64_t kk = key(cx + dxc, cy + dyc, cz + dzc, scene[k]);
                        auto it = std::lower_bound(cells.begin(), cells.end(), std::make_pair(kk, -1));
                        for (; it != cells.end() && it->first == kk; ++it) {
                            const int t = it->second;
                            const int j = segs[t];
                            if (j == k || scene[j] != scene[k]) continue;
                            bool ov = true;
                            for (int a = 0; a < 3; a++)
                                ov = ov && bmn[3 * s + a] <= bmx[3 * t + a] && bmn[3 * t + a] <= bmx[3 * s + a];
                            if (!ov) continue;
                            if (keep(std::min(j, k), std::max(j, k))) out.push_back(j);
                        }
                    }
            std::sort(out.begin(), out.end());
            if ((int)out.size() > MAXC) {
                overflow = 1;
                out.resize(MAXC);
            }
        }
        for (int i = 0; i < n; i++) cols[i].clear();
        for (int s = 0; s < m; s++) cols[segs[s]] = std::move(found[s]);
        return overflow;
    }

    // recomputeStepLimitKernel, collision.cu:121-159
    void step_limit() {
        int64_t pen = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pen)
        for (int k = 0; k < n; k++) {
            T m = T(INFINITY);
            if (seg(k)) {
                const Par<T>& p = par[scene[k]];
                const v3<T> a0 = pos[k];
                const v3<T> a1 = pos[k + 1] - a0;
                m = p.stepBase;
                if (p.useVelRadius) m = m + std::sqrt(len2(dx[k]));
                const T safe = (T(1) - T(0.1f)) * T(0.5f);
                for (int o : cols[k]) {
                    const v3<T> b0 = pos[o] - a0;
                    const v3<T> b1 = pos[o + 1] - a0;
                    T u, v;
                    closest(a1, b0, b1, islands, u, v);
                    const v3<T> nrm = u * a1 - mixv(b0, b1, v);
                    const T l = std::sqrt(len2(nrm));
                    m = std::min(m, safe * l);
                    if (o > k && l <= p.twoR) pen++;
                }
                if (!p.useStepLimit) m = T(INFINITY);
            }
            stepLim[k] = m;
        }
        penetrations += pen;
    }

    // Barrier terms (cosserat.cu:118-125); FP64 below d = 1e-2 in the mixed mode.
    void barrier(T d, const Par<T>& p, T& dH, T& ff) const {
        if (sizeof(T) == 4 && islands && d < T(1e-2)) {
            const double dd = d, invd = 1.0 / dd, logd = std::log(dd);
            dH = (T)((-3.0 + (2.0 + invd) * invd - 2.0 * logd) * (double)p.kCol * (double)p.invb);
            ff = (T)(-(1.0 - dd) * (dd - 1.0 + 2.0 * dd * logd) * invd * (double)p.kCol);
        } else {
            const T invd = T(1) / d;
            const T logd = std::log(d);
            dH = (T(-3) + (T(2) + invd) * invd - T(2) * logd) * p.kCol * p.invb;
            ff = -(T(1) - d) * (d - T(1) + T(2) * d * logd) * invd * p.kCol;
        }
    }

    // cosseratItr (cosserat.cu:20-207) as two strict-Jacobi passes: segment terms, then
    // the per-vertex gather and solve.
    void cosserat_itr() {
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; i++) {
            const Par<T>& p = par[scene[i]];
            const T D = p.D;
            v3<T> f = mk(T(0), T(0), T(0)), f2 = f;
            hs3<T> H, H2;
            hzero(H); hzero(H2);
            const v3<T> p0 = pos[i], d0 = dx[i];
            if (invMass[i] != T(0)) {
                hdiag(H, T(1) / (invMass[i] * p.h * p.h));
                f = (T(1) / (p.h * p.h * invMass[i])) * (y[i] - d0);
            }
            if (cid[i] >= 0) {
                const T stiff = T(40);
                const v3<T> pc = pos[cid[i]], dc = dx[cid[i]];
                f = f - stiff * ((p0 - pc) + (d0 - dc) + D * d0);
                hdiag(H, stiff * (T(1) + D));
            }
            if (seg(i)) {
                const v3<T> p1 = pos[i + 1], d1 = dx[i + 1];
                const T invl = T(1) / lRest[i];
                const v3<T> c = ((p1 - p0) + (d1 - d0)) * invl - rrotate(q[i], mk(T(1), T(0), T(0)));
                const T k = kStretch[i] * invl;
                T dd = k * invl;
                f = f + k * c - (D * dd) * d0;
                f2 = f2 + (-k) * c - (D * dd) * d1;
                dd = dd * (T(1) + D);
                hdiag(H, dd);
                hdiag(H2, dd);
                for (int j : cols[i]) {
                    const v3<T> b0 = pos[j], b1 = pos[j + 1], db0 = dx[j], db1 = dx[j + 1];
                    T u, v;
                    closest((p1 - p0) + (d1 - d0), (b0 - p0) + (db0 - d0), (b1 - p0) + (db1 - d0), islands, u, v);
                    const v3<T> dpos = mixv(p0, p1, u) - mixv(b0, b1, v);
                    const v3<T> ddpos = mixv(d0, d1, u) - mixv(db0, db1, v);
                    v3<T> nrm = dpos + ddpos;
                    const T dist = len(nrm);
                    nrm = nrm * (T(1) / dist);
                    const T wa = T(1) - u, wb = u;
                    T g = (dist - p.twoR) * p.invb;
                    if (g > T(1)) continue;
                    g = std::max(g, T(1e-3f));
                    T dH, ff;
                    barrier(g, p, dH, ff);
                    f = f + (ff * wa - D * dH * wa * wa * dot(nrm, d0)) * nrm;
                    f2 = f2 + (ff * wb - D * dH * wb * wb * dot(nrm, d1)) * nrm;
                    dH = dH * (T(1) + D);
                    houter(H, nrm, dH * wa * wa);
                    houter(H2, nrm, dH * wb * wb);
                    const v3<T> uu = ddpos - dot(nrm, ddpos) * nrm;
                    const T ul = len(uu);
                    if (ul > T(0)) {
                        const T f1 = std::min(p.fricK, p.fricMu * ff / ul);
                        f = f - (f1 * wa) * uu;
                        f2 = f2 - (f1 * wb) * uu;
                        const T sa = wa * wa * f1, sb = wb * wb * f1;
                        hdiag(H, sa); houter(H, nrm, -sa);
                        hdiag(H2, sb); houter(H2, nrm, -sb);
                    }
                }
            }
            fA[i] = f; HA[i] = H; fB[i] = f2; HB[i] = H2;
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            const Par<T>& p = par[scene[i]];
            v3<T> f = fA[i];
            hs3<T> H = HA[i];
            T sl = seg(i) ? stepLim[i] : T(INFINITY);
            if (flags[i] & HAS_PREV) {
                f = f + fB[i - 1];
                for (int e = 0; e < 6; e++) H.d[e] += HB[i - 1].d[e];
                sl = std::min(sl, stepLim[i - 1]);
            }
            v3<T> d = dx[i];
            if (invMass[i] != T(0)) {
                d = d + p.accel * hsolve(H, f);
                const T l = len(d);
                if (l > sl && l > T(0)) d = d * (sl / l);
            }
            dxn[i] = d;
        }
        dx.swap(dxn);
    }

    // quaternionLambdaItr, cosserat.cu:209-253 (strict Jacobi on the orientations)
    void quaternion_itr() {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            rot<T> q0 = q[i];
            const uint32_t fl = flags[i];
            if (!(fl & FIX_ORI) && (fl & HAS_NEXT)) {
                v3<T> v = ((pos[i + 1] - pos[i]) + (dx[i + 1] - dx[i])) * (T(1) / lRest[i]);
                v = (T(-2) * kStretch[i]) * v;
                rot<T> b{T(0), T(0), T(0), T(0)};
                if (fl & HAS_PREV) {
                    const rot<T> qr = qRest[i - 1], qq = q[i - 1];
                    const T s = rdot(rmul(rinv(qq), q0), qr) > T(0) ? T(1) : T(-1);
                    b = radd(b, rscale(s, rmul(qq, qr)));
                }
                if (fl & HAS_NEXT_ORI) {
                    const rot<T> qr = qRest[i], qq = q[i + 1];
                    const T s = rdot(rmul(rinv(q0), qq), qr) > T(0) ? T(1) : T(-1);
                    b = radd(b, rscale(s, rmul(qq, rinv(qr))));
                }
                // b = 0 (a yarn of one segment) makes the closed form 0/0; the orientation
                // is kept there (the reference's expression yields NaN).
                const T bl = rlen(b);
                if (bl > T(0)) {
                    const T lambda = len(v) + bl;
                    const rot<T> t = rmul(rmul(rot<T>{v.x, v.y, v.z, T(0)}, b), rot<T>{T(1), T(0), T(0), T(0)});
                    const rot<T> r = radd(t, rscale(lambda, b));
                    q0 = rscale(T(1) / rlen(r), r);
                }
            }
            qn[i] = q0;
        }
        q.swap(qn);
    }

    // endItr, iteration.cu:48-61 (Kahan-compensated position sum in the mixed mode)
    void end_itr() {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            const Par<T>& p = par[scene[i]];
            const v3<T> d = dx[i];
            if (invMass[i] != T(0)) vel[i] = mk(d.x * p.invH * p.dragFactor, d.y * p.invH * p.dragFactor, d.z * p.invH * p.dragFactor);
            if (kahan) {
                v3<T>& c = posC[i];
                const v3<T> yy = d - c;
                const v3<T> t = pos[i] + yy;
                c = (t - pos[i]) - yy;
                pos[i] = t;
            } else {
                pos[i] = pos[i] + d;
            }
        }
    }

    int num_itr() const {
        int it = 0;
        for (auto& m : meta) it = std::max(it, (int)m.numItr);
        return it;
    }

    int advance(float dt, float maxH) override {
        if (!(dt > 0)) return 0;
        const int steps = std::max(1, (int)std::ceil(dt / maxH));
        for (size_t s = 0; s < meta.size(); s++) {
            meta[s].lastH = meta[s].h;
            meta[s].h = dt / steps;
            orc_upload_meta(&meta[s]);
            par[s] = params_of<T>(meta[s]);
        }
        int err = 0;
        const int I = num_itr();
        for (int s = 0; s < steps; s++, stepCounter++) {
            init_itr();
            if (meta[0].detectionPeriod > 0 && stepCounter % (uint64_t)meta[0].detectionPeriod == 0) err |= detect();
            step_limit();
            for (int it = 0; it < I; it++) {
                cosserat_itr();
                quaternion_itr();
            }
            end_itr();
        }
        for (auto& m : meta) m.time += dt;
        return err;
    }

    int phases(int mask, float h) override {
        if (h > 0) {
            for (size_t s = 0; s < meta.size(); s++) {
                meta[s].lastH = meta[s].h;
                meta[s].h = h;
                orc_upload_meta(&meta[s]);
                par[s] = params_of<T>(meta[s]);
            }
        }
        int err = 0;
        if (mask & 1) init_itr();
        if (mask & 6) err |= detect();
        if (mask & 6) step_limit();
        if (mask & 8) step_limit();
        if (mask & 16) { cosserat_itr(); quaternion_itr(); }
        if (mask & 32) end_itr();
        return err;
    }

    void get_state(double* p, double* v, double* qq, double* d, double* lv) override {
        for (int i = 0; i < n; i++) {
            if (p) { p[3 * i] = pos[i].x; p[3 * i + 1] = pos[i].y; p[3 * i + 2] = pos[i].z; }
            if (v) { v[3 * i] = vel[i].x; v[3 * i + 1] = vel[i].y; v[3 * i + 2] = vel[i].z; }
            if (qq) { qq[4 * i] = q[i].x; qq[4 * i + 1] = q[i].y; qq[4 * i + 2] = q[i].z; qq[4 * i + 3] = q[i].w; }
            if (d) { d[4 * i] = dx[i].x; d[4 * i + 1] = dx[i].y; d[4 * i + 2] = dx[i].z; d[4 * i + 3] = 0; }
            if (lv) { lv[3 * i] = lastVel[i].x; lv[3 * i + 1] = lastVel[i].y; lv[3 * i + 2] = lastVel[i].z; }
        }
    }

    void get_contacts(int32_t* nc, int32_t* cl, double* sl) override {
        for (int i = 0; i < n; i++) {
            if (nc) nc[i] = (int32_t)cols[i].size();
            if (cl)
                for (size_t k = 0; k < cols[i].size(); k++) cl[i + (size_t)n * k] = cols[i][k];
            if (sl) sl[i] = (double)stepLim[i];
        }
    }

    // Same definitions as the engine's diagnostics (k_io.cu).
    void diagnostics(double* out) override {
        double e[8] = {0, 0, 0, 0, 0, 0, INFINITY, 0};
        for (int i = 0; i < n; i++) {
            const Par<T>& p = par[scene[i]];
            const double vx = vel[i].x, vy = vel[i].y, vz = vel[i].z;
            if (invMass[i] != T(0)) {
                const double m = 1.0 / (double)invMass[i];
                e[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
                e[1] += -m * ((double)p.gx * pos[i].x + (double)p.gy * pos[i].y + (double)p.gz * pos[i].z);
            }
            e[5] = std::max(e[5], std::sqrt(vx * vx + vy * vy + vz * vz));
            if (!seg(i)) continue;
            const rot<double> qd{(double)q[i].x, (double)q[i].y, (double)q[i].z, (double)q[i].w};
            const v3<double> t = rrotate(qd, mk(1.0, 0.0, 0.0));
            const double il = 1.0 / (double)lRest[i];
            const v3<double> c = mk(((double)pos[i + 1].x - pos[i].x) * il - t.x, ((double)pos[i + 1].y - pos[i].y) * il - t.y,
                                    ((double)pos[i + 1].z - pos[i].z) * il - t.z);
            e[2] += 0.5 * (double)kStretch[i] * len2(c);
            if (flags[i] & HAS_NEXT_ORI) {
                const rot<double> r{(double)qRest[i].x, (double)qRest[i].y, (double)qRest[i].z, (double)qRest[i].w};
                const rot<double> q1{(double)q[i + 1].x, (double)q[i + 1].y, (double)q[i + 1].z, (double)q[i + 1].w};
                e[3] += rlen(r) - std::fabs(rdot(rmul(qd, r), q1));
            }
            for (int j : cols[i]) {
                if (j < i) continue;
                const v3<double> a0 = mk<double>(pos[i].x, pos[i].y, pos[i].z), a1 = mk<double>(pos[i + 1].x, pos[i + 1].y, pos[i + 1].z);
                const v3<double> b0 = mk<double>(pos[j].x, pos[j].y, pos[j].z), b1 = mk<double>(pos[j + 1].x, pos[j + 1].y, pos[j + 1].z);
                double u, v;
                closest(a1 - a0, b0 - a0, b1 - a0, false, u, v);
                const double dist = len(mixv(a0, a1, u) - mixv(b0, b1, v));
                double g = (dist - (double)p.twoR) * (double)p.invb;
                e[6] = std::min(e[6], g);
                e[7] += 1.0;
                if (g < 1.0) {
                    g = std::max(g, 1e-3);
                    e[4] += -(double)p.kCol / (double)p.invb * (g - 1.0) * (g - 1.0) * std::log(g);
                }
            }
        }
        std::memcpy(out, e, sizeof(e));
    }
};

}  // namespace

struct orc_sim {
    SimBase* s;
};

extern "C" {

// ---- host setup (FP32, exactly as the reference host code) ----------------------------
static inline rot<float> from_to(v3<float> from, v3<float> to) {
    // Rotor::fromTo, Rotor.h:57-64; orthoBasisX (Common.h:235-251) when from == -to
    v3<float> h = (from + to) * 0.5f;
    const float l = len2(h);
    if (l > 0) {
        h = h * (1.0f / std::sqrt(l));
    } else {
        const v3<float> nn = from;
        if (nn.z >= nn.y) {
            const float a = 1.0f / (1.0f + nn.z);
            const float b = -nn.x * nn.y * a;
            h = mk(b, 1.0f - nn.y * nn.y * a, -nn.y);
        } else {
            const float a = 1.0f / (1.0f + nn.y);
            const float b = -nn.x * nn.z * a;
            h = mk(1.0f - nn.x * nn.x * a, -nn.x, b);
        }
    }
    const v3<float> c = cross(from, h);
    return rot<float>{c.x, c.y, c.z, dot(from, h)};
}

// The oracle's FP32 math helpers over arrays, with the argument layout of the reference-kernel
// harness (oracle/refbuild/ref_host.cpp, ref_math) so that tests can compare them bit for bit:
// op 0 closest points (a0, a1, b0, b1 -> uv; relative to a0, as every kernel calls it),
// 1 rotor product, 2 rotor rotation, 3 fromTo, 4 rotor normalisation, 5 hess3 outer-product
// update and local solve.
int orc_math(int op, int n, const float* a, const float* b, const float* c, const float* d, float* out, float* out2) {
    for (int i = 0; i < n; i++) {
        switch (op) {
            case 0: {
                const float* p = a + 12 * (size_t)i;
                const v3<float> a0 = mk(p[0], p[1], p[2]);
                float u, v;
                closest(mk(p[3], p[4], p[5]) - a0, mk(p[6], p[7], p[8]) - a0, mk(p[9], p[10], p[11]) - a0, false, u, v);
                out[2 * i] = u;
                out[2 * i + 1] = v;
                break;
            }
            case 1: {
                const float* l = a + 4 * (size_t)i;
                const float* r = b + 4 * (size_t)i;
                const rot<float> q = rmul(rot<float>{l[0], l[1], l[2], l[3]}, rot<float>{r[0], r[1], r[2], r[3]});
                out[4 * i] = q.x; out[4 * i + 1] = q.y; out[4 * i + 2] = q.z; out[4 * i + 3] = q.w;
                break;
            }
            case 2: {
                const float* q = a + 4 * (size_t)i;
                const float* v = b + 3 * (size_t)i;
                const v3<float> r = rrotate(rot<float>{q[0], q[1], q[2], q[3]}, mk(v[0], v[1], v[2]));
                out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
                break;
            }
            case 3: {
                const float* f = a + 3 * (size_t)i;
                const float* t = b + 3 * (size_t)i;
                const rot<float> q = from_to(mk(f[0], f[1], f[2]), mk(t[0], t[1], t[2]));
                out[4 * i] = q.x; out[4 * i + 1] = q.y; out[4 * i + 2] = q.z; out[4 * i + 3] = q.w;
                break;
            }
            case 4: {
                const float* v = a + 4 * (size_t)i;
                const rot<float> r{v[0], v[1], v[2], v[3]};
                const rot<float> q = rscale(1.0f / rlen(r), r);
                out[4 * i] = q.x; out[4 * i + 1] = q.y; out[4 * i + 2] = q.z; out[4 * i + 3] = q.w;
                break;
            }
            case 5: {
                hs3<float> H;
                for (int k = 0; k < 6; k++) H.d[k] = a[6 * (size_t)i + k];
                const float* nn = b + 3 * (size_t)i;
                houter(H, mk(nn[0], nn[1], nn[2]), c[i]);
                for (int k = 0; k < 6; k++) out[6 * (size_t)i + k] = H.d[k];
                const float* f = d + 3 * (size_t)i;
                const v3<float> x = hsolve(H, mk(f[0], f[1], f[2]));
                out2[3 * i] = x.x; out2[3 * i + 1] = x.y; out2[3 * i + 2] = x.z;
                break;
            }
            default:
                return -2;
        }
    }
    return 0;
}

int orc_configure(int n, float density, orc_vertex* verts, float* qs, float* qRests, float* initialInvMasses,
                  float* maxSegLen, float* minSegLen) {
    float mx = 0, mn = FLT_MAX;
    verts[n - 1].flags &= ~(uint32_t)(HAS_NEXT | HAS_NEXT_ORI);
    verts[0].flags &= ~(uint32_t)HAS_PREV;
    rot<float> lastQ{0, 0, 0, 1};
    for (int i = 0; i < n; i++) {
        orc_vertex& v = verts[i];
        if (i < n - 1) {
            const bool hasNext = (v.flags & HAS_NEXT) != 0;
            verts[i + 1].flags = hasNext ? (verts[i + 1].flags | HAS_PREV) : (verts[i + 1].flags & ~(uint32_t)HAS_PREV);
            const bool hasNextNext = hasNext && (verts[i + 1].flags & HAS_NEXT);
            v.flags = hasNextNext ? (v.flags | HAS_NEXT_ORI) : (v.flags & ~(uint32_t)HAS_NEXT_ORI);
            if (!hasNext) v.flags |= FIX_ORI;
        }
        if (!(v.flags & HAS_PREV) && !(v.flags & HAS_NEXT)) return 4;
        v.lRest = 1.f / n;
        float mass = 0;
        if (v.flags & HAS_PREV) mass += verts[i - 1].lRest;
        if (v.flags & HAS_NEXT) {
            const v3<float> seg0 = mk(verts[i + 1].pos[0], verts[i + 1].pos[1], verts[i + 1].pos[2]) -
                                   mk(v.pos[0], v.pos[1], v.pos[2]);
            v.lRest = len(seg0);
            if (v.lRest == 0 || !std::isfinite(v.lRest)) return 5;
            const v3<float> dir = seg0 * (1.0f / std::sqrt(len2(seg0)));
            const rot<float> qq = from_to(mk(1.f, 0.f, 0.f), dir);
            rot<float> t = rmul(rinv(qq), lastQ);
            t = rot<float>{t.x, 0.f, 0.f, t.w};
            t = rscale(1.0f / rlen(t), t);
            lastQ = rmul(qq, t);
            mass += v.lRest;
            mx = std::max(mx, v.lRest);
            mn = std::min(mn, v.lRest);
        }
        qs[4 * i] = lastQ.x; qs[4 * i + 1] = lastQ.y; qs[4 * i + 2] = lastQ.z; qs[4 * i + 3] = lastQ.w;
        mass *= 0.5f * density;
        if (mass != 0)
            v.invMass *= 1 / mass;
        else
            v.invMass = 0;
        if (initialInvMasses) initialInvMasses[i] = v.invMass;
    }
    for (int i = 0; i < n - 1; i++) {
        const rot<float> a{qs[4 * i], qs[4 * i + 1], qs[4 * i + 2], qs[4 * i + 3]};
        const rot<float> b{qs[4 * i + 4], qs[4 * i + 5], qs[4 * i + 6], qs[4 * i + 7]};
        const rot<float> r{qRests[4 * i], qRests[4 * i + 1], qRests[4 * i + 2], qRests[4 * i + 3]};
        const rot<float> o = rscale(rlen(r), rmul(rinv(a), b));
        qRests[4 * i] = o.x; qRests[4 * i + 1] = o.y; qRests[4 * i + 2] = o.z; qRests[4 * i + 3] = o.w;
    }
    if (maxSegLen) *maxSegLen = mx;
    if (minSegLen) *minSegLen = mn;
    return 0;
}

void orc_set_kstretch(int n, orc_vertex* verts, float k) {
    for (int i = 0; i < n; i++) verts[i].kStretch = k * verts[i].lRest;
}

void orc_set_kbend(int n, const orc_vertex* verts, float* qr, float k) {
    k *= 4;
    for (int i = 0; i < n; i++) {
        rot<float> r{qr[4 * i], qr[4 * i + 1], qr[4 * i + 2], qr[4 * i + 3]};
        r = rscale(1.0f / rlen(r), r);
        r = rscale(k / verts[i].lRest, r);
        qr[4 * i] = r.x; qr[4 * i + 1] = r.y; qr[4 * i + 2] = r.z; qr[4 * i + 3] = r.w;
    }
}

int orc_upload_meta(orc_meta* m) {
    m->detectionRadius = m->radius + 0.5f * m->barrierThickness;
    m->scaledDetectionRadius = m->detectionRadius * m->detectionScaler;
    if (m->detectionScaler <= 1) return 6;
    if (2 * m->minSegLen < 2 * m->radius + m->barrierThickness) return 7;
    return 0;
}

orc_sim* orc_create(int n, int mode) {
    orc_sim* s = new orc_sim();
    if (mode == ORC_FP64)
        s->s = new Sim<double>(n, false, false);
    else if (mode == ORC_FP32)
        s->s = new Sim<float>(n, false, false);
    else
        s->s = new Sim<float>(n, true, true);
    return s;
}

void orc_destroy(orc_sim* s) {
    if (!s) return;
    delete s->s;
    delete s;
}

void orc_set_state(orc_sim* s, const orc_vertex* verts, const float* vels, const float* qs, const float* qRests,
                   const int32_t* sceneOf, int numScenes, const orc_meta* meta) {
    s->s->set_state(verts, vels, qs, qRests, sceneOf, numScenes, meta);
}
void orc_set_meta(orc_sim* s, int scene, const orc_meta* meta) { s->s->set_meta(scene, meta); }
void orc_set_last_vel(orc_sim* s, const double* lv) { s->s->set_last_vel(lv); }
void orc_set_schedule(orc_sim* s, uint64_t stepCounter) { s->s->stepCounter = stepCounter; }
int orc_advance(orc_sim* s, float dt, float maxH) { return s->s->advance(dt, maxH); }
int orc_phases(orc_sim* s, int mask, float h) { return s->s->phases(mask, h); }
void orc_get_state(orc_sim* s, double* pos, double* vel, double* q, double* dx, double* lastVel) {
    s->s->get_state(pos, vel, q, dx, lastVel);
}
void orc_get_contacts(orc_sim* s, int32_t* numCols, int32_t* cols, double* stepLimit) {
    s->s->get_contacts(numCols, cols, stepLimit);
}
void orc_diagnostics(orc_sim* s, double out[8]) { s->s->diagnostics(out); }
int64_t orc_penetrations(orc_sim* s) { return s->s->penetrations; }
void orc_set_threads(int t) { omp_set_num_threads(t > 0 ? t : 1); }
int orc_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
