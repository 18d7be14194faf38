// scenes.cpp - seeded synthetic yarn geometry for the benchmark and test workloads.
//
// No reference counterpart: the reference reads curves from .bcc/.obj/.poly files
// (KittenEngine/YarnBall/io/reader.cpp); the workloads here are synthetic random walks:
//   * RNG: SplitMix64 expands the seed into the state of xoshiro256** (Blackman & Vigna);
//     normal deviates by Box-Muller;
//   * a yarn starts uniformly in the cube with a uniform direction; each step of length
//     segLen turns the direction by an angle ~ N(0, turnSigma) about a uniformly random
//     perpendicular axis; a step that would leave the cube has the offending direction
//     components reflected (so every segment keeps length segLen);
//   * a step is rejected when the new segment comes closer than minDist to any existing
//     segment other than its two predecessors on the same yarn (uniform-grid search);
//     after maxTries rejections in a row the walk backtracks, and a yarn that keeps failing
//     is discarded and restarted.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

#include "yarnball_b200_scenes.h"

namespace {

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t& x) {
        uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
        for (auto& v : s) v = splitmix(seed);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    double normal() {
        const double u1 = 1.0 - uniform();  // (0,1]
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct D3 {
    double x, y, z;
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline D3 unit(D3 a) { return (1.0 / std::sqrt(dot(a, a))) * a; }
inline double get(const D3& a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
inline void set(D3& a, int i, double v) { (i == 0 ? a.x : (i == 1 ? a.y : a.z)) = v; }

// Distance between segments [p0,p1] and [q0,q1] (clamped closest points, FP64).
double seg_dist(D3 p0, D3 p1, D3 q0, D3 q1) {
    const D3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
    const double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    double s, t;
    const double c = dot(d1, r), b = dot(d1, d2), den = a * e - b * b;
    s = den > 1e-300 ? std::fmin(std::fmax((b * f - c * e) / den, 0.0), 1.0) : 0.0;
    t = (b * s + f) / e;
    if (t < 0.0) {
        t = 0.0;
        s = std::fmin(std::fmax(-c / a, 0.0), 1.0);
    } else if (t > 1.0) {
        t = 1.0;
        s = std::fmin(std::fmax((b - c) / a, 0.0), 1.0);
    }
    const D3 cp = (p0 + s * d1) - (q0 + t * d2);
    return std::sqrt(dot(cp, cp));
}

struct Grid {
    double cell;
    std::unordered_map<uint64_t, std::vector<int>> cells;
    static uint64_t key(int64_t x, int64_t y, int64_t z) {
        return ((uint64_t)(x & 0x1FFFFF) << 42) | ((uint64_t)(y & 0x1FFFFF) << 21) | (uint64_t)(z & 0x1FFFFF);
    }
    int64_t c(double v) const { return (int64_t)std::floor(v / cell); }
    template <typename F>
    void for_cells(D3 a, D3 b, double pad, F f) const {
        const int64_t x0 = c(std::fmin(a.x, b.x) - pad), x1 = c(std::fmax(a.x, b.x) + pad);
        const int64_t y0 = c(std::fmin(a.y, b.y) - pad), y1 = c(std::fmax(a.y, b.y) + pad);
        const int64_t z0 = c(std::fmin(a.z, b.z) - pad), z1 = c(std::fmax(a.z, b.z) + pad);
        for (int64_t x = x0; x <= x1; x++)
            for (int64_t y = y0; y <= y1; y++)
                for (int64_t z = z0; z <= z1; z++) f(key(x, y, z));
    }
};

// Generates one scene; returns 0 or -1 when a yarn could not be placed.  When a step
// fails maxTries times in a row the walk backtracks (drops its last few vertices, more
// on repeated failures) before giving up on the yarn and restarting it.
int walk_scene(uint64_t seed, int numYarns, const int* vertsPerYarn, double segLen, double cube, double sigma,
               double minDist, int maxTries, int maxRestarts, float* out) {
    Rng rng(seed);
    Grid g;
    g.cell = segLen + minDist;
    std::vector<D3> s0, s1;   // segment endpoints
    std::vector<int> yarnOf;  // owning yarn attempt id
    std::vector<int> segPos;  // index of the segment within its yarn
    std::vector<char> alive;
    size_t o = 0;
    int attemptId = 0;
    for (int y = 0; y < numYarns; y++) {
        const int m = vertsPerYarn[y];
        bool placed = false;
        for (int restart = 0; restart <= maxRestarts && !placed; restart++) {
            const int id = attemptId++;
            std::vector<D3> pts, dirs;
            std::vector<int> segIds;  // global segment id of segment v-1 (ending at vertex v)
            pts.reserve(m);
            D3 p{cube * rng.uniform(), cube * rng.uniform(), cube * rng.uniform()};
            D3 dir = unit(D3{rng.normal(), rng.normal(), rng.normal()});
            pts.push_back(p);
            dirs.push_back(dir);
            int backtracks = 0, depth = 4;
            bool ok = true;
            while ((int)pts.size() < m) {
                const int v = (int)pts.size();
                p = pts.back();
                dir = dirs.back();
                bool stepOk = false;
                for (int t = 0; t < maxTries && !stepOk; t++) {
                    const double th = sigma * rng.normal();
                    D3 r{rng.normal(), rng.normal(), rng.normal()};
                    D3 ax = r - dot(r, dir) * dir;
                    const double al = std::sqrt(dot(ax, ax));
                    if (!(al > 1e-12)) continue;
                    ax = (1.0 / al) * ax;
                    D3 nd = unit(std::cos(th) * dir + std::sin(th) * cross(ax, dir));
                    D3 q = p + segLen * nd;
                    for (int a = 0; a < 3; a++) {
                        if (get(q, a) < 0.0 || get(q, a) > cube) set(nd, a, -get(nd, a));
                    }
                    q = p + segLen * nd;
                    bool clash = false;
                    const int segIdx = v - 1;  // index of the new segment within this yarn
                    g.for_cells(p, q, minDist, [&](uint64_t k) {
                        if (clash) return;
                        auto it = g.cells.find(k);
                        if (it == g.cells.end()) return;
                        for (int sidx : it->second) {
                            if (!alive[sidx]) continue;
                            if (yarnOf[sidx] == id && segPos[sidx] >= segIdx - 2) continue;
                            if (seg_dist(p, q, s0[sidx], s1[sidx]) < minDist) {
                                clash = true;
                                return;
                            }
                        }
                    });
                    if (clash) continue;
                    const int sidx = (int)s0.size();
                    s0.push_back(p);
                    s1.push_back(q);
                    yarnOf.push_back(id);
                    segPos.push_back(segIdx);
                    alive.push_back(1);
                    g.for_cells(p, q, 0.0, [&](uint64_t k) { g.cells[k].push_back(sidx); });
                    pts.push_back(q);
                    dirs.push_back(nd);
                    segIds.push_back(sidx);
                    stepOk = true;
                }
                if (!stepOk) {
                    if (++backtracks > 400) {
                        ok = false;
                        break;
                    }
                    const int drop = std::min((int)pts.size() - 1, depth);
                    for (int k = 0; k < drop; k++) {
                        alive[segIds.back()] = 0;
                        segIds.pop_back();
                        pts.pop_back();
                        dirs.pop_back();
                    }
                    depth = std::min(depth * 2, 256);
                } else if (depth > 4 && (int)pts.size() % 64 == 0) {
                    depth /= 2;
                }
            }
            if (ok) {
                placed = true;
                for (int v = 0; v < m; v++) {
                    out[3 * (o + v)] = (float)pts[v].x;
                    out[3 * (o + v) + 1] = (float)pts[v].y;
                    out[3 * (o + v) + 2] = (float)pts[v].z;
                }
                o += m;
            } else {
                for (int sidx : segIds) alive[sidx] = 0;
            }
        }
        if (!placed) return -1;
    }
    return 0;
}

}  // namespace

extern "C" {

int yb_scene_random_walks(uint64_t seed, int32_t numYarns, const int32_t* vertsPerYarn, float segLen, float cube,
                          float turnSigma, float minDist, float* posOut) {
    if (numYarns < 0 || (numYarns > 0 && (!vertsPerYarn || !posOut)) || !(segLen > 0) || !(cube > 4 * segLen))
        return -2;
    for (int y = 0; y < numYarns; y++)
        if (vertsPerYarn[y] < 2) return -2;
    return walk_scene(seed, numYarns, vertsPerYarn, segLen, cube, turnSigma, minDist, 64, 64, posOut);
}

int yb_scene_random_walks_batch(uint64_t seed, int32_t numScenes, const int32_t* yarnsPerScene,
                                const int32_t* vertsPerYarn, float segLen, float cube, float turnSigma, float minDist,
                                float* posOut, int32_t threads) {
    if (numScenes < 0 || (numScenes > 0 && (!yarnsPerScene || !vertsPerYarn || !posOut))) return -2;
    std::vector<size_t> yarnOff(numScenes + 1, 0), vertOff(numScenes + 1, 0);
    for (int s = 0; s < numScenes; s++) {
        yarnOff[s + 1] = yarnOff[s] + yarnsPerScene[s];
        size_t v = 0;
        for (size_t y = yarnOff[s]; y < yarnOff[s + 1]; y++) {
            if (vertsPerYarn[y] < 2) return -2;
            v += vertsPerYarn[y];
        }
        vertOff[s + 1] = vertOff[s] + v;
    }
    int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    std::vector<int> status(numScenes, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; t++) {
        pool.emplace_back([&, t]() {
            for (int s = t; s < numScenes; s += nt) {
                // Scene s is seeded by (seed, s) so that its geometry does not depend on the
                // thread count or on the other scenes.
                uint64_t mix = seed ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(s + 1));
                status[s] = walk_scene(Rng::splitmix(mix), yarnsPerScene[s], vertsPerYarn + yarnOff[s], segLen,
                                       cube, turnSigma, minDist, 64, 64, posOut + 3 * vertOff[s]);
            }
        });
    }
    for (auto& th : pool) th.join();
    for (int s = 0; s < numScenes; s++)
        if (status[s] != 0) return -1 - s;
    return 0;
}

uint64_t yb_rng_u64(uint64_t seed, int32_t index) {
    Rng r(seed);
    uint64_t v = 0;
    for (int i = 0; i <= index; i++) v = r.next();
    return v;
}

}  // extern "C"
