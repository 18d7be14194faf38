// mesher.cu - fibre mesh export, Sim::exportFiberMesh (io/fiberMesher.cpp:9-157).
//
// Every yarn segment is drawn as 8 twisted fibres (Catmull-Rom centre line through the
// segment's neighbours, frame blended between the neighbouring rotors, fibres orbiting the
// centre line with a twist of 1200 rad/m and a random frizz) plus random fuzz strands, written
// as OBJ polylines ("o fiber", then "o fuzz").  The reference draws its random numbers from one
// sequential stream in a fixed order, and the number of fuzz strands of a segment is itself a
// draw, so the host replays that stream exactly (xoroshiro128+ seeded by chained SplitMix64,
// seed 0x12345678) together with the running twist angle (a sequential float sum reduced
// modulo 2 pi); the GPU then evaluates every fibre and fuzz vertex in parallel, and host
// threads format the text in order.  Counts, indices and the random stream match the
// reference exactly; positions agree to float rounding (the GPU's sin/cos and the host's).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "yarnball_b200.h"
#include "ybmath.cuh"

namespace yb {
void set_io_error(const std::string& msg);  // curves.cpp

namespace {

constexpr int NUM_FIBERS = 8;

// The reference mesher's random stream (Blackman & Vigna's xoroshiro128+ with rotations
// 24 / 16 / 37; the state is two chained SplitMix64 outputs of the seed).
struct MeshRng {
    uint64_t s0, s1;
    static uint64_t splitmix(uint64_t v) {
        uint64_t z = v + 0x9e3779b97f4a7c15ull;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    explicit MeshRng(uint64_t seed) {
        s0 = splitmix(seed);
        s1 = splitmix(s0);
    }
    uint64_t next() {
        const uint64_t r = s0 + s1;
        s1 ^= s0;
        s0 = rotl(s0, 24) ^ s1 ^ (s1 << 16);
        s1 = rotl(s1, 37);
        return r;
    }
    // low 32 bits over (float)UINT32_MAX, clamped to [0, 1]
    float uniform() {
        const float x = (float)(uint32_t)next() / (float)UINT32_MAX;
        return x < 0.f ? 0.f : (x > 1.f ? 1.f : x);
    }
};

struct MeshParams {
    float fiberFrizz, fiberTwist, fiberOrbit, fuzzLength;
};

struct SegIn {  // one segment with its Catmull-Rom neighbours and frames
    float pa[3], p0[3], p1[3], pb[3];
    float q0[4], q1[4], q2[4];
    float lRest, twist;  // rest length, running twist angle at the segment start
    int numH;            // fibre vertices along the segment
};

__device__ inline V3<float> cmr3(const float* a, const float* b, const float* c, const float* d, float t) {
    // Kit::cmrSpline in float: repeated linear interpolation
    auto mix = [](float x, float y, float s) { return x * (1.f - s) + y * s; };
    float r[3];
    for (int i = 0; i < 3; i++) {
        const float a0 = mix(a[i], b[i], t + 1), a1 = mix(b[i], c[i], t + 0), a2 = mix(c[i], d[i], t - 1);
        const float b0 = mix(a0, a1, (t + 1) * 0.5f), b1 = mix(a1, a2, (t + 0) * 0.5f);
        r[i] = mix(b0, b1, t);
    }
    return V3<float>(r[0], r[1], r[2]);
}

// Frame at parameter t: the segment's rotor blended toward the previous (t < 0.5) or the next
// one, as normalize(mix(q_a.v, q_b.v, s)).
__device__ inline Q<float> frame_at(const SegIn& s, float t) {
    const float* a = t < 0.5f ? s.q0 : s.q1;
    const float* b = t < 0.5f ? s.q1 : s.q2;
    const float w = t < 0.5f ? t + 0.5f : t - 0.5f;
    float v[4];
    float n2 = 0.f;
    for (int i = 0; i < 4; i++) {
        v[i] = a[i] * (1.f - w) + b[i] * w;
    }
    n2 = (v[0] * v[0] + v[1] * v[1]) + (v[2] * v[2] + v[3] * v[3]);
    const float inv = 1.f / sqrtf(n2);
    return qmk(v[0] * inv, v[1] * inv, v[2] * inv, v[3] * inv);
}

// One thread per (fibre, segment): its numH vertices, written at out[base ...].
__global__ void k_fibers(const SegIn* __restrict__ segs, int nseg, const int* __restrict__ base,
                         const float* __restrict__ frizz, MeshParams mp, float3* __restrict__ out) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nseg * NUM_FIBERS) return;
    const int fid = id / nseg, si = id % nseg;
    const SegIn s = segs[si];
    const int b0 = base[id];
    const float twoPi = 2.f * 3.14159265358979323846f;
    for (int hi = 0; hi < s.numH; hi++) {
        const float t = hi / (float)s.numH;
        const V3<float> pos = cmr3(s.pa, s.p0, s.p1, s.pb, t);
        const Q<float> fr = frame_at(s, t);
        float ang = s.twist + mp.fiberTwist * t * s.lRest;
        ang += fid / (float)NUM_FIBERS * twoPi;
        V3<float> tw(0.f, cosf(ang), sinf(ang));
        tw = mp.fiberOrbit * tw;
        if (hi) {
            const float* r = frizz + 3 * (size_t)(b0 + hi);
            tw = tw + mp.fiberFrizz * V3<float>(r[0] * 2.f - 1.f, r[1] * 2.f - 1.f, r[2] * 2.f - 1.f);
        }
        const V3<float> w = pos + qrotate(fr, tw);
        out[b0 + hi] = make_float3(w.x, w.y, w.z);
    }
}

// One thread per fuzz strand: its two vertices.
__global__ void k_fuzz(const SegIn* __restrict__ segs, const int* __restrict__ fuzzSeg, int nfuzz,
                       const float* __restrict__ draws, MeshParams mp, float3* __restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfuzz) return;
    const SegIn s = segs[fuzzSeg[f]];
    const float* r = draws + 8 * (size_t)f;  // t, fuzzDir xyz, offset xyz, length
    const float t = r[0];
    const V3<float> pos = cmr3(s.pa, s.p0, s.p1, s.pb, t);
    const Q<float> fr = frame_at(s, t);
    V3<float> dir(r[1] * 2.f - 1.f, r[2] * 2.f - 1.f, r[3] * 2.f - 1.f);
    V3<float> off = dir + V3<float>(r[4] * 2.f - 1.f, r[5] * 2.f - 1.f, r[6] * 2.f - 1.f);
    off.x *= 0.1f;
    const float ol = sqrtf((off.x * off.x + off.y * off.y) + off.z * off.z);
    off = (0.9f * mp.fiberOrbit) * ((1.f / ol) * off);
    dir = (mp.fuzzLength * (0.8f + 0.2f * r[7])) * dir;
    const V3<float> w0 = pos + qrotate(fr, off);
    const V3<float> w1 = pos + qrotate(fr, dir + off);
    out[2 * (size_t)f] = make_float3(w0.x, w0.y, w0.z);
    out[2 * (size_t)f + 1] = make_float3(w1.x, w1.y, w1.z);
}

template <typename T>
cudaError_t to_device(T** d, const std::vector<T>& h) {
    *d = nullptr;
    if (h.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(d, sizeof(T) * h.size());
    if (e == cudaSuccess) e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return e;
}

void append_v(std::string& s, const float3& p) {
    char buf[96];
    const int m = std::snprintf(buf, sizeof(buf), "v %.8f %.8f %.8f\n", p.x, p.y, p.z);
    s.append(buf, (size_t)m);
}

}  // namespace
}  // namespace yb

using namespace yb;

extern "C" yb_status yb_export_fiber_mesh(yb_sim* sim, const char* path) {
    if (!sim || !path) return YB_ERR_INVALID_ARGUMENT;
    yb_meta m;
    yb_status st = yb_get_meta(sim, 0, &m);
    if (st != YB_OK) return st;
    FILE* file = std::fopen(path, "w");
    if (!file) {
        set_io_error("Failed to open file for writing");
        return YB_ERR_IO;
    }
    std::fputs("o fiber\n", file);
    st = yb_download(sim);
    if (st != YB_OK) {
        std::fclose(file);
        return st;
    }
    yb_vertex* v = nullptr;
    float *qs = nullptr, *qr = nullptr, *vel = nullptr;
    yb_host_arrays(sim, &v, &qs, &qr, &vel);
    int32_t n = 0, ns = 0, prec = 0;
    yb_info(sim, &n, &ns, &prec);

    // constants of fiberMesher.cpp:14-30
    const float r = m.radius + 0.5f * m.barrierThickness;
    const float fiberFrizz = 0.2f * r, fiberTwist = 1200.f, fuzzDensity = 1.25e4f, fuzzLength = 1.f * r;
    const float fiberRadius = 0.6f * r / std::sqrt((float)NUM_FIBERS);
    const float heightSegLen = 0.3f * r;
    const float fiberOrbit = 0.9f * r - fiberRadius - fiberFrizz;
    const float twoPi = 2.f * 3.14159265358979323846f;

    // segments in vertex order, with neighbours, frames, vertex counts and the running twist
    std::vector<SegIn> segs;
    std::vector<int> segOf(n, -1);
    float curTwist = 0.f;
    for (int i = 0; i < n; i++) {
        if (!(v[i].flags & YB_HAS_NEXT)) continue;
        SegIn s;
        const int a = (v[i].flags & YB_HAS_PREV) ? i - 1 : i;
        const int b = (v[i + 1].flags & YB_HAS_NEXT) ? i + 2 : i + 1;
        std::memcpy(s.pa, v[a].pos, 12);
        std::memcpy(s.p0, v[i].pos, 12);
        std::memcpy(s.p1, v[i + 1].pos, 12);
        std::memcpy(s.pb, v[b].pos, 12);
        std::memcpy(s.q1, qs + 4 * (size_t)i, 16);
        std::memcpy(s.q0, (v[i].flags & YB_HAS_PREV) ? qs + 4 * (size_t)(i - 1) : s.q1, 16);
        std::memcpy(s.q2, (v[i + 1].flags & YB_HAS_NEXT) ? qs + 4 * (size_t)(i + 1) : s.q1, 16);
        s.lRest = v[i].lRest;
        s.numH = std::max((int)std::ceil(v[i].lRest / heightSegLen), 1);
        s.twist = curTwist;
        curTwist += fiberTwist * v[i].lRest;
        curTwist = curTwist - twoPi * std::floor(curTwist / twoPi);  // glm::mod
        segOf[i] = (int)segs.size();
        segs.push_back(s);
    }
    const int nseg = (int)segs.size();

    // the random stream, in the reference's order: fibre frizz, then fuzz
    MeshRng rng(0x12345678ull);
    std::vector<int> base((size_t)nseg * NUM_FIBERS);
    size_t fiberVerts = 0;
    for (int fid = 0; fid < NUM_FIBERS; fid++)
        for (int si = 0; si < nseg; si++) {
            base[(size_t)fid * nseg + si] = (int)fiberVerts;
            fiberVerts += segs[si].numH;
        }
    if (fiberVerts > (size_t)INT32_MAX / 3) {
        std::fclose(file);
        return YB_ERR_INVALID_ARGUMENT;
    }
    std::vector<float> frizz(3 * fiberVerts, 0.f);
    for (int fid = 0; fid < NUM_FIBERS; fid++)
        for (int si = 0; si < nseg; si++) {
            const int b0 = base[(size_t)fid * nseg + si];
            for (int hi = 1; hi < segs[si].numH; hi++)
                for (int c = 0; c < 3; c++) frizz[3 * (size_t)(b0 + hi) + c] = rng.uniform();
        }
    std::vector<int> fuzzSeg;
    std::vector<float> fuzzDraws;
    for (int si = 0; si < nseg; si++) {
        const int nf = (int)std::round(2 * rng.uniform() * segs[si].lRest * fuzzDensity);
        for (int f = 0; f < nf; f++) {
            fuzzSeg.push_back(si);
            for (int c = 0; c < 8; c++) fuzzDraws.push_back(rng.uniform());
        }
    }
    const int nfuzz = (int)fuzzSeg.size();

    // geometry on the GPU
    std::vector<float3> fib(fiberVerts), fz(2 * (size_t)nfuzz);
    SegIn* dSegs = nullptr;
    int *dBase = nullptr, *dFuzzSeg = nullptr;
    float *dFrizz = nullptr, *dDraws = nullptr;
    float3 *dFib = nullptr, *dFz = nullptr;
    const MeshParams mp{fiberFrizz, fiberTwist, fiberOrbit, fuzzLength};
    cudaError_t e = to_device(&dSegs, segs);
    if (e == cudaSuccess) e = to_device(&dBase, base);
    if (e == cudaSuccess) e = to_device(&dFrizz, frizz);
    if (e == cudaSuccess) e = to_device(&dFuzzSeg, fuzzSeg);
    if (e == cudaSuccess) e = to_device(&dDraws, fuzzDraws);
    if (e == cudaSuccess && fiberVerts) e = cudaMalloc(&dFib, sizeof(float3) * fiberVerts);
    if (e == cudaSuccess && nfuzz) e = cudaMalloc(&dFz, sizeof(float3) * 2 * (size_t)nfuzz);
    if (e == cudaSuccess && nseg) {
        k_fibers<<<(nseg * NUM_FIBERS + 127) / 128, 128>>>(dSegs, nseg, dBase, dFrizz, mp, dFib);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && nfuzz) {
        k_fuzz<<<(nfuzz + 127) / 128, 128>>>(dSegs, dFuzzSeg, nfuzz, dDraws, mp, dFz);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && fiberVerts) e = cudaMemcpy(fib.data(), dFib, sizeof(float3) * fiberVerts, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nfuzz) e = cudaMemcpy(fz.data(), dFz, sizeof(float3) * 2 * (size_t)nfuzz, cudaMemcpyDeviceToHost);
    cudaFree(dSegs); cudaFree(dBase); cudaFree(dFrizz); cudaFree(dFuzzSeg); cudaFree(dDraws);
    cudaFree(dFib); cudaFree(dFz);
    if (e != cudaSuccess) {
        std::fclose(file);
        return e == cudaErrorMemoryAllocation ? YB_ERR_OUT_OF_MEMORY : YB_ERR_CUDA;
    }

    // text, in the reference's order: per fibre, each yarn's vertices then its polyline
    struct Unit {  // one yarn of one fibre
        int fid, first, last;  // vertex range [first, last] of the yarn (last = vertex without hasNext)
    };
    std::vector<Unit> units;
    for (int fid = 0; fid < NUM_FIBERS; fid++) {
        int start = 0;
        for (int i = 0; i < n; i++)
            if (!(v[i].flags & YB_HAS_NEXT)) {
                units.push_back({fid, start, i});
                start = i + 1;
            }
        if (start < n) units.push_back({fid, start, -1});  // trailing segments without an end vertex
    }
    auto fmt_unit = [&](const Unit& u, std::string& out) {
        const int lastV = u.last < 0 ? n - 1 : u.last;
        int vs = -1, ve = -1;  // OBJ indices (0-based) of this unit's vertices
        for (int i = u.first; i <= lastV; i++) {
            if (!(v[i].flags & YB_HAS_NEXT)) continue;
            const int si = segOf[i];
            const int b0 = base[(size_t)u.fid * nseg + si];
            if (vs < 0) vs = b0;
            ve = b0 + segs[si].numH;
            for (int hi = 0; hi < segs[si].numH; hi++) append_v(out, fib[b0 + hi]);
        }
        if (u.last >= 0 && vs >= 0 && ve - vs > 2) {
            out += "l";
            char buf[24];
            for (int k = vs; k < ve; k++) {
                const int m2 = std::snprintf(buf, sizeof(buf), " %d", k + 1);
                out.append(buf, (size_t)m2);
            }
            out += "\n";
        }
    };
    const int nthreads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    auto parallel_text = [&](size_t count, auto&& body) {
        std::vector<std::string> parts(nthreads);
        std::vector<std::thread> th;
        for (int t = 0; t < nthreads; t++)
            th.emplace_back([&, t] {
                const size_t a = count * t / nthreads, b = count * (t + 1) / nthreads;
                for (size_t k = a; k < b; k++) body(k, parts[t]);
            });
        for (auto& x : th) x.join();
        bool ok = true;
        for (auto& p : parts) ok = ok && std::fwrite(p.data(), 1, p.size(), file) == p.size();
        return ok;
    };
    bool ok = parallel_text(units.size(), [&](size_t k, std::string& out) { fmt_unit(units[k], out); });
    ok = ok && std::fputs("o fuzz\n", file) >= 0;
    ok = ok && parallel_text((size_t)nfuzz, [&](size_t f, std::string& out) {
        append_v(out, fz[2 * f]);
        append_v(out, fz[2 * f + 1]);
        char buf[48];
        const long long a = (long long)fiberVerts + 2 * (long long)f;
        const int m2 = std::snprintf(buf, sizeof(buf), "l %lld %lld\n", a + 1, a + 2);
        out.append(buf, (size_t)m2);
    });
    std::fclose(file);
    return ok ? YB_OK : YB_ERR_IO;
}
