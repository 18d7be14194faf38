// ref_host.cpp - host side that runs the reference's own simulator kernels on the GPU
// (test infrastructure; built by oracle/refbuild/build.py into oracle/_ref/libyb_ref.so).
//
// The kernels come unchanged from the reference (see ref_device.cu), loaded from a fatbin with
// the CUDA runtime's library API.  This file restates the host side of the reference's
// schedule around them - the parts GCC cannot compile from the reference itself:
//   device allocation and upload      YarnBall.cu:159-200, 226-262 (configure, uploadMeta, upload)
//   Sim::advance                      sim/step.cpp:36-55 (substeps, detection cadence)
//   Sim::detectCollisions             sim/collision.cu:94-119 (AABBs, BVH query, lists)
//   Sim::recomputeStepLimit           sim/collision.cu:161-171
//   Sim::iterateCosserat              sim/cosserat.cu:255-258 (launch shapes)
//   Sim::startIterate / endIterate    sim/iteration.cu:43-45, 63-65
//   Sim::checkErrors                  YarnBall.cu:276-304
// with the same launch shapes, in the same order, on one stream (the reference's graph holds
// the step limit, the iterations and the advection; launching them directly is equivalent).
// The host arrays (vertices after configure, rotors, rest rotors) are the caller's: the tests
// take them from the oracle's restatement of configure.  The BVH query is the brute-force
// stand-in refk_pairs (ref_device.cu); a query with no candidate pair launches no list kernel
// (the reference would launch an empty grid, which its error check turns into an exit).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../yb_oracle.h"

namespace {

constexpr int MAXC = 128;  // MAX_COLLISIONS_PER_SEGMENT, YarnBall.h:20

// The reference's MetaData: 14 device pointers (YarnBall.h:64-79), then the parameter fields,
// whose order and types are orc_meta's.  Checked against the compiled layout at load time.
struct MetaHost {
    void* d_verts;
    void* d_qs;
    void* d_qRests;
    void* d_dx;
    void* d_vels;
    void* d_lastVels;
    void* d_lastPos;
    void* d_lastFlags;
    void* d_lastCID;
    void* d_numCols;
    void* d_maxStepSize;
    void* d_collisions;
    void* d_bounds;
    void* d_boundColList;
    orc_meta p;
};

struct Lib {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t initItr, endItr, aabbs[2], lists[2], limit[2][2], cosserat, quaternion, copyTemp, pairs;
    cudaKernel_t closest, rmul, rrotate, rfromto, norm4, hess3;
    std::string error;
};

std::mutex g_mu;
std::vector<std::pair<std::string, Lib*>> g_libs;  // loaded fatbins by path
std::string g_err;

Lib* lib_at(int id) {
    std::lock_guard<std::mutex> lock(g_mu);
    return id >= 0 && id < (int)g_libs.size() ? g_libs[id].second : nullptr;
}

bool get(Lib* L, cudaKernel_t* k, const char* name) {
    if (cudaLibraryGetKernel(k, L->lib, name) != cudaSuccess) {
        cudaGetLastError();
        L->error = std::string("kernel not found: ") + name;
        return false;
    }
    return true;
}

// Itanium names of the reference's kernels (namespace YarnBall; MetaData and Vertex are typedef
// names of unnamed structs, which name them for linkage).
bool resolve(Lib* L) {
    return get(L, &L->initItr, "_ZN8YarnBall7initItrEPNS_8MetaDataE") &&
           get(L, &L->endItr, "_ZN8YarnBall6endItrEPNS_8MetaDataE") &&
           get(L, &L->aabbs[0], "_ZN8YarnBall10buildAABBsILb0EEEvPNS_8MetaDataEPi") &&
           get(L, &L->aabbs[1], "_ZN8YarnBall10buildAABBsILb1EEEvPNS_8MetaDataEPi") &&
           get(L, &L->lists[0], "_ZN8YarnBall18buildCollisionListILb0EEEvPNS_8MetaDataEiPi") &&
           get(L, &L->lists[1], "_ZN8YarnBall18buildCollisionListILb1EEEvPNS_8MetaDataEiPi") &&
           get(L, &L->limit[0][0], "_ZN8YarnBall24recomputeStepLimitKernelILb0ELb0EEEvPNS_8MetaDataE") &&
           get(L, &L->limit[0][1], "_ZN8YarnBall24recomputeStepLimitKernelILb0ELb1EEEvPNS_8MetaDataE") &&
           get(L, &L->limit[1][0], "_ZN8YarnBall24recomputeStepLimitKernelILb1ELb0EEEvPNS_8MetaDataE") &&
           get(L, &L->limit[1][1], "_ZN8YarnBall24recomputeStepLimitKernelILb1ELb1EEEvPNS_8MetaDataE") &&
           get(L, &L->cosserat, "_ZN8YarnBall11cosseratItrEPNS_8MetaDataE") &&
           get(L, &L->quaternion, "_ZN8YarnBall19quaternionLambdaItrEPNS_8MetaDataE") &&
           get(L, &L->copyTemp, "_ZN8YarnBall12copyTempDataEPNS_6VertexEPjPii") &&
           get(L, &L->pairs, "refk_pairs") && get(L, &L->closest, "refk_closest") &&
           get(L, &L->rmul, "refk_rotor_mul") && get(L, &L->rrotate, "refk_rotor_rotate") &&
           get(L, &L->rfromto, "refk_rotor_from_to") && get(L, &L->norm4, "refk_normalize4") &&
           get(L, &L->hess3, "refk_hess3");
}

bool check_layout(Lib* L) {
    void* p = nullptr;
    size_t bytes = 0;
    if (cudaLibraryGetGlobal(&p, &bytes, L->lib, "refk_layout") != cudaSuccess || bytes != 10 * 8) {
        cudaGetLastError();
        L->error = "refk_layout missing";
        return false;
    }
    unsigned long long lay[10];
    if (cudaMemcpy(lay, p, sizeof(lay), cudaMemcpyDeviceToHost) != cudaSuccess) {
        L->error = "refk_layout unreadable";
        return false;
    }
    const unsigned long long want[10] = {sizeof(MetaHost), offsetof(MetaHost, p), 32, 24, 16, 12, 8,
                                         offsetof(MetaHost, d_boundColList),
                                         offsetof(MetaHost, p) + offsetof(orc_meta, useVelocityRadius), MAXC};
    for (int i = 0; i < 10; i++)
        if (lay[i] != want[i]) {
            char b[128];
            snprintf(b, sizeof(b), "reference layout entry %d is %llu, expected %llu", i, lay[i], want[i]);
            L->error = b;
            return false;
        }
    return true;
}

#define RCK(x)                                                       \
    do {                                                             \
        cudaError_t e_ = (x);                                        \
        if (e_ != cudaSuccess) {                                     \
            g_err = std::string(#x) + ": " + cudaGetErrorString(e_); \
            return -1;                                               \
        }                                                            \
    } while (0)

struct RefSim {
    Lib* L;
    int n;
    MetaHost m{};
    MetaHost* d_meta = nullptr;
    int* d_error = nullptr;
    unsigned long long* d_count = nullptr;
    float maxH = 1e-3f;
    float lastBVHRebuild = std::numeric_limits<float>::infinity();
    uint64_t stepCounter = 0;
    int lastErrorCode = 0, lastWarningCode = 0;
    bool truncated = false;
    uint64_t pairCandidates = 0;
    cudaStream_t st = 0;

    int launch(cudaKernel_t k, int grid, int block, void** args) {
        if (grid <= 0) return 0;
        RCK(cudaLaunchKernel((const void*)k, dim3(grid), dim3(block), args, 0, st));
        return 0;
    }
    int upload_meta() {
        // YarnBall.cu:226-237 (the parameter checks are the caller's: the oracle's orc_upload_meta)
        m.p.detectionRadius = m.p.radius + 0.5f * m.p.barrierThickness;
        m.p.scaledDetectionRadius = m.p.detectionRadius * m.p.detectionScaler;
        RCK(cudaMemcpyAsync(d_meta, &m, sizeof(MetaHost), cudaMemcpyHostToDevice, st));
        RCK(cudaStreamSynchronize(st));
        return 0;
    }
    int start_iterate() {
        void* a[] = {&d_meta};
        return launch(L->initItr, (n + 255) / 256, 256, a);
    }
    int end_iterate() {
        void* a[] = {&d_meta};
        return launch(L->endItr, (n + 255) / 256, 256, a);
    }
    int detect() {
        const int vr = m.p.useVelocityRadius ? 1 : 0;
        void* a[] = {&d_meta, &d_error};
        if (launch(L->aabbs[vr], (n + 255) / 256, 256, a)) return -1;
        if (lastBVHRebuild >= m.p.bvhRebuildPeriod) lastBVHRebuild = 0;
        else lastBVHRebuild += m.p.h * m.p.detectionPeriod;
        // stand-in query into d_boundColList (capacity n * MAXC ints = n * 64 pairs)
        unsigned long long cap = (unsigned long long)n * (MAXC / 2);
        RCK(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st));
        void* b[] = {&m.d_bounds, &n, &m.d_boundColList, &cap, &d_count};
        if (launch(L->pairs, (n + 255) / 256, 256, b)) return -1;
        unsigned long long cnt = 0;
        RCK(cudaMemcpyAsync(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost, st));
        RCK(cudaStreamSynchronize(st));
        pairCandidates = cnt;
        truncated = truncated || cnt > cap;
        int numCols = (int)(cnt > cap ? cap : cnt);
        RCK(cudaMemsetAsync(m.d_numCols, 0, sizeof(int) * n, st));
        void* c[] = {&d_meta, &numCols, &d_error};
        return launch(L->lists[vr], (numCols + 127) / 128, 128, c);
    }
    int step_limit() {
        void* a[] = {&d_meta};
        return launch(L->limit[m.p.useStepSizeLimit ? 1 : 0][m.p.useVelocityRadius ? 1 : 0], (n + 127) / 128, 128, a);
    }
    int iterate() {
        void* a[] = {&d_meta};
        if (launch(L->cosserat, (n + 64 - 2) / (64 - 1), 128, a)) return -1;
        return launch(L->quaternion, (n + 127) / 128, 128, a);
    }
    int check_errors() {
        RCK(cudaGetLastError());
        int e[2];
        RCK(cudaMemcpyAsync(e, d_error, sizeof(e), cudaMemcpyDeviceToHost, st));
        RCK(cudaStreamSynchronize(st));
        if (e[0] != 0) lastErrorCode = e[0];
        if (e[1] != 0) lastWarningCode = e[1];
        if (e[0] || e[1]) RCK(cudaMemsetAsync(d_error, 0, sizeof(e), st));
        return e[0] == 1 ? 8 : (e[0] != 0 ? 11 : 0);
    }
    int advance(float dt) {
        if (!(dt > 0)) return 0;
        const int steps = std::max(1, (int)std::ceil(dt / maxH));
        m.p.lastH = m.p.h;
        m.p.h = dt / steps;
        if (upload_meta()) return -1;
        for (int s = 0; s < steps; s++, stepCounter++) {
            if (start_iterate()) return -1;
            if (m.p.detectionPeriod > 0 && stepCounter % (uint64_t)m.p.detectionPeriod == 0)
                if (detect()) return -1;
            if (step_limit()) return -1;
            for (int i = 0; i < m.p.numItr; i++)
                if (iterate()) return -1;
            if (end_iterate()) return -1;
        }
        m.p.time += dt;
        return check_errors();
    }
};

int library(const char* fatbinPath) {
    std::lock_guard<std::mutex> lock(g_mu);
    for (size_t i = 0; i < g_libs.size(); i++)
        if (g_libs[i].first == fatbinPath) return (int)i;
    FILE* f = fopen(fatbinPath, "rb");
    if (!f) {
        g_err = std::string("cannot open ") + fatbinPath;
        return -1;
    }
    std::vector<char> img;
    char buf[1 << 16];
    size_t r;
    while ((r = fread(buf, 1, sizeof(buf), f)) > 0) img.insert(img.end(), buf, buf + r);
    fclose(f);
    Lib* L = new Lib();
    if (cudaLibraryLoadData(&L->lib, img.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
        g_err = std::string("cudaLibraryLoadData: ") + cudaGetErrorString(cudaGetLastError());
        delete L;
        return -1;
    }
    if (!resolve(L) || !check_layout(L)) {
        g_err = L->error;
        cudaLibraryUnload(L->lib);
        delete L;
        return -1;
    }
    g_libs.push_back({fatbinPath, L});
    return (int)g_libs.size() - 1;
}

int alloc(void** p, size_t bytes) {
    RCK(cudaMalloc(p, bytes));
    return 0;
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// Loads the reference kernels from fatbinPath (once per path and process); returns the
// library id (>= 0) for ref_create / ref_math, or -1 (ref_last_error has the reason).
int ref_init(const char* fatbinPath) { return library(fatbinPath); }

void ref_destroy(void* h);

// A reference simulation of n vertices from configured host arrays (32-byte vertices, 3 floats
// of velocity, 4 of rotor and of rest rotor per vertex) and its parameters; NULL on failure.
void* ref_create(int lib, int n, const orc_vertex* verts, const float* vels, const float* qs, const float* qRests,
                 const orc_meta* meta, float maxH) {
    Lib* L = lib_at(lib);
    if (!L || n < 3) return nullptr;
    RefSim* s = new RefSim();
    s->L = L;
    s->n = n;
    s->m.p = *meta;
    s->m.p.numVerts = n;
    s->maxH = maxH;
    const size_t N = (size_t)n;
    int bad = 0;
    bad |= alloc((void**)&s->d_meta, sizeof(MetaHost));
    bad |= alloc((void**)&s->d_error, 2 * sizeof(int));
    bad |= alloc((void**)&s->d_count, sizeof(unsigned long long));
    bad |= alloc(&s->m.d_dx, 12 * N);
    bad |= alloc(&s->m.d_verts, 32 * N);
    bad |= alloc(&s->m.d_qs, 16 * N);
    bad |= alloc(&s->m.d_lastVels, 12 * N);
    bad |= alloc(&s->m.d_vels, 12 * N);
    bad |= alloc(&s->m.d_qRests, 16 * N);
    bad |= alloc(&s->m.d_lastPos, 12 * N);
    bad |= alloc(&s->m.d_lastCID, 4 * N);
    bad |= alloc(&s->m.d_lastFlags, 4 * N);
    bad |= alloc(&s->m.d_maxStepSize, 4 * N);
    bad |= alloc(&s->m.d_numCols, 4 * N);
    bad |= alloc(&s->m.d_collisions, 4 * N * MAXC);
    bad |= alloc(&s->m.d_bounds, 24 * N);
    bad |= alloc(&s->m.d_boundColList, 4 * N * MAXC);
    if (bad) {
        ref_destroy(s);
        return nullptr;
    }
    cudaMemset(s->d_error, 0, 2 * sizeof(int));
    cudaMemset(s->m.d_lastVels, 0, 12 * N);
    cudaMemset(s->m.d_numCols, 0, 4 * N);
    // upload (YarnBall.cu:247-254)
    cudaMemcpy(s->m.d_verts, verts, 32 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(s->m.d_vels, vels, 12 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(s->m.d_qs, qs, 16 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(s->m.d_qRests, qRests, 16 * N, cudaMemcpyHostToDevice);
    void* a[] = {&s->m.d_verts, &s->m.d_lastFlags, &s->m.d_lastCID, &s->n};
    if (s->upload_meta() || s->launch(s->L->copyTemp, (n + 511) / 512, 512, a) ||
        cudaDeviceSynchronize() != cudaSuccess) {
        if (g_err.empty()) g_err = cudaGetErrorString(cudaGetLastError());
        ref_destroy(s);
        return nullptr;
    }
    return s;
}

void ref_destroy(void* h) {
    RefSim* s = (RefSim*)h;
    if (!s) return;
    cudaDeviceSynchronize();
    void* ptrs[] = {s->d_meta, s->d_error, s->d_count, s->m.d_dx, s->m.d_verts, s->m.d_qs, s->m.d_lastVels,
                    s->m.d_vels, s->m.d_qRests, s->m.d_lastPos, s->m.d_lastCID, s->m.d_lastFlags,
                    s->m.d_maxStepSize, s->m.d_numCols, s->m.d_collisions, s->m.d_bounds, s->m.d_boundColList};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete s;
}

// Sim::advance(dt): 0, 8 (MAX_COLLISIONS_PER_SEGMENT exceeded) or -1 (CUDA error).
int ref_advance(void* h, float dt) { return ((RefSim*)h)->advance(dt); }

// One phase of a substep: 0 set h (lastH = h_old, h = value, uploadMeta), 1 initItr,
// 2 detectCollisions, 3 recomputeStepLimit, 4 one iterateCosserat, 5 endItr.  Synchronises.
int ref_phase(void* hnd, int phase, float value) {
    RefSim* s = (RefSim*)hnd;
    int r = 0;
    switch (phase) {
        case 0:
            s->m.p.lastH = s->m.p.h;
            s->m.p.h = value;
            r = s->upload_meta();
            break;
        case 1: r = s->start_iterate(); break;
        case 2: r = s->detect(); break;
        case 3: r = s->step_limit(); break;
        case 4: r = s->iterate(); break;
        case 5: r = s->end_iterate(); break;
        default: return -2;
    }
    if (r) return r;
    RCK(cudaStreamSynchronize(s->st));
    RCK(cudaGetLastError());
    return 0;
}

// Copies a device array to host memory: 0 dx (3n floats), 1 vels (3n; holds y between initItr
// and endItr), 2 lastVels (3n), 3 lastPos (3n), 4 numCols (n ints), 5 collisions (n*128 ints,
// entry k of segment i at i + n*k), 6 maxStepSize (n floats), 7 qs (4n floats), 8 verts
// (n 32-byte vertices).
int ref_read(void* hnd, int what, void* out) {
    RefSim* s = (RefSim*)hnd;
    const size_t N = (size_t)s->n;
    const void* src[] = {s->m.d_dx, s->m.d_vels, s->m.d_lastVels, s->m.d_lastPos, s->m.d_numCols,
                         s->m.d_collisions, s->m.d_maxStepSize, s->m.d_qs, s->m.d_verts};
    const size_t bytes[] = {12 * N, 12 * N, 12 * N, 12 * N, 4 * N, 4 * N * MAXC, 4 * N, 16 * N, 32 * N};
    if (what < 0 || what > 8) return -2;
    RCK(cudaStreamSynchronize(s->st));
    RCK(cudaMemcpy(out, src[what], bytes[what], cudaMemcpyDeviceToHost));
    return 0;
}

// Replaces device state arrays (vertices, velocities, previous velocities, rotors) with host
// copies, e.g. to start a substep from another simulation's state; NULL leaves one unchanged.
int ref_write_state(void* hnd, const orc_vertex* verts, const float* vels, const float* lastVels, const float* qs) {
    RefSim* s = (RefSim*)hnd;
    const size_t N = (size_t)s->n;
    RCK(cudaStreamSynchronize(s->st));
    if (verts) RCK(cudaMemcpy(s->m.d_verts, verts, 32 * N, cudaMemcpyHostToDevice));
    if (vels) RCK(cudaMemcpy(s->m.d_vels, vels, 12 * N, cudaMemcpyHostToDevice));
    if (lastVels) RCK(cudaMemcpy(s->m.d_lastVels, lastVels, 12 * N, cudaMemcpyHostToDevice));
    if (qs) RCK(cudaMemcpy(s->m.d_qs, qs, 16 * N, cudaMemcpyHostToDevice));
    return 0;
}

int ref_get_meta(void* hnd, orc_meta* out) {
    *out = ((RefSim*)hnd)->m.p;
    return 0;
}
int ref_set_meta(void* hnd, const orc_meta* in) {
    RefSim* s = (RefSim*)hnd;
    const int n = s->m.p.numVerts;
    s->m.p = *in;
    s->m.p.numVerts = n;
    return s->upload_meta();
}
void ref_info(void* hnd, uint64_t* stepCounter, int* lastError, int* lastWarning, int* truncated,
              uint64_t* pairCandidates) {
    RefSim* s = (RefSim*)hnd;
    if (stepCounter) *stepCounter = s->stepCounter;
    if (lastError) *lastError = s->lastErrorCode;
    if (lastWarning) *lastWarning = s->lastWarningCode;
    if (truncated) *truncated = s->truncated ? 1 : 0;
    if (pairCandidates) *pairCandidates = s->pairCandidates;
}

// advance(dt) `frames` times between CUDA events on the simulation's stream; *ms receives the
// device time.  Returns as ref_advance.
int ref_time_advance(void* hnd, float dt, int frames, float* ms) {
    RefSim* s = (RefSim*)hnd;
    cudaEvent_t e0, e1;
    RCK(cudaEventCreate(&e0));
    RCK(cudaEventCreate(&e1));
    RCK(cudaEventRecord(e0, s->st));
    int r = 0;
    for (int f = 0; f < frames && r == 0; f++) r = s->advance(dt);
    RCK(cudaEventRecord(e1, s->st));
    RCK(cudaEventSynchronize(e1));
    float t = 0.f;
    RCK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t;
    return r;
}

// The reference's math helpers evaluated on the device over n inputs (host arrays in and out):
// op 0 segmentClosestPoints (12 floats in -> 2 out), 1 rotor product (4 + 4 -> 4), 2 rotor
// rotation (4 + 3 -> 3), 3 Rotor::fromTo (3 + 3 -> 4), 4 normalize(vec4) (4 -> 4),
// 5 hess3 (h 6 + n 3 + s 1 + f 3 -> H 6 + solve 3).
int ref_math(int lib, int op, int n, const float* a, const float* b, const float* c, const float* d, float* out,
             float* out2) {
    Lib* L = lib_at(lib);
    if (!L || n <= 0) return -1;
    static const int inW[6][4] = {{12, 0, 0, 0}, {4, 4, 0, 0}, {4, 3, 0, 0}, {3, 3, 0, 0}, {4, 0, 0, 0}, {6, 3, 1, 3}};
    static const int outW[6][2] = {{2, 0}, {4, 0}, {3, 0}, {4, 0}, {4, 0}, {6, 3}};
    if (op < 0 || op > 5) return -2;
    const float* in[4] = {a, b, c, d};
    float* dIn[4] = {nullptr, nullptr, nullptr, nullptr};
    float* dOut[2] = {nullptr, nullptr};
    for (int k = 0; k < 4; k++)
        if (inW[op][k]) {
            RCK(cudaMalloc(&dIn[k], sizeof(float) * inW[op][k] * (size_t)n));
            RCK(cudaMemcpy(dIn[k], in[k], sizeof(float) * inW[op][k] * (size_t)n, cudaMemcpyHostToDevice));
        }
    for (int k = 0; k < 2; k++)
        if (outW[op][k]) RCK(cudaMalloc(&dOut[k], sizeof(float) * outW[op][k] * (size_t)n));
    const dim3 grid((n + 127) / 128), block(128);
    cudaError_t e;
    switch (op) {
        case 0: { void* args[] = {&dIn[0], &dOut[0], &n}; e = cudaLaunchKernel((const void*)L->closest, grid, block, args, 0, 0); break; }
        case 1: { void* args[] = {&dIn[0], &dIn[1], &dOut[0], &n}; e = cudaLaunchKernel((const void*)L->rmul, grid, block, args, 0, 0); break; }
        case 2: { void* args[] = {&dIn[0], &dIn[1], &dOut[0], &n}; e = cudaLaunchKernel((const void*)L->rrotate, grid, block, args, 0, 0); break; }
        case 3: { void* args[] = {&dIn[0], &dIn[1], &dOut[0], &n}; e = cudaLaunchKernel((const void*)L->rfromto, grid, block, args, 0, 0); break; }
        case 4: { void* args[] = {&dIn[0], &dOut[0], &n}; e = cudaLaunchKernel((const void*)L->norm4, grid, block, args, 0, 0); break; }
        default: { void* args[] = {&dIn[0], &dIn[1], &dIn[2], &dIn[3], &dOut[0], &dOut[1], &n}; e = cudaLaunchKernel((const void*)L->hess3, grid, block, args, 0, 0); break; }
    }
    RCK(e);
    RCK(cudaDeviceSynchronize());
    RCK(cudaMemcpy(out, dOut[0], sizeof(float) * outW[op][0] * (size_t)n, cudaMemcpyDeviceToHost));
    if (outW[op][1]) RCK(cudaMemcpy(out2, dOut[1], sizeof(float) * outW[op][1] * (size_t)n, cudaMemcpyDeviceToHost));
    for (float* p : dIn)
        if (p) cudaFree(p);
    for (float* p : dOut)
        if (p) cudaFree(p);
    return 0;
}

}  // extern "C"
