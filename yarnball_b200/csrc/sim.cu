// sim.cu - host side of the substep engine and the C ABI (include/yarnball_b200.h).
//
// Reference interfaces replaced here (KittenEngine/YarnBall/...):
//   Sim::Sim / ~Sim                     YarnBall.cu:11-85
//   Sim::configure                      YarnBall.cu:91-200
//   Sim::setKStretch / setKBend         YarnBall.cu:202-224
//   Sim::uploadMeta                     YarnBall.cu:226-237
//   Sim::upload / download / zeroVel    YarnBall.cu:239-274
//   Sim::checkErrors                    YarnBall.cu:276-304
//   Sim::rebuildCUDAGraph / advance     sim/step.cpp:5-59
//   Sim::detectCollisions               sim/collision.cu:94-119
//   Sim::printCollisionStats            sim/statistics.cpp:5-23
//
// One substep on the device is: predictor -> [detection: BVH rebuild or refit, traversal
// (+ step limit)] or [step limit] -> numItr fused Newton/orientation iterations ->
// advection.  No step reads anything back to the host (the reference's BVH query returns
// its pair count to the host every detection); each of the three substep shapes is captured
// once as a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "yarnball_b200.h"
#include "engine.cuh"
#include "io.cuh"

using namespace yb;

namespace {

constexpr int GRAPH_TYPES = 3;  // 0: detect + rebuild, 1: detect + refit, 2: no detection

struct EngineBase {
    virtual ~EngineBase() {}
    virtual yb_status upload() = 0;
    virtual yb_status download() = 0;
    virtual yb_status zero_vel() = 0;
    virtual void write_params() = 0;
    virtual uint64_t enqueue_substep(bool detect, bool rebuild, unsigned long long* slots = nullptr) = 0;
    virtual yb_status run_substep(int type) = 0;
    virtual void invalidate_graphs() = 0;
    virtual yb_status check_errors() = 0;
    virtual yb_status read_state_f64(double* pos, double* vel, double* q, double* dx, int buf) = 0;
    virtual yb_status contacts(int* numCols, int* cols, float* stepLimit) = 0;
    virtual yb_status bounds(int scene, float* out) = 0;
    virtual yb_status diagnostics(double* out) = 0;
    virtual uint64_t debug_phases(int mask, int& buf) = 0;
    virtual int64_t penetrations() = 0;
    virtual double min_distance() = 0;
    virtual yb_status profile_substep(bool detect, bool rebuild, double* ms, uint64_t* launches) = 0;
    virtual yb_status time_iter(int threads, int lanes, int pipe, int reps, float* ms) = 0;
    virtual yb_status download_range(int first, int count) = 0;
    virtual yb_status gather(int count, yb_sim* const* src, const int* srcScenes) = 0;
    virtual size_t device_bytes() const = 0;
    virtual yb_status set_pins(const unsigned char* group, int numMotions, const PinMotion* motions) = 0;
    virtual yb_status save_device(FILE* f) = 0;
    virtual yb_status load_device(FILE* f) = 0;
    virtual yb_status drive_pins(double dt) = 0;
    virtual yb_status residual_substep(int type, double* out, int cap, int* count) = 0;
    virtual yb_status read_last_vel(double* out) = 0;
    virtual void set_traversal(int packet) = 0;
    virtual bool small_fits() const = 0;
    virtual yb_status run_small(int steps) = 0;
    virtual yb_status packed_contacts(uint32_t* off, int32_t* cols, int64_t capacity) = 0;
};

}  // namespace

struct yb_sim {
    int n = 0;
    int numScenes = 1;
    int capVerts = 0;   // host arrays and device buffers hold this many vertices
    int capScenes = 0;  // ... and this many scenes (a recycled batch may use fewer)
    int precision = YB_PRECISION_FP32;
    std::vector<int> sceneOff;  // numScenes + 1
    std::vector<yb_meta> meta;  // per scene
    float maxH = 1e-3f;
    yb_vertex* verts = nullptr;
    float* qs = nullptr;
    float* qRests = nullptr;
    float* vels = nullptr;
    bool pinned = false;
    std::vector<float> initialInvMasses;
    bool configured = false;
    float lastBVHRebuild = INFINITY;
    uint64_t stepCounter = 0;
    int lastErrorCode = 0, lastWarningCode = 0;
    int iterThreads = 128;
    int iterLanes = 0;
    int iterPipe = 0;
    int useGraphs = 1;
    int travPacket = 2;  // broadphase walk: 2 per query with cooperative loads, 1 per warp of 32 queries, 0 per query
    int useSmall = 1;    // advance small simulations with the one-block kernel
    uint64_t launches = 0;
    cudaStream_t stream = nullptr;     // active stream (own or the caller's)
    cudaStream_t ownStream = nullptr;  // created by configure, destroyed by yb_destroy
    EngineBase* eng = nullptr;
    int dbgBuf = 0;
    std::vector<int> segs;  // host copy of the segment list
};

namespace {

inline bool has(uint32_t f, uint32_t bit) { return (f & bit) != 0; }
inline uint32_t setf(uint32_t f, uint32_t bit, bool on) { return on ? (f | bit) : (f & ~bit); }

yb_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return YB_OK;
    if (e == cudaErrorMemoryAllocation) return YB_ERR_OUT_OF_MEMORY;
    return YB_ERR_CUDA;
}
#define YB_CUDA(x)                                     \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

void default_meta(yb_meta& m, int n, float maxH) {
    // Sim::Sim, YarnBall.cu:14-35
    std::memset(&m, 0, sizeof(m));
    m.numVerts = n;
    m.gravity[0] = 0.f; m.gravity[1] = -9.8f; m.gravity[2] = 0.f;
    m.h = maxH;
    m.drag = 0.2f;
    m.damping = 1e-6f;
    m.time = 0.f;
    m.radius = 1e-4f;
    m.barrierThickness = 8e-4f;
    m.accelerationRatio = 1.f;
    m.kCollision = 1e-5f;
    m.detectionScaler = 1.2f;
    m.frictionCoeff = 0.1f;
    m.kFriction = 5.f;
    m.detectionPeriod = 1;
    m.useStepSizeLimit = 1;
    m.useVelocityRadius = 1;
    m.bvhRebuildPeriod = 1 / 10.f;
    m.numItr = 8;
}

// ---- host rotor helpers for configure (FP32, separately rounded: -ffp-contract=off) ----
struct HQ { float x, y, z, w; };
inline HQ hq_mul(HQ l, HQ r) {
    // Rotor.h:185-188
    const float cx = l.y * r.z - r.y * l.z, cy = l.z * r.x - r.z * l.x, cz = l.x * r.y - r.x * l.y;
    HQ o;
    o.x = l.w * r.x + r.w * l.x + cx;
    o.y = l.w * r.y + r.w * l.y + cy;
    o.z = l.w * r.z + r.w * l.z + cz;
    o.w = l.w * r.w - (l.x * r.x + l.y * r.y + l.z * r.z);
    return o;
}
inline HQ hq_inv(HQ q) { return HQ{-q.x, -q.y, -q.z, q.w}; }
inline float hq_len(HQ q) { return std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w); }
inline HQ hq_normalize(HQ q) {
    const float s = 1.f / hq_len(q);
    return HQ{q.x * s, q.y * s, q.z * s, q.w * s};
}
// Rotor::fromTo(from, to), Rotor.h:57-64, with orthoBasisX (Common.h:235-251) for opposite vectors.
inline HQ hq_from_to(const float f[3], const float t[3]) {
    float h[3] = {(f[0] + t[0]) * 0.5f, (f[1] + t[1]) * 0.5f, (f[2] + t[2]) * 0.5f};
    const float l = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
    if (l > 0) {
        const float s = 1.f / std::sqrt(l);
        h[0] *= s; h[1] *= s; h[2] *= s;
    } else {
        const float* nn = f;
        if (nn[2] >= nn[1]) {
            const float a = 1.0f / (1.0f + nn[2]);
            const float b = -nn[0] * nn[1] * a;
            h[0] = b; h[1] = 1.0f - nn[1] * nn[1] * a; h[2] = -nn[1];
        } else {
            const float a = 1.0f / (1.0f + nn[1]);
            const float b = -nn[0] * nn[2] * a;
            h[0] = 1.0f - nn[0] * nn[0] * a; h[1] = -nn[0]; h[2] = b;
        }
    }
    HQ o;
    o.x = f[1] * h[2] - h[1] * f[2];
    o.y = f[2] * h[0] - h[2] * f[0];
    o.z = f[0] * h[1] - h[0] * f[1];
    o.w = f[0] * h[0] + f[1] * h[1] + f[2] * h[2];
    return o;
}

// Sim::configure host part for one scene's vertex range, YarnBall.cu:91-157.
yb_status configure_scene(yb_sim* S, int o, int m, float density, float& maxSeg, float& minSeg) {
    yb_vertex* V = S->verts + o;
    float* qs = S->qs + 4 * (size_t)o;
    float* qr = S->qRests + 4 * (size_t)o;
    maxSeg = 0.f;
    minSeg = FLT_MAX;
    // The last vertex of a scene cannot start a segment (the reference leaves this to the
    // caller; a stray hasNext there would read past the scene).
    V[m - 1].flags &= ~(uint32_t)(YB_HAS_NEXT | YB_HAS_NEXT_ORIENTATION);
    V[0].flags &= ~(uint32_t)YB_HAS_PREV;
    HQ lastQ{0.f, 0.f, 0.f, 1.f};
    for (int i = 0; i < m; i++) {
        yb_vertex& v = V[i];
        if (i < m - 1) {
            const bool hasNext = has(v.flags, YB_HAS_NEXT);
            V[i + 1].flags = setf(V[i + 1].flags, YB_HAS_PREV, hasNext);
            const bool hasNextNext = hasNext && has(V[i + 1].flags, YB_HAS_NEXT);
            v.flags = setf(v.flags, YB_HAS_NEXT_ORIENTATION, hasNextNext);
            if (!hasNext) v.flags |= (uint32_t)YB_FIX_ORIENTATION;
        }
        if (!has(v.flags, YB_HAS_PREV) && !has(v.flags, YB_HAS_NEXT)) return YB_ERR_DANGLING_SEGMENT;
        v.lRest = 1.f / m;
        float mass = 0;
        if (has(v.flags, YB_HAS_PREV)) mass += V[i - 1].lRest;
        if (has(v.flags, YB_HAS_NEXT)) {
            const yb_vertex& v1 = V[i + 1];
            const float seg[3] = {v1.pos[0] - v.pos[0], v1.pos[1] - v.pos[1], v1.pos[2] - v.pos[2]};
            v.lRest = std::sqrt(seg[0] * seg[0] + seg[1] * seg[1] + seg[2] * seg[2]);
            if (v.lRest == 0 || !std::isfinite(v.lRest)) return YB_ERR_ZERO_LENGTH_SEGMENT;
            const float inv = 1.f / std::sqrt(seg[0] * seg[0] + seg[1] * seg[1] + seg[2] * seg[2]);
            const float dir[3] = {seg[0] * inv, seg[1] * inv, seg[2] * inv};
            const float e1[3] = {1.f, 0.f, 0.f};
            const HQ qq = hq_from_to(e1, dir);
            HQ t = hq_mul(hq_inv(qq), lastQ);
            t = hq_normalize(HQ{t.x, 0.f, 0.f, t.w});
            lastQ = hq_mul(qq, t);
            mass += v.lRest;
            maxSeg = std::max(maxSeg, v.lRest);
            minSeg = std::min(minSeg, v.lRest);
        }
        qs[4 * i] = lastQ.x; qs[4 * i + 1] = lastQ.y; qs[4 * i + 2] = lastQ.z; qs[4 * i + 3] = lastQ.w;
        mass *= 0.5f * density;
        if (mass != 0)
            v.invMass *= 1 / mass;
        else
            v.invMass = 0;
        S->initialInvMasses[o + i] = v.invMass;
    }
    for (int i = 0; i < m - 1; i++) {
        const HQ a{qs[4 * i], qs[4 * i + 1], qs[4 * i + 2], qs[4 * i + 3]};
        const HQ b{qs[4 * i + 4], qs[4 * i + 5], qs[4 * i + 6], qs[4 * i + 7]};
        const HQ r{qr[4 * i], qr[4 * i + 1], qr[4 * i + 2], qr[4 * i + 3]};
        const float l = hq_len(r);
        const HQ d = hq_mul(hq_inv(a), b);
        qr[4 * i] = l * d.x; qr[4 * i + 1] = l * d.y; qr[4 * i + 2] = l * d.z; qr[4 * i + 3] = l * d.w;
    }
    return YB_OK;
}

// uploadMeta's derived radii and validation, YarnBall.cu:226-234.
yb_status upload_meta_checks(yb_meta& m) {
    m.detectionRadius = m.radius + 0.5f * m.barrierThickness;
    m.scaledDetectionRadius = m.detectionRadius * m.detectionScaler;
    if (m.detectionScaler <= 1) return YB_ERR_DETECTION_SCALER;
    if (2 * m.minSegLen < 2 * m.radius + m.barrierThickness) return YB_ERR_SEGMENT_TOO_SHORT;
    return YB_OK;
}

template <typename R>
SceneParams<R> scene_params_of(const yb_meta& m) {
    SceneParams<R> p;
    std::memset(&p, 0, sizeof(p));
    const R h = (R)m.h;
    p.h = h;
    p.lastH = (R)m.lastH;
    p.invH = R(1) / h;
    p.hh = h * h;
    p.gx = (R)m.gravity[0]; p.gy = (R)m.gravity[1]; p.gz = (R)m.gravity[2];
    p.g2 = (p.gx * p.gx + p.gy * p.gy) + p.gz * p.gz;
    p.dragFactor = R(1) - (R)m.drag * h;
    p.D = (R)m.damping / h;
    p.accel = (R)m.accelerationRatio;
    p.twoR = R(2) * (R)m.radius;
    p.invb = R(1) / (R)m.barrierThickness;
    p.kCol = (R)m.kCollision * p.invb;
    p.fricK = (R)m.kFriction;
    p.fricMu = (R)m.frictionCoeff;
    const R dr = (R)m.radius + R(0.5f) * (R)m.barrierThickness;
    p.sdr = dr * (R)m.detectionScaler;
    p.stepBase = dr * ((R)m.detectionScaler - R(1));
    p.useStepLimit = m.useStepSizeLimit ? 1 : 0;
    p.useVelRadius = m.useVelocityRadius ? 1 : 0;
    p.time = m.time;
    return p;
}

int scene_bits(int numScenes) {
    int b = 0;
    while ((1 << b) < numScenes) b++;
    return b;
}

template <typename R>
struct Engine : EngineBase {
    yb_sim* S;
    Dev<R> d{};
    void* block = nullptr;  // one device allocation, sub-allocated
    void* sortScratch = nullptr;
    size_t sortBytes = 0;
    int* sceneOf = nullptr;
    char* stage = nullptr;  // host-layout staging: verts | vels | qs | qRests
    float* rootBoxes = nullptr;
    double* diagPart = nullptr;
    int* sceneDelta = nullptr;
    SceneParams<R>* spDev = nullptr;
    SceneParams<R>* spHost = nullptr;
    int* errHost = nullptr;
    cudaGraphExec_t graphs[GRAPH_TYPES] = {nullptr, nullptr, nullptr};
    uint64_t graphLaunches[GRAPH_TYPES] = {0, 0, 0};
    int graphItr = -1, graphThreads = -1, graphLanes = -1, graphPipe = -1, graphNseg = -1;
    int keyBits = 30;
    int64_t penTotal = 0;
    float minDist = INFINITY;

    explicit Engine(yb_sim* s) : S(s) {}

    ~Engine() override {
        for (auto& g : graphs)
            if (g) cudaGraphExecDestroy(g);
        if (block) cudaFree(block);
        if (pinMem) cudaFree(pinMem);
        if (spHost) cudaFreeHost(spHost);
        if (errHost) cudaFreeHost(errHost);
    }

    size_t allocBytes = 0;

    yb_status alloc() {
        const size_t n = (size_t)S->capVerts;
        const size_t ns = (size_t)S->capScenes;
        const size_t nn = n > 1 ? n - 1 : 1;
        sortBytes = radix_sort_scratch_bytes((int)n);
        size_t off = 0;
        std::vector<std::pair<void**, size_t>> req;
        auto want = [&](void** p, size_t bytes) { req.push_back({p, bytes}); };
        want((void**)&d.pos, sizeof(V4<R>) * n);
        want((void**)&d.posC, sizeof(V4<R>) * n);
        want((void**)&d.vel, sizeof(V4<R>) * n);
        want((void**)&d.lastVel, sizeof(V4<R>) * n);
        want((void**)&d.dx[0], sizeof(D2<R>) * n);
        want((void**)&d.dx[1], sizeof(D2<R>) * n);
        want((void**)&d.q[0], sizeof(V4<R>) * n);
        want((void**)&d.q[1], sizeof(V4<R>) * n);
        want((void**)&d.qRest, sizeof(V4<R>) * n);
        want((void**)&d.vp, sizeof(VP<R>) * n);
        want((void**)&d.stepLim, sizeof(R) * n);
        want((void**)&d.numCols, sizeof(int) * n);
        want((void**)&d.cols, sizeof(int) * n * MAX_COLS);
        want((void**)&d.relA, sizeof(V4<R>) * n * RELCAP);
        want((void**)&d.relB, sizeof(R2<R>) * n * RELCAP);
        // packed contacts: every list at its cap fits (slot indices are 32-bit)
        const size_t csrCap = std::min(n * (size_t)MAX_COLS, (size_t)0xffffffffu);
        const size_t listTiles = (n + LIST_THREADS - 1) / LIST_THREADS;
        want((void**)&d.csrOff, sizeof(unsigned) * (n + 1));
        want((void**)&d.csrCols, sizeof(int) * csrCap);
        want((void**)&d.listStatus, sizeof(unsigned long long) * (1 + listTiles));
        want((void**)&d.segs, sizeof(int) * n);
        want((void**)&spDev, sizeof(SceneParams<R>) * ns);
        want((void**)&d.err, sizeof(int) * EW_COUNT);
        want((void**)&d.nodes, sizeof(BNode<R>) * nn);
        want((void**)&d.wide, sizeof(WNode<R>) * nn);
        want((void**)&d.depJump[0], sizeof(int) * nn);
        want((void**)&d.depJump[1], sizeof(int) * nn);
        want((void**)&d.depDist[0], sizeof(int) * nn);
        want((void**)&d.depDist[1], sizeof(int) * nn);
        want((void**)&d.wideUsed, nn);
        want((void**)&d.wideAll, sizeof(int));
        want((void**)&d.qrec, sizeof(QRec<R>) * n);
        want((void**)&d.nodeLast, sizeof(int) * nn);
        want((void**)&d.leafParent, sizeof(int) * n);
        want((void**)&d.refitCount, sizeof(unsigned) * nn);
        want((void**)&d.sceneRoot, sizeof(int) * ns);
        want((void**)&d.sceneLast, sizeof(int) * ns);
        want((void**)&d.travNext, sizeof(unsigned) * 4);
        want((void**)&d.keys[0], sizeof(unsigned long long) * n);
        want((void**)&d.keys[1], sizeof(unsigned long long) * n);
        want((void**)&d.vals[0], sizeof(int) * n);
        want((void**)&d.vals[1], sizeof(int) * n);
        want((void**)&d.sceneBox, sizeof(unsigned) * 6 * ns);
        want((void**)&sortScratch, sortBytes);
        want((void**)&sceneOf, sizeof(int) * n);
        want((void**)&stage, (sizeof(yb_vertex) + 12 + 16 + 16) * n);
        want((void**)&rootBoxes, sizeof(float) * 6 * ns);
        want((void**)&diagPart, sizeof(double) * 8 * ((n + 255) / 256 + 1));
        want((void**)&sceneDelta, sizeof(int) * ns);
        for (auto& r : req) off += (r.second + 255) & ~(size_t)255;
        YB_CUDA(cudaMalloc(&block, off));
        allocBytes = off;
        off = 0;
        for (auto& r : req) {
            *r.first = (char*)block + off;
            off += (r.second + 255) & ~(size_t)255;
        }
        d.n = S->n;
        d.numScenes = S->numScenes;
        d.nseg = 0;
        d.sp = spDev;
        d.csrCap = (unsigned)csrCap;
        d.relCap = (unsigned)(n * RELCAP);
        {
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            for (int m = 0; m < 3; m++) d.travBlocks[m] = sms * traverse_blocks_per_sm<R>(m);
        }
        d.travPacket = S->travPacket;
        YB_CUDA(cudaHostAlloc((void**)&spHost, sizeof(SceneParams<R>) * ns, cudaHostAllocDefault));
        YB_CUDA(cudaHostAlloc((void**)&errHost, sizeof(int) * EW_COUNT, cudaHostAllocDefault));
        YB_CUDA(cudaMemsetAsync(d.err, 0, sizeof(int) * EW_COUNT, S->stream));
        static const int kInfBits = 0x7f800000;  // EW_MIN_DIST starts at +inf
        YB_CUDA(cudaMemcpyAsync(d.err + EW_MIN_DIST, &kInfBits, sizeof(int), cudaMemcpyHostToDevice, S->stream));
        YB_CUDA(cudaMemsetAsync(d.numCols, 0, sizeof(int) * n, S->stream));
        // no packed contacts until the first list pass (a Newton launch before it reads none)
        YB_CUDA(cudaMemsetAsync(d.csrOff, 0, sizeof(unsigned) * (n + 1), S->stream));
        YB_CUDA(cudaMemsetAsync(d.lastVel, 0, sizeof(V4<R>) * n, S->stream));
        YB_CUDA(cudaMemsetAsync(d.refitCount, 0, sizeof(unsigned) * nn, S->stream));
        // records never built read as empty (last = 0 prunes every entry); until the first
        // rebuild marks the nodes, every record is built
        YB_CUDA(cudaMemsetAsync(d.wide, 0, sizeof(WNode<R>) * nn, S->stream));
        {
            static const int kAll = 1;
            YB_CUDA(cudaMemcpyAsync(d.wideAll, &kAll, sizeof(int), cudaMemcpyHostToDevice, S->stream));
        }
        YB_CUDA(upload_layout());
        launch_bvh_reset(d, S->stream);
        YB_CUDA(cudaStreamSynchronize(S->stream));
        return YB_OK;
    }

    // Scene of every vertex and the sort key width for the current scene layout.
    cudaError_t upload_layout() {
        std::vector<int> so((size_t)S->n);
        for (int s = 0; s < S->numScenes; s++)
            for (int i = S->sceneOff[s]; i < S->sceneOff[s + 1]; i++) so[i] = s;
        d.n = S->n;
        d.numScenes = S->numScenes;
        keyBits = 30 + scene_bits(S->numScenes);
        cudaError_t e = cudaMemcpyAsync(sceneOf, so.data(), sizeof(int) * so.size(), cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
        return e;
    }

    size_t device_bytes() const override { return allocBytes; }

    // Kinematic pin driver state (allocated on first use).
    void* pinMem = nullptr;
    float4* pinInit = nullptr;
    unsigned char* pinGroup = nullptr;
    PinMotion* pinMotion = nullptr;
    bool pinsOn = false;

    yb_status set_pins(const unsigned char* group, int numMotions, const PinMotion* motions) override {
        if (!group) {
            pinsOn = false;
            return YB_OK;
        }
        const size_t cap = (size_t)S->capVerts;
        if (!pinMem) {
            const size_t bytes = (sizeof(float4) * cap + 255) / 256 * 256 + (cap + 255) / 256 * 256 +
                                 sizeof(PinMotion) * 255;
            YB_CUDA(cudaMalloc(&pinMem, bytes));
            pinInit = (float4*)pinMem;
            pinGroup = (unsigned char*)pinMem + (sizeof(float4) * cap + 255) / 256 * 256;
            pinMotion = (PinMotion*)(pinGroup + (cap + 255) / 256 * 256);
        }
        const size_t n = (size_t)S->n;
        cudaStream_t st = S->stream;
        // reference positions: the current device positions
        std::vector<double> pos(3 * n);
        YB_CUDA(read_state_f64(pos.data(), nullptr, nullptr, nullptr, 0) == YB_OK ? cudaSuccess : cudaErrorUnknown);
        std::vector<float4> init(n);
        for (size_t i = 0; i < n; i++) init[i] = make_float4((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2], 0.f);
        YB_CUDA(cudaMemcpyAsync(pinInit, init.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, st));
        YB_CUDA(cudaMemcpyAsync(pinGroup, group, n, cudaMemcpyHostToDevice, st));
        YB_CUDA(cudaMemcpyAsync(pinMotion, motions, sizeof(PinMotion) * numMotions, cudaMemcpyHostToDevice, st));
        YB_CUDA(cudaStreamSynchronize(st));
        pinsOn = true;
        return YB_OK;
    }

    // Checkpoint: the device state in the simulation's precision, in a fixed order, then the
    // contact lists (kept across substeps without detection when detectionPeriod > 1).
    std::vector<std::pair<void*, size_t>> state_arrays() {
        const size_t n = (size_t)S->n;
        return {{d.pos, sizeof(V4<R>) * n},     {d.posC, sizeof(V4<R>) * n}, {d.vel, sizeof(V4<R>) * n},
                {d.lastVel, sizeof(V4<R>) * n}, {d.q[0], sizeof(V4<R>) * n}, {d.qRest, sizeof(V4<R>) * n},
                {d.vp, sizeof(VP<R>) * n},      {d.numCols, sizeof(int) * n}};
    }

    yb_status save_device(FILE* f) override {
        YB_CUDA(cudaStreamSynchronize(S->stream));
        int32_t maxNc = 0;
        for (auto& a : state_arrays()) {
            std::vector<char> h(a.second);
            YB_CUDA(cudaMemcpy(h.data(), a.first, a.second, cudaMemcpyDeviceToHost));
            if (a.first == (void*)d.numCols)
                for (int i = 0; i < S->n; i++) maxNc = std::max(maxNc, ((const int32_t*)h.data())[i]);
            if (fwrite(h.data(), 1, a.second, f) != a.second) return YB_ERR_INVALID_ARGUMENT;
        }
        // cols holds one row of MAX_COLS per segment: the first maxNc entries of every row
        // hold every listed contact.
        const size_t colBytes = sizeof(int) * (size_t)S->n * (size_t)maxNc;
        std::vector<char> h(colBytes);
        if (colBytes)
            YB_CUDA(cudaMemcpy2D(h.data(), sizeof(int) * maxNc, d.cols, sizeof(int) * MAX_COLS, sizeof(int) * maxNc,
                                 (size_t)S->n, cudaMemcpyDeviceToHost));
        if (fwrite(&maxNc, 4, 1, f) != 1 || fwrite(h.data(), 1, colBytes, f) != colBytes) return YB_ERR_INVALID_ARGUMENT;
        return YB_OK;
    }

    yb_status load_device(FILE* f) override {
        for (auto& a : state_arrays()) {
            std::vector<char> h(a.second);
            if (fread(h.data(), 1, a.second, f) != a.second) return YB_ERR_INVALID_ARGUMENT;
            YB_CUDA(cudaMemcpy(a.first, h.data(), a.second, cudaMemcpyHostToDevice));
        }
        int32_t maxNc = -1;
        if (fread(&maxNc, 4, 1, f) != 1 || maxNc < 0 || maxNc > MAX_COLS) return YB_ERR_INVALID_ARGUMENT;
        const size_t colBytes = sizeof(int) * (size_t)S->n * (size_t)maxNc;
        std::vector<char> h(colBytes);
        if (fread(h.data(), 1, colBytes, f) != colBytes) return YB_ERR_INVALID_ARGUMENT;
        if (colBytes)
            YB_CUDA(cudaMemcpy2D(d.cols, sizeof(int) * MAX_COLS, h.data(), sizeof(int) * maxNc, sizeof(int) * maxNc,
                                 (size_t)S->n, cudaMemcpyHostToDevice));
        // Host arrays and the segment list from the restored state (not convert_in, which
        // would reset the compensation terms); the BVH is rebuilt by the next detection.
        const yb_status st = download();
        return st == YB_OK ? refresh_segments() : st;
    }

    yb_status drive_pins(double dt) override {
        if (!pinsOn) return YB_OK;
        launch_pin_drive(d, pinInit, pinGroup, pinMotion, dt, S->stream);
        S->launches++;
        YB_CUDA(cudaGetLastError());
        return YB_OK;
    }

    // Segment list from the host flags (the rule of upload()).
    yb_status refresh_segments() {
        std::vector<int> segs;
        segs.reserve((size_t)S->n);
        for (int s = 0; s < S->numScenes; s++)
            for (int i = S->sceneOff[s]; i + 1 < S->sceneOff[s + 1]; i++)
                if (has(S->verts[i].flags, YB_HAS_NEXT)) segs.push_back(i);
        if (!segs.empty())
            YB_CUDA(cudaMemcpyAsync(d.segs, segs.data(), sizeof(int) * segs.size(), cudaMemcpyHostToDevice, S->stream));
        YB_CUDA(cudaStreamSynchronize(S->stream));
        d.nseg = (int)segs.size();
        S->segs.swap(segs);
        S->lastBVHRebuild = INFINITY;
        invalidate_graphs();
        return YB_OK;
    }

    yb_status download_range(int first, int count) override {
        char* sv = stage;
        char* svel = sv + sizeof(yb_vertex) * (size_t)S->capVerts;
        char* sq = svel + 12 * (size_t)S->capVerts;
        cudaStream_t st = S->stream;
        launch_convert_out(d, sv, (float*)svel, (float*)sq, first, count, st);
        S->launches++;
        YB_CUDA(cudaGetLastError());
        YB_CUDA(cudaMemcpyAsync(S->verts + first, sv + sizeof(yb_vertex) * first, sizeof(yb_vertex) * count,
                                cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaMemcpyAsync(S->vels + 3 * (size_t)first, svel + 12 * (size_t)first, 12 * (size_t)count,
                                cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaMemcpyAsync(S->qs + 4 * (size_t)first, sq + 16 * (size_t)first, 16 * (size_t)count,
                                cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaStreamSynchronize(st));
        return YB_OK;
    }

    // Copies scene srcScenes[i] of src[i] into scene i of this simulation's current layout
    // (device to device), then fixes scene ids and connection indices.
    yb_status gather(int count, yb_sim* const* src, const int* srcScenes) override {
        cudaStream_t st = S->stream;
        YB_CUDA(upload_layout());
        std::vector<int> delta(count);
        for (int i = 0; i < count; i++) {
            yb_sim* Sx = src[i];
            YB_CUDA(cudaStreamSynchronize(Sx->stream));
            const Dev<R>& sd = static_cast<Engine<R>*>(Sx->eng)->d;
            const size_t so = (size_t)Sx->sceneOff[srcScenes[i]];
            const size_t m = (size_t)(Sx->sceneOff[srcScenes[i] + 1] - Sx->sceneOff[srcScenes[i]]);
            const size_t to = (size_t)S->sceneOff[i];
            delta[i] = (int)to - (int)so;
            const size_t v4b = sizeof(V4<R>) * m;
            YB_CUDA(cudaMemcpyAsync(d.pos + to, sd.pos + so, v4b, cudaMemcpyDeviceToDevice, st));
            YB_CUDA(cudaMemcpyAsync(d.posC + to, sd.posC + so, v4b, cudaMemcpyDeviceToDevice, st));
            YB_CUDA(cudaMemcpyAsync(d.vel + to, sd.vel + so, v4b, cudaMemcpyDeviceToDevice, st));
            YB_CUDA(cudaMemcpyAsync(d.lastVel + to, sd.lastVel + so, v4b, cudaMemcpyDeviceToDevice, st));
            YB_CUDA(cudaMemcpyAsync(d.q[0] + to, sd.q[0] + so, v4b, cudaMemcpyDeviceToDevice, st));
            YB_CUDA(cudaMemcpyAsync(d.qRest + to, sd.qRest + so, v4b, cudaMemcpyDeviceToDevice, st));
            YB_CUDA(cudaMemcpyAsync(d.vp + to, sd.vp + so, sizeof(VP<R>) * m, cudaMemcpyDeviceToDevice, st));
        }
        YB_CUDA(cudaMemcpyAsync(sceneDelta, delta.data(), sizeof(int) * count, cudaMemcpyHostToDevice, st));
        launch_relayout(d, sceneOf, sceneDelta, st);
        S->launches++;
        YB_CUDA(cudaMemsetAsync(d.numCols, 0, sizeof(int) * (size_t)S->n, st));
        YB_CUDA(cudaGetLastError());
        YB_CUDA(cudaStreamSynchronize(st));
        return refresh_segments();
    }

    yb_status upload() override {
        const size_t n = (size_t)S->n;
        const size_t cap = (size_t)S->capVerts;
        char* sv = stage;
        char* svel = sv + sizeof(yb_vertex) * cap;
        char* sq = svel + 12 * cap;
        char* sqr = sq + 16 * cap;
        cudaStream_t st = S->stream;
        // The copies into the staging buffers run while the host validates connections and
        // rebuilds the segment list; the device state changes only in convert_in, launched
        // after the host pass has accepted the input.
        YB_CUDA(cudaMemcpyAsync(sv, S->verts, sizeof(yb_vertex) * n, cudaMemcpyHostToDevice, st));
        YB_CUDA(cudaMemcpyAsync(svel, S->vels, 12 * n, cudaMemcpyHostToDevice, st));
        YB_CUDA(cudaMemcpyAsync(sq, S->qs, 16 * n, cudaMemcpyHostToDevice, st));
        YB_CUDA(cudaMemcpyAsync(sqr, S->qRests, 16 * n, cudaMemcpyHostToDevice, st));
        bool changed = false;
        const bool ok = host_segments(changed);
        if (!ok) {
            cudaStreamSynchronize(st);
            return YB_ERR_INVALID_ARGUMENT;
        }
        if (changed && !S->segs.empty())
            YB_CUDA(cudaMemcpyAsync(d.segs, S->segs.data(), sizeof(int) * S->segs.size(), cudaMemcpyHostToDevice, st));
        launch_convert_in(d, sv, (const float*)svel, (const float*)sq, (const float*)sqr, sceneOf, st);
        S->launches++;
        YB_CUDA(cudaGetLastError());
        YB_CUDA(cudaStreamSynchronize(st));
        if (changed) {
            d.nseg = (int)S->segs.size();
            S->lastBVHRebuild = INFINITY;  // topology must be rebuilt
            invalidate_graphs();
        }
        return YB_OK;
    }

    // Segment list (vertices with hasNext that are not the last of their scene) and
    // connection-index validation from the host arrays, on host threads.  Replaces S->segs and
    // sets `changed` when the list differs from the previous one; false on an invalid index.
    bool host_segments(bool& changed) {
        const int n = S->n;
        const int T = std::max(1, std::min<int>(16, std::min<int>((int)std::thread::hardware_concurrency(),
                                                                   (n + 262143) / 262144)));
        std::vector<int> cnt(T, 0);
        std::vector<char> bad(T, 0);
        auto seg_here = [&](int i, int sceneEnd) { return i + 1 < sceneEnd && has(S->verts[i].flags, YB_HAS_NEXT); };
        auto scene_end = [&](int i) {  // end of the scene holding vertex i
            return *std::upper_bound(S->sceneOff.begin(), S->sceneOff.end(), i);
        };
        auto run = [&](auto&& body) {
            std::vector<std::thread> th;
            for (int t = 1; t < T; t++) th.emplace_back(body, t);
            body(0);
            for (auto& x : th) x.join();
        };
        run([&](int t) {
            const int a = (int)((long long)n * t / T), b = (int)((long long)n * (t + 1) / T);
            int c = 0, end = a < n ? scene_end(a) : n;
            for (int i = a; i < b; i++) {
                if (i >= end) end = scene_end(i);
                const int ci = S->verts[i].connectionIndex;
                if (ci >= n || ci < -1) bad[t] = 1;
                c += seg_here(i, end);
            }
            cnt[t] = c;
        });
        for (int t = 0; t < T; t++)
            if (bad[t]) return false;
        std::vector<int> off(T + 1, 0);
        for (int t = 0; t < T; t++) off[t + 1] = off[t] + cnt[t];
        std::vector<int> segs(off[T]);
        const bool sameSize = S->segs.size() == segs.size();
        std::vector<char> diff(T, 0);
        run([&](int t) {
            const int a = (int)((long long)n * t / T), b = (int)((long long)n * (t + 1) / T);
            int k = off[t], end = a < n ? scene_end(a) : n;
            for (int i = a; i < b; i++) {
                if (i >= end) end = scene_end(i);
                if (seg_here(i, end)) segs[k++] = i;
            }
            if (sameSize) diff[t] = !std::equal(segs.begin() + off[t], segs.begin() + off[t + 1], S->segs.begin() + off[t]);
        });
        changed = !sameSize;
        for (int t = 0; t < T; t++) changed = changed || diff[t];
        if (changed) S->segs.swap(segs);
        return true;
    }

    yb_status download() override {
        const size_t n = (size_t)S->n;
        char* sv = stage;
        char* svel = sv + sizeof(yb_vertex) * (size_t)S->capVerts;
        char* sq = svel + 12 * (size_t)S->capVerts;
        cudaStream_t st = S->stream;
        launch_convert_out(d, sv, (float*)svel, (float*)sq, 0, S->n, st);
        S->launches++;
        YB_CUDA(cudaGetLastError());
        YB_CUDA(cudaMemcpyAsync(S->verts, sv, sizeof(yb_vertex) * n, cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaMemcpyAsync(S->vels, svel, 12 * n, cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaMemcpyAsync(S->qs, sq, 16 * n, cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaStreamSynchronize(st));
        return YB_OK;
    }

    yb_status zero_vel() override {
        launch_zero_vel(d, S->stream);
        S->launches++;
        YB_CUDA(cudaGetLastError());
        return YB_OK;
    }

    void write_params() override {
        for (int s = 0; s < S->numScenes; s++) spHost[s] = scene_params_of<R>(S->meta[s]);
        cudaMemcpyAsync(spDev, spHost, sizeof(SceneParams<R>) * S->numScenes, cudaMemcpyHostToDevice, S->stream);
    }

    // Newton iterations per substep: shared by every scene (validate_all_meta).
    int num_itr() const { return (int)S->meta[0].numItr; }

    // Enqueues one substep on the stream; returns the number of kernels it launches.
    // One substep's kernels on S->stream; returns how many were launched.  With slots, the
    // largest iterate change of Newton iteration it is reduced into slots[it] after it.
    uint64_t enqueue_substep(bool detect, bool rebuild, unsigned long long* slots = nullptr) override {
        cudaStream_t st = S->stream;
        uint64_t k = 0;
        launch_init(d, st); k++;
        if (detect && d.nseg > 0) {
            if (rebuild) {  // the schedule rebuilds first after any path that did not use the tree
                launch_bvh_rebuild(d, st, sortScratch, sortBytes, keyBits);
                bvhBuilt = true;
                const int passes = d.nseg > 1 ? (keyBits + 7) / 8 : 0;
                k += 3 + (d.nseg > 1 ? 2 + passes : 0) + 1 + DEPTH_LAUNCHES + 2;
            } else {
                launch_bvh_refit(d, st);
                k += 2;
            }
            launch_traverse(d, st); k += 2;
        } else {
            launch_lists_step_limit(d, st); k++;
        }
        const int I = num_itr();
        for (int it = 0; it < I; it++) {
            launch_iter(d, it & 1, S->iterThreads, S->iterLanes, S->iterPipe, st);
            k++;
            if (slots) { launch_iter_delta(d, it & 1, slots + it, st); k++; }
        }
        launch_end(d, I & 1, (I & 1) != 0, sizeof(R) == 4, st); k++;
        return k;
    }

    void invalidate_graphs() override {
        for (auto& g : graphs) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
        graphItr = graphThreads = graphLanes = graphPipe = graphNseg = -1;
    }

    yb_status run_substep(int type) override {
        const bool detect = type != 2, rebuild = type == 0;
        if (!S->useGraphs) {
            S->launches += enqueue_substep(detect, rebuild);
            YB_CUDA(cudaGetLastError());
            return YB_OK;
        }
        if (graphItr != num_itr() || graphThreads != S->iterThreads || graphLanes != S->iterLanes ||
            graphPipe != S->iterPipe || graphNseg != d.nseg) {
            invalidate_graphs();
            graphItr = num_itr();
            graphThreads = S->iterThreads;
            graphLanes = S->iterLanes;
            graphPipe = S->iterPipe;
            graphNseg = d.nseg;
        }
        if (!graphs[type]) {
            cudaGraph_t g = nullptr;
            YB_CUDA(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
            graphLaunches[type] = enqueue_substep(detect, rebuild);
            cudaError_t e = cudaStreamEndCapture(S->stream, &g);
            if (e != cudaSuccess) return cuda_status(e);
            e = cudaGraphInstantiate(&graphs[type], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                graphs[type] = nullptr;
                return cuda_status(e);
            }
        }
        YB_CUDA(cudaGraphLaunch(graphs[type], S->stream));
        S->launches += graphLaunches[type];
        return YB_OK;
    }

    yb_status check_errors() override {
        YB_CUDA(cudaGetLastError());
        YB_CUDA(cudaMemcpyAsync(errHost, d.err, sizeof(int) * EW_COUNT, cudaMemcpyDeviceToHost, S->stream));
        YB_CUDA(cudaStreamSynchronize(S->stream));
        yb_status st = YB_OK;
        penTotal = errHost[EW_PENETRATIONS];
        std::memcpy(&minDist, &errHost[EW_MIN_DIST], sizeof(float));
        if (errHost[EW_ERROR] != 0) {
            S->lastErrorCode = errHost[EW_ERROR];
            st = YB_ERR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED;
        }
        if (errHost[EW_WARNING] != 0) S->lastWarningCode = errHost[EW_WARNING];
        if (errHost[EW_INTERNAL] != 0 && st == YB_OK) st = YB_ERR_INTERNAL;
        if (errHost[EW_ERROR] || errHost[EW_WARNING] || errHost[EW_INTERNAL])
            YB_CUDA(cudaMemsetAsync(d.err, 0, sizeof(int) * 3, S->stream));
        return st;
    }

    int64_t penetrations() override { return penTotal; }
    double min_distance() override { return minDist; }

    yb_status read_state_f64(double* pos, double* vel, double* q, double* dx, int buf) override {
        const size_t n = (size_t)S->n;
        double* tmp = nullptr;
        YB_CUDA(cudaMalloc(&tmp, sizeof(double) * 14 * n));
        double *dp = tmp, *dv = tmp + 3 * n, *dq = tmp + 6 * n, *ddx = tmp + 10 * n;
        launch_state_f64(d, buf, pos ? dp : nullptr, vel ? dv : nullptr, q ? dq : nullptr, dx ? ddx : nullptr,
                         S->stream);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess && pos) e = cudaMemcpyAsync(pos, dp, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, S->stream);
        if (e == cudaSuccess && vel) e = cudaMemcpyAsync(vel, dv, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, S->stream);
        if (e == cudaSuccess && q) e = cudaMemcpyAsync(q, dq, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, S->stream);
        if (e == cudaSuccess && dx) e = cudaMemcpyAsync(dx, ddx, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, S->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
        cudaFree(tmp);
        return cuda_status(e);
    }

    bool bvhBuilt = false;  // the tree exists (a refit needs one)

    bool small_fits() const override { return small_path_fits(d); }

    // All substeps of an advance in one launch of the one-block kernel; the BVH is not used,
    // so the next detection on the multi-block path rebuilds it.
    yb_status run_small(int steps) override {
        launch_small(d, steps, num_itr(), (unsigned long long)S->stepCounter, S->meta[0].detectionPeriod,
                     sizeof(R) == 4, S->stream);
        S->launches++;
        bvhBuilt = false;
        S->lastBVHRebuild = INFINITY;
        YB_CUDA(cudaGetLastError());
        return YB_OK;
    }

    void set_traversal(int packet) override {
        if (d.travPacket != packet) invalidate_graphs();
        d.travPacket = packet;
    }

    yb_status read_last_vel(double* out) override {
        const size_t n = (size_t)S->n;
        std::vector<V4<R>> h(n);
        YB_CUDA(cudaMemcpyAsync(h.data(), d.lastVel, sizeof(V4<R>) * n, cudaMemcpyDeviceToHost, S->stream));
        YB_CUDA(cudaStreamSynchronize(S->stream));
        for (size_t i = 0; i < n; i++) {
            out[3 * i] = (double)h[i].x;
            out[3 * i + 1] = (double)h[i].y;
            out[3 * i + 2] = (double)h[i].z;
        }
        return YB_OK;
    }

    // The packed lists the Newton kernels read: n + 1 offsets, then up to capacity partner ids.
    yb_status packed_contacts(uint32_t* off, int32_t* cols, int64_t capacity) override {
        const size_t n = (size_t)S->n;
        cudaStream_t st = S->stream;
        std::vector<uint32_t> o(n + 1);
        YB_CUDA(cudaMemcpyAsync(o.data(), d.csrOff, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
        YB_CUDA(cudaStreamSynchronize(st));
        if (off) std::memcpy(off, o.data(), sizeof(uint32_t) * (n + 1));
        const size_t total = std::min((size_t)o[n], (size_t)std::max<int64_t>(capacity, 0));
        if (cols && total) {
            YB_CUDA(cudaMemcpyAsync(cols, d.csrCols, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, st));
            YB_CUDA(cudaStreamSynchronize(st));
        }
        return YB_OK;
    }

    yb_status contacts(int* numCols, int* cols, float* stepLimit) override {
        const size_t n = (size_t)S->n;
        cudaStream_t st = S->stream;
        if (numCols) YB_CUDA(cudaMemcpyAsync(numCols, d.numCols, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
        if (cols) YB_CUDA(cudaMemcpyAsync(cols, d.cols, sizeof(int) * n * MAX_COLS, cudaMemcpyDeviceToHost, st));
        if (stepLimit) {
            if (sizeof(R) == 4) {
                YB_CUDA(cudaMemcpyAsync(stepLimit, d.stepLim, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
            } else {
                std::vector<R> tmp(n);
                YB_CUDA(cudaMemcpyAsync(tmp.data(), d.stepLim, sizeof(R) * n, cudaMemcpyDeviceToHost, st));
                YB_CUDA(cudaStreamSynchronize(st));
                for (size_t i = 0; i < n; i++) stepLimit[i] = (float)tmp[i];
            }
        }
        YB_CUDA(cudaStreamSynchronize(st));
        return YB_OK;
    }

    yb_status bounds(int scene, float* out) override {
        if (!bvhBuilt && d.nseg > 0) {  // the one-block path does not keep a tree: build one now
            launch_bvh_rebuild(d, S->stream, sortScratch, sortBytes, keyBits);
            bvhBuilt = true;
        }
        launch_scene_root_box(d, rootBoxes, S->stream);
        S->launches++;
        std::vector<float> b(6 * (size_t)S->numScenes);
        YB_CUDA(cudaMemcpyAsync(b.data(), rootBoxes, sizeof(float) * b.size(), cudaMemcpyDeviceToHost, S->stream));
        YB_CUDA(cudaStreamSynchronize(S->stream));
        float r[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (int s = 0; s < S->numScenes; s++) {
            if (scene >= 0 && s != scene) continue;
            for (int a = 0; a < 3; a++) {
                r[a] = std::min(r[a], b[6 * s + a]);
                r[3 + a] = std::max(r[3 + a], b[6 * s + 3 + a]);
            }
        }
        std::memcpy(out, r, sizeof(r));
        return YB_OK;
    }

    yb_status diagnostics(double* out) override {
        write_params();
        const int nb = launch_diag(d, diagPart, S->stream);
        S->launches++;
        std::vector<double> part(8 * (size_t)nb);
        YB_CUDA(cudaGetLastError());
        if (nb) YB_CUDA(cudaMemcpyAsync(part.data(), diagPart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, S->stream));
        YB_CUDA(cudaStreamSynchronize(S->stream));
        double r[8] = {0, 0, 0, 0, 0, 0, INFINITY, 0};
        for (int b = 0; b < nb; b++) {
            for (int a = 0; a < 8; a++) {
                const double v = part[8 * (size_t)b + a];
                if (a == 5) r[a] = std::max(r[a], v);
                else if (a == 6) r[a] = std::min(r[a], v);
                else r[a] += v;
            }
        }
        std::memcpy(out, r, sizeof(r));
        return YB_OK;
    }

    // One substep with each kernel class bracketed by events (see yb_profile_advance).
    yb_status profile_substep(bool detect, bool rebuild, double* ms, uint64_t* launches) override {
        cudaStream_t st = S->stream;
        cudaEvent_t ev[16];
        int cls[16];
        int ne = 0;
        for (auto& e : ev) YB_CUDA(cudaEventCreate(&e));
        auto mark = [&](int c) {
            cls[ne] = c;
            cudaEventRecord(ev[ne++], st);
        };
        const int I = num_itr();
        mark(0);
        launch_init(d, st); launches[0]++;
        if (detect && d.nseg > 0) {
            if (rebuild || !bvhBuilt) {
                mark(1);
                launch_bvh_rebuild(d, st, sortScratch, sortBytes, keyBits);
                bvhBuilt = true;
                const int passes = d.nseg > 1 ? (keyBits + 7) / 8 : 0;
                launches[1] += 3 + (d.nseg > 1 ? 2 + passes : 0) + 1 + DEPTH_LAUNCHES + 2;
            } else {
                mark(2);
                launch_bvh_refit(d, st);
                launches[2] += 2;
            }
            mark(3);
            launch_traverse(d, st); launches[3] += 2;
        } else {
            mark(4);
            launch_lists_step_limit(d, st); launches[4]++;
        }
        mark(5);
        for (int it = 0; it < I; it++) launch_iter(d, it & 1, S->iterThreads, S->iterLanes, S->iterPipe, st);
        launches[5] += I;
        mark(6);
        launch_end(d, I & 1, (I & 1) != 0, sizeof(R) == 4, st); launches[6]++;
        mark(-1);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[ne - 1]);
        for (int i = 0; e == cudaSuccess && i + 1 < ne; i++) {
            float t = 0.f;
            e = cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            ms[cls[i]] += t;
        }
        for (auto& x : ev) cudaEventDestroy(x);
        S->launches += 0;
        return cuda_status(e);
    }

    // Average device time of one Newton iteration launch of the given shape on the current
    // state.  Reads dx[0]/q[0] and writes only dx[1]/q[1], which hold nothing between
    // substeps, so the simulation state is unchanged.
    yb_status time_iter(int threads, int lanes, int pipe, int reps, float* ms) override {
        cudaStream_t st = S->stream;
        cudaEvent_t e0, e1;
        YB_CUDA(cudaEventCreate(&e0));
        YB_CUDA(cudaEventCreate(&e1));
        launch_iter(d, 0, threads, lanes, pipe, st);
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps; r++) launch_iter(d, 0, threads, lanes, pipe, st);
        cudaEventRecord(e1, st);
        S->launches += reps + 1;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float t = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = t / reps;
        return cuda_status(e);
    }

    // One substep of the given shape, launched kernel by kernel (no graph) in the order of
    // enqueue_substep, with the largest iterate change of every Newton iteration recorded.
    yb_status residual_substep(int type, double* out, int cap, int* count) override {
        cudaStream_t st = S->stream;
        const bool detect = type != 2, rebuild = type == 0;
        const int I = num_itr();
        unsigned long long* slots = nullptr;
        YB_CUDA(cudaMalloc(&slots, sizeof(unsigned long long) * (size_t)std::max(I, 1)));
        cudaError_t e = cudaMemsetAsync(slots, 0, sizeof(unsigned long long) * (size_t)std::max(I, 1), st);
        uint64_t k = 0;
        if (e == cudaSuccess) {
            k = enqueue_substep(detect, rebuild, slots);
            e = cudaGetLastError();
        }
        std::vector<unsigned long long> h((size_t)std::max(I, 1));
        if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), slots, sizeof(unsigned long long) * h.size(),
                                                  cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(slots);
        if (e != cudaSuccess) return cuda_status(e);
        S->launches += k;
        for (int it = 0; it < I && it < cap; it++) std::memcpy(out + it, &h[it], sizeof(double));
        *count = I;
        return YB_OK;
    }

    uint64_t debug_phases(int mask, int& buf) override {
        cudaStream_t st = S->stream;
        uint64_t k = 0;
        if (mask & 1) { launch_init(d, st); k++; buf = 0; }
        if ((mask & 6) && d.nseg > 0) {
            if ((mask & 2) || !bvhBuilt) {  // a refit needs a tree
                launch_bvh_rebuild(d, st, sortScratch, sortBytes, keyBits);
                bvhBuilt = true;
                k += 3 + (d.nseg > 1 ? 2 + (keyBits + 7) / 8 : 0) + 1 + DEPTH_LAUNCHES + 2;
            } else {
                launch_bvh_refit(d, st);
                k += 2;
            }
            launch_traverse(d, st);
            k += 2;
        }
        if (mask & 8) { launch_lists_step_limit(d, st); k++; }
        if (mask & 16) { launch_iter(d, buf, S->iterThreads, S->iterLanes, S->iterPipe, st); buf ^= 1; k++; }
        if (mask & 32) { launch_end(d, buf, buf != 0, sizeof(R) == 4, st); buf = 0; k++; }
        return k;
    }
};

EngineBase* make_engine(yb_sim* S) {
    if (S->precision == YB_PRECISION_FP64) return new (std::nothrow) Engine<double>(S);
    return new (std::nothrow) Engine<float>(S);
}

yb_status engine_alloc(yb_sim* S) {
    if (S->precision == YB_PRECISION_FP64) return static_cast<Engine<double>*>(S->eng)->alloc();
    return static_cast<Engine<float>*>(S->eng)->alloc();
}

// Every scene of a batch advances on one schedule: the substep loop, the detection cadence
// and the BVH rebuild clock are shared, and every Newton launch covers all scenes.  The
// reference keeps numItr, detectionPeriod and bvhRebuildPeriod per Sim (YarnBall.h:63-114,
// step.cpp:46-49), so a batch whose scenes disagree on them is refused rather than run on
// one scene's values.
yb_status validate_schedule(const yb_sim* S) {
    const yb_meta& m0 = S->meta[0];
    for (const auto& m : S->meta)
        if (m.numItr != m0.numItr || m.detectionPeriod != m0.detectionPeriod ||
            !(m.bvhRebuildPeriod == m0.bvhRebuildPeriod))
            return YB_ERR_INVALID_ARGUMENT;
    return YB_OK;
}

yb_status validate_all_meta(yb_sim* S) {
    for (auto& m : S->meta) {
        const yb_status st = upload_meta_checks(m);
        if (st != YB_OK) return st;
    }
    return validate_schedule(S);
}

}  // namespace

// =========================================================================================
extern "C" {

static yb_status create_internal(int32_t numScenes, const int32_t* vertsPerScene, int32_t precision,
                                 long long capVerts, int32_t capScenes, yb_sim** out);

yb_status yb_create_batch(int32_t numScenes, const int32_t* vertsPerScene, int32_t precision, yb_sim** out) {
    return create_internal(numScenes, vertsPerScene, precision, 0, 0, out);
}

static yb_status create_internal(int32_t numScenes, const int32_t* vertsPerScene, int32_t precision,
                                 long long capVerts, int32_t capScenes, yb_sim** out) {
    if (!out || numScenes < 1 || !vertsPerScene) return YB_ERR_INVALID_ARGUMENT;
    if (precision != YB_PRECISION_FP32 && precision != YB_PRECISION_FP64) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    long long total = 0;
    for (int s = 0; s < numScenes; s++) {
        if (vertsPerScene[s] < 3) return YB_ERR_TOO_FEW_VERTICES;
        total += vertsPerScene[s];
    }
    if (capVerts < total) capVerts = total;
    if (capScenes < numScenes) capScenes = numScenes;
    if (capVerts > (1LL << 31) / YB_MAX_COLLISIONS_PER_SEGMENT) return YB_ERR_INVALID_ARGUMENT;
    yb_sim* S = new (std::nothrow) yb_sim();
    if (!S) return YB_ERR_OUT_OF_MEMORY;
    S->n = (int)total;
    S->numScenes = numScenes;
    S->capVerts = (int)capVerts;
    S->capScenes = capScenes;
    S->precision = precision;
    S->sceneOff.resize(numScenes + 1, 0);
    for (int s = 0; s < numScenes; s++) S->sceneOff[s + 1] = S->sceneOff[s] + vertsPerScene[s];
    S->meta.resize(numScenes);
    for (int s = 0; s < numScenes; s++) default_meta(S->meta[s], vertsPerScene[s], S->maxH);
    const size_t n = (size_t)capVerts;
    const size_t bytes = n * (sizeof(yb_vertex) + 12 + 16 + 16);
    void* host = nullptr;
    if (cudaHostAlloc(&host, bytes, cudaHostAllocDefault) == cudaSuccess) {
        S->pinned = true;
    } else {
        cudaGetLastError();
        host = std::malloc(bytes);
        if (!host) { delete S; return YB_ERR_OUT_OF_MEMORY; }
    }
    S->verts = (yb_vertex*)host;
    S->vels = (float*)((char*)host + sizeof(yb_vertex) * n);
    S->qs = (float*)((char*)S->vels + 12 * n);
    S->qRests = (float*)((char*)S->qs + 16 * n);
    // Per-vertex defaults, YarnBall.cu:42-50
    for (size_t i = 0; i < n; i++) {
        yb_vertex& v = S->verts[i];
        v.pos[0] = v.pos[1] = v.pos[2] = 0.f;
        v.invMass = 1.f;
        v.lRest = 1.f;
        v.kStretch = 100.f;
        v.connectionIndex = -1;
        v.flags = YB_HAS_NEXT;
        S->vels[3 * i] = S->vels[3 * i + 1] = S->vels[3 * i + 2] = 0.f;
        S->qs[4 * i] = S->qs[4 * i + 1] = S->qs[4 * i + 2] = 0.f;
        S->qs[4 * i + 3] = 1.f;
        S->qRests[4 * i] = S->qRests[4 * i + 1] = S->qRests[4 * i + 2] = 0.f;
        S->qRests[4 * i + 3] = 5.f;
    }
    for (int s = 0; s < numScenes; s++) S->verts[S->sceneOff[s + 1] - 1].flags = 0;
    *out = S;
    return YB_OK;
}

yb_status yb_create(int32_t numVerts, yb_sim** out) {
    return create_internal(1, &numVerts, YB_PRECISION_FP32, 0, 0, out);
}

void yb_destroy(yb_sim* S) {
    if (!S) return;
    if (S->stream) cudaStreamSynchronize(S->stream);
    delete S->eng;
    if (S->ownStream) {
        cudaStreamSynchronize(S->ownStream);
        cudaStreamDestroy(S->ownStream);
    }
    if (S->pinned)
        cudaFreeHost(S->verts);
    else
        std::free(S->verts);
    delete S;
}

yb_status yb_host_arrays(yb_sim* S, yb_vertex** verts, float** qs, float** qRests, float** vels) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (verts) *verts = S->verts;
    if (qs) *qs = S->qs;
    if (qRests) *qRests = S->qRests;
    if (vels) *vels = S->vels;
    return YB_OK;
}

yb_status yb_get_meta(yb_sim* S, int32_t scene, yb_meta* out) {
    if (!S || !out || scene < 0 || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    *out = S->meta[scene];
    return YB_OK;
}

yb_status yb_set_meta(yb_sim* S, int32_t scene, const yb_meta* in) {
    if (!S || !in || scene < 0 || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    const int n = S->meta[scene].numVerts;
    S->meta[scene] = *in;
    S->meta[scene].numVerts = n;  // fixed at creation
    return YB_OK;
}

yb_status yb_get_max_h(yb_sim* S, float* maxH) {
    if (!S || !maxH) return YB_ERR_INVALID_ARGUMENT;
    *maxH = S->maxH;
    return YB_OK;
}

yb_status yb_set_max_h(yb_sim* S, float maxH) {
    if (!S || !(maxH > 0)) return YB_ERR_INVALID_ARGUMENT;
    S->maxH = maxH;
    return YB_OK;
}

yb_status yb_configure(yb_sim* S, float density) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    S->initialInvMasses.assign(S->n, 0.f);
    for (int s = 0; s < S->numScenes; s++) {
        float mx = 0, mn = 0;
        const yb_status st = configure_scene(S, S->sceneOff[s], S->sceneOff[s + 1] - S->sceneOff[s], density, mx, mn);
        if (st != YB_OK) return st;
        S->meta[s].maxSegLen = mx;
        S->meta[s].minSegLen = mn;
    }
    {
        const yb_status st = validate_schedule(S);
        if (st != YB_OK) return st;
    }
    if (S->eng) {  // re-configure: start from a fresh device state
        if (S->stream) cudaStreamSynchronize(S->stream);
        delete S->eng;
        S->eng = nullptr;
        S->configured = false;
    }
    if (!S->ownStream) {
        cudaError_t e = cudaStreamCreateWithFlags(&S->ownStream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            S->ownStream = nullptr;
            return cuda_status(e);
        }
    }
    if (!S->stream) S->stream = S->ownStream;
    S->eng = make_engine(S);
    if (!S->eng) return YB_ERR_OUT_OF_MEMORY;
    yb_status st = engine_alloc(S);
    if (st != YB_OK) {
        delete S->eng;
        S->eng = nullptr;
        return st;
    }
    S->configured = true;
    st = validate_all_meta(S);
    if (st != YB_OK) return st;
    S->eng->write_params();
    return S->eng->upload();
}

yb_status yb_set_kstretch(yb_sim* S, int32_t scene, float k) {
    if (!S || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    const int s0 = scene < 0 ? 0 : scene, s1 = scene < 0 ? S->numScenes : scene + 1;
    for (int i = S->sceneOff[s0]; i < S->sceneOff[s1]; i++) S->verts[i].kStretch = k * S->verts[i].lRest;
    return YB_OK;
}

yb_status yb_set_kbend(yb_sim* S, int32_t scene, float k) {
    if (!S || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    const int s0 = scene < 0 ? 0 : scene, s1 = scene < 0 ? S->numScenes : scene + 1;
    k *= 4;
    for (int i = S->sceneOff[s0]; i < S->sceneOff[s1]; i++) {
        float* r = S->qRests + 4 * (size_t)i;
        const float l = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
        const float inv = 1.f / l;
        const float s = k / S->verts[i].lRest;
        const float a = r[0] * inv, b = r[1] * inv, c = r[2] * inv, w = r[3] * inv;
        r[0] = s * a; r[1] = s * b; r[2] = s * c; r[3] = s * w;
    }
    return YB_OK;
}

yb_status yb_upload(yb_sim* S) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->upload();
}

yb_status yb_download(yb_sim* S) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->download();
}

yb_status yb_zero_velocities(yb_sim* S) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->zero_vel();
}

yb_status yb_advance(yb_sim* S, float dt, float* advanced) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (advanced) *advanced = 0.f;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    if (!(dt > 0)) return YB_OK;
    // step.cpp:36-55
    const int steps = std::max(1, (int)std::ceil(dt / S->maxH));
    for (auto& m : S->meta) {
        m.lastH = m.h;
        m.h = dt / steps;
    }
    yb_status st = validate_all_meta(S);
    if (st != YB_OK) return st;
    S->eng->write_params();
    st = S->eng->drive_pins(dt);
    if (st != YB_OK) return st;
    const yb_meta& m0 = S->meta[0];
    if (S->useSmall && S->eng->small_fits()) {
        // a small simulation: every substep in one launch of the one-block kernel
        st = S->eng->run_small(steps);
        if (st != YB_OK) return st;
        S->stepCounter += (uint64_t)steps;
        for (auto& m : S->meta) m.time += dt;
        st = S->eng->check_errors();
        if (advanced) *advanced = dt;
        return st;
    }
    for (int s = 0; s < steps; s++, S->stepCounter++) {
        int type = 2;
        if (m0.detectionPeriod > 0 && S->stepCounter % (uint64_t)m0.detectionPeriod == 0) {
            // collision.cu:101-108
            if (S->lastBVHRebuild >= m0.bvhRebuildPeriod) {
                type = 0;
                S->lastBVHRebuild = 0;
            } else {
                type = 1;
                S->lastBVHRebuild += m0.h * m0.detectionPeriod;
            }
        }
        st = S->eng->run_substep(type);
        if (st != YB_OK) return st;
    }
    for (auto& m : S->meta) m.time += dt;
    st = S->eng->check_errors();
    if (advanced) *advanced = dt;
    return st;
}

yb_status yb_step(yb_sim* S, float) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    return yb_advance(S, S->maxH, nullptr);
}

yb_status yb_step_count(yb_sim* S, uint64_t* out) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = S->stepCounter;
    return YB_OK;
}

yb_status yb_bounds(yb_sim* S, int32_t scene, float minmax[6]) {
    if (!S || !minmax || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->bounds(scene, minmax);
}

yb_status yb_collision_stats(yb_sim* S, uint64_t* totalPairs, int32_t* segmentsWithContacts, int32_t* maxPerSegment) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    std::vector<int> nc(S->n);
    const yb_status st = S->eng->contacts(nc.data(), nullptr, nullptr);
    if (st != YB_OK) return st;
    uint64_t tot = 0;
    int segs = 0, mx = 0;
    for (int c : nc) {
        if (c > 0) { tot += c; segs++; }
        mx = std::max(mx, c);
    }
    if (totalPairs) *totalPairs = tot / 2;
    if (segmentsWithContacts) *segmentsWithContacts = segs;
    if (maxPerSegment) *maxPerSegment = mx;
    return YB_OK;
}

yb_status yb_last_error(yb_sim* S, int32_t* errorCode, int32_t* warningCode) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (errorCode) *errorCode = S->lastErrorCode;
    if (warningCode) *warningCode = S->lastWarningCode;
    return YB_OK;
}

yb_status yb_initial_inv_masses(yb_sim* S, const float** out, int32_t* count) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = S->initialInvMasses.empty() ? nullptr : S->initialInvMasses.data();
    if (count) *count = (int32_t)S->initialInvMasses.size();
    return YB_OK;
}

const char* yb_status_string(yb_status s) {
    switch (s) {
        case YB_OK: return "ok";
        case YB_ERR_INVALID_ARGUMENT: return "invalid argument";
        case YB_ERR_TOO_FEW_VERTICES: return "Too little vertices";
        case YB_ERR_NOT_CONFIGURED: return "No rest length. Must call configure()";
        case YB_ERR_DANGLING_SEGMENT: return "Dangling segment. Yarns must be atleast 2 segments long";
        case YB_ERR_ZERO_LENGTH_SEGMENT: return "0 length segment";
        case YB_ERR_DETECTION_SCALER: return "Detection scaler must be greater than 1.";
        case YB_ERR_SEGMENT_TOO_SHORT:
            return "Use thinner yarn or use longer segments. (2 * Min seg length must be at least 2 * radius + barrierThickness";
        case YB_ERR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED: return "MAX_COLLISIONS_PER_SEGMENT exceeded";
        case YB_ERR_CUDA: return "CUDA error";
        case YB_ERR_OUT_OF_MEMORY: return "out of device or host memory";
        case YB_ERR_INTERNAL: return "internal error: a bounded device wait expired or the BVH stack overflowed";
        case YB_ERR_ALREADY_CONFIGURED: return "already configured";
        case YB_ERR_SCRATCH_TOO_SMALL:
            return "request exceeds the fixed scratch area of the allocation-free entry point (n > YB_SORT_NOALLOC_MAX_N)";
        case YB_ERR_IO: return "Could not open file";
        case YB_ERR_FORMAT: return "malformed file (see yb_last_io_error)";
    }
    return "unknown status";
}

static bool valid_shape(int threads, int lanes, int pipe) {
    if (lanes == 0) return threads == 128;
    if (pipe) return (lanes == 1 && (threads == 128 || threads == 256)) || (lanes == 4 && threads == 256);
    return (lanes == 1 && (threads == 128 || threads == 256)) || (lanes == 2 && threads == 256) ||
           ((lanes == 4 || lanes == 8) && (threads == 256 || threads == 512));
}

yb_status yb_set_tuning(yb_sim* S, int32_t iterThreads, int32_t lanesPerVertex, int32_t pipelined, int32_t useGraphs) {
    if (!S || !valid_shape(iterThreads, lanesPerVertex, pipelined)) return YB_ERR_INVALID_ARGUMENT;
    S->iterThreads = iterThreads;
    S->iterLanes = lanesPerVertex;
    S->iterPipe = pipelined ? 1 : 0;
    S->useGraphs = useGraphs ? 1 : 0;
    if (S->eng) S->eng->invalidate_graphs();
    return YB_OK;
}

yb_status yb_get_tuning(yb_sim* S, int32_t* iterThreads, int32_t* lanesPerVertex, int32_t* pipelined,
                        int32_t* useGraphs) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (iterThreads) *iterThreads = S->iterThreads;
    if (lanesPerVertex) *lanesPerVertex = S->iterLanes;
    if (pipelined) *pipelined = S->iterPipe;
    if (useGraphs) *useGraphs = S->useGraphs;
    return YB_OK;
}

yb_status yb_autotune(yb_sim* S, int32_t* bestThreads, int32_t* bestLanes, int32_t* bestPipelined, float* bestMs) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    static const int shapes[][3] = {{256, 1, 0}, {128, 1, 0}, {256, 2, 0}, {256, 4, 0}, {512, 4, 0}, {256, 8, 0},
                                    {512, 8, 0}, {128, 1, 1}, {256, 1, 1}, {256, 4, 1}, {128, 0, 0}, {128, 0, 1}};
    constexpr int NS = sizeof(shapes) / sizeof(shapes[0]);
    float best = INFINITY;
    int bt = S->iterThreads, bl = S->iterLanes, bp = S->iterPipe;
    S->eng->write_params();
    // Three rounds over all shapes (8 timed launches each), keeping each shape's fastest
    // round: interleaving the rounds cancels drift, and the minimum discards launches that
    // another stream or a clock change slowed down.
    float shapeMs[NS];
    for (int i = 0; i < NS; i++) shapeMs[i] = INFINITY;
    for (int round = 0; round < 3; round++) {
        for (int i = 0; i < NS; i++) {
            float ms = 0.f;
            const yb_status st = S->eng->time_iter(shapes[i][0], shapes[i][1], shapes[i][2], 8, &ms);
            if (st != YB_OK) return st;
            shapeMs[i] = std::min(shapeMs[i], ms);
        }
    }
    for (int i = 0; i < NS; i++) {
        if (shapeMs[i] < best) {
            best = shapeMs[i];
            bt = shapes[i][0];
            bl = shapes[i][1];
            bp = shapes[i][2];
        }
    }
    const yb_status st = yb_set_tuning(S, bt, bl, bp, S->useGraphs);
    if (bestThreads) *bestThreads = bt;
    if (bestLanes) *bestLanes = bl;
    if (bestPipelined) *bestPipelined = bp;
    if (bestMs) *bestMs = best;
    return st;
}

yb_status yb_set_small_path(yb_sim* S, int32_t enable) {
    if (!S || (enable != 0 && enable != 1)) return YB_ERR_INVALID_ARGUMENT;
    S->useSmall = enable;
    return YB_OK;
}

yb_status yb_set_traversal(yb_sim* S, int32_t packet) {
    if (!S || packet < 0 || packet > 2) return YB_ERR_INVALID_ARGUMENT;
    S->travPacket = packet;
    if (S->eng) S->eng->set_traversal(packet);
    return YB_OK;
}

yb_status yb_get_traversal(yb_sim* S, int32_t* packet) {
    if (!S || !packet) return YB_ERR_INVALID_ARGUMENT;
    *packet = S->travPacket;
    return YB_OK;
}

yb_status yb_set_stream(yb_sim* S, void* stream) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (S->stream) {
        cudaError_t e = cudaStreamSynchronize(S->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    S->stream = stream ? (cudaStream_t)stream : S->ownStream;
    return YB_OK;
}

yb_status yb_profile_advance(yb_sim* S, float dt, double* msByClass, uint64_t* launchesByClass) {
    if (!S || !msByClass || !launchesByClass) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    if (!(dt > 0)) return YB_OK;
    const int steps = std::max(1, (int)std::ceil(dt / S->maxH));
    for (auto& m : S->meta) {
        m.lastH = m.h;
        m.h = dt / steps;
    }
    yb_status st = validate_all_meta(S);
    if (st != YB_OK) return st;
    S->eng->write_params();
    const yb_meta& m0 = S->meta[0];
    for (int s = 0; s < steps; s++, S->stepCounter++) {
        bool detect = false, rebuild = false;
        if (m0.detectionPeriod > 0 && S->stepCounter % (uint64_t)m0.detectionPeriod == 0) {
            detect = true;
            if (S->lastBVHRebuild >= m0.bvhRebuildPeriod) {
                rebuild = true;
                S->lastBVHRebuild = 0;
            } else {
                S->lastBVHRebuild += m0.h * m0.detectionPeriod;
            }
        }
        uint64_t before[YB_PROFILE_CLASSES];
        std::memcpy(before, launchesByClass, sizeof(before));
        st = S->eng->profile_substep(detect, rebuild, msByClass, launchesByClass);
        for (int c = 0; c < YB_PROFILE_CLASSES; c++) S->launches += launchesByClass[c] - before[c];
        if (st != YB_OK) return st;
    }
    for (auto& m : S->meta) m.time += dt;
    return S->eng->check_errors();
}

yb_status yb_download_scene(yb_sim* S, int32_t scene) {
    if (!S || scene < 0 || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->download_range(S->sceneOff[scene], S->sceneOff[scene + 1] - S->sceneOff[scene]);
}

yb_status yb_set_pin_motion(yb_sim* S, const uint8_t* group, int32_t numMotions, const yb_pin_motion* motions) {
    if (!S || (group && (numMotions < 1 || numMotions > 255 || !motions))) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    std::vector<PinMotion> m(group ? numMotions : 0);
    for (size_t g = 0; g < m.size(); g++) {
        const yb_pin_motion& x = motions[g];
        double a[3] = {x.axis[0], x.axis[1], x.axis[2]};
        const double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (!(l > 0) && x.omega != 0.f) return YB_ERR_INVALID_ARGUMENT;
        for (int i = 0; i < 3; i++) {
            m[g].c[i] = x.center[i];
            m[g].a[i] = l > 0 ? a[i] / l : 0.0;
            m[g].v[i] = x.velocity[i];
        }
        m[g].omega = x.omega;
        m[g].t0 = x.tStart;
        m[g].t1 = x.tEnd;
    }
    if (group)
        for (int i = 0; i < S->n; i++)
            if (group[i] > numMotions) return YB_ERR_INVALID_ARGUMENT;
    return S->eng->set_pins(group, (int)m.size(), m.data());
}

// ---- files: BCC / OBJ export (fileExport.cpp:6-100) and full-state checkpoints ----------

// Runs of consecutive segment vertices [start, end] (end = the first vertex without hasNext).
static std::vector<std::pair<int, int>> curve_runs(const yb_sim* S) {
    std::vector<std::pair<int, int>> runs;
    bool last = false;
    int start = 0;
    for (int i = 0; i < S->n; i++) {
        const bool seg = (S->verts[i].flags & YB_HAS_NEXT) != 0;
        if (seg && !last) start = i;
        if (!seg && last) runs.push_back({start, i});
        last = seg;
    }
    return runs;
}

yb_status yb_export_bcc(yb_sim* S, const char* path, int32_t asPolyline) {
    if (!S || !path) return YB_ERR_INVALID_ARGUMENT;
    yb_status st = yb_download(S);
    if (st != YB_OK) return st;
    FILE* f = std::fopen(path, "wb");
    if (!f) return YB_ERR_INVALID_ARGUMENT;
    unsigned char hdr[64];
    std::memset(hdr, 0, sizeof(hdr));
    hdr[0] = 'B'; hdr[1] = 'C'; hdr[2] = 'C';
    hdr[3] = 0x44;
    hdr[4] = asPolyline ? 'P' : 'C';
    hdr[5] = asPolyline ? 'L' : '0';
    hdr[6] = 3;  // dimensions
    hdr[7] = 1;  // up dimension
    const auto runs = curve_runs(S);
    uint64_t curves = runs.size(), points = 0;
    for (auto& r : runs) points += (uint64_t)(r.second - r.first + 1);
    std::memcpy(hdr + 8, &curves, 8);
    std::memcpy(hdr + 16, &points, 8);
    bool ok = std::fwrite(hdr, 1, 64, f) == 64;
    for (auto& r : runs) {
        const int32_t np = r.second - r.first + 1;
        ok = ok && std::fwrite(&np, 4, 1, f) == 1;
        for (int i = r.first; i <= r.second; i++) ok = ok && std::fwrite(S->verts[i].pos, 4, 3, f) == 3;
    }
    std::fclose(f);
    return ok ? YB_OK : YB_ERR_INVALID_ARGUMENT;
}

yb_status yb_export_obj(yb_sim* S, const char* path) {
    if (!S || !path) return YB_ERR_INVALID_ARGUMENT;
    yb_status st = yb_download(S);
    if (st != YB_OK) return st;
    FILE* f = std::fopen(path, "w");
    if (!f) return YB_ERR_INVALID_ARGUMENT;
    std::fprintf(f, "# YarnBall Sim\n\no YarnBall\n\n# Vertices (in meters)\n");
    for (int i = 0; i < S->n; i++)
        std::fprintf(f, "v %.16f %.16f %.16f\n", S->verts[i].pos[0], S->verts[i].pos[1], S->verts[i].pos[2]);
    std::fprintf(f, "\n# Curves\n");
    bool last = false;
    for (int i = 0; i < S->n; i++) {
        const bool seg = (S->verts[i].flags & YB_HAS_NEXT) != 0;
        if (seg) {
            if (!last) std::fprintf(f, "l %d", i + 1);
            std::fprintf(f, " %d", i + 2);
        } else if (last) {
            std::fprintf(f, "\n");
        }
        last = seg;
    }
    std::fclose(f);
    return YB_OK;
}

static const char CKPT_MAGIC[8] = {'Y', 'B', 'C', 'K', 'P', 'T', '0', '1'};

yb_status yb_save_state(yb_sim* S, const char* path) {
    if (!S || !path) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    FILE* f = std::fopen(path, "wb");
    if (!f) return YB_ERR_INVALID_ARGUMENT;
    bool ok = std::fwrite(CKPT_MAGIC, 1, 8, f) == 8;
    const int32_t hdr[3] = {S->precision, S->n, S->numScenes};
    ok = ok && std::fwrite(hdr, 4, 3, f) == 3;
    std::vector<int32_t> counts(S->numScenes);
    for (int s = 0; s < S->numScenes; s++) counts[s] = S->sceneOff[s + 1] - S->sceneOff[s];
    ok = ok && std::fwrite(counts.data(), 4, counts.size(), f) == counts.size();
    ok = ok && std::fwrite(S->meta.data(), sizeof(yb_meta), S->meta.size(), f) == S->meta.size();
    ok = ok && std::fwrite(&S->maxH, 4, 1, f) == 1;
    ok = ok && std::fwrite(&S->stepCounter, 8, 1, f) == 1;
    ok = ok && std::fwrite(&S->lastBVHRebuild, 4, 1, f) == 1;
    const int32_t tune[4] = {S->iterThreads, S->iterLanes, S->iterPipe, S->useGraphs};
    ok = ok && std::fwrite(tune, 4, 4, f) == 4;
    ok = ok && std::fwrite(S->qRests, 16, S->n, f) == (size_t)S->n;
    ok = ok && std::fwrite(S->initialInvMasses.data(), 4, S->initialInvMasses.size(), f) == S->initialInvMasses.size();
    yb_status st = ok ? S->eng->save_device(f) : YB_ERR_INVALID_ARGUMENT;
    std::fclose(f);
    return st;
}

yb_status yb_load_state(const char* path, yb_sim** out) {
    if (!path || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return YB_ERR_INVALID_ARGUMENT;
    char magic[8];
    int32_t hdr[3];
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, CKPT_MAGIC, 8) == 0 &&
              std::fread(hdr, 4, 3, f) == 3 && hdr[1] > 0 && hdr[2] > 0;
    std::vector<int32_t> counts(ok ? hdr[2] : 0);
    ok = ok && std::fread(counts.data(), 4, counts.size(), f) == counts.size();
    yb_sim* S = nullptr;
    yb_status st = ok ? create_internal(hdr[2], counts.data(), hdr[0], 0, 0, &S) : YB_ERR_INVALID_ARGUMENT;
    if (st != YB_OK) {
        std::fclose(f);
        return st;
    }
    ok = std::fread(S->meta.data(), sizeof(yb_meta), S->meta.size(), f) == S->meta.size();
    ok = ok && std::fread(&S->maxH, 4, 1, f) == 1 && std::fread(&S->stepCounter, 8, 1, f) == 1 &&
         std::fread(&S->lastBVHRebuild, 4, 1, f) == 1;
    int32_t tune[4] = {256, 4, 0, 1};
    ok = ok && std::fread(tune, 4, 4, f) == 4;
    S->iterThreads = tune[0]; S->iterLanes = tune[1]; S->iterPipe = tune[2]; S->useGraphs = tune[3];
    ok = ok && std::fread(S->qRests, 16, S->n, f) == (size_t)S->n;
    S->initialInvMasses.resize(S->n);
    ok = ok && std::fread(S->initialInvMasses.data(), 4, S->n, f) == (size_t)S->n;
    if (ok) {
        cudaError_t e = cudaStreamCreateWithFlags(&S->ownStream, cudaStreamNonBlocking);
        st = cuda_status(e);
        if (st == YB_OK) {
            S->stream = S->ownStream;
            S->eng = make_engine(S);
            st = S->eng ? engine_alloc(S) : YB_ERR_OUT_OF_MEMORY;
        }
        if (st == YB_OK) {
            S->configured = true;
            st = S->eng->load_device(f);
        }
    } else {
        st = YB_ERR_INVALID_ARGUMENT;
    }
    std::fclose(f);
    if (st == YB_OK) S->eng->write_params();
    if (st != YB_OK) {
        yb_destroy(S);
        return st;
    }
    *out = S;
    return YB_OK;
}

yb_status yb_scene_range(yb_sim* S, int32_t scene, int32_t* first, int32_t* count) {
    if (!S || scene < 0 || scene >= S->numScenes) return YB_ERR_INVALID_ARGUMENT;
    if (first) *first = S->sceneOff[scene];
    if (count) *count = S->sceneOff[scene + 1] - S->sceneOff[scene];
    return YB_OK;
}

yb_status yb_device_bytes(yb_sim* S, uint64_t* out) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = S->eng ? (uint64_t)S->eng->device_bytes() : 0;
    return YB_OK;
}

yb_status yb_batch_gather(int32_t count, yb_sim* const* srcSims, const int32_t* srcScenes, yb_sim* recycle,
                          int64_t capacityVerts, yb_sim** out) {
    if (!out || count < 1 || !srcSims || !srcScenes) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const int prec = srcSims[0] ? srcSims[0]->precision : -1;
    std::vector<int32_t> counts(count);
    long long total = 0;
    for (int i = 0; i < count; i++) {
        yb_sim* x = srcSims[i];
        if (!x || x == recycle || x->precision != prec) return YB_ERR_INVALID_ARGUMENT;
        if (!x->configured) return YB_ERR_NOT_CONFIGURED;
        if (srcScenes[i] < 0 || srcScenes[i] >= x->numScenes) return YB_ERR_INVALID_ARGUMENT;
        counts[i] = x->sceneOff[srcScenes[i] + 1] - x->sceneOff[srcScenes[i]];
        total += counts[i];
    }
    if (total > (1LL << 31) / YB_MAX_COLLISIONS_PER_SEGMENT) return YB_ERR_INVALID_ARGUMENT;
    yb_sim* S = nullptr;
    if (recycle && recycle->configured && recycle->precision == prec && recycle->capVerts >= total &&
        recycle->capScenes >= count) {
        S = recycle;
        cudaStreamSynchronize(S->stream);
    } else {
        const yb_status st = create_internal(count, counts.data(), prec, capacityVerts,
                                             (int32_t)std::max<int64_t>(count, capacityVerts / 64), &S);
        if (st != YB_OK) return st;
    }
    // host-side layout, parameters and host arrays follow the sources
    S->n = (int)total;
    S->numScenes = count;
    S->sceneOff.assign(count + 1, 0);
    S->meta.resize(count);
    S->initialInvMasses.resize(total);
    S->maxH = srcSims[0]->maxH;
    for (int i = 0; i < count; i++) {
        yb_sim* x = srcSims[i];
        const int so = x->sceneOff[srcScenes[i]], m = counts[i];
        const int to = S->sceneOff[i];
        S->sceneOff[i + 1] = to + m;
        S->meta[i] = x->meta[srcScenes[i]];
        std::memcpy(S->verts + to, x->verts + so, sizeof(yb_vertex) * m);
        std::memcpy(S->vels + 3 * (size_t)to, x->vels + 3 * (size_t)so, 12 * (size_t)m);
        std::memcpy(S->qs + 4 * (size_t)to, x->qs + 4 * (size_t)so, 16 * (size_t)m);
        std::memcpy(S->qRests + 4 * (size_t)to, x->qRests + 4 * (size_t)so, 16 * (size_t)m);
        if ((int)x->initialInvMasses.size() >= so + m)
            std::memcpy(S->initialInvMasses.data() + to, x->initialInvMasses.data() + so, sizeof(float) * m);
        for (int v = to; v < to + m; v++)
            if (S->verts[v].connectionIndex >= 0) S->verts[v].connectionIndex += to - so;
    }
    S->stepCounter = 0;
    S->lastBVHRebuild = INFINITY;
    S->iterThreads = srcSims[0]->iterThreads;
    S->iterLanes = srcSims[0]->iterLanes;
    S->iterPipe = srcSims[0]->iterPipe;
    S->travPacket = srcSims[0]->travPacket;
    S->useSmall = srcSims[0]->useSmall;
    if (!S->configured) {
        cudaError_t e = cudaStreamCreateWithFlags(&S->ownStream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            yb_destroy(S);
            return cuda_status(e);
        }
        S->stream = S->ownStream;
        S->eng = make_engine(S);
        yb_status st = S->eng ? engine_alloc(S) : YB_ERR_OUT_OF_MEMORY;
        if (st != YB_OK) {
            yb_destroy(S);
            return st;
        }
        S->configured = true;
    }
    S->eng->set_traversal(S->travPacket);
    yb_status st = S->eng->gather(count, srcSims, srcScenes);
    if (st == YB_OK) st = validate_all_meta(S);
    if (st == YB_OK) S->eng->write_params();
    if (st != YB_OK) {
        if (S != recycle) yb_destroy(S);
        return st;
    }
    *out = S;
    return YB_OK;
}

yb_status yb_launch_count(yb_sim* S, uint64_t* out) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = S->launches;
    return YB_OK;
}

yb_status yb_info(yb_sim* S, int32_t* numVerts, int32_t* numScenes, int32_t* precision) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (numVerts) *numVerts = S->n;
    if (numScenes) *numScenes = S->numScenes;
    if (precision) *precision = S->precision;
    return YB_OK;
}

yb_status yb_penetration_count(yb_sim* S, int64_t* out) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    const yb_status st = S->eng->check_errors();
    *out = S->eng->penetrations();
    return st == YB_ERR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED ? YB_OK : st;
}

yb_status yb_min_pair_distance(yb_sim* S, double* out) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    const yb_status st = S->eng->check_errors();
    *out = S->eng->min_distance();
    return st == YB_ERR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED ? YB_OK : st;
}

yb_status yb_diagnostics(yb_sim* S, double out[8]) {
    if (!S || !out) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->diagnostics(out);
}

yb_status yb_read_state_f64(yb_sim* S, double* pos, double* vel, double* q) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->read_state_f64(pos, vel, q, nullptr, 0);
}

yb_status yb_debug_contacts(yb_sim* S, int32_t* numCols, int32_t* cols, float* stepLimit) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->contacts(numCols, cols, stepLimit);
}

yb_status yb_debug_packed_contacts(yb_sim* S, uint32_t* offsets, int32_t* cols, int64_t capacity) {
    if (!S || !offsets || capacity < 0 || (capacity > 0 && !cols)) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->packed_contacts(offsets, cols, capacity);
}

yb_status yb_debug_last_vel(yb_sim* S, double* lastVel3) {
    if (!S || !lastVel3) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->read_last_vel(lastVel3);
}

yb_status yb_debug_dx(yb_sim* S, double* dx4) {
    if (!S || !dx4) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    return S->eng->read_state_f64(nullptr, nullptr, nullptr, dx4, S->dbgBuf);
}

yb_status yb_step_residuals(yb_sim* S, double* maxDelta, int32_t capacity, int32_t* numIterations) {
    if (!S || !numIterations || capacity < 0 || (capacity > 0 && !maxDelta)) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    // one substep of maxH with the schedule of yb_advance (step.cpp:36-55)
    const float dt = S->maxH;
    for (auto& m : S->meta) {
        m.lastH = m.h;
        m.h = dt;
    }
    yb_status st = validate_all_meta(S);
    if (st != YB_OK) return st;
    S->eng->write_params();
    st = S->eng->drive_pins(dt);
    if (st != YB_OK) return st;
    const yb_meta& m0 = S->meta[0];
    int type = 2;
    if (m0.detectionPeriod > 0 && S->stepCounter % (uint64_t)m0.detectionPeriod == 0) {
        if (S->lastBVHRebuild >= m0.bvhRebuildPeriod) {
            type = 0;
            S->lastBVHRebuild = 0;
        } else {
            type = 1;
            S->lastBVHRebuild += m0.h * m0.detectionPeriod;
        }
    }
    int count = 0;
    st = S->eng->residual_substep(type, maxDelta, capacity, &count);
    if (st != YB_OK) return st;
    S->stepCounter++;
    for (auto& m : S->meta) m.time += dt;
    *numIterations = count;
    return S->eng->check_errors();
}

yb_status yb_debug_phases(yb_sim* S, int32_t mask, float h) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    if (!S->configured) return YB_ERR_NOT_CONFIGURED;
    if (h > 0) {
        for (auto& m : S->meta) {
            m.lastH = m.h;
            m.h = h;
        }
    }
    yb_status st = validate_all_meta(S);
    if (st != YB_OK) return st;
    S->eng->write_params();
    S->launches += S->eng->debug_phases(mask, S->dbgBuf);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    return S->eng->check_errors();
}

yb_status yb_debug_sort_pairs(const uint64_t* keys, const int32_t* vals, int32_t n, int32_t bits, uint64_t* keysOut,
                              int32_t* valsOut) {
    if (n < 0 || (n > 0 && (!keys || !vals || !keysOut || !valsOut)) || bits < 0 || bits > 64)
        return YB_ERR_INVALID_ARGUMENT;
    if (n == 0) return YB_OK;
    const size_t scratch = radix_sort_scratch_bytes(n);
    char* mem = nullptr;
    const size_t kb = sizeof(unsigned long long) * (size_t)n, vb = sizeof(int) * (size_t)n;
    YB_CUDA(cudaMalloc(&mem, 2 * kb + 2 * vb + scratch + 256));
    unsigned long long* k[2] = {(unsigned long long*)mem, (unsigned long long*)(mem + kb)};
    int* v[2] = {(int*)(mem + 2 * kb), (int*)(mem + 2 * kb + vb)};
    void* scr = mem + 2 * kb + 2 * vb;
    int* err = (int*)((char*)scr + scratch);
    cudaError_t e = cudaMemcpy(k[0], keys, kb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(v[0], vals, vb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(int));
    int buf = 0;
    if (e == cudaSuccess) {
        buf = radix_sort_pairs(k, v, n, bits, scr, err, 0);
        e = cudaGetLastError();
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(keysOut, k[buf], kb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(valsOut, v[buf], vb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(mem);
    if (e != cudaSuccess) return cuda_status(e);
    return herr ? YB_ERR_INTERNAL : YB_OK;
}

}  // extern "C"
