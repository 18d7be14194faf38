// YarnBall.h - C++ drop-in for YarnBall::Sim over the C ABI of yarnball_b200.
//
// Mirrors the reference's public interface (KittenEngine/YarnBall/YarnBall.h:16-206): the
// same namespace, types, field names, method names, defaults and error behaviour
// (std::runtime_error), so application code written against the reference compiles
// unchanged for the simulation path.  Link with -lyarnball_b200.
//
// Differences that a caller can observe:
//   * advance() returns dt (the reference declares float but returns nothing);
//   * when <glm/glm.hpp> is available vec3/vec4 are glm's, otherwise minimal POD structs
//     with the same layout; Rotor is a POD {x, y, z, w} (w scalar), like Kit::Rotor's layout;
//   * rendering is not part of this library; the file readers and
//     buildFromJSON are free functions here, as in the reference (YarnBall.h:208-211).
#pragma once
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../yarnball_b200.h"

#if __has_include(<glm/glm.hpp>)
#include <glm/glm.hpp>
namespace YarnBall {
using vec3 = glm::vec3;
using vec4 = glm::vec4;
using mat4 = glm::mat4;
inline const float* mat4_data(const mat4& m) { return &m[0][0]; }
}  // namespace YarnBall
#else
namespace YarnBall {
struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float& operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
};
struct vec4 {
    float x, y, z, w;
    vec4() : x(0), y(0), z(0), w(0) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float& operator[](int i) { return (&x)[i]; }
    float operator[](int i) const { return (&x)[i]; }
};
// Column-major 4x4 matrix like glm::mat4: m[column][row]; mat4(d) is d times the identity.
struct mat4 {
    vec4 c[4];
    explicit mat4(float d = 1.f) : c{vec4(d, 0, 0, 0), vec4(0, d, 0, 0), vec4(0, 0, d, 0), vec4(0, 0, 0, d)} {}
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};
inline const float* mat4_data(const mat4& m) { return &m.c[0].x; }
}  // namespace YarnBall
#endif

namespace YarnBall {

constexpr int MAX_COLLISIONS_PER_SEGMENT = YB_MAX_COLLISIONS_PER_SEGMENT;

enum class VertexFlags {
    hasPrev = YB_HAS_PREV,
    hasNext = YB_HAS_NEXT,
    hasNextOrientation = YB_HAS_NEXT_ORIENTATION,
    fixOrientation = YB_FIX_ORIENTATION,
    colliding = YB_COLLIDING,
};

inline bool hasFlag(const uint32_t flags, const VertexFlags flag) { return (flags & (uint32_t)flag) != 0; }
inline uint32_t setFlag(const uint32_t flags, const VertexFlags flag, const bool state) {
    return state ? flags | (uint32_t)flag : flags & ~(uint32_t)flag;
}

struct Vertex {
    vec3 pos;
    float invMass;
    float lRest;
    float kStretch;
    int connectionIndex;
    uint32_t flags;
};
static_assert(sizeof(Vertex) == sizeof(yb_vertex), "Vertex layout");

struct Rotor {
    float x, y, z, w;
};

// MetaData: the parameter fields of the reference (device pointers are internal here).
struct MetaData {
    vec3 gravity;
    int numItr;
    vec3 worldFloorNormal;
    float worldFloorPos;
    float h;
    float lastH;
    float time;
    int numVerts;
    float damping;
    float drag;
    float frictionCoeff;
    float kCollision;
    float kFriction;
    float detectionRadius;
    float scaledDetectionRadius;
    float radius;
    float accelerationRatio;
    float barrierThickness;
    float detectionScaler;
    float bvhRebuildPeriod;
    int detectionPeriod;
    float maxSegLen;
    float minSegLen;
    int useStepSizeLimit;
    int useVelocityRadius;
};
static_assert(sizeof(MetaData) == sizeof(yb_meta), "MetaData layout");

// The box type Sim::bounds() returns: the reference returns Kitten::LBVH::aabb, the 3-D
// float Kitten::Bound (KittenEngine/includes/modules/Bound.h:7-72), whose members and methods
// are restated here so code that grows, pads or tests the returned box compiles unchanged.
struct aabb {
    vec3 min, max;
    aabb() : min(fill(__builtin_huge_valf())), max(fill(-__builtin_huge_valf())) {}
    explicit aabb(const vec3& c) : min(c), max(c) {}
    aabb(const vec3& mn, const vec3& mx) : min(mn), max(mx) {}
    vec3 center() const { return vec3((min[0] + max[0]) * 0.5f, (min[1] + max[1]) * 0.5f, (min[2] + max[2]) * 0.5f); }
    void absorb(const aabb& b) {
        for (int a = 0; a < 3; a++) {
            min[a] = b.min[a] < min[a] ? b.min[a] : min[a];
            max[a] = max[a] < b.max[a] ? b.max[a] : max[a];
        }
    }
    void absorb(const vec3& p) { absorb(aabb(p)); }
    bool contains(const vec3& p) const {
        for (int a = 0; a < 3; a++)
            if (!(min[a] <= p[a] && p[a] <= max[a])) return false;
        return true;
    }
    bool contains(const aabb& b) const {
        for (int a = 0; a < 3; a++)
            if (!(min[a] <= b.min[a] && b.max[a] <= max[a])) return false;
        return true;
    }
    bool intersects(const aabb& b) const {
        for (int a = 0; a < 3; a++)
            if (max[a] <= b.min[a] || min[a] >= b.max[a]) return false;
        return true;
    }
    void pad(float p) { pad(vec3(p, p, p)); }
    void pad(const vec3& p) {
        for (int a = 0; a < 3; a++) {
            min[a] -= p[a];
            max[a] += p[a];
        }
    }
    float volume() const { return (max[0] - min[0]) * (max[1] - min[1]) * (max[2] - min[2]); }

   private:
    static vec3 fill(float v) { return vec3(v, v, v); }
};
using Bounds = aabb;

class Sim {
   public:
    enum { ERROR_NONE = 0, ERROR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED, WARNING_SEGMENT_INTERPENETRATION };

    Vertex* verts = nullptr;
    Rotor* qs = nullptr;
    vec4* qRests = nullptr;
    vec3* vels = nullptr;

    MetaData meta;
    float maxH = 1e-3f;
    std::vector<float> initialInvMasses;

    int lastErrorCode = ERROR_NONE;
    int lastWarningCode = ERROR_NONE;
    bool printErrors = true;

    explicit Sim(int numVerts) {
        check(yb_create(numVerts, &h_));
        bind();
    }
    ~Sim() { yb_destroy(h_); }
    Sim(const Sim&) = delete;
    Sim& operator=(const Sim&) = delete;

    size_t stepCount() {
        uint64_t c = 0;
        check(yb_step_count(h_, &c));
        return (size_t)c;
    }

    void configure(float density = 1e-3f) {
        push();
        check(yb_configure(h_, density));
        pull();
        const float* im = nullptr;
        int32_t cnt = 0;
        check(yb_initial_inv_masses(h_, &im, &cnt));
        initialInvMasses.assign(im, im + cnt);
    }
    void setKBend(float k = 3e-9f) { check(yb_set_kbend(h_, -1, k)); }
    void setKStretch(float k = 1e-2f) { check(yb_set_kstretch(h_, -1, k)); }

    void upload() {
        push();
        check(yb_upload(h_));
    }
    void download() { check(yb_download(h_)); }
    void zeroVelocities() { check(yb_zero_velocities(h_)); }

    void step(float dt) {
        (void)dt;
        advance(maxH);
    }
    float advance(float dt) {
        push();
        float done = 0;
        const yb_status st = yb_advance(h_, dt, &done);
        pull();
        int32_t e = 0, w = 0;
        yb_last_error(h_, &e, &w);
        if (printErrors && w == WARNING_SEGMENT_INTERPENETRATION && w != lastWarningCode)
            fprintf(stderr, "WARNING: Interpenetration detection. This can be due to unstable contacts\n");
        lastErrorCode = e;
        lastWarningCode = w;
        if (st == YB_ERR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED && printErrors)
            fprintf(stderr, "ERROR: MAX_COLLISIONS_PER_SEGMENT exceeded. Current simulation state may be corrupted!\n");
        check(st);
        return done;
    }

    aabb bounds() {
        float b[6];
        check(yb_bounds(h_, -1, b));
        return aabb(vec3(b[0], b[1], b[2]), vec3(b[3], b[4], b[5]));
    }

    void printCollisionStats() {
        uint64_t tot = 0;
        int32_t segs = 0, mx = 0;
        check(yb_collision_stats(h_, &tot, &segs, &mx));
        printf("Total collisions: %llu\n", (unsigned long long)tot);
        printf("Segments with collisions: %d/%d\n", segs, meta.numVerts);
    }

    // io/fileExport.cpp:6-100.  Like the reference, a path that cannot be opened prints
    // "Error opening file" and returns.
    void exportToBCC(std::string path, bool exportAsPolyline = false) {
        push();
        report_file(yb_export_bcc(h_, path.c_str(), exportAsPolyline ? 1 : 0));
    }
    void exportToOBJ(std::string path) {
        push();
        report_file(yb_export_obj(h_, path.c_str()));
    }
    // io/fiberMesher.cpp:9-157; throws like the reference when the file cannot be opened.
    void exportFiberMesh(std::string path) {
        push();
        const yb_status st = yb_export_fiber_mesh(h_, path.c_str());
        if (st == YB_ERR_IO) throw std::runtime_error("Failed to open file for writing");
        check(st);
    }

    // Sim::glueEndpoints (io/jsonBuilder.cpp:174-212), on the host arrays.
    void glueEndpoints(float searchRadius) {
        push();
        check(yb_glue_endpoints(h_, searchRadius));
    }

    yb_sim* handle() { return h_; }

    // A Sim around a handle made by the C ABI (the readers below).
    static Sim* adopt(yb_sim* h) { return new Sim(h); }

   private:
    yb_sim* h_ = nullptr;

    explicit Sim(yb_sim* h) : h_(h) { bind(); }
    void bind() {
        yb_vertex* v = nullptr;
        float *q = nullptr, *qr = nullptr, *vel = nullptr;
        check(yb_host_arrays(h_, &v, &q, &qr, &vel));
        verts = reinterpret_cast<Vertex*>(v);
        qs = reinterpret_cast<Rotor*>(q);
        qRests = reinterpret_cast<vec4*>(qr);
        vels = reinterpret_cast<vec3*>(vel);
        pull();
        const float* im = nullptr;
        int32_t cnt = 0;
        if (yb_initial_inv_masses(h_, &im, &cnt) == YB_OK && im) initialInvMasses.assign(im, im + cnt);
    }

    static void check(yb_status st) {
        if (st != YB_OK) throw std::runtime_error(yb_status_string(st));
    }
    static void report_file(yb_status st) {
        if (st == YB_ERR_INVALID_ARGUMENT) {
            fprintf(stdout, "Error opening file\n");
            return;
        }
        check(st);
    }
    void push() {
        check(yb_set_meta(h_, 0, reinterpret_cast<const yb_meta*>(&meta)));
        check(yb_set_max_h(h_, maxH));
    }
    void pull() {
        check(yb_get_meta(h_, 0, reinterpret_cast<yb_meta*>(&meta)));
        check(yb_get_max_h(h_, &maxH));
    }
};

// ---- scene construction (io/reader.cpp:49-293, io/jsonBuilder.cpp:8-172) -----------------
// Errors throw std::runtime_error with the reference's messages.
namespace detail {
inline Sim* adopt_or_throw(yb_status st, yb_sim* h) {
    if (st != YB_OK) {
        const char* m = yb_last_io_error();
        throw std::runtime_error(m && *m ? m : yb_status_string(st));
    }
    return Sim::adopt(h);
}
}  // namespace detail

inline Sim* readFromOBJ(std::string path, float targetSegLen, mat4 transform, bool breakUpClosedCurves = false,
                        bool allowResample = true) {
    yb_sim* h = nullptr;
    const yb_status st = yb_read_obj(path.c_str(), targetSegLen, mat4_data(transform), breakUpClosedCurves,
                                     allowResample, &h);
    return detail::adopt_or_throw(st, h);
}
inline Sim* readFromBCC(std::string path, float targetSegLen, mat4 transform, bool breakUpClosedCurves = false,
                        bool allowResample = true) {
    yb_sim* h = nullptr;
    const yb_status st = yb_read_bcc(path.c_str(), targetSegLen, mat4_data(transform), breakUpClosedCurves,
                                     allowResample, &h);
    return detail::adopt_or_throw(st, h);
}
inline Sim* readFromPoly(std::string path, float targetSegLen, mat4 transform, bool breakUpClosedCurves = false,
                         bool allowResample = true) {
    yb_sim* h = nullptr;
    const yb_status st = yb_read_poly(path.c_str(), targetSegLen, mat4_data(transform), breakUpClosedCurves,
                                      allowResample, &h);
    return detail::adopt_or_throw(st, h);
}
inline Sim* buildFromJSON(std::string path) {
    yb_sim* h = nullptr;
    const yb_status st = yb_build_from_json(path.c_str(), &h);
    return detail::adopt_or_throw(st, h);
}

}  // namespace YarnBall
