/*
 * yb_oracle.h - CPU oracle for the Stable Cosserat Rods substep (test infrastructure).
 *
 * This is the checker, not the product: only the tests, the smoke check and the benchmark's
 * CPU-baseline leg use it.  It is a plain C++/OpenMP restatement of the reference's
 * algorithm (YarnBall::Sim::advance and the kernels it launches), written independently of
 * the CUDA engine, evaluated in FP64 (the accuracy oracle) or FP32 (the CPU baseline).
 *
 * Pinned to the reference: oracle/refbuild compiles the reference's own kernels and math
 * headers unchanged for the GPU (against a restatement of the absent glm and a stand-in for
 * the absent LBVH), and the GPU tests compare them with this restatement (tests/
 * test_gpu_reference.py).  It is also checked against independent derivations (finite
 * differences, brute-force minimisation, FP64 LU solves, geometric invariants) and against a
 * second, pure-numpy restatement in the CPU tests.
 *
 * Semantic choices (the reference's own kernels are scheduling dependent):
 *   - strict Jacobi: iteration k reads only iteration k-1's dx and orientations;
 *   - each segment's contact list is sorted by partner id;
 *   - the contact set is defined after the narrow-phase filter, so it does not depend on
 *     how the broadphase enumerates overlapping boxes (a uniform grid here).
 */
#ifndef YB_ORACLE_H
#define YB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference Vertex / MetaData host fields. */
typedef struct orc_vertex {
    float pos[3];
    float invMass, lRest, kStretch;
    int32_t connectionIndex;
    uint32_t flags;
} orc_vertex;

typedef struct orc_meta {
    float gravity[3];
    int32_t numItr;
    float worldFloorNormal[3];
    float worldFloorPos;
    float h, lastH, time;
    int32_t numVerts;
    float damping, drag, frictionCoeff, kCollision, kFriction;
    float detectionRadius, scaledDetectionRadius, radius, accelerationRatio;
    float barrierThickness, detectionScaler, bvhRebuildPeriod;
    int32_t detectionPeriod;
    float maxSegLen, minSegLen;
    int32_t useStepSizeLimit, useVelocityRadius;
} orc_meta;

/* Modes: FP64 (accuracy oracle), FP32 as the reference writes it, and FP32 with the
 * engine's precision policy (FP64 closest points for near-parallel pairs, FP64 barrier
 * terms near the clamp, Kahan-compensated positions). */
enum { ORC_FP64 = 0, ORC_FP32 = 1, ORC_FP32_MIXED = 2 };

/* Host setup of one scene (YarnBall.cu:91-157, 202-224, 226-234), FP32 as the reference. */
int orc_configure(int n, float density, orc_vertex* verts, float* qs, float* qRests, float* initialInvMasses,
                  float* maxSegLen, float* minSegLen);
void orc_set_kstretch(int n, orc_vertex* verts, float k);
void orc_set_kbend(int n, const orc_vertex* verts, float* qRests, float k);
int orc_upload_meta(orc_meta* m); /* derives the detection radii; 0 or an error code */
/* The FP32 math helpers over n inputs (op 0 closest points, 1 rotor product, 2 rotation,
 * 3 fromTo, 4 rotor normalisation, 5 hess3 update + solve); see yb_oracle.cpp. */
int orc_math(int op, int n, const float* a, const float* b, const float* c, const float* d, float* out, float* out2);

typedef struct orc_sim orc_sim;
orc_sim* orc_create(int n, int mode);
void orc_destroy(orc_sim* s);
/* sceneOf may be NULL (one scene); meta holds numScenes entries. */
void orc_set_state(orc_sim* s, const orc_vertex* verts, const float* vels, const float* qs, const float* qRests,
                   const int32_t* sceneOf, int numScenes, const orc_meta* meta);
void orc_set_meta(orc_sim* s, int scene, const orc_meta* meta);
void orc_set_last_vel(orc_sim* s, const double* lastVel);
void orc_set_schedule(orc_sim* s, uint64_t stepCounter);
/* Sim::advance (step.cpp:36-55); returns 0 or 1 (contact overflow). */
int orc_advance(orc_sim* s, float dt, float maxH);
/* Phases: 1 predictor, 2 detection (+ step limit), 8 step limit, 16 one iteration, 32 advection.
 * h > 0 first sets lastH = h_old, h = h for every scene. */
int orc_phases(orc_sim* s, int mask, float h);
void orc_get_state(orc_sim* s, double* pos, double* vel, double* q, double* dx, double* lastVel);
void orc_get_contacts(orc_sim* s, int32_t* numCols, int32_t* cols, double* stepLimit);
void orc_diagnostics(orc_sim* s, double out[8]);
int64_t orc_penetrations(orc_sim* s);
void orc_set_threads(int threads);
int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
