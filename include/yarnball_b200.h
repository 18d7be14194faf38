/*
 * yarnball_b200.h - C ABI of the B200-native Stable Cosserat Rods substep.
 *
 * This is the boundary that replaces the static-library link to YarnBall::Sim
 * (reference: KittenEngine/YarnBall/YarnBall.h:116-206).  Every entry point takes plain
 * pointers and sizes, returns a yb_status and never calls exit(); the C++ drop-in header
 * <yarnball/YarnBall.h> turns non-zero statuses back into std::runtime_error, as the
 * reference does.
 *
 * Data model (identical to the reference's host side):
 *   - a simulation owns host arrays verts (yb_vertex, 32 B each), qs (4 floats: x,y,z
 *     bivector + w scalar), qRests (4 floats) and vels (3 floats), obtained with
 *     yb_host_arrays(); the caller fills them, then configure/upload/download move data;
 *   - parameters live in yb_meta, the non-pointer part of YarnBall::MetaData.
 * A simulation may hold several independent scenes packed in one flat vertex array
 * (yb_create_batch); scenes never collide with each other and each has its own yb_meta
 * material parameters, while all of them advance with one time step.
 *
 * Threading: a yb_sim is not thread-safe; calls on one yb_sim are stream-ordered on its
 * own CUDA stream.
 */
#ifndef YARNBALL_B200_H
#define YARNBALL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum yb_status {
    YB_OK = 0,
    YB_ERR_INVALID_ARGUMENT = 1,
    YB_ERR_TOO_FEW_VERTICES = 2,       /* Sim::Sim, YarnBall.cu:12 */
    YB_ERR_NOT_CONFIGURED = 3,         /* setKStretch/setKBend before configure, YarnBall.cu:203,213 */
    YB_ERR_DANGLING_SEGMENT = 4,       /* configure, YarnBall.cu:115-116 */
    YB_ERR_ZERO_LENGTH_SEGMENT = 5,    /* configure, YarnBall.cu:128-129 */
    YB_ERR_DETECTION_SCALER = 6,       /* uploadMeta, YarnBall.cu:230-231 */
    YB_ERR_SEGMENT_TOO_SHORT = 7,      /* uploadMeta, YarnBall.cu:233-234 */
    YB_ERR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED = 8, /* checkErrors, YarnBall.cu:283-286 */
    YB_ERR_CUDA = 9,                   /* replaces checkCudaErrors' exit(), Common.h:15-21 */
    YB_ERR_OUT_OF_MEMORY = 10,
    YB_ERR_INTERNAL = 11,              /* a bounded device wait expired or the BVH stack overflowed */
    YB_ERR_ALREADY_CONFIGURED = 12,
    YB_ERR_SCRATCH_TOO_SMALL = 13,     /* request larger than a fixed scratch area */
    YB_ERR_IO = 14,                    /* a file could not be opened (io/reader.cpp, io/jsonBuilder.cpp) */
    YB_ERR_FORMAT = 15                 /* a file could not be parsed; yb_last_io_error() has the message */
} yb_status;

/* VertexFlags, YarnBall.h:34-40 */
enum {
    YB_HAS_PREV = 1,
    YB_HAS_NEXT = 2,
    YB_HAS_NEXT_ORIENTATION = 4,
    YB_FIX_ORIENTATION = 8,
    YB_COLLIDING = 16
};

/* Sim::ERROR_* / WARNING_*, YarnBall.h:118-122 */
enum {
    YB_ERROR_NONE = 0,
    YB_ERROR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED = 1,
    YB_WARNING_SEGMENT_INTERPENETRATION = 2
};

#define YB_MAX_COLLISIONS_PER_SEGMENT 128 /* YarnBall.h:20 */

/* Vertex, YarnBall.h:52-61 (same field order and size: 32 bytes). */
typedef struct yb_vertex {
    float pos[3];
    float invMass;
    float lRest;
    float kStretch;
    int32_t connectionIndex;
    uint32_t flags;
} yb_vertex;

/* MetaData without its device pointers, YarnBall.h:63-114 (same field order). */
typedef struct yb_meta {
    float gravity[3];
    int32_t numItr;
    float worldFloorNormal[3];
    float worldFloorPos;
    float h;
    float lastH;
    float time;
    int32_t numVerts;
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
    int32_t detectionPeriod;
    float maxSegLen;
    float minSegLen;
    int32_t useStepSizeLimit;
    int32_t useVelocityRadius;
} yb_meta;

typedef struct yb_sim yb_sim;

enum { YB_PRECISION_FP32 = 0, YB_PRECISION_FP64 = 1 };

/* Sim::Sim(int numVerts), YarnBall.cu:11-51: defaults for meta and every vertex. */
yb_status yb_create(int32_t numVerts, yb_sim** out);

/* Several scenes in one flat array (no reference counterpart; the batched form).
 * Scene s owns vertices [sum(vertsPerScene[0..s)), +vertsPerScene[s]).  precision is
 * YB_PRECISION_FP32 (production) or YB_PRECISION_FP64 (the FP64 build of the same kernels).
 * The scenes of a batch share one schedule: their yb_meta must agree on numItr,
 * detectionPeriod and bvhRebuildPeriod, else configure, advance and gather return
 * YB_ERR_INVALID_ARGUMENT (material and contact parameters may differ per scene). */
yb_status yb_create_batch(int32_t numScenes, const int32_t* vertsPerScene, int32_t precision, yb_sim** out);

/* Sim::~Sim, YarnBall.cu:53-85. */
void yb_destroy(yb_sim* sim);

/* Host arrays Sim::verts/qs/qRests/vels, YarnBall.h:124-127.  Owned by the simulation
 * (page-locked when a GPU is present); valid until yb_destroy. */
yb_status yb_host_arrays(yb_sim* sim, yb_vertex** verts, float** qs, float** qRests, float** vels);

/* Sim::meta, YarnBall.h:129.  scene selects the scene of a batch (0 for a plain Sim). */
yb_status yb_get_meta(yb_sim* sim, int32_t scene, yb_meta* out);
yb_status yb_set_meta(yb_sim* sim, int32_t scene, const yb_meta* in);

/* Sim::maxH, YarnBall.h:130. */
yb_status yb_get_max_h(yb_sim* sim, float* maxH);
yb_status yb_set_max_h(yb_sim* sim, float maxH);

/* Sim::configure(float density), YarnBall.cu:91-200: flags, rest lengths, masses, frames,
 * rest Darboux rotors, device allocation, uploadMeta and upload.  Applies to every scene. */
yb_status yb_configure(yb_sim* sim, float density);

/* Sim::setKStretch / Sim::setKBend, YarnBall.cu:202-224 (host arrays only, like the
 * reference; call yb_upload afterwards).  scene < 0 applies to all scenes. */
yb_status yb_set_kstretch(yb_sim* sim, int32_t scene, float k);
yb_status yb_set_kbend(yb_sim* sim, int32_t scene, float k);

/* Sim::upload / download / zeroVelocities, YarnBall.cu:247-274 (blocking, like the reference). */
yb_status yb_upload(yb_sim* sim);
yb_status yb_download(yb_sim* sim);
yb_status yb_zero_velocities(yb_sim* sim);

/* Sim::advance(float h), step.cpp:36-55: ceil(dt/maxH) substeps, then the error check.
 * *advanced receives dt (the reference declares float but returns nothing). */
yb_status yb_advance(yb_sim* sim, float dt, float* advanced);

/* Sim::step(float), step.cpp:57-59: one advance(maxH). */
yb_status yb_step(yb_sim* sim, float dt);

/* Sim::stepCount, YarnBall.h:163. */
yb_status yb_step_count(yb_sim* sim, uint64_t* out);

/* Sim::bounds, YarnBall.cu:87-89: root box of the BVH (padded segment boxes) after the
 * last detection; minmax = {min x,y,z, max x,y,z}.  scene < 0 gives the union. */
yb_status yb_bounds(yb_sim* sim, int32_t scene, float minmax[6]);

/* Sim::printCollisionStats, statistics.cpp:5-23, returned instead of printed:
 * unordered contact pairs, segments with at least one contact, largest list. */
yb_status yb_collision_stats(yb_sim* sim, uint64_t* totalPairs, int32_t* segmentsWithContacts,
                             int32_t* maxPerSegment);

/* Sim::lastErrorCode / lastWarningCode, YarnBall.h:134-135. */
yb_status yb_last_error(yb_sim* sim, int32_t* errorCode, int32_t* warningCode);

/* Sim::initialInvMasses, YarnBall.h:131 (filled by configure). */
yb_status yb_initial_inv_masses(yb_sim* sim, const float** out, int32_t* count);

/* Human-readable text of a status (replaces the reference's fprintf messages). */
const char* yb_status_string(yb_status s);

/* ---- Additions without a reference counterpart ---------------------------------- */

/* Engine tuning of the Newton kernel: threads per block, lanes per vertex (lanes split a
 * segment's contact loop; 0 selects a load-balanced kernel that flattens contact lists) and
 * software pipelining of the contact loop (with lanes 0: flatten per warp instead of per
 * block); valid shapes: (128, 0, 0|1), (128|256, 1, 0|1), (256, 2, 0), (256, 4, 0|1),
 * (512, 4, 0), (256|512, 8, 0).  useGraphs: replay captured CUDA graphs per substep.
 * Default (128, 0, 0), the load-balanced kernel, graphs on. */
yb_status yb_set_tuning(yb_sim* sim, int32_t iterThreads, int32_t lanesPerVertex, int32_t pipelined,
                        int32_t useGraphs);
yb_status yb_get_tuning(yb_sim* sim, int32_t* iterThreads, int32_t* lanesPerVertex, int32_t* pipelined,
                        int32_t* useGraphs);

/* Autotuner: times every Newton-kernel shape on the current device state (which it leaves
 * unchanged; three interleaved rounds of 8 launches per shape, each shape's fastest round),
 * keeps the fastest and returns it with its time per launch.  Call after at least one
 * advance(). */
yb_status yb_autotune(yb_sim* sim, int32_t* bestThreads, int32_t* bestLanes, int32_t* bestPipelined,
                      float* bestMs);

/* Broadphase walk of the BVH: packet = 2 (default) walks the tree once per query with the
 * warp's node records loaded cooperatively (whole 128-byte lines per load, through shared
 * memory; in the FP64 build each lane loads its own), packet = 1 once per warp for 32
 * consecutive queries, packet = 0 once per query.  The contact lists are identical. */
yb_status yb_set_traversal(yb_sim* sim, int32_t packet);
yb_status yb_get_traversal(yb_sim* sim, int32_t* packet);

/* Simulations of at most 256 vertices advance all substeps of an advance() in one launch of a
 * one-block kernel (enable = 1, the default); enable = 0 uses the multi-block kernels and the
 * BVH.  Both run the same device functions in the same order (the load-balanced Newton
 * kernel's summation order); they agree to rounding, since the compiler may fuse multiply-adds
 * differently inside the one kernel. */
yb_status yb_set_small_path(yb_sim* sim, int32_t enable);

/* Launch the simulation's work on `stream` (a cudaStream_t; NULL returns to the simulation's
 * own stream).  Lets a caller order the engine with its own work and time it with events. */
yb_status yb_set_stream(yb_sim* sim, void* stream);

/* advance(dt) with every kernel class bracketed by CUDA events on the simulation's stream
 * (no graphs): msByClass[c] accumulates device milliseconds and launchesByClass[c] the
 * launches of class c: 0 predictor, 1 BVH rebuild (bounds, Morton, sort, Karras, refit),
 * 2 BVH refit, 3 traversal + step limit, 4 step limit alone, 5 Newton/orientation
 * iteration, 6 advection.  Arrays hold YB_PROFILE_CLASSES entries. */
#define YB_PROFILE_CLASSES 7
yb_status yb_profile_advance(yb_sim* sim, float dt, double* msByClass, uint64_t* launchesByClass);

/* Continuous batching (no reference counterpart).  Builds a batch whose scene i is a copy of
 * scene srcScenes[i] of srcSims[i], copying the device state device to device (nothing goes
 * through the host); sources stay valid and unchanged.  If `recycle` is a batch with enough
 * capacity (vertices and scenes) its device allocation is reused and *out == recycle;
 * otherwise a new batch with room for max(total, capacityVerts) vertices is created and the
 * caller still owns `recycle`.  The new batch starts with a BVH rebuild and a detection on
 * its first substep, so a scene evolves identically alone and inside a batch when
 * detectionPeriod is 1 and the Newton kernel shape is the same.  All sources must share a
 * precision. */
yb_status yb_batch_gather(int32_t count, yb_sim* const* srcSims, const int32_t* srcScenes, yb_sim* recycle,
                          int64_t capacityVerts, yb_sim** out);

/* download() restricted to one scene of a batch (its range of the host arrays). */
yb_status yb_download_scene(yb_sim* sim, int32_t scene);

/* Kinematic driver for pinned vertices, on the device.  It performs the reference's
 * per-frame twist and pull scenarios (KittenEngine/main.cpp:54-121: download, move the pinned
 * vertices, set their velocity, upload) without the host round trip.  group[v] = 0 leaves
 * vertex v alone; g in 1..numMotions makes it follow motions[g-1] from its current position
 * x0:  x(t) = c + Rot(axis, omega s) (x0 - c) + velocity s,  s = clamp(t - tStart, 0, tEnd - tStart),
 * t being its scene's simulated time.  At the start of every advance(dt) each driven vertex is
 * placed at x(t) with velocity (x(t+dt) - x(t)) / dt.  Driven vertices are normally pinned
 * (invMass 0).  group = NULL switches the driver off. */
typedef struct yb_pin_motion {
    float center[3];
    float axis[3];
    float omega;
    float velocity[3];
    float tStart;
    float tEnd;
} yb_pin_motion;
yb_status yb_set_pin_motion(yb_sim* sim, const uint8_t* group, int32_t numMotions, const yb_pin_motion* motions);

/* Sim::exportToBCC (io/fileExport.cpp:6-63): download(), then a 64-byte BCC header ('BCC',
 * 0x44, curve type "PL" when asPolyline else "C0", 3 dimensions, up axis 1, curve and control
 * point counts, 40 zero bytes) and each curve (a run of vertices with hasNext plus the vertex
 * that ends it) as an int32 point count followed by float32 xyz per point.  Every scene of a
 * batch is written into the one file.  An unopenable path gives YB_ERR_INVALID_ARGUMENT where
 * the reference prints "Error opening file" and returns. */
yb_status yb_export_bcc(yb_sim* sim, const char* path, int32_t asPolyline);

/* Sim::exportToOBJ (io/fileExport.cpp:65-100): download(), then "v x y z" lines with 16
 * decimals and one "l i j ..." polyline (1-based) per curve. */
yb_status yb_export_obj(yb_sim* sim, const char* path);

/* Sim::exportFiberMesh (io/fiberMesher.cpp:9-157): download(), then every segment as 8 twisted
 * fibres (Catmull-Rom centre line, frame blended between neighbouring rotors, random frizz)
 * and random fuzz strands, written as OBJ polylines ("o fiber", "o fuzz").  The random stream
 * is the reference's (xoroshiro128+, seed 0x12345678, the same draws in the same order, the
 * three draws of one vector taken x, y, z), so vertex and line counts and indices match it;
 * vertex positions are evaluated on the GPU and agree to float rounding.  Uses meta of scene 0
 * for the yarn radius.  An unopenable path gives YB_ERR_IO ("Failed to open file for
 * writing" in yb_last_io_error). */
yb_status yb_export_fiber_mesh(yb_sim* sim, const char* path);

/* Full-state checkpoint (no reference counterpart; the exporters above keep positions only).
 * Writes the device state in the simulation's precision (positions with their compensation
 * terms, velocities, last velocities, rotors, rest rotors, per-vertex constants, the contact
 * lists), every scene's meta, maxH, the step counter and the Newton kernel shape.  A
 * simulation restored by yb_load_state continues bit-identically to one that never stopped.
 * Pin motions (yb_set_pin_motion) are not saved.  Requires a configured simulation. */
yb_status yb_save_state(yb_sim* sim, const char* path);
yb_status yb_load_state(const char* path, yb_sim** out);

/* ---- scene construction from files (io/reader.cpp, io/resample.h, io/jsonBuilder.cpp) ----
 * readFromBCC / readFromOBJ / readFromPoly: curves from a file, each point mapped by
 * `transform` (4x4, column major like glm::mat4; NULL = identity) as vec3(T * vec4(p, 1)),
 * Catmull-Rom curves resampled to about `targetSegLen` spacing when allowResample is set, and
 * turned into a new, unconfigured simulation by createFromCurves (io/reader.cpp:13-47): one
 * yarn per curve, closed curves glued end to end through connectionIndex unless
 * breakUpClosedCurves.  Curves that end up with fewer than 3 (.bcc) or 4 (.obj, .poly) points
 * are dropped.  A file that cannot be opened gives YB_ERR_IO and a malformed one
 * YB_ERR_FORMAT; yb_last_io_error() returns the reference's exception message for either. */
yb_status yb_read_bcc(const char* path, float targetSegLen, const float transform[16], int32_t breakUpClosedCurves,
                      int32_t allowResample, yb_sim** out);
yb_status yb_read_obj(const char* path, float targetSegLen, const float transform[16], int32_t breakUpClosedCurves,
                      int32_t allowResample, yb_sim** out);
yb_status yb_read_poly(const char* path, float targetSegLen, const float transform[16], int32_t breakUpClosedCurves,
                       int32_t allowResample, yb_sim** out);

/* buildFromJSON (io/jsonBuilder.cpp:8-172): reads the scene description (curveFile,
 * transform (3x4 rows; default scale 0.01), resampleLength, breakUpClosedCurves, curveRadius,
 * the "simulation" block, glueEndpoints, fixBorders, fixVertex), then configures, sets
 * kStretch/kBend, glues, pins and uploads.  The file may hold // and block comments and
 * trailing commas.  Relative curve paths are relative to the working directory. */
yb_status yb_build_from_json(const char* path, yb_sim** out);

/* Sim::glueEndpoints (io/jsonBuilder.cpp:174-212) on the host arrays: every yarn endpoint is
 * joined (connectionIndex both ways, both moved to their midpoint) to the nearest vertex of its
 * scene with |i - j| > 2 when that vertex is within searchRadius and neither is joined yet.
 * The nearest-vertex search runs on the GPU over the positions at the call (ties: the lowest
 * index); joins are applied in ascending endpoint order. */
yb_status yb_glue_endpoints(yb_sim* sim, float searchRadius);

/* Resample::resampleCMR (io/resample.h:143-187): `count` float xyz points of a uniform
 * Catmull-Rom curve resampled between parameters start and end to about targetSegLen spacing.
 * *outCount receives the number of points; they are written to `out` when capacity allows
 * (else YB_ERR_SCRATCH_TOO_SMALL; out = NULL only queries the count).  Curves with fewer than 4
 * points are returned unchanged. */
yb_status yb_resample_cmr(const float* points, int32_t count, double start, double end, double targetSegLen,
                          float* out, int32_t capacity, int32_t* outCount);

/* Message of the last failed file reader or JSON build on the calling thread. */
const char* yb_last_io_error(void);

/* First vertex and vertex count of a scene. */
yb_status yb_scene_range(yb_sim* sim, int32_t scene, int32_t* first, int32_t* count);

/* Device memory held by the simulation (bytes). */
yb_status yb_device_bytes(yb_sim* sim, uint64_t* out);

/* Kernels launched on the device so far (each graph node counts once per replay). */
yb_status yb_launch_count(yb_sim* sim, uint64_t* out);

/* Number of vertices, scenes and precision of a simulation. */
yb_status yb_info(yb_sim* sim, int32_t* numVerts, int32_t* numScenes, int32_t* precision);

/* Contacts with centre-line distance <= 2 * radius seen since creation (interpenetrations). */
yb_status yb_penetration_count(yb_sim* sim, int64_t* out);

/* Smallest centre-line distance (metres, rounded to float) between the two segments of any
 * listed contact, at the start of every substep since creation; +inf while no contact has
 * been listed.  The segments' centre-lines have crossed when it reaches 0. */
yb_status yb_min_pair_distance(yb_sim* sim, double* out);

/* Convergence of the Newton iteration: advances by one substep of maxH exactly as yb_step
 * does (same schedule, same kernels in the same order, launched without a graph) and writes,
 * for each of its Newton iterations, the largest change of the iterate over all vertices,
 * max |dx_new - dx_old| in FP64 (metres), to maxDelta[0..min(numItr, capacity)).
 * *numIterations receives numItr. */
yb_status yb_step_residuals(yb_sim* sim, double* maxDelta, int32_t capacity, int32_t* numIterations);

/* FP64 diagnostics of the current device state (substep start), computed on the device:
 * out[0] kinetic, out[1] gravity potential, out[2] stretch, out[3] bend, out[4] barrier
 * energy (each contact pair once), out[5] max |v|, out[6] min normalised contact gap,
 * out[7] contact pairs.  Energies follow the definitions written beside the kernel. */
yb_status yb_diagnostics(yb_sim* sim, double out[8]);

/* State access in the simulation's precision widened to double (for accuracy studies):
 * pos (3n), vel (3n), q (4n); any pointer may be NULL. */
yb_status yb_read_state_f64(yb_sim* sim, double* pos, double* vel, double* q);

/* Device-side debugging views used by the parity tests (copies to host buffers):
 *   numCols (n int32), cols (n*128 int32, one row per segment: seg*128 + k), stepLimit (n float),
 *   dx (4n in state precision widened to double).  NULL pointers are skipped. */
yb_status yb_debug_contacts(yb_sim* sim, int32_t* numCols, int32_t* cols, float* stepLimit);
yb_status yb_debug_dx(yb_sim* sim, double* dx4);
/* Velocity of the previous substep (the predictor's lastVels, iteration.cu:19-20), 3n doubles. */
yb_status yb_debug_last_vel(yb_sim* sim, double* lastVel3);
/* The contact lists packed in vertex order by the last list pass (what the Newton kernels read):
 * offsets (n + 1 uint32; vertex k's partners are cols[offsets[k] .. offsets[k+1])), then up to
 * capacity partner ids into cols. */
yb_status yb_debug_packed_contacts(yb_sim* sim, uint32_t* offsets, int32_t* cols, int64_t capacity);

/* Runs only the substep phases selected by mask on the current device state:
 * 1 = predictor (initItr), 2 = detection with BVH rebuild, 4 = detection with refit only,
 * 8 = step limit, 16 = one Newton+orientation iteration, 32 = advection (endItr).
 * Meant for phase-by-phase parity tests; advance() is the production path. */
yb_status yb_debug_phases(yb_sim* sim, int32_t mask, float h);

/* Stable radix sort of (key, value) pairs on host buffers through the device sort used by
 * the BVH build (ascending by the low `bits` key bits). */
yb_status yb_debug_sort_pairs(const uint64_t* keys, const int32_t* vals, int32_t n, int32_t bits,
                              uint64_t* keysOut, int32_t* valsOut);

/* Allocation-free variant of the sort above (no counterpart in the reference).  For callers
 * that may not allocate device memory where they sort - code running inside another
 * framework that owns the device-memory budget through its own pool, or a fixed-budget loop
 * in which an allocation (which can synchronise the device or fail under fragmentation) is
 * an error.  keysIn/valsIn/keysOut/valsOut are DEVICE pointers owned by the caller (inputs
 * are only read; an output that overlaps its input gives YB_ERR_INVALID_ARGUMENT, so the
 * sort is never in place); stream is a cudaStream_t (NULL = legacy default).  Scratch is a fixed
 * array compiled into the library (about 4.2 MB held on every GPU that loads it), so n is
 * limited to YB_SORT_NOALLOC_MAX_N; larger n returns YB_ERR_SCRATCH_TOO_SMALL.  No
 * cudaMalloc/cudaFree or allocating library call is made; under lazy module loading the first
 * call on a device loads the library's kernels and the scratch array there (once), so make
 * that first call where loading is allowed.  Each call synchronises `stream` (it reads back an
 * error word), so it cannot be captured in a CUDA graph.  Calls share the scratch: calls that
 * overlap on the GPU race and must be serialised.  Returns after the sort has completed on
 * `stream`. */
#define YB_SORT_NOALLOC_MAX_N 262144
yb_status yb_sort_pairs_noalloc(const uint64_t* keysIn, const int32_t* valsIn, uint64_t* keysOut,
                                int32_t* valsOut, int32_t n, int32_t bits, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* YARNBALL_B200_H */
