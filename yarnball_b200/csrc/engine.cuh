// engine.cuh - device data layout and kernel entry points of the substep engine.
//
// Layout in HBM (structure of arrays, one element per vertex unless noted; R = float|double):
//   pos      V4<R>  xyz = position at the start of the substep, w = invMass
//   posC     V4<R>  Kahan compensation of pos (xyz), FP32 build only
//   vel      V4<R>  xyz = velocity (kept intact during the iterations; y = h v + h^2 g is
//                   formed on the fly instead of overwriting vel as YarnBall.cu does)
//   lastVel  V4<R>  velocity of the previous substep (acceleration-aware initial guess)
//   dx[2]    D2<R>  Newton iterate of k and k+1 (double buffered: strict Jacobi)
//   q[2]     V4<R>  segment orientation rotor (double buffered)
//   qRest    V4<R>  rest Darboux rotor; its magnitude is the bending stiffness
//   vp       VP<R>  {lRest, kStretch, connectionIndex, flags | scene << 8}
//   stepLim  R      per-segment displacement limit (collision.cu:121-159)
//   numCols  int    contacts of each segment
//   cols     int    contact partner ids, one row per segment: cols[seg * MAX_COLS + k]
//                   (the broadphase appends here; the list pass sorts each row)
//   csrOff   u32    n + 1: the contacts of vertex k, packed in vertex order by the list pass
//                   every substep, are slots [csrOff[k], csrOff[k+1]) of
//   csrCols  int    partner ids (sorted within each vertex's range)
//   relA/B   V4,R2  partner endpoints relative to p0, staged per substep in the same slots
//                   while the slot is below relCap (the one-block path stages rows of RELCAP)
// Segments are the vertices with hasNext; segs[] lists them and is the leaf set of the BVH.
#pragma once
#include "ybmath.cuh"

namespace yb {

constexpr int MAX_COLS = 128;  // MAX_COLLISIONS_PER_SEGMENT, YarnBall.h:20

enum : uint32_t {
    F_HAS_PREV = 1,
    F_HAS_NEXT = 2,
    F_HAS_NEXT_ORI = 4,
    F_FIX_ORI = 8,
    F_COLLIDING = 16,
    F_USER_MASK = 0xFFu,
};
YB_HD int scene_of(uint32_t f) { return (int)(f >> 8); }

// Error word slots (device int[8]).
enum {
    EW_ERROR = 0,        // 1 = max collisions per segment exceeded (collision.cu:81-90)
    EW_WARNING = 1,      // 2 = segment interpenetration (YarnBall.h:121)
    EW_INTERNAL = 2,     // bit mask of IE_* below
    EW_PENETRATIONS = 3, // number of contacts seen with distance <= 2 * radius (cumulative)
    EW_MAX_COLS = 4,     // largest contact count of any segment (cumulative max)
    EW_MIN_DIST = 5,     // float bits of the smallest centre-line distance of any listed contact
                         // at substep start (cumulative min; +inf before the first contact)
    EW_COUNT = 8
};
enum { IE_BVH_STACK = 1, IE_SORT_WAIT = 2, IE_GRID_WAIT = 4, IE_REFIT = 8, IE_LIST_WAIT = 16, IE_CONTACT = 32 };

// The Newton iterate of vertex k stored together with that of vertex k+1, so that a segment's
// two endpoints come from one 32-byte sector (one gather per contact partner).
template <typename R>
struct alignas(sizeof(R) * 8) D2 {
    V4<R> a;  // dx[k]
    V4<R> b;  // dx[k+1] (zero for the last vertex)
};

template <typename R>
struct alignas(sizeof(R) * 2) R2 {
    R x, y;
};

constexpr int RELCAP = 8;  // staged relative partner positions: RELCAP x vertices slots in all
constexpr int LIST_THREADS = 128;  // vertices per block of the list pass (one packed-offset tile)

// Wide records are built only for the nodes the walk loads: those at an even depth below
// their scene's root (a record's entries are grandchildren).  Depths come from pointer jumping
// over the parent links at rebuild (DEPTH_ROUNDS rounds: depths below 2^DEPTH_ROUNDS); a
// deeper tree gets every record.
constexpr int DEPTH_ROUNDS = 7;
constexpr int DEPTH_LAUNCHES = 1 + DEPTH_ROUNDS + 1;  // init, jumps, marks

// Contact-list addressing: each segment owns a row of MAX_COLS partner ids and a row of RELCAP
// staged partner positions, so the contacts of one segment are contiguous (the flattened
// contact loop of the Newton kernel reads consecutive contacts of one owner together).
__host__ __device__ __forceinline__ size_t col_at(int seg, int c) { return (size_t)seg * MAX_COLS + c; }
__host__ __device__ __forceinline__ size_t rel_at(int seg, int c) { return (size_t)seg * RELCAP + c; }

template <typename R>
struct VP {
    R lRest, kStretch;
    int cid;
    uint32_t flags;
};

template <typename R>
struct SceneParams {
    R h, lastH, invH, hh;           // h, previous h, 1/h, h*h
    R gx, gy, gz, g2;               // gravity and |g|^2
    R dragFactor;                   // 1 - drag * h
    R D;                            // damping / h
    R accel;                        // accelerationRatio
    R twoR;                         // 2 * radius
    R invb;                         // 1 / barrierThickness
    R kCol;                         // kCollision / barrierThickness
    R fricK, fricMu;                // kFriction, frictionCoeff
    R sdr;                          // scaledDetectionRadius
    R stepBase;                     // detectionRadius * (detectionScaler - 1)
    int useStepLimit, useVelRadius;
    double time;                    // simulated time at the start of the current advance()
};

// Prescribed rigid motion of a group of pinned vertices (see yb_set_pin_motion).
struct PinMotion {
    double c[3], a[3];  // rotation centre and unit axis
    double omega;       // rad/s
    double v[3];        // translation velocity
    double t0, t1;      // motion active for simulated time in [t0, t1]
};

template <typename R>
struct alignas(16) BNode {         // internal BVH node: boxes of both children + links
    R lmin[3], lmax[3], rmin[3], rmax[3];
    int left, right;               // child code: >= 0 internal node, < 0 leaf -(seg + 1)
    int parent;
    int split;                     // sorted position of the left child's last leaf
};

// 4-wide view of the binary tree for traversal: entry e of node i is a grandchild of binary
// node i (or a child, when that child is a leaf), with its box, child code and the sorted
// position of the last leaf below it.  Unused entries have code WIDE_NONE and an empty box.
// An entry is contiguous (32 bytes in FP32), so a walk can read one entry at a time.
constexpr int WIDE_NONE = -2147483647 - 1;
template <typename R>
struct WEntry {
    R mn[3], mx[3];
    int code, last;
};
template <typename R>
struct alignas(16) WNode {
    WEntry<R> e[4];
};

// Query record of a sorted leaf, written by the refit for the traversal: the segment's padded
// box, the segment and its scene (one coalesced load when a lane starts a query).
template <typename R>
struct alignas(16) QRec {
    R mn[3], mx[3];
    int k, sc;
};

template <typename R>
struct Dev {
    int n;            // vertices
    int nseg;         // segments (= BVH leaves)
    int numScenes;
    V4<R>* pos;
    V4<R>* posC;
    V4<R>* vel;
    V4<R>* lastVel;
    D2<R>* dx[2];     // iterate pairs (dx[k], dx[k+1]), double buffered
    V4<R>* q[2];
    V4<R>* qRest;
    VP<R>* vp;
    R* stepLim;
    int* numCols;
    int* cols;
    V4<R>* relA;      // staged per substep in the packed slots below relCap:
    R2<R>* relB;      //   relA = (b0 - p0, (b1 - p0).x), relB = (b1 - p0).yz
    unsigned* csrOff; // n + 1 packed offsets (see the layout above)
    int* csrCols;     // csrCap packed partner ids
    unsigned csrCap;  // slots of csrCols
    unsigned relCap;  // slots of relA / relB
    unsigned long long* listStatus;  // list pass: [0] tile ticket, [1 + tile] look-back status
    int* segs;        // segment -> vertex index, ascending (scene-contiguous)
    const SceneParams<R>* sp;
    int* err;         // EW_COUNT ints
    // BVH
    BNode<R>* nodes;  // nseg - 1 internal nodes
    WNode<R>* wide;   // nseg - 1 wide nodes (rebuilt after every refit)
    int* depJump[2];  // rebuild scratch: pointer-jumping parent links and distances
    int* depDist[2];
    unsigned char* wideUsed;  // 1: the walk can load this node's record
    int* wideAll;     // 1: build every record (tree too deep for the depth marks)
    QRec<R>* qrec;    // per sorted leaf: box, segment, scene (written by the refit)
    int* nodeLast;    // sorted position of the last leaf of each internal node's range
    int* leafParent;  // per sorted leaf position
    unsigned* refitCount;
    int* sceneRoot;   // child code of each scene's subtree root (or INT_MIN when empty)
    int* sceneLast;   // sorted position of the last leaf of each scene's subtree
    unsigned* travNext;   // next query (sorted position) handed out by the traversal
    int travBlocks[3];    // persistent traversal grid of each walk mode (travPacket)
    int travPacket;       // 2: one walk per lane with warp-cooperative record loads (default),
                          // 1: one walk per warp for 32 queries (k_traverse_packet), 0: one per lane
    unsigned long long* keys[2];
    int* vals[2];
    unsigned* sceneBox;   // 6 ordered-uint per scene: min xyz, max xyz of segment midpoints
};

// Hint: bring the line holding p into L1 (no register is held until the data is used).
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// --- kernel launchers (stream-ordered; no host synchronisation) ---
template <typename R> void launch_init(const Dev<R>& d, cudaStream_t s);
template <typename R> void launch_end(const Dev<R>& d, int finalBuf, bool copyQ, bool kahan, cudaStream_t s);
template <typename R> void launch_iter(const Dev<R>& d, int srcBuf, int threads, int lanes, int pipe, cudaStream_t s);
template <typename R> void launch_bvh_rebuild(const Dev<R>& d, cudaStream_t s, void* sortScratch, size_t sortScratchBytes, int keyBits);
template <typename R> void launch_bvh_refit(const Dev<R>& d, cudaStream_t s);
template <typename R> void launch_traverse(const Dev<R>& d, cudaStream_t s);  // + list sort + step limit (2 kernels)
template <typename R> int traverse_blocks_per_sm(int mode);  // resident traversal blocks per SM (persistent grid)
template <typename R> void launch_lists_step_limit(const Dev<R>& d, cudaStream_t s);  // step limit over segments
template <typename R> void launch_bvh_reset(const Dev<R>& d, cudaStream_t s);
// Places driven vertices on their prescribed motion at the start of an advance of length dt.
template <typename R>
void launch_pin_drive(const Dev<R>& d, const float4* init, const unsigned char* group, const PinMotion* m, double dt,
                      cudaStream_t s);  // scene roots := empty

// One block advances a small simulation (n <= 256 vertices) through `steps` substeps in one launch.
template <typename R> bool small_path_fits(const Dev<R>& d);
template <typename R>
void launch_small(const Dev<R>& d, int steps, int numItr, unsigned long long step0, int detectionPeriod, bool kahan,
                  cudaStream_t s);

// Radix sort of (u64 key, int value) pairs, ascending by the low `bits` key bits, stable.
// keys/vals ping-pong between [0] and [1]; the result lands in buffer (passes & 1).
size_t radix_sort_scratch_bytes(int n);
int radix_sort_pairs(unsigned long long* keys[2], int* vals[2], int n, int bits, void* scratch, int* err, cudaStream_t s);

}  // namespace yb
