// k_bvh.cu - linear BVH over segment AABBs and the broadphase that emits contact lists.
//
// The reference calls an LBVH library whose source is not part of the reference project
// (KittenEngine/KittenGpuLBVH is an empty submodule; call sites collision.cu:94-119).  This
// is a new implementation of the published method:
//   * leaf keys: 30-bit Morton code of the segment midpoint, normalised by its scene's
//     bounds, with the scene id above bit 30 so that every scene is one subtree;
//   * stable LSD radix sort of (key, segment) pairs (k_sort.cu);
//   * Karras 2012 binary radix tree emission, one thread per internal node, ties between
//     equal keys broken by leaf position;
//   * bottom-up AABB refit with one atomic arrival counter per internal node;
//   * traversal: every segment walks its own scene's subtree with its own padded box and
//     keeps the partners that pass the narrow-phase filter (detect.cuh).  Each segment
//     writes only its own list (no atomics on other segments' lists); the list is then
//     sorted by partner id and the step-size limit is computed from it in the same thread.
#include <cuda/atomic>

#include "detect.cuh"

namespace yb {

__device__ __forceinline__ unsigned f2ord(float f) {
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

template <typename R>
__global__ void k_scene_box_init(Dev<R> d) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.numScenes) return;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        d.sceneBox[6 * s + a] = 0xFFFFFFFFu;
        d.sceneBox[6 * s + 3 + a] = 0u;
    }
    d.sceneRoot[s] = INT_MIN;
}

// Per-scene bounds of segment midpoints (Morton normalisation).
template <typename R>
__global__ void __launch_bounds__(256) k_scene_bounds(Dev<R> d) {
    const int si = blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= d.nseg) return;
    const int k = d.segs[si];
    const int sc = scene_of(d.vp[k].flags);
    const V4<R> p0 = d.pos[k], p1 = d.pos[k + 1];
    const float m[3] = {(float)((p0.x + p1.x) * R(0.5)), (float)((p0.y + p1.y) * R(0.5)),
                        (float)((p0.z + p1.z) * R(0.5))};
    // Warp-level pre-reduction when the whole warp belongs to one scene (the common case).
    const unsigned mask = __activemask();
    const int sc0 = __shfl_sync(mask, sc, __ffs(mask) - 1);
    const bool uniform = __all_sync(mask, sc == sc0);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        unsigned lo = f2ord(m[a]), hi = lo;
        if (uniform) {
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(mask, lo, o));
                hi = max(hi, __shfl_xor_sync(mask, hi, o));
            }
            if ((threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1)) {
                atomicMin(&d.sceneBox[6 * sc + a], lo);
                atomicMax(&d.sceneBox[6 * sc + 3 + a], hi);
            }
        } else {
            atomicMin(&d.sceneBox[6 * sc + a], lo);
            atomicMax(&d.sceneBox[6 * sc + 3 + a], hi);
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_morton(Dev<R> d) {
    const int si = blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= d.nseg) return;
    const int k = d.segs[si];
    const int sc = scene_of(d.vp[k].flags);
    const V4<R> p0 = d.pos[k], p1 = d.pos[k + 1];
    const float m[3] = {(float)((p0.x + p1.x) * R(0.5)), (float)((p0.y + p1.y) * R(0.5)),
                        (float)((p0.z + p1.z) * R(0.5))};
    uint32_t code = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float lo = ord2f(d.sceneBox[6 * sc + a]);
        const float hi = ord2f(d.sceneBox[6 * sc + 3 + a]);
        const float ext = hi - lo;
        float c = ext > 0.f ? (m[a] - lo) / ext : 0.5f;
        int qv = (int)(c * 1024.f);
        qv = qv < 0 ? 0 : (qv > 1023 ? 1023 : qv);
        code |= morton_spread10((uint32_t)qv) << (2 - a);
    }
    d.keys[0][si] = ((unsigned long long)sc << 30) | code;
    d.vals[0][si] = k;
}

__device__ __forceinline__ int kdelta(const unsigned long long* __restrict__ keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(i ^ j);
    return __clzll(a ^ b);
}

// Karras 2012 internal-node emission + scene subtree roots.
template <typename R>
__global__ void __launch_bounds__(256) k_karras(Dev<R> d, const unsigned long long* __restrict__ keys,
                                                const int* __restrict__ vals) {
    const int n = d.nseg;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // single-leaf scenes
    {
        const unsigned long long sc = keys[i] >> 30;
        const bool lo = (i == 0) || ((keys[i - 1] >> 30) != sc);
        const bool hi = (i == n - 1) || ((keys[i + 1] >> 30) != sc);
        if (lo && hi) d.sceneRoot[sc] = -(vals[i] + 1);
    }
    if (i >= n - 1) return;
    const int dir = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(keys, n, i, i - dir);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * dir) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * dir) > dmin) l += t;
    const int j = i + l * dir;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (kdelta(keys, n, i, i + (s + t) * dir) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * dir + (dir < 0 ? -1 : 0);
    const int first = min(i, j), last = max(i, j);
    BNode<R>& nd = d.nodes[i];
    nd.split = gamma;
    d.nodeLast[i] = last;
    if (first == gamma) {
        nd.left = -(vals[gamma] + 1);
        d.leafParent[gamma] = i;
    } else {
        nd.left = gamma;
        d.nodes[gamma].parent = i;
    }
    if (last == gamma + 1) {
        nd.right = -(vals[gamma + 1] + 1);
        d.leafParent[gamma + 1] = i;
    } else {
        nd.right = gamma + 1;
        d.nodes[gamma + 1].parent = i;
    }
    if (i == 0) nd.parent = -1;
    const unsigned long long sc = keys[first] >> 30;
    if ((keys[last] >> 30) == sc && (first == 0 || (keys[first - 1] >> 30) != sc) &&
        (last == n - 1 || (keys[last + 1] >> 30) != sc)) {
        d.sceneRoot[sc] = i;
        d.sceneLast[sc] = last;
    }
}

template <typename R>
__device__ __forceinline__ void store_child_box(BNode<R>& nd, bool left, const Box<R>& b) {
    R* mn = left ? nd.lmin : nd.rmin;
    R* mx = left ? nd.lmax : nd.rmax;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        __stcg(mn + a, b.mn[a]);
        __stcg(mx + a, b.mx[a]);
    }
}

// Bottom-up refit: leaf boxes from the current positions/velocity radius, unions upward.
// refitCount must be zero on entry (cleared by the launcher).
template <typename R>
__global__ void __launch_bounds__(256) k_refit(Dev<R> d, const int* __restrict__ sortedVals) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= d.nseg) return;
    const int k = sortedVals[p];
    const int sc = scene_of(d.vp[k].flags);
    const SceneParams<R>& sp = d.sp[sc];
    Box<R> b = segment_box(d, k, sp);
    {
        QRec<R> r;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            r.mn[a] = b.mn[a];
            r.mx[a] = b.mx[a];
        }
        r.k = k;
        r.sc = sc;
        d.qrec[p] = r;
    }
    int code = -(k + 1);
    if (d.nseg == 1) return;
    int node = d.leafParent[p];
    int guard = 0;
    while (node >= 0) {
        if (node >= d.nseg - 1) {  // only a corrupt tree gets here: report, touch nothing
            atomicOr(&d.err[EW_INTERNAL], IE_REFIT);
            return;
        }
        BNode<R>& nd = d.nodes[node];
        const bool isLeft = (nd.left == code);
        store_child_box(nd, isLeft, b);
        // device-scope acquire-release: the first arrival's box stores are visible to the
        // second arrival, which finishes the node
        const unsigned old =
            cuda::atomic_ref<unsigned, cuda::thread_scope_device>(d.refitCount[node]).fetch_add(
                1u, cuda::memory_order_acq_rel);
        if (old == 0u) return;  // first arrival: the sibling finishes this node
        const R* omn = isLeft ? nd.rmin : nd.lmin;
        const R* omx = isLeft ? nd.rmax : nd.lmax;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            b.mn[a] = ymin(b.mn[a], __ldcg(omn + a));
            b.mx[a] = ymax(b.mx[a], __ldcg(omx + a));
        }
        code = node;
        node = nd.parent;
        if (++guard > 4096) {  // a cycle would mean a corrupt tree: stop and report
            atomicOr(&d.err[EW_INTERNAL], IE_REFIT);
            return;
        }
    }
}

// Depth marks for the wide records (rebuild).  Pointer jumping: after round r every node
// knows its distance to the ancestor 2^r levels up (or to the root, with link -1).  A node's
// record is used when its depth below its scene's root is even; a link left after the last
// round (a tree 2^DEPTH_ROUNDS deep or more) makes every record built.
template <typename R>
__global__ void __launch_bounds__(256) k_depth_init(Dev<R> d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nseg - 1) return;
    const int p = d.nodes[i].parent;
    d.depJump[0][i] = p;
    d.depDist[0][i] = p >= 0 ? 1 : 0;
}

template <typename R>
__global__ void __launch_bounds__(256) k_depth_jump(Dev<R> d, int src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nseg - 1) return;
    const int j = d.depJump[src][i];
    int dist = d.depDist[src][i], jj = -1;
    if (j >= 0) {
        dist += d.depDist[src][j];
        jj = d.depJump[src][j];
    }
    d.depDist[src ^ 1][i] = dist;
    d.depJump[src ^ 1][i] = jj;
}

template <typename R>
__global__ void __launch_bounds__(256) k_depth_mark(Dev<R> d, int fin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nseg - 1) return;
    if (d.depJump[fin][i] >= 0) *d.wideAll = 1;
    // internal node i's leaf range has leaf i at one end, so leaf i's key names its scene
    const int root = d.sceneRoot[(int)(d.keys[0][i] >> 30)];
    int used = 0;
    if (root >= 0) {
        const int rel = d.depDist[fin][i] - d.depDist[fin][root];
        used = rel >= 0 && (rel & 1) == 0;
    }
    d.wideUsed[i] = (unsigned char)used;
}

// Wide nodes from the refitted binary tree: node i's entries are the children of its two
// children (a leaf child is an entry itself), so a walk over wide nodes loads one node per
// two binary levels.  Entry order: left child's left, left child's right, right child's left,
// right child's right.
template <typename R>
__global__ void __launch_bounds__(256) k_widen(Dev<R> d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nseg - 1) return;
    if (!d.wideUsed[i] && !*d.wideAll) return;  // a record the walk never loads
    const BNode<R> nd = d.nodes[i];
    WNode<R> w;
    int e = 0;
    auto put = [&](int code, const R* mn, const R* mx, int last) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            w.e[e].mn[a] = mn[a];
            w.e[e].mx[a] = mx[a];
        }
        w.e[e].code = code;
        w.e[e].last = last;
        e++;
    };
    const int lastI = d.nodeLast[i];
    // left child covers [first, split], right child [split + 1, last]
    const int kid[2] = {nd.left, nd.right};
    const int kidLast[2] = {nd.split, lastI};
    const R* kmn[2] = {nd.lmin, nd.rmin};
    const R* kmx[2] = {nd.lmax, nd.rmax};
#pragma unroll
    for (int c = 0; c < 2; c++) {
        if (kid[c] < 0) {
            put(kid[c], kmn[c], kmx[c], kidLast[c]);
            R emn[3] = {yinf<R>(), yinf<R>(), yinf<R>()}, emx[3] = {-yinf<R>(), -yinf<R>(), -yinf<R>()};
            put(WIDE_NONE, emn, emx, -1);
        } else {
            const BNode<R>& ch = d.nodes[kid[c]];
            put(ch.left, ch.lmin, ch.lmax, ch.split);
            put(ch.right, ch.rmin, ch.rmax, kidLast[c]);
        }
    }
    d.wide[i] = w;
}

constexpr int BVH_STACK = 96;
constexpr int TRAV_THREADS = 128;
constexpr int TRAV_WARPS = TRAV_THREADS / 32;
constexpr int TRAV_QCAP = 160;      // < 32 left over + up to 4 candidates per lane
constexpr int TRAV_GRAB = 32;       // queries a warp takes from the counter at a time

// Appends y to x's contact list.  The count keeps growing past MAX_COLS so that the list
// kernel can report the overflow (collision.cu:80-90).
template <typename R>
__device__ __forceinline__ void list_append(const Dev<R>& d, int x, int y) {
    const int pos = atomicAdd(&d.numCols[x], 1);
    if (pos < MAX_COLS) d.cols[col_at(x, pos)] = y;
}

// Broadphase + narrow phase.  Every segment queries the tree once with its own box (the
// sorted leaves of the last rebuild, taken in Morton order, so neighbouring lanes start on
// neighbouring queries).  Each unordered pair is found by exactly one of its two segments:
// the one with the lower sorted position, whose walk skips every entry holding only leaves at
// or before its own position.  The walk runs over the wide nodes (four grandchildren per
// node), so a query takes half as many dependent node loads as on the binary tree.  Lanes walk
// independently, with a per-lane stack; a lane that finishes takes the next query of its
// warp's range of TRAV_GRAB queries (ranges come from a global counter, the next one requested
// while the current one is used), so a warp keeps all 32 lanes busy until the queries run out
// (persistent grid) with one atomic per TRAV_GRAB queries.  A leaf entry that overlaps a lane's box
// becomes a candidate pair in a per-warp queue; whenever 32 candidates are queued the warp
// runs the separately rounded narrow-phase test on them, one pair per lane, with the lower
// segment index as segment A, and appends kept pairs to both lists.  The pair set is the same
// as an all-pairs test: the test is symmetric and every overlapping pair is visited once.
template <typename R>
__device__ __forceinline__ void trav_load_wide(const WNode<R>* wide, int node, WNode<R>& w) {
    if constexpr (sizeof(R) == 4) {  // one wide node = eight 16-byte loads
        const float4* src = reinterpret_cast<const float4*>(wide + node);
        float4* dst = reinterpret_cast<float4*>(&w);
#pragma unroll
        for (int k = 0; k < 8; k++) dst[k] = __ldg(src + k);
    } else {
        w = wide[node];
    }
}

// Warp-cooperative load of the 32 lanes' current records (FP32 records: eight 16-byte
// pieces, one 128-byte line).  Loading its own record, each lane would touch 32 different lines
// with each of its 8 loads (256 L1 wavefronts per step of the warp); here load r fetches piece
// (lane & 7) of the record of lane 4r + (lane >> 3), so each load covers 4 whole lines (32
// wavefronts per step), and the pieces reach their lanes through shared memory (rows padded to
// 9 pieces, so the reads back are free of bank conflicts).  node < 0: the lane loads nothing.
constexpr int COOP_ROW = 9;

__device__ __forceinline__ void coop_load_wide(const WNode<float>* wide, int node, float4 (*rows)[COOP_ROW], int lane) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const int owner = 4 * r + (lane >> 3);
        const int on = __shfl_sync(0xffffffffu, node, owner);
        if (on >= 0) rows[owner][lane & 7] = __ldg(reinterpret_cast<const float4*>(wide + on) + (lane & 7));
    }
    __syncwarp();
}

// Entry e of a wide record: from the lane's shared-memory row (cooperative load) or from
// the record in registers.
template <typename R>
__device__ __forceinline__ WEntry<R> wide_entry(const WNode<R>& w, const float4* row, int e, bool fromRow) {
    if constexpr (sizeof(R) == 4) {
        if (fromRow) {
            const float4 A = row[2 * e], B = row[2 * e + 1];  // (mn xyz, mx x), (mx yz, code, last)
            WEntry<R> x;
            x.mn[0] = A.x; x.mn[1] = A.y; x.mn[2] = A.z;
            x.mx[0] = A.w; x.mx[1] = B.x; x.mx[2] = B.y;
            x.code = __float_as_int(B.z);
            x.last = __float_as_int(B.w);
            return x;
        }
    }
    return w.e[e];
}

template <typename R, bool COOP>
__global__ void __launch_bounds__(TRAV_THREADS) k_traverse(Dev<R> d) {
    __shared__ int sQx[TRAV_WARPS][TRAV_QCAP];
    __shared__ int sQy[TRAV_WARPS][TRAV_QCAP];
    __shared__ float4 sRec[COOP ? TRAV_WARPS : 1][COOP ? 32 : 1][COOP_ROW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int nseg = d.nseg;
    int stack[BVH_STACK];
    int top = 0;
    int qi = 0, k = -1, node = -1;  // query: sorted position, segment, walk state
    int steps = 0;                  // wide nodes visited by this query (a valid walk visits fewer than nseg)
    bool walking = false;
    Box<R> qb;
    int qn = 0;        // queued candidates (identical in every lane)
    bool more = true;  // the counter has not run out (warp-uniform)
    // Queries are handed out TRAV_GRAB at a time: the warp's current range [poolNext, poolEnd)
    // and, in lane 0, the start of the next range, requested one range ahead so that a refill
    // rarely waits on the counter.  Ranges come from one counter in increasing order, so a
    // warp whose current range reaches nseg holds no later valid query.
    int poolNext = 0, poolEnd = 0;
    int pend = 0;
    if (lane == 0) pend = (int)atomicAdd(d.travNext, (unsigned)TRAV_GRAB);
    while (true) {
        // Refill lanes without a walk.
        const unsigned idle = __ballot_sync(0xffffffffu, !walking);
        if (more && idle) {
            const int need = __popc(idle);  // <= 32 <= TRAV_GRAB: at most one new range
            const int avail = poolEnd - poolNext;
            int next = 0;
            if (avail < need) {
                next = __shfl_sync(0xffffffffu, pend, 0);
                if (lane == 0) pend = (int)atomicAdd(d.travNext, (unsigned)TRAV_GRAB);
            }
            if (!walking) {
                const int rank = __popc(idle & lt);
                qi = rank < avail ? poolNext + rank : next + (rank - avail);
                if (qi < nseg) {
                    QRec<R> r;
                    if constexpr (sizeof(R) == 4) {
                        const float4* src = reinterpret_cast<const float4*>(d.qrec + qi);
                        float4* dst = reinterpret_cast<float4*>(&r);
                        dst[0] = __ldg(src);
                        dst[1] = __ldg(src + 1);
                    } else {
                        r = d.qrec[qi];
                    }
                    k = r.k;
                    const int sc = r.sc;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        qb.mn[a] = r.mn[a];
                        qb.mx[a] = r.mx[a];
                    }
                    node = d.sceneRoot[sc];
                    top = 0;
                    steps = 0;
                    walking = node >= 0 && d.sceneLast[sc] > qi;  // a leaf root has no pairs
                }
            }
            if (avail >= need) {
                poolNext += need;
            } else {
                poolNext = next + (need - avail);
                poolEnd = next + TRAV_GRAB;
            }
            if (poolNext >= nseg) more = false;
        }
        if (!more && !__any_sync(0xffffffffu, walking) && qn == 0) break;
        int cand[4];
        int nc = 0;
        if (walking && (node >= nseg - 1 || ++steps > nseg)) {  // only a corrupt tree gets here
            atomicOr(&d.err[EW_INTERNAL], IE_BVH_STACK);
            walking = false;
        }
        constexpr bool ROW = COOP && sizeof(R) == 4;
        WNode<R> w;
        if constexpr (ROW) coop_load_wide(d.wide, walking ? node : -1, sRec[warp], lane);
        if (walking) {
            if constexpr (!ROW) trav_load_wide(d.wide, node, w);
            int next = -1;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const WEntry<R> x = wide_entry(w, sRec[COOP ? warp : 0][COOP ? lane : 0], e, ROW);
                const bool hit = x.last > qi && qb.mn[0] <= x.mx[0] && x.mn[0] <= qb.mx[0] && qb.mn[1] <= x.mx[1] &&
                                 x.mn[1] <= qb.mx[1] && qb.mn[2] <= x.mx[2] && x.mn[2] <= qb.mx[2];
                if (!hit) continue;
                const int c = x.code;
                if (c < 0) {
                    cand[nc++] = -c - 1;
                } else if (next < 0) {
                    next = c;
                } else if (top < BVH_STACK) {
                    stack[top++] = c;
                } else {
                    atomicOr(&d.err[EW_INTERNAL], IE_BVH_STACK);
                }
            }
            if (next >= 0) {
                node = next;
            } else if (top > 0) {
                node = stack[--top];
            } else {
                walking = false;
            }
        }
        // queue this lane's candidates at its offset (warp scan of the counts)
        int incl = nc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int at = qn + incl - nc;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if (e < nc) {
                sQx[warp][at + e] = min(k, cand[e]);
                sQy[warp][at + e] = max(k, cand[e]);
            }
        }
        qn += __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();  // also: every lane has read its record row before the next load fills it
        const bool drain = !more && !__any_sync(0xffffffffu, walking);
        while (qn >= 32 || (drain && qn > 0)) {
            const int m = min(qn, 32);
            if (lane < m) {
                const int x = sQx[warp][qn - m + lane];
                const int y = sQy[warp][qn - m + lane];
                if (pair_keep(d, x, y, d.sp[scene_of(d.vp[x].flags)])) {
                    list_append(d, x, y);
                    list_append(d, y, x);
                }
            }
            qn -= m;
            __syncwarp();
        }
    }
}

// Sorts segment k's contact list (n <= MAX_COLS distinct partner ids) ascending, in place.
// Called by all 32 lanes of a warp (k < 0 or n = 0 for lanes without a list).  A list of up to
// 16 entries is sorted by its own thread with a bitonic network on 16 registers; a longer one
// by the whole warp, one list at a time, as a bitonic sort of 128 entries held four per lane
// (entry i = 32 r + lane): steps with a stride of 32 or more swap within a lane, smaller ones
// exchange between lanes.  Padding entries are INT_MAX and sort to the end.
template <typename R>
__device__ __forceinline__ void sort_list(const Dev<R>& d, int k, int n) {
    constexpr int PAD = 0x7fffffff;
    const int lane = threadIdx.x & 31;
    if (k >= 0 && n > 1 && n <= 16) {
        int* __restrict__ cl = d.cols + col_at(k, 0);
        int v[16];
#pragma unroll
        for (int a = 0; a < 16; a++) v[a] = a < n ? cl[a] : PAD;
#pragma unroll
        for (int sz = 2; sz <= 16; sz <<= 1) {
#pragma unroll
            for (int st = sz >> 1; st > 0; st >>= 1) {
#pragma unroll
                for (int a = 0; a < 16; a++) {
                    const int b = a ^ st;
                    if (b > a) {
                        const bool up = (a & sz) == 0;
                        const int x = v[a], y = v[b];
                        const bool sw = up ? (x > y) : (x < y);
                        v[a] = sw ? y : x;
                        v[b] = sw ? x : y;
                    }
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 16; a++)
            if (a < n) cl[a] = v[a];
    }
    unsigned longLists = __ballot_sync(0xffffffffu, k >= 0 && n > 16);
    while (longLists) {
        const int src = __ffs(longLists) - 1;
        longLists &= longLists - 1;
        const int kk = __shfl_sync(0xffffffffu, k, src);
        const int m = __shfl_sync(0xffffffffu, n, src);
        int* __restrict__ cl = d.cols + col_at(kk, 0);
        int v[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = 32 * r + lane;
            v[r] = i < m ? cl[i] : PAD;
        }
#pragma unroll
        for (int sz = 2; sz <= 128; sz <<= 1) {
#pragma unroll
            for (int st = sz >> 1; st > 0; st >>= 1) {
                if (st >= 32) {
                    const int rs = st >> 5;
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        if (r & rs) continue;
                        const int r2 = r | rs;
                        const bool up = ((32 * r + lane) & sz) == 0;
                        const int x = v[r], y = v[r2];
                        const bool sw = up ? (x > y) : (x < y);
                        v[r] = sw ? y : x;
                        v[r2] = sw ? x : y;
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        const int i = 32 * r + lane;
                        const int x = v[r];
                        const int y = __shfl_xor_sync(0xffffffffu, x, st);
                        const bool up = (i & sz) == 0;
                        const bool lower = (i & st) == 0;  // the lower index of the pair
                        v[r] = (lower == up) ? min(x, y) : max(x, y);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = 32 * r + lane;
            if (i < m) cl[i] = v[r];
        }
        __syncwarp();
    }
}

// List pass, every substep, over tiles of LIST_THREADS consecutive vertices.  Per segment after
// the broadphase: clamp and check the count, sort the list by partner id (fixed summation order
// in the Newton iteration); with sortLists = 0 the lists are kept (substeps without detection,
// collision.cu:121-172).  Then the lists of all vertices are packed in vertex order (csrOff,
// csrCols): a tile takes its index from a ticket counter, scans its counts and resolves its
// first slot by decoupled look-back over the tiles before it, 32 at a time (they hold smaller
// tickets, so they are running or done; each wait is bounded and a timeout sets
// IE_LIST_WAIT).  The tile's
// contacts are then evaluated 128 at a time, one per thread: the packed partner id, the
// partner endpoints staged relative to p0 in the same slot, and the step-size limit
// (collision.cu:121-159), of which each segment takes the minimum over its contacts in list
// order (the minimum is exact, so this equals a per-segment loop).  The packed slots are
// contiguous per tile, so the Newton iteration reads them coalesced.
constexpr int LIST_SPIN_LIMIT = 1 << 22;
constexpr unsigned long long LS_AGG = 1ull << 62;
constexpr unsigned long long LS_PRE = 2ull << 62;
constexpr unsigned long long LS_VAL = (1ull << 62) - 1;

template <typename R>
__global__ void __launch_bounds__(LIST_THREADS) k_lists(Dev<R> d, int sortLists) {
    constexpr int B = LIST_THREADS;
    __shared__ int sOff[B + 1];
    __shared__ int sWarp[B / 32];
    __shared__ int sTile;
    __shared__ unsigned long long sBase;
    __shared__ R sA0[3][B], sA1[3][B];
    __shared__ int sScene[B];
    __shared__ R sLim[B];
    const int t = threadIdx.x;
    if (t == 0) sTile = (int)atomicAdd(d.listStatus, 1ull);
    __syncthreads();
    const int tile = sTile;
    const int k = tile * B + t;
    const bool inRange = k < d.n;
    bool valid = false;  // k is a segment
    int nc = 0, sc = 0, rawCount = 0;
    V3<R> a0(R(0)), a1(R(0));
    if (inRange) {
        const uint32_t fl = d.vp[k].flags;
        valid = (fl & F_HAS_NEXT) != 0;
        if (valid) {
            sc = scene_of(fl);
            nc = d.numCols[k];
            rawCount = nc;
            if (sortLists && nc > MAX_COLS) d.err[EW_ERROR] = 1;
            nc = min(nc, MAX_COLS);
            if (sortLists) d.numCols[k] = nc;
            a0 = xyz(d.pos[k]);
            a1 = xsub(xyz(d.pos[k + 1]), a0);
        }
    }
    {
        const int lane = t & 31, w = t >> 5;
        int x = nc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sWarp[w] = x;
        __syncthreads();
        int wo = 0;
        for (int i = 0; i < w; i++) wo += sWarp[i];
        sOff[t] = wo + x - nc;
        if (t == B - 1) sOff[B] = wo + x;
        __syncthreads();
    }
    // The tile's count is published before the sort, so that a later tile's look-back rarely
    // has to wait for it.
    volatile unsigned long long* st = d.listStatus + 1;
    if (t == 0) st[tile] = (tile == 0 ? LS_PRE : LS_AGG) | (unsigned long long)sOff[B];
    if (sortLists) {
        // largest list of the warp (before the clamp), one atomic per warp
        int m = rawCount;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((t & 31) == 0 && m) atomicMax(&d.err[EW_MAX_COLS], m);
        sort_list(d, valid ? k : -1, nc);
    }
    sScene[t] = sc;
    sA0[0][t] = a0.x; sA0[1][t] = a0.y; sA0[2][t] = a0.z;
    sA1[0][t] = a1.x; sA1[1][t] = a1.y; sA1[2][t] = a1.z;
    // first packed slot of this tile: decoupled look-back by warp 0, 32 predecessors at a time
    // (lane l reads tile hi - l; the window ends at the nearest tile that holds a prefix)
    if (t < 32) {
        const unsigned FULL = 0xffffffffu;
        const unsigned long long agg = (unsigned long long)sOff[B];
        unsigned long long excl = 0;
        bool timedOut = false;
        if (tile > 0) {
            for (int hi = tile - 1; hi >= 0; hi -= 32) {
                const int p = hi - t;
                unsigned long long w = LS_PRE;  // before tile 0: an inclusive prefix of 0
                if (p >= 0) {
                    w = st[p];
                    int spins = 0;
                    while ((w >> 62) == 0ull) {
                        if (++spins > LIST_SPIN_LIMIT) {
                            timedOut = true;
                            break;
                        }
                        if (spins > 64) __nanosleep(32);
                        w = st[p];
                    }
                }
                if (__any_sync(FULL, timedOut)) {
                    timedOut = true;
                    break;
                }
                const unsigned pre = __ballot_sync(FULL, (w & LS_PRE) != 0ull);
                const int stop = pre ? __ffs(pre) - 1 : 31;
                unsigned long long v = t <= stop ? (w & LS_VAL) : 0ull;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
                excl += v;
                if (pre) break;
            }
            if (t == 0) {
                if (timedOut) atomicOr(&d.err[EW_INTERNAL], IE_LIST_WAIT);
                st[tile] = LS_PRE | (excl + agg);
            }
        }
        if (t == 0) {
            if (excl + agg > (unsigned long long)d.csrCap) atomicOr(&d.err[EW_INTERNAL], IE_CONTACT);
            sBase = excl;
        }
    }
    __syncthreads();
    const unsigned long long base = sBase;
    const int total = sOff[B];
    const int myOff = sOff[t];
    if (inRange) {
        d.csrOff[k] = (unsigned)(base + myOff);
        if (k == d.n - 1) d.csrOff[d.n] = (unsigned)(base + myOff + nc);
    }
    R m = R(0);
    if (valid) m = step_limit_base(d, k, d.sp[sc]);
    int pens = 0;
    float dmin = INFINITY;
    for (int b0 = 0; b0 < total; b0 += B) {
        const int f = b0 + t;
        R lim = yinf<R>();
        if (f < total) {
            int lo = 0, hi = B - 1;  // owner: the last slot whose offset is <= f
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sOff[mid] <= f) lo = mid; else hi = mid - 1;
            }
            const int s = lo, c = f - sOff[s];
            const int ks = tile * B + s;
            const int o = d.cols[col_at(ks, c)];
            const unsigned long long g = base + (unsigned long long)f;
            if (g < (unsigned long long)d.csrCap) d.csrCols[g] = o;
            const V3<R> oa0(sA0[0][s], sA0[1][s], sA0[2][s]);
            const V3<R> oa1(sA1[0][s], sA1[1][s], sA1[2][s]);
            bool pen = false;
            R dist;
            lim = contact_step_limit(d, ks, g < (unsigned long long)d.relCap ? (size_t)g : NO_STAGE, o, oa0, oa1,
                                     d.sp[sScene[s]], pen, dist);
            pens += pen;
            dmin = fminf(dmin, (float)dist);
        }
        sLim[t] = lim;
        __syncthreads();
        const int f0 = max(myOff, b0), f1 = min(myOff + nc, b0 + B);
        for (int g = f0; g < f1; g++) m = ymin(m, sLim[g - b0]);
        __syncthreads();
    }
    if (pens) {
        atomicAdd(&d.err[EW_PENETRATIONS], pens);
        d.err[EW_WARNING] = 2;
    }
    // distances are >= 0, whose float bit patterns order like the integers
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmin = fminf(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
    if ((t & 31) == 0 && dmin < INFINITY) atomicMin(&d.err[EW_MIN_DIST], __float_as_int(dmin));
    if (valid) d.stepLim[k] = d.sp[sc].useStepLimit ? m : yinf<R>();
}

// Packet traversal: a warp walks the tree once for 32 consecutive queries (consecutive sorted
// positions, so neighbouring segments in Morton order).  Every lane tests its own box against
// the entries of the node the warp has loaded (one record, read by all lanes at the same
// address); the warp descends into an internal entry when any of its lanes overlaps it, keeping
// one stack per warp in shared memory.  The walk is the union of the 32 walks of k_traverse,
// but each node is loaded once per warp instead of once per lane, so the chain of dependent
// node loads is paid once per 32 queries.  Each lane keeps exactly the leaves k_traverse keeps
// for it (its own box, leaves after its sorted position), so the pair set is identical; lanes
// of different scenes in one warp walk their scenes one after the other.
constexpr int PK_STACK = 64;

template <typename R>
__global__ void __launch_bounds__(TRAV_THREADS) k_traverse_packet(Dev<R> d) {
    __shared__ int sQx[TRAV_WARPS][TRAV_QCAP];
    __shared__ int sQy[TRAV_WARPS][TRAV_QCAP];
    __shared__ int sStack[TRAV_WARPS][PK_STACK];
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nseg = d.nseg;
    int* stack = sStack[warp];
    int qn = 0;  // queued candidates (identical in every lane)
    auto drain = [&](bool all) {
        while (qn >= 32 || (all && qn > 0)) {
            const int m = min(qn, 32);
            if (lane < m) {
                const int x = sQx[warp][qn - m + lane];
                const int y = sQy[warp][qn - m + lane];
                if (pair_keep(d, x, y, d.sp[scene_of(d.vp[x].flags)])) {
                    list_append(d, x, y);
                    list_append(d, y, x);
                }
            }
            qn -= m;
            __syncwarp();
        }
    };
    while (true) {
        int base = 0;
        if (lane == 0) base = (int)atomicAdd(d.travNext, 32u);
        base = __shfl_sync(FULL, base, 0);
        if (base >= nseg) break;
        const int qi = base + lane;
        bool live = qi < nseg;
        int k = -1, sc = -1;
        Box<R> qb;
        if (live) {
            QRec<R> r;
            if constexpr (sizeof(R) == 4) {
                const float4* src = reinterpret_cast<const float4*>(d.qrec + qi);
                float4* dst = reinterpret_cast<float4*>(&r);
                dst[0] = __ldg(src);
                dst[1] = __ldg(src + 1);
            } else {
                r = d.qrec[qi];
            }
            k = r.k;
            sc = r.sc;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                qb.mn[a] = r.mn[a];
                qb.mx[a] = r.mx[a];
            }
            live = d.sceneRoot[sc] >= 0 && d.sceneLast[sc] > qi;  // a leaf root has no pairs
        }
        unsigned todo = __ballot_sync(FULL, live);
        while (todo) {
            const int leader = __ffs(todo) - 1;
            const int wsc = __shfl_sync(FULL, sc, leader);
            const bool mine = live && sc == wsc;
            todo &= ~__ballot_sync(FULL, mine);
            int node = d.sceneRoot[wsc];
            int top = 0, steps = 0;
            while (node >= 0) {
                if (node >= nseg - 1 || ++steps > nseg) {  // only a corrupt tree gets here
                    if (lane == 0) atomicOr(&d.err[EW_INTERNAL], IE_BVH_STACK);
                    break;
                }
                WNode<R> w;
                trav_load_wide(d.wide, node, w);
                int cand[4];
                int nc = 0;
                int next = -1;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const WEntry<R>& x = w.e[e];
                    const bool hit = mine && x.last > qi && qb.mn[0] <= x.mx[0] && x.mn[0] <= qb.mx[0] &&
                                     qb.mn[1] <= x.mx[1] && x.mn[1] <= qb.mx[1] && qb.mn[2] <= x.mx[2] &&
                                     x.mn[2] <= qb.mx[2];
                    const int c = x.code;  // the same in every lane
                    if (c < 0) {
                        if (hit) cand[nc++] = -c - 1;
                    } else if (__any_sync(FULL, hit)) {
                        if (next < 0) {
                            next = c;
                        } else if (top < PK_STACK) {
                            if (lane == 0) stack[top] = c;
                            top++;
                        } else if (lane == 0) {
                            atomicOr(&d.err[EW_INTERNAL], IE_BVH_STACK);
                        }
                    }
                }
                // queue this lane's candidates at its offset (warp scan of the counts)
                int incl = nc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += y;
                }
                const int at = qn + incl - nc;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    if (e < nc) {
                        sQx[warp][at + e] = min(k, cand[e]);
                        sQy[warp][at + e] = max(k, cand[e]);
                    }
                }
                qn += __shfl_sync(FULL, incl, 31);
                __syncwarp();
                drain(false);
                if (next >= 0) {
                    node = next;
                } else if (top > 0) {
                    node = stack[--top];
                } else {
                    node = -1;
                }
            }
            __syncwarp();
        }
    }
    drain(true);
}

template <typename R>
void launch_bvh_rebuild(const Dev<R>& d, cudaStream_t s, void* sortScratch, size_t, int keyBits) {
    if (d.nseg <= 0) return;
    const int nb = (d.nseg + 255) / 256;
    k_scene_box_init<R><<<(d.numScenes + 127) / 128, 128, 0, s>>>(d);
    k_scene_bounds<R><<<nb, 256, 0, s>>>(d);
    k_morton<R><<<nb, 256, 0, s>>>(d);
    unsigned long long* keys[2] = {d.keys[0], d.keys[1]};
    int* vals[2] = {d.vals[0], d.vals[1]};
    const int buf = radix_sort_pairs(keys, vals, d.nseg, keyBits, sortScratch, d.err + EW_INTERNAL, s);
    // After sorting, buffer 0 must hold the sorted pairs (refit/karras read it).
    if (buf != 0) {
        cudaMemcpyAsync(d.keys[0], d.keys[1], sizeof(unsigned long long) * d.nseg, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d.vals[0], d.vals[1], sizeof(int) * d.nseg, cudaMemcpyDeviceToDevice, s);
    }
    k_karras<R><<<nb, 256, 0, s>>>(d, d.keys[0], d.vals[0]);
    // DEPTH_LAUNCHES kernels: which wide records the walk can load
    const int ib = (max(d.nseg - 1, 1) + 255) / 256;
    cudaMemsetAsync(d.wideAll, 0, sizeof(int), s);
    k_depth_init<R><<<ib, 256, 0, s>>>(d);
    for (int r = 0; r < DEPTH_ROUNDS; r++) k_depth_jump<R><<<ib, 256, 0, s>>>(d, r & 1);
    k_depth_mark<R><<<ib, 256, 0, s>>>(d, DEPTH_ROUNDS & 1);
    launch_bvh_refit(d, s);
}

template <typename R>
void launch_bvh_reset(const Dev<R>& d, cudaStream_t s) {
    if (d.numScenes > 0) k_scene_box_init<R><<<(d.numScenes + 127) / 128, 128, 0, s>>>(d);
}

template <typename R>
void launch_bvh_refit(const Dev<R>& d, cudaStream_t s) {
    if (d.nseg <= 0) return;  // one segment: no internal node, but its query record is written
    if (d.nseg > 1) cudaMemsetAsync(d.refitCount, 0, sizeof(unsigned) * (d.nseg - 1), s);
    k_refit<R><<<(d.nseg + 255) / 256, 256, 0, s>>>(d, d.vals[0]);
    k_widen<R><<<(d.nseg + 255) / 256, 256, 0, s>>>(d);  // at least one block; the kernel bounds itself
}

template <typename R>
void launch_lists(const Dev<R>& d, int sortLists, cudaStream_t s) {
    const int tiles = (d.n + LIST_THREADS - 1) / LIST_THREADS;
    cudaMemsetAsync(d.listStatus, 0, sizeof(unsigned long long) * (1 + (size_t)tiles), s);
    k_lists<R><<<tiles, LIST_THREADS, 0, s>>>(d, sortLists);
}

template <typename R>
void launch_traverse(const Dev<R>& d, cudaStream_t s) {
    if (d.nseg <= 0) return;
    cudaMemsetAsync(d.numCols, 0, sizeof(int) * d.n, s);
    cudaMemsetAsync(d.travNext, 0, sizeof(unsigned), s);
    const int blocks = min((d.nseg + TRAV_THREADS - 1) / TRAV_THREADS, max(d.travBlocks[d.travPacket], 1));
    if (d.travPacket == 1)
        k_traverse_packet<R><<<blocks, TRAV_THREADS, 0, s>>>(d);
    else if (d.travPacket == 2)
        k_traverse<R, true><<<blocks, TRAV_THREADS, 0, s>>>(d);
    else
        k_traverse<R, false><<<blocks, TRAV_THREADS, 0, s>>>(d);
    launch_lists(d, 1, s);
}

template <typename R>
void launch_lists_step_limit(const Dev<R>& d, cudaStream_t s) {
    if (d.nseg <= 0) {  // no segment, no contact: the packed lists are empty
        if (d.n > 0) cudaMemsetAsync(d.csrOff, 0, sizeof(unsigned) * (d.n + 1), s);
        return;
    }
    launch_lists(d, 0, s);
}

template void launch_bvh_rebuild<float>(const Dev<float>&, cudaStream_t, void*, size_t, int);
template void launch_bvh_rebuild<double>(const Dev<double>&, cudaStream_t, void*, size_t, int);
template void launch_bvh_refit<float>(const Dev<float>&, cudaStream_t);
template void launch_bvh_refit<double>(const Dev<double>&, cudaStream_t);
template void launch_bvh_reset<float>(const Dev<float>&, cudaStream_t);
template void launch_bvh_reset<double>(const Dev<double>&, cudaStream_t);
template <typename R>
int traverse_blocks_per_sm(int mode) {  // resident blocks of the traversal kernel of a walk mode
    int b = 0;
    const cudaError_t e =
        mode == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_traverse_packet<R>, TRAV_THREADS, 0)
        : mode == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_traverse<R, true>, TRAV_THREADS, 0)
                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_traverse<R, false>, TRAV_THREADS, 0);
    if (e != cudaSuccess || b < 1) {
        cudaGetLastError();
        return 4;
    }
    return b;
}
template int traverse_blocks_per_sm<float>(int);
template int traverse_blocks_per_sm<double>(int);
template void launch_traverse<float>(const Dev<float>&, cudaStream_t);
template void launch_lists_step_limit<float>(const Dev<float>&, cudaStream_t);
template void launch_lists_step_limit<double>(const Dev<double>&, cudaStream_t);
template void launch_traverse<double>(const Dev<double>&, cudaStream_t);

}  // namespace yb
