// k_sort.cu - stable LSD radix sort of (u64 key, int value) pairs, one kernel per 8-bit
// digit ("onesweep": Adinets & Merrill 2022).
//
//   1. one histogram kernel counts every digit of every pass in a single read of the keys;
//   2. a one-block kernel turns the histograms into per-pass digit offsets;
//   3. per pass, each CTA takes the next tile (2048 keys) from an atomic counter, ranks its
//      keys per digit with warp match (stable: warp-striped order = input order), publishes its
//      per-digit count, and resolves its global offset by decoupled look-back over the
//      predecessors' published counts/prefixes, then scatters.
// Tiles only wait on tiles that obtained a smaller index from the counter, i.e. that are
// already running, so the look-back always completes; every wait is still bounded and a
// timeout sets IE_SORT_WAIT in the error word instead of hanging.

#include "engine.cuh"
#include "yarnball_b200.h"

namespace yb {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_MAX_PASSES = 8;
constexpr unsigned ST_AGG = 1u << 30;
constexpr unsigned ST_PRE = 2u << 30;
constexpr unsigned ST_CNT = (1u << 30) - 1;
constexpr int SORT_SPIN_LIMIT = 1 << 22;

static inline int sort_tiles(int n) { return (n + SORT_TILE - 1) / SORT_TILE; }

size_t radix_sort_scratch_bytes(int n) {
    const size_t tiles = (size_t)sort_tiles(n < 1 ? 1 : n);
    return sizeof(unsigned) * (SORT_MAX_PASSES * 256 + SORT_MAX_PASSES + SORT_MAX_PASSES * tiles * 256);
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(const unsigned long long* __restrict__ keys, int n,
                                                            int passes, unsigned* __restrict__ hist) {
    __shared__ unsigned sh[SORT_MAX_PASSES][256];
    for (int i = threadIdx.x; i < SORT_MAX_PASSES * 256; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        for (int p = 0; p < passes; p++) atomicAdd(&sh[p][(unsigned)(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
        const unsigned v = (&sh[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
}

// Exclusive scan of each pass's 256 digit counts (in place).  One block of 256 threads.
__global__ void __launch_bounds__(256) k_sort_scan(unsigned* __restrict__ hist, int passes) {
    __shared__ unsigned warpSum[8];
    const int d = threadIdx.x, lane = d & 31, w = d >> 5;
    for (int p = 0; p < passes; p++) {
        const unsigned v = hist[p * 256 + d];
        unsigned x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSum[w] = x;
        __syncthreads();
        unsigned off = 0;
        for (int i = 0; i < w; i++) off += warpSum[i];
        hist[p * 256 + d] = off + x - v;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_pass(const unsigned long long* __restrict__ kin,
                                                            const int* __restrict__ vin,
                                                            unsigned long long* __restrict__ kout,
                                                            int* __restrict__ vout, int n, int shift,
                                                            const unsigned* __restrict__ digitOff,
                                                            unsigned* status, unsigned* tileCounter, int* err) {
    __shared__ unsigned sTile;
    __shared__ unsigned sWarp[SORT_WARPS][256];
    __shared__ unsigned sBase[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sTile = atomicAdd(tileCounter, 1u);
    for (int i = tid; i < SORT_WARPS * 256; i += SORT_THREADS) (&sWarp[0][0])[i] = 0u;
    __syncthreads();
    const int tile = (int)sTile;
    const long long base = (long long)tile * SORT_TILE + (long long)warp * 32 * SORT_ITEMS;
    const unsigned ltmask = (1u << lane) - 1u;

    unsigned long long key[SORT_ITEMS];
    int val[SORT_ITEMS];
    unsigned rank[SORT_ITEMS];
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; i++) {
        const long long idx = base + i * 32 + lane;
        const bool valid = idx < n;
        key[i] = valid ? kin[idx] : 0ull;
        val[i] = valid ? vin[idx] : 0;
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        rank[i] = 0;
        if (valid) {
            const unsigned dig = (unsigned)(key[i] >> shift) & 255u;
            const unsigned peers = __match_any_sync(vmask, dig);
            const unsigned cnt = sWarp[warp][dig];
            rank[i] = cnt + __popc(peers & ltmask);
            __syncwarp(vmask);
            if (lane == __ffs(peers) - 1) sWarp[warp][dig] = cnt + __popc(peers);
            __syncwarp(vmask);
        }
    }
    __syncthreads();
    {
        const int d = tid;
        unsigned run = 0;
#pragma unroll
        for (int w = 0; w < SORT_WARPS; w++) {
            const unsigned c = sWarp[w][d];
            sWarp[w][d] = run;
            run += c;
        }
        volatile unsigned* st = status;
        unsigned excl = 0;
        if (tile == 0) {
            st[d] = ST_PRE | run;
        } else {
            st[(size_t)tile * 256 + d] = ST_AGG | run;
            int t = tile - 1;
            bool timedOut = false;
            while (t >= 0 && !timedOut) {
                unsigned wv = st[(size_t)t * 256 + d];
                int spins = 0;
                while ((wv >> 30) == 0u) {
                    if (++spins > SORT_SPIN_LIMIT) {
                        timedOut = true;
                        break;
                    }
                    __nanosleep(32);
                    wv = st[(size_t)t * 256 + d];
                }
                if (timedOut) break;
                excl += wv & ST_CNT;
                if (wv & ST_PRE) break;
                t--;
            }
            if (timedOut) atomicOr(err, IE_SORT_WAIT);
            __threadfence();
            st[(size_t)tile * 256 + d] = ST_PRE | (excl + run);
        }
        sBase[d] = digitOff[d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; i++) {
        const long long idx = base + i * 32 + lane;
        if (idx < n) {
            const unsigned dig = (unsigned)(key[i] >> shift) & 255u;
            const unsigned pos = sBase[dig] + sWarp[warp][dig] + rank[i];
            if (pos < (unsigned)n) {  // always true unless a look-back wait expired
                kout[pos] = key[i];
                vout[pos] = val[i];
            } else {
                atomicOr(err, IE_SORT_WAIT);
            }
        }
    }
}

int radix_sort_pairs(unsigned long long* keys[2], int* vals[2], int n, int bits, void* scratch, int* err,
                     cudaStream_t s) {
    if (n <= 1 || bits <= 0) return 0;
    const int passes = (bits + 7) / 8 > SORT_MAX_PASSES ? SORT_MAX_PASSES : (bits + 7) / 8;
    const int tiles = sort_tiles(n);
    unsigned* hist = (unsigned*)scratch;
    unsigned* counters = hist + SORT_MAX_PASSES * 256;
    unsigned* status = counters + SORT_MAX_PASSES;
    cudaMemsetAsync(scratch, 0, sizeof(unsigned) * (SORT_MAX_PASSES * 256 + SORT_MAX_PASSES + (size_t)passes * tiles * 256), s);
    int hb = (n + SORT_THREADS * 4 - 1) / (SORT_THREADS * 4);
    if (hb > 148 * 8) hb = 148 * 8;
    k_sort_hist<<<hb, SORT_THREADS, 0, s>>>(keys[0], n, passes, hist);
    k_sort_scan<<<1, 256, 0, s>>>(hist, passes);
    for (int p = 0; p < passes; p++) {
        const int src = p & 1;
        k_sort_pass<<<tiles, SORT_THREADS, 0, s>>>(keys[src], vals[src], keys[src ^ 1], vals[src ^ 1], n, 8 * p,
                                                   hist + p * 256, status + (size_t)p * tiles * 256, counters + p,
                                                   err);
    }
    return passes & 1;
}

}  // namespace yb

// =========================================================================================
// Allocation-free sort (yb_sort_pairs_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a sort: code that
// runs inside a host framework which owns the whole device-memory budget through its own
// pool, or a fixed-budget simulation/render loop where an allocation (which may synchronise
// the device, or fail once memory is fragmented) is treated as an error.  This variant uses
// only the caller's input/output buffers plus one fixed scratch area compiled into the
// library as a file-scope __device__ array.  Every GPU that loads the library holds that
// array (about 4.2 MB) until the process exits.  Each call looks its address up with
// cudaGetSymbolAddress (host code may not use the symbol itself as a device address).  With
// lazy module loading the first call on a device loads the library's kernels and this array
// there, once; later calls allocate nothing.  Each call reads back an error word and
// synchronises its stream, so it cannot be captured in a CUDA graph.  All calls share the
// array: calls whose GPU work overlaps (two streams, or two host threads at once) race on it
// and must be serialised by the caller.
namespace yb {
namespace {

constexpr int NOALLOC_MAX_N = 1 << 18;  // 262,144 pairs (YB_SORT_NOALLOC_MAX_N)
constexpr int NOALLOC_TILES = (NOALLOC_MAX_N + SORT_TILE - 1) / SORT_TILE;
constexpr int NOALLOC_WORDS = SORT_MAX_PASSES * 256 + SORT_MAX_PASSES + SORT_MAX_PASSES * NOALLOC_TILES * 256;

struct NoAllocScratch {
    unsigned long long keys[NOALLOC_MAX_N];
    int vals[NOALLOC_MAX_N];
    unsigned words[NOALLOC_WORDS];  // histograms | tile counters | look-back status words
    int err;
};

static __device__ __align__(256) unsigned char g_sort_scratch[sizeof(NoAllocScratch)];

// Device address of g_sort_scratch in the current context, looked up on every call (a
// driver table lookup), so no address outlives a device reset.
cudaError_t scratch_address(NoAllocScratch** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess) return e;
    *out = (NoAllocScratch*)p;
    return cudaSuccess;
}

}  // namespace
}  // namespace yb

extern "C" yb_status yb_sort_pairs_noalloc(const uint64_t* keysIn, const int32_t* valsIn, uint64_t* keysOut,
                                           int32_t* valsOut, int32_t n, int32_t bits, void* stream) {
    using namespace yb;
    if (n < 0 || bits < 0 || bits > 64) return YB_ERR_INVALID_ARGUMENT;
    if (n > NOALLOC_MAX_N) return YB_ERR_SCRATCH_TOO_SMALL;
    if (n == 0) return YB_OK;
    if (!keysIn || !valsIn || !keysOut || !valsOut) return YB_ERR_INVALID_ARGUMENT;
    // The passes read the input while other blocks scatter into the output, so the output
    // may not overlap the input (an in-place call would corrupt the keys).
    auto overlap = [](const void* a, const void* b, size_t bytes) {
        const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
        return x < y + bytes && y < x + bytes;
    };
    if (overlap(keysIn, keysOut, sizeof(uint64_t) * (size_t)n) || overlap(valsIn, valsOut, sizeof(int32_t) * (size_t)n))
        return YB_ERR_INVALID_ARGUMENT;
    NoAllocScratch* S = nullptr;
    cudaError_t e = scratch_address(&S);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? YB_ERR_OUT_OF_MEMORY : YB_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned long long* kin = (const unsigned long long*)keysIn;
    unsigned long long* kout = (unsigned long long*)keysOut;
    const int passes = n == 1 ? 0 : (bits + 7) / 8;
    if (passes == 0) {
        e = cudaMemcpyAsync(kout, kin, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(valsOut, valsIn, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? YB_OK : YB_ERR_CUDA;
    }
    const int tiles = sort_tiles(n);
    unsigned* hist = S->words;
    unsigned* counters = hist + SORT_MAX_PASSES * 256;
    unsigned* status = counters + SORT_MAX_PASSES;
    // The scratch keeps the previous call's contents: clear what must start at zero.
    e = cudaMemsetAsync(S->words, 0, sizeof(unsigned) * (SORT_MAX_PASSES * 256 + SORT_MAX_PASSES), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(unsigned) * (size_t)passes * tiles * 256, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&S->err, 0, sizeof(int), st);
    if (e != cudaSuccess) return YB_ERR_CUDA;
    int hb = (n + SORT_THREADS * 4 - 1) / (SORT_THREADS * 4);
    k_sort_hist<<<hb, SORT_THREADS, 0, st>>>(kin, n, passes, hist);
    k_sort_scan<<<1, 256, 0, st>>>(hist, passes);
    // Pass p writes the output buffers when (passes-1-p) is even and the scratch otherwise,
    // so the last pass lands in the caller's output; pass 0 reads the caller's input.
    const unsigned long long* srcK = kin;
    const int* srcV = valsIn;
    for (int p = 0; p < passes; p++) {
        const bool toOut = ((passes - 1 - p) & 1) == 0;
        unsigned long long* dstK = toOut ? kout : S->keys;
        int* dstV = toOut ? valsOut : S->vals;
        k_sort_pass<<<tiles, SORT_THREADS, 0, st>>>(srcK, srcV, dstK, dstV, n, 8 * p, hist + p * 256,
                                                    status + (size_t)p * tiles * 256, counters + p, &S->err);
        srcK = dstK;
        srcV = dstV;
    }
    int herr = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, &S->err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return YB_ERR_CUDA;
    return herr ? YB_ERR_INTERNAL : YB_OK;
}
