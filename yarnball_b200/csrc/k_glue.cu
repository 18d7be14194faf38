// k_glue.cu - nearest vertex of every yarn endpoint, for Sim::glueEndpoints
// (io/jsonBuilder.cpp:174-212, where it is an O(endpoints x vertices) OpenMP loop).
//
// For endpoint i the candidate set is every vertex j of its scene with |i - j| > 2; the
// distance is glm::length(p_i - p_j) in float, evaluated with separately rounded operations
// ((dx dx + dy dy) + dz dz, then a correctly rounded square root) so that it equals the host
// evaluation bit for bit.  The result is packed as (distance bits << 32) | j: distances are
// non-negative, so their bit patterns order like the values, and the 64-bit minimum is the
// smallest distance with the smallest index among ties, i.e. the first minimum the
// reference's strict "<" scan keeps.  Each block holds 128 endpoints (one per thread) and
// walks one slice of the vertex array through shared memory; slices are combined with a
// 64-bit atomicMin.
#include <cuda_runtime.h>

#include <cstdint>

namespace yb {

namespace {

constexpr int GLUE_THREADS = 128;
constexpr int GLUE_TILE = 1024;

__global__ void __launch_bounds__(GLUE_THREADS) k_glue_nearest(const float4* __restrict__ pos, int n,
                                                               const int* __restrict__ ends,
                                                               const int* __restrict__ lo,
                                                               const int* __restrict__ hi, int count,
                                                               int sliceLen, unsigned long long* __restrict__ keys) {
    __shared__ float4 tile[GLUE_TILE];
    const int e = blockIdx.x * GLUE_THREADS + threadIdx.x;
    const bool active = e < count;
    int i = 0, a = 0, b = 0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
        i = ends[e];
        a = lo[e];
        b = hi[e];
        pi = pos[i];
    }
    const int s0 = blockIdx.y * sliceLen;
    const int s1 = min(n, s0 + sliceLen);
    unsigned long long best = ~0ull;
    for (int t0 = s0; t0 < s1; t0 += GLUE_TILE) {
        const int tn = min(GLUE_TILE, s1 - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < tn; k += GLUE_THREADS) tile[k] = pos[t0 + k];
        __syncthreads();
        if (!active) continue;
        const int k0 = max(a - t0, 0), k1 = min(b - t0, tn);
        for (int k = k0; k < k1; k++) {
            const int j = t0 + k;
            if (abs(i - j) <= 2) continue;
            const float4 pj = tile[k];
            const float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y), dz = __fsub_rn(pi.z, pj.z);
            const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            const float d = __fsqrt_rn(d2);
            if (!(d == d)) continue;  // NaN positions take no part
            const unsigned long long key = ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)j;
            best = key < best ? key : best;
        }
    }
    if (active && best != ~0ull) atomicMin(keys + e, best);
}

}  // namespace

cudaError_t glue_nearest(const float* pos4, int n, const int* endpoints, const int* lo, const int* hi, int count,
                         unsigned long long* keys) {
    if (count <= 0) return cudaSuccess;
    float4* dPos = nullptr;
    int* dInt = nullptr;
    unsigned long long* dKeys = nullptr;
    cudaError_t e = cudaMalloc(&dPos, sizeof(float4) * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dInt, sizeof(int) * 3 * (size_t)count);
    if (e == cudaSuccess) e = cudaMalloc(&dKeys, sizeof(unsigned long long) * (size_t)count);
    if (e == cudaSuccess) e = cudaMemcpy(dPos, pos4, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dInt, endpoints, sizeof(int) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dInt + count, lo, sizeof(int) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dInt + 2 * count, hi, sizeof(int) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dKeys, 0xff, sizeof(unsigned long long) * (size_t)count);
    if (e == cudaSuccess) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int bx = (count + GLUE_THREADS - 1) / GLUE_THREADS;
        // enough vertex slices for about 8 blocks per SM, each slice at least one tile
        int slices = (8 * sms + bx - 1) / bx;
        const int maxSlices = (n + GLUE_TILE - 1) / GLUE_TILE;
        slices = slices < 1 ? 1 : (slices > maxSlices ? maxSlices : slices);
        if (slices > 65535) slices = 65535;
        const int sliceLen = (n + slices - 1) / slices;
        k_glue_nearest<<<dim3(bx, slices), GLUE_THREADS>>>(dPos, n, dInt, dInt + count, dInt + 2 * count, count,
                                                            sliceLen, dKeys);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(keys, dKeys, sizeof(unsigned long long) * (size_t)count, cudaMemcpyDeviceToHost);
    cudaFree(dPos);
    cudaFree(dInt);
    cudaFree(dKeys);
    return e;
}

}  // namespace yb
