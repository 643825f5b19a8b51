// bandwidth.cu -- copy-bandwidth probe used as a roofline denominator.
//
// The substep kernel's population array of a 101^3 lattice (78 MB in FP32,
// 39 MB in FP16) fits in the 126 MB L2, so its achieved bandwidth is reported
// against a measured L2 copy bandwidth as well as against the HBM copy
// bandwidth.  This probe copies a buffer back and forth `reps` times inside
// one launch: with a footprint (2 x bytes) well below the L2 size every rep
// after the first is served by L2, with a footprint well above it by HBM.
// Loads and stores go through L2 only (ld.global.cg / st.global.cg), so L1
// never serves a re-read.
//
// A second probe measures the ceiling of the substep kernel's own access
// pattern: every cell of a lattice reads its 19 populations and writes them
// back with nothing computed in between, in the even AA form (the cell's own
// slots, written to the opposite direction's plane) and in the odd form
// (gathered from the 18 neighbours' slots, scattered back to them), with the
// substep kernel's layout (19 planes, one per direction) and element size.
// One population array, 19 read and 19 write streams: what a collision-free
// substep could reach on this device.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdio>

#include "glsm_b200.h"
#include "d3q19.cuh"

namespace {

using glsm::qcx;
using glsm::qcy;
using glsm::qcz;
using glsm::qopp;

// even AA form without the collision: cell i moves slot q to slot opp(q)
template <typename T>
__global__ void __launch_bounds__(256) aa_even_probe_kernel(T* P, unsigned n, size_t S) {
    const unsigned i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    T v[19];
#pragma unroll
    for (int q = 0; q < 19; q++) v[q] = P[q * S + i];
#pragma unroll
    for (int q = 0; q < 19; q++) P[qopp(q) * S + i] = v[q];
}

// odd AA form without the collision, for the cells whose 18 neighbours lie
// inside the array ([lo, hi)): gather slot opp(q) at i - off_q, scatter to
// slot q at i + off_q
template <typename T>
__global__ void __launch_bounds__(256) aa_odd_probe_kernel(T* P, unsigned lo, unsigned hi, size_t S, int nx,
                                                           int nxy) {
    const unsigned i = lo + blockIdx.x * 256 + threadIdx.x;
    if (i >= hi) return;
    T v[19];
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int off = qcx(q) + qcy(q) * nx + qcz(q) * nxy;
        v[q] = P[qopp(q) * S + i - off];
    }
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int off = qcx(q) + qcy(q) * nx + qcz(q) * nxy;
        P[q * S + i + off] = v[q];
    }
}

// Every thread copies the same elements in every rep, so a rep reads only what
// the same thread wrote in the rep before: no synchronisation between threads.
__global__ void __launch_bounds__(256) copy_reps_kernel(float4* a, float4* b, size_t n, int reps) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int r = 0; r < reps; r++) {
        const float4* src = (r & 1) ? b : a;
        float4* dst = (r & 1) ? a : b;
        size_t i = t;
        for (; i + 3 * stride < n; i += 4 * stride) {
            const float4 v0 = __ldcg(src + i);
            const float4 v1 = __ldcg(src + i + stride);
            const float4 v2 = __ldcg(src + i + 2 * stride);
            const float4 v3 = __ldcg(src + i + 3 * stride);
            __stcg(dst + i, v0);
            __stcg(dst + i + stride, v1);
            __stcg(dst + i + 2 * stride, v2);
            __stcg(dst + i + 3 * stride, v3);
        }
        for (; i < n; i += stride) __stcg(dst + i, __ldcg(src + i));
    }
}

thread_local char g_err[256];

int bw_fail(const char* what, cudaError_t e) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, e == cudaSuccess ? "bad argument" : cudaGetErrorString(e));
    return e == cudaSuccess ? GLSM_ERR_ARG : GLSM_ERR_CUDA;
}

template <typename T>
int pattern_probe(int nx, int ny, int nz, int reps, double* gbs_even, double* gbs_odd) {
    const unsigned n = (unsigned)nx * ny * nz, nxy = (unsigned)nx * ny;
    const size_t S = ((size_t)n + 63) / 64 * 64, bytes = 19 * S * sizeof(T);
    const unsigned lo = nxy + nx + 1, hi = n - nxy - nx - 1;
    T* P = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaError_t e = cudaMalloc(&P, bytes);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    for (int k = 0; k < 4 && e == cudaSuccess; k++) e = cudaEventCreate(&ev[k]);
    if (e == cudaSuccess) e = cudaMemsetAsync(P, 0, bytes, s);
    const unsigned ge = (n + 255) / 256, go = (hi - lo + 255) / 256;
    auto even = [&] { aa_even_probe_kernel<T><<<ge, 256, 0, s>>>(P, n, S); };
    auto odd = [&] { aa_odd_probe_kernel<T><<<go, 256, 0, s>>>(P, lo, hi, S, nx, (int)nxy); };
    for (int k = 0; k < 4 && e == cudaSuccess; k++) {  // warm-up: the array into L2 where it fits
        even();
        odd();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], s);
    for (int k = 0; k < reps && e == cudaSuccess; k++) even();
    if (e == cudaSuccess) e = cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], s);
    for (int k = 0; k < reps && e == cudaSuccess; k++) odd();
    if (e == cudaSuccess) e = cudaEventRecord(ev[3], s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms_even = 0.f, ms_odd = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_even, ev[0], ev[1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_odd, ev[2], ev[3]);
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    if (s) cudaStreamDestroy(s);
    if (P) cudaFree(P);
    if (e != cudaSuccess) return bw_fail("pattern probe", e);
    const double per_cell = 2.0 * 19.0 * sizeof(T);
    *gbs_even = (double)reps * n * per_cell / ((double)ms_even * 1e-3) / 1e9;
    *gbs_odd = (double)reps * (hi - lo) * per_cell / ((double)ms_odd * 1e-3) / 1e9;
    return GLSM_OK;
}

}  // namespace

extern "C" {

const char* glsm_copy_bandwidth_error(void) { return g_err; }

int glsm_copy_bandwidth(size_t bytes, int reps, double* gbs) {
    if (!gbs || bytes < 16 || bytes % 16 != 0 || bytes > ((size_t)8 << 30) || reps < 1 || reps > 100000)
        return bw_fail("glsm_copy_bandwidth: bytes must be a multiple of 16 in [16, 8 GiB], reps in [1, 100000]",
                       cudaSuccess);
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, copy_reps_kernel, 256, 0);
    if (e != cudaSuccess) return bw_fail("device query", e);
    const size_t n = bytes / 16;
    float4 *a = nullptr, *b = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaMalloc(&a, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&b, bytes);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemsetAsync(a, 0, bytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b, 0, bytes, s);
    const unsigned grid = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
    float ms = 0.f;
    if (e == cudaSuccess) {
        copy_reps_kernel<<<grid, 256, 0, s>>>(a, b, n, 2);  // warm-up: brings the buffers into L2 when they fit
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) {
        copy_reps_kernel<<<grid, 256, 0, s>>>(a, b, n, reps);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    if (e != cudaSuccess) return bw_fail("copy probe", e);
    *gbs = (double)reps * 2.0 * (double)bytes / ((double)ms * 1e-3) / 1e9;
    return GLSM_OK;
}

int glsm_pattern_bandwidth(int nx, int ny, int nz, int storage, int reps, double* gbs_even, double* gbs_odd) {
    if (!gbs_even || !gbs_odd || nx < 4 || ny < 4 || nz < 4 || reps < 1 || reps > 10000 ||
        (long long)nx * ny * nz > 200000000LL || storage < GLSM_STORE_F32 || storage > GLSM_STORE_BF16)
        return bw_fail("glsm_pattern_bandwidth: lattice >= 4 per axis and <= 2e8 cells, storage 0-2, reps in [1, 10000]",
                       cudaSuccess);
    // 16-bit storages share one element size
    return storage == GLSM_STORE_F32 ? pattern_probe<float>(nx, ny, nz, reps, gbs_even, gbs_odd)
                                     : pattern_probe<__half>(nx, ny, nz, reps, gbs_even, gbs_odd);
}

}  // extern "C"
