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
#include <cuda_runtime.h>

#include <cstdio>

#include "glsm_b200.h"

namespace {

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

}  // extern "C"
