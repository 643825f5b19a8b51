// noalloc.cu -- glsm_substep_noalloc: one LBM substep with immersed-boundary
// forcing on caller-owned device buffers, using no device allocation at all.
//
// Who needs it: callers that cannot call cudaMalloc -- code running inside a
// host framework that owns all device memory through its own pool (and forbids
// raw allocations), plug-ins loaded into a process whose allocator must see
// every byte, and hard real-time loops where an allocation (which may
// synchronise the device) is not allowed.  Such a caller cannot create the
// gel / coupler / fluid handles, which own their buffers.  This entry point
// takes the populations, velocity field and marker arrays from the caller and
// keeps its scratch (the spread force field and the per-marker stencil cache)
// in one file-scope __device__ array of fixed size.
//
// Limits: at most kNaMaxCells lattice cells and kNaMaxMarkers markers per
// call; every GPU that loads the library holds the 5,308,416-byte array until
// the process exits.  All calls on a device share the array: calls that
// overlap on the GPU (different streams without ordering) race on it.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress and caches it together with
// the device's current context; a later call on a new context of that device
// (after cudaDeviceReset, or a primary context released and re-created, where
// the module and its array are loaded anew) repeats the look-up.  Make the
// first call on a device before any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/glsm_b200.h"
#include "d3q19.cuh"

namespace {

constexpr long long kNaMaxCells = 1LL << 18;  // 262,144 lattice cells, e.g. 64^3
constexpr int kNaMaxMarkers = 16384;
constexpr size_t kNaForceBytes = (size_t)kNaMaxCells * sizeof(float4);
constexpr size_t kNaBaseBytes = (size_t)kNaMaxMarkers * sizeof(int4);
constexpr size_t kNaWeightBytes = (size_t)kNaMaxMarkers * sizeof(float4) * 3;
constexpr size_t kNaSumBytes = (size_t)kNaMaxMarkers * sizeof(float);
constexpr size_t kNaScratchBytes = kNaForceBytes + kNaBaseBytes + kNaWeightBytes + kNaSumBytes;
static_assert(kNaScratchBytes == 5308416, "documented scratch size");

// the scratch of glsm_substep_noalloc; host code needs its device address from
// cudaGetSymbolAddress (the name itself is a host-side stand-in there)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

struct NaScratch {
    float4* force;   // spread IBM force per lattice cell
    int4* base;      // first stencil cell of each marker and a validity word
    float4* ph[3];   // delta-4 weights of the 4 stencil columns per axis
    float* wsum;     // sum of the clipped stencil's weights
};

__host__ __device__ inline NaScratch carve(unsigned char* p) {
    NaScratch s;
    s.force = reinterpret_cast<float4*>(p);
    s.base = reinterpret_cast<int4*>(p + kNaForceBytes);
    for (int k = 0; k < 3; k++)
        s.ph[k] = reinterpret_cast<float4*>(p + kNaForceBytes + kNaBaseBytes + k * (size_t)kNaMaxMarkers * 16);
    s.wsum = reinterpret_cast<float*>(p + kNaForceBytes + kNaBaseBytes + kNaWeightBytes);
    return s;
}

__device__ __forceinline__ float na_delta4(float r) {
    r = fabsf(r);
    if (r <= 1.f) return 0.125f * (3.f - 2.f * r + sqrtf(1.f + 4.f * r - 4.f * r * r));
    if (r <= 2.f) return 0.125f * (5.f - 2.f * r - sqrtf(-7.f + 12.f * r - 4.f * r * r));
    return 0.f;
}

__device__ __forceinline__ float na_comp(const float4& v, int a) {
    return a == 0 ? v.x : (a == 1 ? v.y : (a == 2 ? v.z : v.w));
}

__global__ void na_zero_force(unsigned char* scratch, unsigned N) {
    const NaScratch s = carve(scratch);
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) s.force[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// per-marker delta-4 stencil, clipped at the lattice (the reference's
// k_ibm_interpolate_velocity loop bounds, src/fluid_kernels.cu:251-262)
__global__ void na_stencil(unsigned char* scratch, const float4* lag, int M, float h, int nx, int ny, int nz) {
    const NaScratch s = carve(scratch);
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= M) return;
    const float4 p = lag[l];
    const int n[3] = {nx, ny, nz};
    // a non-finite or far-out position gives a fully clipped stencil (the
    // marker then neither samples nor spreads); within 8 cells of the lattice
    // the position is used as it is (a stencil reaches 2 cells)
    const bool fin = isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
    float g[3] = {p.x / h, p.y / h, p.z / h};
    for (int d = 0; d < 3; d++) g[d] = fin ? fminf(fmaxf(g[d], -8.f), (float)n[d] + 8.f) : -8.f;
    int b0[3], valid = 0;
    float ph[3][4];
    for (int d = 0; d < 3; d++) {
        const int ic = (int)floorf(g[d]);
        b0[d] = ic - 1;
        for (int k = 0; k < 4; k++) {
            const int c = ic - 1 + k;
            const bool in = c >= 0 && c < n[d];
            ph[d][k] = in ? na_delta4(g[d] - (float)c) : 0.f;
            if (in) valid |= 1 << (4 * d + k);
        }
    }
    float ws = 0.f;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++)
                if (((valid >> i) & 1) && ((valid >> (4 + j)) & 1) && ((valid >> (8 + k)) & 1))
                    ws += ph[0][i] * ph[1][j] * ph[2][k];
    s.base[l] = make_int4(b0[0], b0[1], b0[2], valid);
    for (int d = 0; d < 3; d++) s.ph[d][l] = make_float4(ph[d][0], ph[d][1], ph[d][2], ph[d][3]);
    s.wsum[l] = ws;
}

// one warp per marker: interpolate u, penalty force beta_eff (V - U), spread
__global__ void na_ibm(unsigned char* scratch, const float4* u4, const float4* vel, int M, float h, float beta_eff,
                       int nx, int ny, float4* Ul, float4* Fdrag) {
    const NaScratch s = carve(scratch);
    const int lane = threadIdx.x & 31;
    const int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (l >= M) return;
    const int4 b = s.base[l];
    const float4 px = s.ph[0][l], py = s.ph[1][l], pz = s.ph[2][l];
    const float ws = s.wsum[l];
    float sx = 0.f, sy = 0.f, sz = 0.f, w[2];
    long long cell[2];
    bool ok[2];
    for (int j = 0; j < 2; j++) {
        const int p = lane + 32 * j;
        const int ax = p >> 4, ay = (p >> 2) & 3, az = p & 3;
        ok[j] = ((b.w >> ax) & 1) && ((b.w >> (4 + ay)) & 1) && ((b.w >> (8 + az)) & 1);
        w[j] = na_comp(px, ax) * na_comp(py, ay) * na_comp(pz, az);
        cell[j] = (long long)(b.x + ax) + (long long)(b.y + ay) * nx + (long long)(b.z + az) * nx * ny;
        if (ok[j]) {
            const float4 uu = u4[cell[j]];
            sx += uu.x * w[j];
            sy += uu.y * w[j];
            sz += uu.z * w[j];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
    }
    const float4 U = ws > 0.f ? make_float4(sx / ws, sy / ws, sz / ws, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 V = vel[l];
    const float4 Fd = make_float4(beta_eff * (V.x - U.x), beta_eff * (V.y - U.y), beta_eff * (V.z - U.z), 0.f);
    if (lane == 0) {
        Ul[l] = U;
        Fdrag[l] = Fd;
    }
    if (ws == 0.f) return;
    const float scale = (float)(1.0 / (double)(h * h * h)) / ws;
    for (int j = 0; j < 2; j++)
        if (ok[j]) {
            const float wg = w[j] * scale;
            atomicAdd(&s.force[cell[j]], make_float4(Fd.x * wg, Fd.y * wg, Fd.z * wg, 0.f));
        }
}

// one cell per thread: AA-pattern gather, BGK + Guo collision in deviation
// form, AA-pattern scatter with half-way bounce-back on all six faces
__global__ void na_lbm(const unsigned char* scratch, float* pop, unsigned S, float4* u4, int nx, int ny, int nz,
                       int parity, float omega, float fpref, float fcx, float fcy, float fcz) {
    using namespace glsm;
    const NaScratch s = carve(const_cast<unsigned char*>(scratch));
    const unsigned N = (unsigned)nx * ny * nz;
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int x = (int)(i % (unsigned)nx), y = (int)((i / (unsigned)nx) % (unsigned)ny),
              z = (int)(i / ((unsigned)nx * ny));
    const int st[3] = {1, nx, nx * ny};
    const int c[3] = {x, y, z}, n[3] = {nx, ny, nz};
    float d[19];
    for (int q = 0; q < 19; q++) {
        if (parity == 0) {
            d[q] = pop[q * S + i];
        } else {
            const int cq[3] = {qcx(q), qcy(q), qcz(q)};
            bool wall = false;
            int off = 0;
            for (int k = 0; k < 3; k++) {
                const int src = c[k] - cq[k];
                if (src < 0 || src >= n[k]) wall = true;
                off -= cq[k] * st[k];
            }
            d[q] = wall ? pop[q * S + i] : pop[qopp(q) * S + (unsigned)((int)i + off)];
        }
    }
    const float4 f = s.force[i];
    const float Fx = fcx + f.x, Fy = fcy + f.y, Fz = fcz + f.z;
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
    for (int q = 0; q < 19; q++) {
        drho += d[q];
        jx += qcx(q) * d[q];
        jy += qcy(q) * d[q];
        jz += qcz(q) * d[q];
    }
    const float rho = 1.0f + drho;
    const float ux = (jx + 0.5f * Fx) / rho, uy = (jy + 0.5f * Fy) / rho, uz = (jz + 0.5f * Fz) / rho;
    const float uu = ux * ux + uy * uy + uz * uz, uF = ux * Fx + uy * Fy + uz * Fz;
    for (int q = 0; q < 19; q++) {
        const float cu = qcx(q) * ux + qcy(q) * uy + qcz(q) * uz;
        const float cF = qcx(q) * Fx + qcy(q) * Fy + qcz(q) * Fz;
        const float deq = qw(q) * (drho + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * uu));
        const float Ft = qw(q) * fpref * (3.0f * cF + 9.0f * cu * cF - 3.0f * uF);
        d[q] = d[q] + omega * (deq - d[q]) + Ft;
    }
    for (int q = 0; q < 19; q++) {
        if (parity == 0) {
            pop[qopp(q) * S + i] = d[q];
        } else {
            const int cq[3] = {qcx(q), qcy(q), qcz(q)};
            bool wall = false;
            int off = 0;
            for (int k = 0; k < 3; k++) {
                const int dst = c[k] + cq[k];
                if (dst < 0 || dst >= n[k]) wall = true;
                off += cq[k] * st[k];
            }
            if (wall)
                pop[qopp(q) * S + i] = d[q];
            else
                pop[q * S + (unsigned)((int)i + off)] = d[q];
        }
    }
    u4[i] = make_float4(ux, uy, uz, rho);
}

thread_local char g_na_err[256] = "";
std::mutex g_na_mutex;
constexpr int kNaMaxDevices = 64;
void* g_na_ptr[kNaMaxDevices] = {};       // the scratch's device address per device
CUcontext g_na_ctx[kNaMaxDevices] = {};   // the context that address belongs to

// cuCtxGetCurrent through the runtime's driver entry point (no link against
// the driver library); null when the driver does not provide it
using CtxGetCurrent = CUresult (*)(CUcontext*);
CtxGetCurrent ctx_get_current() {
    static const CtxGetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        cudaGetLastError();
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    return fn;
}

int na_fail(int code, const char* msg) {
    snprintf(g_na_err, sizeof(g_na_err), "%s", msg);
    return code;
}

}  // namespace

extern "C" {

const char* glsm_noalloc_last_error(void) { return g_na_err; }

size_t glsm_noalloc_scratch_bytes(void) { return kNaScratchBytes; }

int glsm_substep_noalloc(float* pop, int64_t plane_stride, float* u4, int nx, int ny, int nz, int parity, float tau,
                         float fx, float fy, float fz, const float* lag4, const float* vel4, int n_markers, float h,
                         float beta_eff, float* Ul4, float* Fdrag4, void* stream) {
    if (!pop || !u4) return na_fail(GLSM_ERR_ARG, "populations and velocity buffers are required");
    if (nx < 4 || ny < 4 || nz < 4) return na_fail(GLSM_ERR_ARG, "lattice must be >= 4 cells per axis");
    const long long N = (long long)nx * ny * nz;
    if (N > kNaMaxCells)
        return na_fail(GLSM_ERR_ARG, "lattice exceeds the no-allocation limit of 262144 cells");
    if (plane_stride < N || plane_stride * 19 >= (1LL << 32))
        return na_fail(GLSM_ERR_ARG, "plane stride must be >= the cell count");
    if (n_markers < 0 || n_markers > kNaMaxMarkers)
        return na_fail(GLSM_ERR_ARG, "marker count exceeds the no-allocation limit of 16384");
    if (n_markers > 0 && (!lag4 || !vel4 || !Ul4 || !Fdrag4))
        return na_fail(GLSM_ERR_ARG, "marker buffers are required when n_markers > 0");
    if (parity != 0 && parity != 1) return na_fail(GLSM_ERR_ARG, "parity must be 0 or 1");
    if (!(tau > 0.5f) || !(h > 0.f)) return na_fail(GLSM_ERR_ARG, "tau must exceed 0.5 and h be positive");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices)
        return na_fail(GLSM_ERR_CUDA, "no current CUDA device");
    unsigned char* scratch = nullptr;
    {
        // set-up, once per device and context, with that device current: the
        // device address of the scratch array (the first call on a device does
        // this, and the first call after the device's context was re-created)
        std::lock_guard<std::mutex> lock(g_na_mutex);
        CUcontext ctx = nullptr;
        const CtxGetCurrent get_ctx = ctx_get_current();
        const bool known_ctx = get_ctx && get_ctx(&ctx) == CUDA_SUCCESS && ctx;
        if (!g_na_ptr[dev] || !known_ctx || ctx != g_na_ctx[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return na_fail(GLSM_ERR_CUDA, "cudaGetSymbolAddress of the scratch failed");
            g_na_ptr[dev] = p;
            g_na_ctx[dev] = known_ctx ? ctx : nullptr;
        }
        scratch = static_cast<unsigned char*>(g_na_ptr[dev]);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned cells = (unsigned)N;
    na_zero_force<<<(cells + 255) / 256, 256, 0, s>>>(scratch, cells);
    if (n_markers > 0) {
        na_stencil<<<(n_markers + 127) / 128, 128, 0, s>>>(scratch, reinterpret_cast<const float4*>(lag4), n_markers, h,
                                                           nx, ny, nz);
        na_ibm<<<(n_markers * 32 + 255) / 256, 256, 0, s>>>(scratch, reinterpret_cast<const float4*>(u4),
                                                            reinterpret_cast<const float4*>(vel4), n_markers, h,
                                                            beta_eff, nx, ny, reinterpret_cast<float4*>(Ul4),
                                                            reinterpret_cast<float4*>(Fdrag4));
    }
    na_lbm<<<(cells + 255) / 256, 256, 0, s>>>(scratch, pop, (unsigned)plane_stride, reinterpret_cast<float4*>(u4), nx,
                                              ny, nz, parity, 1.0f / tau, 1.0f - 0.5f / tau, fx, fy, fz);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(GLSM_ERR_CUDA, cudaGetErrorString(e));
    return GLSM_OK;
}

}  // extern "C"
