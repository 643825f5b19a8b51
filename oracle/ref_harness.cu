// ref_harness.cu -- drives the reference's OWN CUDA code (lasite/gLSM_fluid_3D
// src/*.cu, compiled unmodified for sm_100a by oracle/Makefile) so that the CPU
// oracle and the product can be compared with it on identical seeded inputs.
//
// TEST INFRASTRUCTURE ONLY (a checker and the timed reference arm of bench.py).
//
// What the harness does on top of the reference's public API (src/gel.h,
// src/fluid.h, src/coupling.h), and why:
//   * lattice dims that the Fluid ctor cannot express (it always makes
//     2*s+1 cells per axis, src/fluid.cu:169-172) are set by building the
//     next larger odd lattice and then narrowing FluidParams::L / N before
//     re-running k_init (buffers are larger than needed, never smaller);
//   * Fluid::Nsub (public) is overridden;
//   * the gel node/element type maps are re-allocated with zero padding so that
//     the reads that calServiceNodesPositionD and calChemBoundaryD make before
//     their bounds checks (src/gel_kernels.cu:623-625, :765-767) stay inside
//     the allocation for every thread of their launch grid;
//   * device buffers that the reference reads before writing (un_robin at the
//     first calUnnormD, F_ibm at the first spread, ...) are zeroed once;
//   * in "ordered" mode each phase is followed by cudaDeviceSynchronize(), so
//     the reference's unsynchronised per-object streams run in program order;
//     the timed mode runs the stock call sequence of src/sim.cpp:97-112.
// recordCenter() is not called (it only feeds the .dat time series).

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "coupling.h"
#include "fluid.h"
#include "gel.h"
#include "orc_noise.h"

__global__ void k_init(float* f, float* rho, float3* u, float* c1, float* c2, FluidParams* fp);

namespace {

struct RefSim {
    int nx, ny, nz, nsub;
    int start_time = 0;  // > 0: gels and fluid restart from the .dat files of that time (setGoonValue)
    std::vector<Gel*> gels;
    std::vector<int> active_from;
    Coupler* coupler = nullptr;
    Fluid* fluid = nullptr;
    float beta = 1.0f;
    cudaEvent_t e0, e1;
};

thread_local char g_err[256];

int check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

// re-allocate a type map so that the launch grid of the kernel that reads it
// (block 8x8x8, grid gdim) never indexes past the end
int pad_map(int*& dmap, const int* hmap, int count, dim3 gdim, int ext_x, int ext_y) {
    long long tx = (long long)gdim.x * 8, ty = (long long)gdim.y * 8, tz = (long long)gdim.z * 8;
    long long need = (tx - 1) + (ty - 1) * ext_x + (tz - 1) * (long long)ext_x * ext_y + 1;
    if (need < count) need = count;
    int* p = nullptr;
    if (check(cudaMalloc(&p, need * sizeof(int)), "pad_map malloc")) return -1;
    cudaMemset(p, 0, need * sizeof(int));
    cudaMemcpy(p, hmap, count * sizeof(int), cudaMemcpyHostToDevice);
    cudaFree(dmap);
    dmap = p;
    return 0;
}

template <typename T>
void zero(T* p, size_t n) {
    if (p) cudaMemset(p, 0, n * sizeof(T));
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err; }

int ref_device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

void* ref_create(int nx, int ny, int nz, int nsub) {
    if (cudaSetDevice(0) != cudaSuccess) return nullptr;
    auto* s = new RefSim;
    s->nx = nx;
    s->ny = ny;
    s->nz = nz;
    s->nsub = nsub;
    cudaEventCreate(&s->e0);
    cudaEventCreate(&s->e1);
    return s;
}

int ref_add_gel(void* p, int sx, int sy, int sz, double px, double py, double pz, int type, int id) {
    auto* s = (RefSim*)p;
    if (s->fluid) return -1;
    Gel* g = new Gel(make_int3(sx, sy, sz), make_double3(px, py, pz), type, id, s->start_time);
    int LX = g->m_gelNodeGrid.x, LY = g->m_gelNodeGrid.y;
    if (pad_map(g->m_dmap_node, g->m_hmap_node, g->m_numGelNodes, g->m_gridDim2, LX + 2, LY + 2)) return -1;
    if (pad_map(g->m_dmap_element, g->m_hmap_element, g->m_numGelElements, g->m_gridDim1, LX + 1, LY + 1))
        return -1;
    size_t nE = g->m_numGelElements, nN = g->m_numGelNodes;
    zero(g->m_dum_norm, nE);
    zero(g->m_dvm_norm, nE);
    zero(g->m_dwmp, nE);
    zero(g->m_dT0m, nE);
    zero(g->m_dT1m, nE);
    zero(g->m_dT2m, nE);
    zero(g->m_dVolm, nE);
    zero(g->m_dPrem, nE);
    zero(g->m_drm, nE);
    zero(g->m_drm_loc, 8 * nE);
    zero(g->m_dnmSm, 6 * nE);
    zero(g->m_dun_norm, nN);
    zero(g->m_dun_robin, nN);
    zero(g->m_dvn_norm, nN);
    zero(g->m_dFn, nN);
    zero(g->m_dFn_robin, nN);
    zero(g->m_dFdrag_robin, nN);
    zero(g->m_dVeln, nN);
    zero(g->m_dVels, nN);
    zero(g->m_dvm_center, 1000);
    zero(g->m_dwm_center, 1000);
    zero(g->m_drm_center, 1000);
    zero(g->m_dFn_center, 1000);
    zero(g->m_dVeln_center, 1000);
    if (check(cudaDeviceSynchronize(), "add_gel")) return -1;
    s->gels.push_back(g);
    s->active_from.push_back(0);
    return (int)s->gels.size() - 1;
}

// same noise definition as the oracle: interior elements, um += amp*n0, vm += amp*n1
int ref_gel_noise(void* p, int gi, unsigned long long seed, double amp) {
    auto* s = (RefSim*)p;
    if (gi < 0 || gi >= (int)s->gels.size()) return -3;
    Gel* g = s->gels[gi];
    int LX = g->m_gelNodeGrid.x, LY = g->m_gelNodeGrid.y, LZ = g->m_gelNodeGrid.z;
    for (int zi = 1; zi < LZ; zi++)
        for (int yi = 1; yi < LY; yi++)
            for (int xi = 1; xi < LX; xi++) {
                int e = g->get_index(xi, yi, zi, 1);
                g->m_hum[e] += amp * orc_noise_pm1(seed, (uint64_t)g->m_gelId, (uint64_t)e, 0);
                g->m_hvm[e] += amp * orc_noise_pm1(seed, (uint64_t)g->m_gelId, (uint64_t)e, 1);
            }
    cudaMemcpy(g->m_dum, g->m_hum, sizeof(double) * g->m_numGelElements, cudaMemcpyHostToDevice);
    cudaMemcpy(g->m_dvm, g->m_hvm, sizeof(double) * g->m_numGelElements, cudaMemcpyHostToDevice);
    return check(cudaDeviceSynchronize(), "noise");
}

int ref_gel_control(void* p, int gi, int what, double value) {
    auto* s = (RefSim*)p;
    if (gi < 0 || gi >= (int)s->gels.size()) return -3;
    Gel* g = s->gels[gi];
    switch (what) {
        case 0: g->resetToQuiescent(); break;
        case 1: g->fireExcitationPulse(); break;
        case 2: g->setAnchorZ(value); break;
        case 3: s->active_from[gi] = (int)value; break;
        case 4: g->buildTubeMask((int)value, false); break;
        case 5: g->buildTubeMask((int)value, true); break;
        default: return -1;
    }
    return check(cudaDeviceSynchronize(), "control");
}

// gels added after this call and the fluid restart from the .dat files of
// time t in the current directory (the constructors' setGoonValue,
// src/gel.cu:221-282, src/fluid.cu:57-83)
int ref_set_start_time(void* p, int t) {
    ((RefSim*)p)->start_time = t;
    return 0;
}

int ref_set_beta(void* p, double beta) {
    ((RefSim*)p)->beta = (float)beta;
    if (((RefSim*)p)->fluid) ((RefSim*)p)->fluid->h_fp->beta = (float)beta;
    return 0;
}

int ref_finalize(void* p) {
    auto* s = (RefSim*)p;
    if (s->fluid) return -1;
    s->coupler = new Coupler(s->gels);
    // smallest odd lattice >= the requested one: 2*fs + 1 cells per axis
    int3 fs = make_int3((s->nx) / 2, (s->ny) / 2, (s->nz) / 2);
    s->fluid = new Fluid(fs, s->start_time, s->coupler);
    Fluid* F = s->fluid;
    F->h_fp->beta = s->beta;
    if (F->fluidNodeGrid.x != s->nx || F->fluidNodeGrid.y != s->ny || F->fluidNodeGrid.z != s->nz) {
        int N = s->nx * s->ny * s->nz;
        F->fluidNodeGrid = make_int3(s->nx, s->ny, s->nz);
        F->N = N;
        F->Nd = 19 * N;
        F->blocksN = (N + F->threads - 1) / F->threads;
        F->h_fp->N = N;
        F->h_fp->L = F->fluidNodeGrid;
        cudaMemcpy(F->d_fp, F->h_fp, sizeof(FluidParams), cudaMemcpyHostToDevice);
        k_init<<<F->blocksN, F->threads, 0, F->fluid_stream>>>(F->d_f, F->d_rho, F->d_u, F->d_c1, F->d_c2, F->d_fp);
    }
    F->Nsub = s->nsub;
    size_t N = F->N;
    zero(F->d_F_ibm, N);
    zero(F->d_F_tot, N);
    zero(F->d_F, N);
    zero(F->d_source, N);
    Coupler* C = s->coupler;
    size_t M = C->sumGelBoundaryCount;
    zero(C->d_Ul_all_, M);
    zero(C->d_Fdrag_all_, M);
    zero(C->d_Frep_all_, M);
    zero(C->d_Dl_all_, M);
    zero(C->d_Sl_all_, M);
    return check(cudaDeviceSynchronize(), "finalize");
}

static int one_iter(RefSim* s, int iter, bool ordered) {
    for (size_t k = 0; k < s->gels.size(); k++)
        if (s->active_from[k] > 0 && iter == s->active_from[k]) s->gels[k]->fireExcitationPulse();
    for (size_t k = 0; k < s->gels.size(); k++) {
        if (s->active_from[k] > 0 && iter < s->active_from[k]) continue;
        s->gels[k]->stepElasticity(iter);
        s->gels[k]->stepChemistry(iter);
    }
    if (ordered && check(cudaDeviceSynchronize(), "gel")) return -1;
    s->coupler->packFromGels();
    if (ordered && check(cudaDeviceSynchronize(), "pack")) return -1;
    s->fluid->stepVelocity(iter);
    if (ordered && check(cudaDeviceSynchronize(), "velocity")) return -1;
    s->fluid->stepConcentration(iter);
    if (ordered && check(cudaDeviceSynchronize(), "concentration")) return -1;
    s->coupler->applyGelRepulsion();
    if (ordered && check(cudaDeviceSynchronize(), "repulsion")) return -1;
    s->coupler->scatterToGels();
    if (ordered && check(cudaDeviceSynchronize(), "scatter")) return -1;
    return 0;
}

// run iterations iter0 .. iter0+n-1 in program order
int ref_run(void* p, int iter0, int n) {
    auto* s = (RefSim*)p;
    if (!s->fluid) return -1;
    for (int k = 0; k < n; k++)
        if (one_iter(s, iter0 + k, true)) return -1;
    return 0;
}

// the stock call sequence (no added synchronisation), timed with events on the
// legacy default stream, which orders after all of the reference's blocking
// streams; returns milliseconds or a negative value on error
double ref_time(void* p, int iter0, int n) {
    auto* s = (RefSim*)p;
    if (!s->fluid) return -1;
    if (check(cudaDeviceSynchronize(), "time pre")) return -1;
    cudaEventRecord(s->e0, 0);
    for (int k = 0; k < n; k++) one_iter(s, iter0 + k, false);
    cudaEventRecord(s->e1, 0);
    if (check(cudaEventSynchronize(s->e1), "time post")) return -1;
    float ms = 0;
    cudaEventElapsedTime(&ms, s->e0, s->e1);
    return ms;
}

// Gel::recordCenter(iter) of every gel.  Its calFilamentD stores up to
// maxFilamentlen crossings per record without a bound check
// (src/gel_kernels.cu:837-866), so only gels with at most that many node faces
// (every crossing lies on its own face) are accepted.
int ref_record_center(void* p, int iter) {
    auto* s = (RefSim*)p;
    for (auto* g : s->gels) {
        const long long faces = (long long)(g->m_gelNodeGrid.x - 1) * (g->m_gelNodeGrid.y - 1) *
                                (g->m_gelNodeGrid.z - 1);
        if (faces > g->m_hgp->maxFilamentlen) {
            snprintf(g_err, sizeof(g_err), "recordCenter: gel with %lld node faces exceeds the filament buffer", faces);
            return -1;
        }
    }
    for (auto* g : s->gels) g->recordCenter(iter);
    return check(cudaDeviceSynchronize(), "recordCenter");
}

// Gel::writeFiles(iter) of every gel and Fluid::writeFiles(iter), written into
// the current directory; the writer threads are joined before returning (the
// reference joins them at the next write or in its destructors)
int ref_write_files(void* p, int iter) {
    auto* s = (RefSim*)p;
    if (!s->fluid) return -1;
    if (check(cudaDeviceSynchronize(), "writeFiles pre")) return -1;
    for (auto* g : s->gels) g->writeFiles(iter);
    s->fluid->writeFiles(iter);
    for (auto* g : s->gels)
        if (g->m_file_writer_thread.joinable()) g->m_file_writer_thread.join();
    if (s->fluid->file_writer_thread.joinable()) s->fluid->file_writer_thread.join();
    return check(cudaDeviceSynchronize(), "writeFiles");
}

int ref_info(void* p, long long* out) {
    auto* s = (RefSim*)p;
    out[0] = s->fluid ? s->fluid->N : 0;
    out[1] = s->coupler ? s->coupler->sumGelBoundaryCount : 0;
    out[2] = (long long)s->gels.size();
    out[3] = s->fluid ? s->fluid->Nsub : s->nsub;
    return 0;
}

// field ids as in glsm_oracle.cpp; values are converted to double
long long ref_field(void* p, int field, int gi, double* buf, long long n) {
    auto* s = (RefSim*)p;
    Fluid* F = s->fluid;
    Coupler* C = s->coupler;
    const void* src = nullptr;
    long long count = 0;
    int is_float = 0;
    long long N = F ? F->N : 0, M = C ? C->sumGelBoundaryCount : 0;
    if (field < 20 && !F) return -1;
    switch (field) {
        case 0: src = F->d_f; count = 19 * N; is_float = 1; break;
        case 1: src = F->d_rho; count = N; is_float = 1; break;
        case 2: src = F->d_u; count = 3 * N; is_float = 1; break;
        case 3: src = F->d_c1; count = N; is_float = 1; break;
        case 4: src = F->d_F_ibm; count = 3 * N; is_float = 1; break;
        case 10: src = C->d_lag_all_; count = 3 * M; is_float = 1; break;
        case 11: src = C->d_Ul_all_; count = 3 * M; is_float = 1; break;
        case 12: src = C->d_Vl_all_; count = 3 * M; is_float = 1; break;
        case 13: src = C->d_Fdrag_all_; count = 3 * M; is_float = 1; break;
        case 14: src = C->d_Frep_all_; count = 3 * M; is_float = 1; break;
        case 15: src = C->d_Cl_all_; count = M; is_float = 1; break;
        case 16: src = C->d_Dl_all_; count = M; is_float = 1; break;
        case 17: src = C->d_Sl_all_; count = M; is_float = 1; break;
        default: break;
    }
    if (field >= 20) {
        if (gi < 0 || gi >= (int)s->gels.size()) return -3;
        Gel* g = s->gels[gi];
        long long nE = g->m_numGelElements, nN = g->m_numGelNodes;
        switch (field) {
            case 20: src = g->m_drn; count = 3 * nN; break;
            case 21: src = g->m_dVeln; count = 3 * nN; break;
            case 22: src = g->m_dVels; count = 3 * nN; break;
            case 23: src = g->m_dFn; count = 3 * nN; break;
            case 24: src = g->m_dum; count = nE; break;
            case 25: src = g->m_dvm; count = nE; break;
            case 26: src = g->m_dwm; count = nE; break;
            case 27: src = g->m_dun_norm; count = nN; break;
            case 28: src = g->m_dvn_norm; count = nN; break;
            case 29: src = g->m_dT0m; count = nE; break;
            case 30: src = g->m_dT1m; count = nE; break;
            case 31: src = g->m_dT2m; count = nE; break;
            case 32: src = g->m_drm; count = 3 * nE; break;
            case 33: src = g->m_dnmSm; count = 18 * nE; break;
            case 34: src = g->m_dVolm; count = nE; break;
            case 35: src = g->m_dPrem; count = nE; break;
            case 36: src = g->m_dun_robin; count = nN; break;
            case 37: src = g->m_dum_norm; count = nE; break;
            case 38: src = g->m_dvm_norm; count = nE; break;
            case 39: src = g->m_dwmp; count = nE; break;
            case 40: src = g->m_dFn_robin; count = 3 * nN; break;
            // the centre-element records of recordCenter, slot (iter / 1000) % 1000
            case 41: src = g->m_dvm_center; count = 1000; break;
            case 42: src = g->m_dwm_center; count = 1000; break;
            case 43: src = g->m_drm_center; count = 3 * 1000; break;
            case 44: src = g->m_dFn_center; count = 3 * 1000; break;
            case 45: src = g->m_dVeln_center; count = 3 * 1000; break;
            default: return -1;
        }
    }
    if (!src) return -1;
    if (!buf) return count;
    if (n < count) return -2;
    if (check(cudaDeviceSynchronize(), "field sync")) return -1;
    if (is_float) {
        std::vector<float> tmp(count);
        if (check(cudaMemcpy(tmp.data(), src, count * sizeof(float), cudaMemcpyDeviceToHost), "field copy"))
            return -1;
        for (long long i = 0; i < count; i++) buf[i] = tmp[i];
    } else {
        if (check(cudaMemcpy(buf, src, count * sizeof(double), cudaMemcpyDeviceToHost), "field copy")) return -1;
    }
    return count;
}

void ref_destroy(void* p) {
    auto* s = (RefSim*)p;
    if (!s) return;
    cudaDeviceSynchronize();
    delete s->fluid;
    delete s->coupler;
    for (auto* g : s->gels) delete g;
    cudaEventDestroy(s->e0);
    cudaEventDestroy(s->e1);
    delete s;
}

}  // extern "C"
