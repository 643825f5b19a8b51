// capi.cu -- the C ABI of libglsm_b200.so (include/glsm_b200.h): object
// lifecycles, host-side gel initialisation, the per-method launches that the
// reference's classes expose, and the graph-captured fused iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/glsm_b200.h"
#include "gel.h"
#include "glsm_internal.h"
#include "lbm.h"

using namespace glsm;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";

static int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            return fail(_e == cudaErrorMemoryAllocation ? GLSM_ERR_NOMEM : GLSM_ERR_CUDA,     \
                        "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e));   \
    } while (0)

// ---------------------------------------------------------------------------
// handle types
// ---------------------------------------------------------------------------
struct glsm_coupler_s;
struct glsm_fluid_s;

// Output snapshot of an object (glsm_fluid_snapshot, glsm_gel_snapshot): the
// fields are copied into `dev` on the object's stream, then to the caller's
// host buffers on the copy stream, so the caller's thread never waits for the
// iterations queued before the snapshot.
struct Snapshot {
    void* dev = nullptr;
    size_t bytes = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t taken = nullptr;  // device-side copy done (recorded on the object's stream)
    cudaEvent_t done = nullptr;   // host buffers filled (recorded on the copy stream)
    bool used = false;            // a snapshot was taken: the next one waits for `done` on the device
};

static int snap_ensure(Snapshot& sn, size_t bytes);
static void snap_release(Snapshot& sn);

struct glsm_gel_s {
    GelDev d{};                 // descriptor with device pointers (host copy)
    GelDev* d_self = nullptr;   // device copy for launches before coupling
    Ctl* d_ctl = nullptr;       // control block before coupling
    void* arena = nullptr;
    size_t bytes = 0;
    cudaStream_t own = nullptr;
    double* series_extra = nullptr;  // a time-series ring larger than the built-in one
    glsm_coupler_s* coupler = nullptr;
    int index = -1;             // position in the coupler
    bool release_with_coupler = false;  // destroyed while coupled: freed with the coupler
    Snapshot snap;              // output snapshot (glsm_gel_snapshot)
    bool ptr_out = false;       // a device pointer was handed out: the fused run gathers every iteration
};

struct glsm_coupler_s {
    std::vector<glsm_gel_s*> gels;
    GelDev* d_gels = nullptr;
    MarkerDev mk{};
    void* arena = nullptr;
    size_t bytes = 0;
    Ctl* d_ctl = nullptr;
    int* d_fresh = nullptr;  // per gel: marker arrays current (kPhGatherStale)
    bool markers_stale = true;  // host: a gel changed since the last fused run (fresh flags to clear)
    Ctl* h_ctl = nullptr;  // pinned mirror for error reads
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    float g2l = 1.0f, l2g = 1.0f;  // CouplerParams gel_to_lbm_vel / lbm_to_gel_vel
    float rep_delta = 1e-4f, rep_gamma = 1.5f;  // src/coupling.cu:75-76
    glsm_fluid_s* fluid = nullptr;
};

// the fused run re-gathers the markers of a coupler whose gels changed
static void mark_markers_stale(glsm_gel_s* g) {
    if (g && g->coupler) g->coupler->markers_stale = true;
}

struct glsm_fluid_s {
    glsm_fluid_desc desc{};
    FluidDev F{};
    glsm_coupler_s* c = nullptr;
    void* arena = nullptr;
    size_t bytes = 0;
    unsigned* d_sync = nullptr;  // tickets[nsub], ibm_done[nsub]
    int cur = 0;                 // current concentration buffer
    long long substeps = 0;      // AA parity bookkeeping
    float* scratch = nullptr;    // 19*N floats, allocated on first use
    int lbm_ctas = 0;            // resident CTAs of the persistent substep kernel (odd substeps)
    int lbm_ctas_even = 0;       // the same for even substeps
    int wait_extra = 0;          // test aid (glsm_test_ibm_wait_extra): > 0 makes the IBM wait run out
    long long dev_iter = -1;     // the device's iteration counter (Ctl::iter) after glsm_fluid_run; -1: unknown
    int device = 0;              // CUDA device the system lives on
    int l2_on = 0;              // keep the population array L2-persisting (glsm_fluid_set_l2_persisting)
    unsigned long long l2_bytes = 0;  // access-policy window of the substep launches (0: none)
    float l2_hit = 0.f;
    double* d_cons = nullptr;    // conservation partial sums (kConsBlocks x 4) and result (4)
    struct glsm_batch_s* batch = nullptr;  // batch this system belongs to
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    Snapshot snap;               // output snapshot (glsm_fluid_snapshot)
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// carve sub-buffers out of one allocation
struct Carver {
    char* base;
    size_t off = 0;
    template <typename T>
    T* take(size_t count) {
        off = align_up(off, 256);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

static uint64_t mix64(uint64_t x) {  // splitmix64 finaliser (Steele, Lea, Flood 2014)
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double noise_unit(uint64_t seed, uint64_t gel_id, uint64_t slot, uint64_t field) {
    const uint64_t h = mix64(mix64(mix64(seed) ^ gel_id) ^ (slot * 2ull + field));
    return 2.0 * ((double)(h >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
}

static cudaStream_t gel_stream(const glsm_gel_s* g) { return g->coupler ? g->coupler->stream : g->own; }

static void mark_markers_stale(glsm_gel_s* g);

static int upload_gel_desc(glsm_gel_s* g) {
    mark_markers_stale(g);
    CK(cudaMemcpyAsync(g->d_self, &g->d, sizeof(GelDev), cudaMemcpyHostToDevice, gel_stream(g)));
    if (g->coupler)
        CK(cudaMemcpyAsync(g->coupler->d_gels + g->index, &g->d, sizeof(GelDev), cudaMemcpyHostToDevice,
                           gel_stream(g)));
    CK(cudaStreamSynchronize(gel_stream(g)));
    return GLSM_OK;
}

struct FieldRef {
    void* ptr;
    size_t count;  // doubles
};
static FieldRef gel_field(const glsm_gel_s* g, int field) {
    const GelDev& d = g->d;
    const size_t nE = d.nE, nN = d.nN;
    switch (field) {
        case GLSM_GEL_RN: return {d.rn, 3 * nN};
        case GLSM_GEL_VELN: return {d.Veln, 3 * nN};
        case GLSM_GEL_VELS: return {d.Vels, 3 * nN};
        case GLSM_GEL_FN: return {d.Fn, 3 * nN};
        case GLSM_GEL_UM: return {d.um, nE};
        case GLSM_GEL_VM: return {d.vm, nE};
        case GLSM_GEL_WM: return {d.wm, nE};
        case GLSM_GEL_UN_NORM: return {d.un_norm, nN};
        case GLSM_GEL_VN_NORM: return {d.vn_norm, nN};
        case GLSM_GEL_T0: return {d.T0, nE};
        case GLSM_GEL_T1: return {d.T1, nE};
        case GLSM_GEL_T2: return {d.T2, nE};
        case GLSM_GEL_RM: return {d.rm, 3 * nE};
        case GLSM_GEL_NMSM: return {d.nmSm, 18 * nE};
        case GLSM_GEL_VOLM: return {d.vol, nE};
        case GLSM_GEL_PREM: return {d.pm, nE};
        case GLSM_GEL_UN_ROBIN: return {d.un_robin, nN};
        case GLSM_GEL_UM_NORM: return {d.um_norm, nE};
        case GLSM_GEL_VM_NORM: return {d.vm_norm, nE};
        case GLSM_GEL_WMP: return {d.wmp, nE};
        case GLSM_GEL_FN_ROBIN: return {d.Fn_robin, 3 * nN};
        case GLSM_GEL_RM_LOC: return {d.rm_loc, 24 * nE};
        case GLSM_GEL_SERIES: return {d.series, 12 * (size_t)d.series_cap};
        default: return {nullptr, 0};
    }
}

static int snap_ensure(Snapshot& sn, size_t bytes) {
    if (!sn.copy) {
        CK(cudaStreamCreateWithFlags(&sn.copy, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&sn.taken, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&sn.done, cudaEventDisableTiming));
    }
    if (bytes > sn.bytes) {
        if (sn.dev) {
            CK(cudaEventSynchronize(sn.done));
            CK(cudaFree(sn.dev));
            sn.dev = nullptr;
            sn.bytes = 0;
        }
        CK(cudaMalloc(&sn.dev, bytes));
        sn.bytes = bytes;
    }
    return GLSM_OK;
}

static void snap_release(Snapshot& sn) {
    if (sn.copy) cudaStreamSynchronize(sn.copy);
    if (sn.dev) cudaFree(sn.dev);
    if (sn.taken) cudaEventDestroy(sn.taken);
    if (sn.done) cudaEventDestroy(sn.done);
    if (sn.copy) cudaStreamDestroy(sn.copy);
    sn = Snapshot{};
}

// steady state of the BZ kinetics at w = FA0 by bisection on v
// (Gel::steadyStateValue / fu_h, src/gel.cu:424-450)
static void bz_steady_state(double f, double q, double FA0, double& u, double& v, double& w) {
    w = FA0;
    const double a = 1.0 - w, aa = a * a;
    auto rate = [&](double vv) {
        const double uu = vv / (1 - w);
        return aa * uu - uu * uu - a * (f * vv + 0.0) * (uu - q * aa) / (uu + q * aa);
    };
    double hi = 1.0, lo = 0.0;
    while (std::fabs(hi - lo) > 1e-10) {
        const double mid = 0.5 * (hi + lo);
        if (rate(mid) * rate(hi) < 0)
            lo = mid;
        else
            hi = mid;
    }
    u = lo / (1.0 - w);
    v = lo;
}

extern "C" {

const char* glsm_last_error(void) { return g_err; }
int glsm_version(void) { return 1; }

// ===========================================================================
// Gel
// ===========================================================================
int glsm_gel_create(int sx, int sy, int sz, double px, double py, double pz, int gel_type, int gel_id,
                    glsm_gel* out) {
    if (!out || sx < 1 || sy < 1 || sz < 1 || sx > 4096 || sy > 4096 || sz > 4096)
        return fail(GLSM_ERR_ARG, "gel size must be >= 1 element per axis");
    if (gel_type != 1 && gel_type != 2) return fail(GLSM_ERR_ARG, "gel type must be 1 or 2");
    auto* g = new glsm_gel_s;
    GelDev& d = g->d;
    d.LX = sx + 1;
    d.LY = sy + 1;
    d.LZ = sz + 1;
    d.nE = (d.LX + 1) * (d.LY + 1) * (d.LZ + 1);
    d.nN = (d.LX + 2) * (d.LY + 2) * (d.LZ + 2);
    d.M = d.LX * d.LY * d.LZ - (d.LX - 2) * (d.LY - 2) * (d.LZ - 2);
    d.gel_id = gel_id;
    d.type = gel_type;
    // GelParams defaults, src/gel.cu:630-653
    d.f = 0.9;
    d.ep = 0.3;
    d.dt = 1e-3;
    d.dtx = 5 * 1e-3;
    d.dx = d.dy = d.dz = 1;
    d.CH0 = 0.338;
    d.CH1 = 0.518;
    d.CHS = 0.1;
    d.C0 = 1.3e-3;
    d.AZ0 = 100.0;
    d.FA0 = 0.139;
    d.c0_bis = 5e-4;
    d.b = 0.01;
    bz_steady_state(d.f, 1e-4, d.FA0, d.uss, d.vss, d.wss);
    d.series_every = 1000;
    d.series_cap = 1000;

    const size_t nE = d.nE, nN = d.nN;
    size_t bytes = 0;
    {
        Carver cv{nullptr};
        for (int i = 0; i < 11; i++) cv.take<double>(nE);
        cv.take<double3>(nE);
        cv.take<double3>(8 * nE);
        cv.take<double3>(6 * nE);
        for (int i = 0; i < 5; i++) cv.take<double3>(nN);
        for (int i = 0; i < 3; i++) cv.take<double>(nN);
        cv.take<int>(d.M);
        cv.take<double>(12 * (size_t)d.series_cap);
        cv.take<GelDev>(1);
        cv.take<Ctl>(1);
        bytes = align_up(cv.off, 256);
    }
    cudaError_t e = cudaMalloc(&g->arena, bytes);
    if (e != cudaSuccess) {
        delete g;
        return fail(GLSM_ERR_NOMEM, "gel allocation of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    g->bytes = bytes;
    Carver cv{(char*)g->arena};
    double** es[11] = {&d.um, &d.vm, &d.wm, &d.wmp, &d.um_norm, &d.vm_norm, &d.T0, &d.T1, &d.T2, &d.vol, &d.pm};
    for (auto p : es) *p = cv.take<double>(nE);
    d.rm = cv.take<double3>(nE);
    d.rm_loc = cv.take<double3>(8 * nE);
    d.nmSm = cv.take<double3>(6 * nE);
    double3** ns[5] = {&d.rn, &d.Veln, &d.Vels, &d.Fn, &d.Fn_robin};
    for (auto p : ns) *p = cv.take<double3>(nN);
    d.un_norm = cv.take<double>(nN);
    d.un_robin = cv.take<double>(nN);
    d.vn_norm = cv.take<double>(nN);
    d.bIndex = cv.take<int>(d.M);
    d.series = cv.take<double>(12 * (size_t)d.series_cap);
    g->d_self = cv.take<GelDev>(1);
    g->d_ctl = cv.take<Ctl>(1);

    // initial state on the host (src/gel.cu:179-219, :161-177)
    std::vector<double> um(nE, 0.0), vm(nE, 0.0), wm(nE, 0.0);
    for (int z = 1; z < d.LZ; z++)
        for (int y = 1; y < d.LY; y++)
            for (int x = 1; x < d.LX; x++) {
                const int i = x + (d.LX + 1) * (y + (d.LY + 1) * z);
                um[i] = d.uss;
                vm[i] = d.vss;
                wm[i] = d.wss;
            }
    const double lam = std::pow(d.FA0 / d.wss, 1 / 3.0);
    std::vector<double3> rn(nN);
    for (int z = 0; z < d.LZ + 2; z++)
        for (int y = 0; y < d.LY + 2; y++)
            for (int x = 0; x < d.LX + 2; x++) {
                double3& r = rn[x + (d.LX + 2) * (y + (d.LY + 2) * z)];
                r.x = px + (2 * double(x) - double(d.LX) - 1) * d.dx * lam / 2;
                r.y = py + (2 * double(y) - double(d.LY) - 1) * d.dy * lam / 2;
                r.z = pz + (2 * double(z) - double(d.LZ) - 1) * d.dz * lam / 2;
            }
    std::vector<int> surf;
    surf.reserve(d.M);
    for (int z = 1; z <= d.LZ; z++)
        for (int y = 1; y <= d.LY; y++)
            for (int x = 1; x <= d.LX; x++)
                if (x == 1 || x == d.LX || y == 1 || y == d.LY || z == 1 || z == d.LZ)
                    surf.push_back(x + (d.LX + 2) * (y + (d.LY + 2) * z));

    // blocking streams, like the reference's: legacy-stream copies order after queued work
    e = cudaStreamCreate(&g->own);
    if (e == cudaSuccess) e = cudaMemset(g->arena, 0, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(d.um, um.data(), nE * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d.vm, vm.data(), nE * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d.wm, wm.data(), nE * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d.rn, rn.data(), nN * sizeof(double3), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d.bIndex, surf.data(), d.M * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(g->d_self, &d, sizeof(GelDev), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (g->own) cudaStreamDestroy(g->own);
        cudaFree(g->arena);
        delete g;
        return fail(GLSM_ERR_CUDA, "gel initialisation: %s", cudaGetErrorString(e));
    }
    *out = g;
    return GLSM_OK;
}

static void gel_release(glsm_gel g) {
    snap_release(g->snap);
    cudaStreamSynchronize(g->own);
    cudaStreamDestroy(g->own);
    if (g->series_extra) cudaFree(g->series_extra);
    cudaFree(g->arena);
    delete g;
}

int glsm_gel_destroy(glsm_gel g) {
    if (!g) return GLSM_OK;
    if (g->coupler) {
        // the reference's drivers delete their gels before the fluid and the
        // coupler (src/sim.cpp:143-146): the gel is released with its coupler
        g->release_with_coupler = true;
        return GLSM_OK;
    }
    gel_release(g);
    return GLSM_OK;
}

int glsm_gel_info(glsm_gel g, int64_t out[8]) {
    if (!g || !out) return fail(GLSM_ERR_ARG, "null argument");
    out[0] = g->d.LX;
    out[1] = g->d.LY;
    out[2] = g->d.LZ;
    out[3] = g->d.nE;
    out[4] = g->d.nN;
    out[5] = g->d.M;
    out[6] = g->d.gel_id;
    out[7] = g->d.type;
    return GLSM_OK;
}

int glsm_gel_steady_state(glsm_gel g, double out[3]) {
    if (!g || !out) return fail(GLSM_ERR_ARG, "null argument");
    out[0] = g->d.uss;
    out[1] = g->d.vss;
    out[2] = g->d.wss;
    return GLSM_OK;
}

static int gel_launch(glsm_gel g, int phases, int iter) {
    if (!g) return fail(GLSM_ERR_ARG, "null gel");
    if (iter < 0) return fail(GLSM_ERR_ARG, "iteration must be >= 0");
    GelArgs a{};
    if (g->coupler) {
        a.gels = g->coupler->d_gels;
        a.first_gel = g->index;
        a.Mk = g->coupler->mk;
        a.ctl = g->coupler->d_ctl;
    } else {
        a.gels = g->d_self;
        a.first_gel = 0;
        a.ctl = g->d_ctl;
    }
    a.phases = phases;
    a.iter_arg = iter;
    mark_markers_stale(g);
    CK(launch_gel(a, 1, gel_stream(g)));
    return GLSM_OK;
}

int glsm_gel_step_elasticity(glsm_gel g, int iter) { return gel_launch(g, kPhElastic, iter); }
int glsm_gel_step_chemistry(glsm_gel g, int iter) { return gel_launch(g, kPhChem, iter); }
int glsm_gel_record_center(glsm_gel g, int iter) { return gel_launch(g, kPhRecord, iter); }

int glsm_gel_series_config(glsm_gel g, int every, int capacity) {
    if (!g || every < 1 || capacity < 1) return fail(GLSM_ERR_ARG, "every and capacity must be >= 1");
    if (capacity > g->d.series_cap) {
        double* p = nullptr;
        CK(cudaStreamSynchronize(gel_stream(g)));
        CK(cudaMalloc(&p, 12 * sizeof(double) * (size_t)capacity));
        CK(cudaMemset(p, 0, 12 * sizeof(double) * (size_t)capacity));
        if (g->series_extra) cudaFree(g->series_extra);
        g->series_extra = p;
        g->d.series = p;
    }
    g->d.series_every = every;
    g->d.series_cap = capacity;
    return upload_gel_desc(g);
}

int glsm_gel_series_read(glsm_gel g, double* dst, size_t count) {
    if (!g || !dst) return fail(GLSM_ERR_ARG, "null argument");
    const size_t n = 12 * (size_t)g->d.series_cap;
    if (count < n) return fail(GLSM_ERR_ARG, "series needs %zu doubles", n);
    CK(cudaStreamSynchronize(gel_stream(g)));
    CK(cudaMemcpy(dst, g->d.series, n * sizeof(double), cudaMemcpyDeviceToHost));
    return GLSM_OK;
}

size_t glsm_gel_field_size(glsm_gel g, int field) { return g ? gel_field(g, field).count : 0; }

int glsm_gel_read(glsm_gel g, int field, double* dst, size_t count) {
    if (!g || !dst) return fail(GLSM_ERR_ARG, "null argument");
    FieldRef f = gel_field(g, field);
    if (!f.ptr) return fail(GLSM_ERR_ARG, "unknown gel field %d", field);
    if (count < f.count) return fail(GLSM_ERR_ARG, "field %d needs %zu doubles", field, f.count);
    CK(cudaMemcpyAsync(dst, f.ptr, f.count * sizeof(double), cudaMemcpyDeviceToHost, gel_stream(g)));
    CK(cudaStreamSynchronize(gel_stream(g)));
    return GLSM_OK;
}

int glsm_gel_snapshot(glsm_gel g, int n_fields, const int* fields, double* const* dst) {
    if (!g || n_fields < 1 || n_fields > 32 || !fields || !dst) return fail(GLSM_ERR_ARG, "bad snapshot arguments");
    FieldRef f[32];
    size_t total = 0;
    for (int k = 0; k < n_fields; k++) {
        f[k] = gel_field(g, fields[k]);
        if (!f[k].ptr || !dst[k]) return fail(GLSM_ERR_ARG, "snapshot field %d: unknown field or null buffer", fields[k]);
        total += f[k].count;
    }
    if (int r = snap_ensure(g->snap, total * sizeof(double))) return r;
    Snapshot& sn = g->snap;
    cudaStream_t s = gel_stream(g);
    // the previous snapshot's transfer reads the device copy: overwrite it after
    if (sn.used) CK(cudaStreamWaitEvent(s, sn.done, 0));
    double* dev = static_cast<double*>(sn.dev);
    size_t off = 0;
    for (int k = 0; k < n_fields; k++) {
        CK(cudaMemcpyAsync(dev + off, f[k].ptr, f[k].count * sizeof(double), cudaMemcpyDeviceToDevice, s));
        off += f[k].count;
    }
    CK(cudaEventRecord(sn.taken, s));
    CK(cudaStreamWaitEvent(sn.copy, sn.taken, 0));
    off = 0;
    for (int k = 0; k < n_fields; k++) {
        CK(cudaMemcpyAsync(dst[k], dev + off, f[k].count * sizeof(double), cudaMemcpyDeviceToHost, sn.copy));
        off += f[k].count;
    }
    CK(cudaEventRecord(sn.done, sn.copy));
    sn.used = true;
    return GLSM_OK;
}

int glsm_gel_snapshot_wait(glsm_gel g) {
    if (!g) return fail(GLSM_ERR_ARG, "null gel");
    if (g->snap.used) CK(cudaEventSynchronize(g->snap.done));
    return GLSM_OK;
}

int glsm_gel_write(glsm_gel g, int field, const double* src, size_t count) {
    if (!g || !src) return fail(GLSM_ERR_ARG, "null argument");
    FieldRef f = gel_field(g, field);
    if (!f.ptr) return fail(GLSM_ERR_ARG, "unknown gel field %d", field);
    if (count != f.count) return fail(GLSM_ERR_ARG, "field %d holds %zu doubles", field, f.count);
    mark_markers_stale(g);
    CK(cudaMemcpyAsync(f.ptr, src, f.count * sizeof(double), cudaMemcpyHostToDevice, gel_stream(g)));
    CK(cudaStreamSynchronize(gel_stream(g)));
    return GLSM_OK;
}

void* glsm_gel_device_ptr(glsm_gel g, int field) {
    if (!g) return nullptr;
    g->ptr_out = true;  // writes through it are invisible to the host
    return gel_field(g, field).ptr;
}

int glsm_gel_filament(glsm_gel g, double* xyz, size_t max_points, size_t* n_points) {
    if (!g || !n_points || (max_points && !xyz)) return fail(GLSM_ERR_ARG, "null argument");
    const size_t faces = (size_t)std::max(0, g->d.LX - 1) * std::max(0, g->d.LY - 1) * std::max(0, g->d.LZ - 1);
    *n_points = 0;
    if (faces == 0) return GLSM_OK;
    cudaStream_t s = gel_stream(g);
    double4* d_out = nullptr;
    CK(cudaMalloc(&d_out, faces * sizeof(double4)));
    std::vector<double4> h(faces);
    cudaError_t e = launch_filament(g->d, d_out, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_out, faces * sizeof(double4), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_out);
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "filament: %s", cudaGetErrorString(e));
    size_t n = 0;
    for (const double4& p : h) {
        if (p.x == 0.0) continue;
        if (n < max_points) {
            xyz[3 * n] = p.y;
            xyz[3 * n + 1] = p.z;
            xyz[3 * n + 2] = p.w;
        }
        n++;
    }
    *n_points = n;
    return GLSM_OK;
}

}  // extern "C"

// element-slot edit on the host: read um, vm, wm, apply fn(x, y, z, u, v, w), write back
template <typename Fn>
static int edit_chemistry(glsm_gel g, Fn fn) {
    const GelDev& d = g->d;
    std::vector<double> u(d.nE), v(d.nE), w(d.nE);
    int r;
    if ((r = glsm_gel_read(g, GLSM_GEL_UM, u.data(), d.nE))) return r;
    if ((r = glsm_gel_read(g, GLSM_GEL_VM, v.data(), d.nE))) return r;
    if ((r = glsm_gel_read(g, GLSM_GEL_WM, w.data(), d.nE))) return r;
    for (int z = 0; z <= d.LZ; z++)
        for (int y = 0; y <= d.LY; y++)
            for (int x = 0; x <= d.LX; x++) {
                const int i = x + (d.LX + 1) * (y + (d.LY + 1) * z);
                fn(x, y, z, u[i], v[i], w[i]);
            }
    if ((r = glsm_gel_write(g, GLSM_GEL_UM, u.data(), d.nE))) return r;
    if ((r = glsm_gel_write(g, GLSM_GEL_VM, v.data(), d.nE))) return r;
    return glsm_gel_write(g, GLSM_GEL_WM, w.data(), d.nE);
}

static bool host_void(const GelDev& d, int y, int z) {
    if (d.tube_mode == 0) return false;
    const float dy = (float)y - d.tube_cy, dz = (float)z - d.tube_cz;
    if (d.tube_mode == 1) return std::fabs(dy) < d.tube_ihy && std::fabs(dz) < d.tube_ihz;
    if (d.tube_ihy < 0.5f || d.tube_ihz < 0.5f) return false;
    return (dy * dy) / (d.tube_ihy * d.tube_ihy) + (dz * dz) / (d.tube_ihz * d.tube_ihz) < 1.0f;
}

extern "C" {

int glsm_gel_reset_quiescent(glsm_gel g) {
    if (!g) return fail(GLSM_ERR_ARG, "null gel");
    const GelDev d = g->d;
    return edit_chemistry(g, [&](int x, int y, int z, double& u, double& v, double& w) {
        if (x >= 1 && y >= 1 && z >= 1) {  // slots 1..LX (src/gel.cu:736-743)
            u = d.uss * 0.01;
            v = d.vss * 0.01;
            w = d.wss;
        }
    });
}

int glsm_gel_fire_pulse(glsm_gel g) {
    if (!g) return fail(GLSM_ERR_ARG, "null gel");
    const GelDev d = g->d;
    const int pw = std::max(1, d.LX / 10);
    return edit_chemistry(g, [&](int x, int y, int z, double& u, double& v, double&) {
        if (x >= 1 && x <= pw && y >= 1 && z >= 1 && !host_void(d, y, z)) {
            u = d.uss * 3.0;
            v = d.vss * 0.1;
        }
    });
}

int glsm_gel_set_anchor_z(glsm_gel g, double anchor_z) {
    if (!g) return fail(GLSM_ERR_ARG, "null gel");
    g->d.use_anchor = 1;
    g->d.anchor_z = anchor_z;
    return upload_gel_desc(g);
}

int glsm_gel_build_tube_mask(glsm_gel g, int wall_thickness, int circular) {
    if (!g || wall_thickness < 0) return fail(GLSM_ERR_ARG, "bad tube mask arguments");
    GelDev& d = g->d;
    const float cy = (d.LY + 1) * 0.5f, cz = (d.LZ + 1) * 0.5f;
    float ihy = (d.LY * 0.5f) - wall_thickness, ihz = (d.LZ * 0.5f) - wall_thickness;
    if (ihy <= 0) ihy = 0;
    if (ihz <= 0) ihz = 0;
    d.tube_mode = circular ? 2 : 1;
    d.tube_cy = cy;
    d.tube_cz = cz;
    d.tube_ihy = ihy;
    d.tube_ihz = ihz;
    int r = upload_gel_desc(g);
    if (r) return r;
    // void elements start at the steady state (src/gel.cu:835-854)
    const GelDev dd = d;
    return edit_chemistry(g, [&](int x, int y, int z, double& u, double& v, double& w) {
        if (x < 1 || y < 1 || z < 1) return;
        const float dy = (float)y - dd.tube_cy, dz = (float)z - dd.tube_cz;
        bool vd;
        if (circular) {
            const float r2 = dy * dy / (dd.tube_ihy * dd.tube_ihy + 1e-6f) + dz * dz / (dd.tube_ihz * dd.tube_ihz + 1e-6f);
            vd = dd.tube_ihy > 0 && dd.tube_ihz > 0 && r2 < 1.0f;
        } else {
            vd = std::fabs(dy) < dd.tube_ihy && std::fabs(dz) < dd.tube_ihz;
        }
        if (vd) {
            u = dd.uss;
            v = dd.vss;
            w = dd.wss;
        }
    });
}

int glsm_gel_set_bz_f(glsm_gel g, double f) {
    if (!g || !(f > 0.0)) return fail(GLSM_ERR_ARG, "f must be positive");
    GelDev& d = g->d;
    d.f = f;
    bz_steady_state(d.f, 1e-4, d.FA0, d.uss, d.vss, d.wss);
    int r = upload_gel_desc(g);
    if (r) return r;
    // the interior starts at the new steady state (src/gel.cu:184-200)
    const GelDev dd = d;
    return edit_chemistry(g, [&](int x, int y, int z, double& u, double& v, double& w) {
        if (x >= 1 && x < dd.LX && y >= 1 && y < dd.LY && z >= 1 && z < dd.LZ) {
            u = dd.uss;
            v = dd.vss;
            w = dd.wss;
        }
    });
}

int glsm_gel_set_active_from(glsm_gel g, int iter) {
    if (!g || iter < 0) return fail(GLSM_ERR_ARG, "iteration must be >= 0");
    g->d.active_from = iter;
    return upload_gel_desc(g);
}

int glsm_gel_add_noise(glsm_gel g, uint64_t seed, double amplitude) {
    if (!g) return fail(GLSM_ERR_ARG, "null gel");
    const GelDev d = g->d;
    return edit_chemistry(g, [&](int x, int y, int z, double& u, double& v, double&) {
        if (x >= 1 && x < d.LX && y >= 1 && y < d.LY && z >= 1 && z < d.LZ) {
            const uint64_t slot = (uint64_t)(x + (d.LX + 1) * (y + (d.LY + 1) * z));
            u += amplitude * noise_unit(seed, (uint64_t)d.gel_id, slot, 0);
            v += amplitude * noise_unit(seed, (uint64_t)d.gel_id, slot, 1);
        }
    });
}

// ===========================================================================
// Coupler
// ===========================================================================
int glsm_coupler_create(const glsm_gel* gels, int n_gels, glsm_coupler* out) {
    if (!out || (n_gels > 0 && !gels) || n_gels < 0) return fail(GLSM_ERR_ARG, "bad gel list");
    if (n_gels > kMaxBoxes) return fail(GLSM_ERR_ARG, "at most %d gels per coupler", kMaxBoxes);
    for (int i = 0; i < n_gels; i++) {
        if (!gels[i]) return fail(GLSM_ERR_ARG, "null gel %d", i);
        if (gels[i]->coupler) return fail(GLSM_ERR_STATE, "gel %d already belongs to a coupler", i);
        for (int j = 0; j < i; j++)
            if (gels[j] == gels[i]) return fail(GLSM_ERR_ARG, "gel %d listed twice", i);
    }
    auto* c = new glsm_coupler_s;
    int M = 0;
    for (int i = 0; i < n_gels; i++) M += gels[i]->d.M;
    c->mk.M = M;
    size_t bytes;
    {
        Carver cv{nullptr};
        cv.take<GelDev>(std::max(1, n_gels));
        for (int i = 0; i < 5; i++) cv.take<float4>(std::max(1, M));
        for (int i = 0; i < 3; i++) cv.take<float>(std::max(1, M));
        cv.take<int>(std::max(1, M));
        cv.take<int4>(std::max(1, M));
        for (int i = 0; i < 3; i++) cv.take<float4>(std::max(1, M));
        cv.take<float>(std::max(1, M));
        cv.take<Box>(kMaxBoxes);
        cv.take<int2>(kMaxBoxes);
        cv.take<Ctl>(1);
        cv.take<int>(kMaxBoxes);
        bytes = align_up(cv.off, 256);
    }
    cudaError_t e = cudaMalloc(&c->arena, bytes);
    if (e != cudaSuccess) {
        delete c;
        return fail(GLSM_ERR_NOMEM, "coupler allocation: %s", cudaGetErrorString(e));
    }
    c->bytes = bytes;
    Carver cv{(char*)c->arena};
    c->d_gels = cv.take<GelDev>(std::max(1, n_gels));
    MarkerDev& mk = c->mk;
    mk.lag = cv.take<float4>(std::max(1, M));
    mk.Vl = cv.take<float4>(std::max(1, M));
    mk.Ul = cv.take<float4>(std::max(1, M));
    mk.Fdrag = cv.take<float4>(std::max(1, M));
    mk.Frep = cv.take<float4>(std::max(1, M));
    mk.Cl = cv.take<float>(std::max(1, M));
    mk.Dl = cv.take<float>(std::max(1, M));
    mk.Sl = cv.take<float>(std::max(1, M));
    mk.owner = cv.take<int>(std::max(1, M));
    mk.base = cv.take<int4>(std::max(1, M));
    mk.phx = cv.take<float4>(std::max(1, M));
    mk.phy = cv.take<float4>(std::max(1, M));
    mk.phz = cv.take<float4>(std::max(1, M));
    mk.wsum = cv.take<float>(std::max(1, M));
    mk.boxes = cv.take<Box>(kMaxBoxes);
    mk.gel_range = cv.take<int2>(kMaxBoxes);
    c->d_ctl = cv.take<Ctl>(1);
    c->d_fresh = cv.take<int>(kMaxBoxes);
    std::vector<int> owner(M);
    int off = 0;
    for (int i = 0; i < n_gels; i++) {
        glsm_gel_s* g = gels[i];
        cudaStreamSynchronize(g->own);
        g->coupler = c;
        g->index = i;
        g->d.marker_off = off;
        for (int l = 0; l < g->d.M; l++) owner[off + l] = i;
        off += g->d.M;
        c->gels.push_back(g);
    }
    e = cudaStreamCreate(&c->stream);
    if (e == cudaSuccess) e = cudaStreamCreate(&c->side);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&c->h_ctl, sizeof(Ctl), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMemset(c->arena, 0, bytes);
    if (e == cudaSuccess && M) e = cudaMemcpy(mk.owner, owner.data(), M * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n_gels) {
        std::vector<int2> ranges(n_gels);
        int m0 = 0;
        for (int i = 0; i < n_gels; i++) {
            ranges[i] = make_int2(m0, m0 + c->gels[i]->d.M);
            m0 += c->gels[i]->d.M;
        }
        e = cudaMemcpy(mk.gel_range, ranges.data(), n_gels * sizeof(int2), cudaMemcpyHostToDevice);
    }
    for (int i = 0; i < n_gels && e == cudaSuccess; i++)
        e = cudaMemcpy(c->d_gels + i, &c->gels[i]->d, sizeof(GelDev), cudaMemcpyHostToDevice);
    for (int i = 0; i < n_gels && e == cudaSuccess; i++)
        e = cudaMemcpy(c->gels[i]->d_self, &c->gels[i]->d, sizeof(GelDev), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        for (auto* g : c->gels) {
            g->coupler = nullptr;
            g->index = -1;
        }
        if (c->ev_fork) cudaEventDestroy(c->ev_fork);
        if (c->ev_join) cudaEventDestroy(c->ev_join);
        if (c->side) cudaStreamDestroy(c->side);
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->h_ctl) cudaFreeHost(c->h_ctl);
        cudaFree(c->arena);
        delete c;
        return fail(GLSM_ERR_CUDA, "coupler initialisation: %s", cudaGetErrorString(e));
    }
    *out = c;
    return GLSM_OK;
}

int glsm_coupler_destroy(glsm_coupler c) {
    if (!c) return GLSM_OK;
    if (c->fluid) return fail(GLSM_ERR_STATE, "destroy the fluid before its coupler");
    cudaStreamSynchronize(c->stream);
    for (auto* g : c->gels) {
        g->coupler = nullptr;
        g->index = -1;
        if (g->release_with_coupler) gel_release(g);
    }
    cudaEventDestroy(c->ev_fork);
    cudaEventDestroy(c->ev_join);
    cudaStreamDestroy(c->side);
    cudaStreamDestroy(c->stream);
    cudaFreeHost(c->h_ctl);
    cudaFree(c->arena);
    delete c;
    return GLSM_OK;
}

int glsm_coupler_markers(glsm_coupler c) { return c ? c->mk.M : 0; }
void* glsm_coupler_stream(glsm_coupler c) { return c ? (void*)c->stream : nullptr; }

static GelArgs coupler_gel_args(glsm_coupler c, int phases, int iter_arg) {
    GelArgs a{};
    a.gels = c->d_gels;
    a.first_gel = 0;
    a.Mk = c->mk;
    a.ctl = c->d_ctl;
    a.phases = phases;
    a.iter_arg = iter_arg;
    if (c->fluid) {
        a.nx = c->fluid->F.nx;
        a.ny = c->fluid->F.ny;
        a.nz = c->fluid->F.nz;
        a.h = c->fluid->F.h;
    }
    a.g2l = c->g2l;
    return a;
}

int glsm_coupler_pack(glsm_coupler c) {
    if (!c) return fail(GLSM_ERR_ARG, "null coupler");
    if (!c->fluid) return fail(GLSM_ERR_STATE, "create the fluid before packing markers");
    CK(launch_gel(coupler_gel_args(c, kPhGather, 0), (int)c->gels.size(), c->stream));
    return GLSM_OK;
}

int glsm_coupler_scatter(glsm_coupler c) {
    if (!c) return fail(GLSM_ERR_ARG, "null coupler");
    CK(launch_scatter(c->d_gels, c->mk, c->stream));
    return GLSM_OK;
}

int glsm_coupler_repulsion(glsm_coupler c) {
    if (!c) return fail(GLSM_ERR_ARG, "null coupler");
    RepulsionArgs r{c->d_gels, c->mk, c->rep_delta, c->rep_gamma, 0, nullptr, (int)c->gels.size(),
                    c->fluid ? c->fluid->F.h : 0.0f};
    CK(launch_repulsion(r, c->stream));
    return GLSM_OK;
}

int glsm_coupler_read(glsm_coupler c, int field, float* dst, size_t count) {
    if (!c || !dst) return fail(GLSM_ERR_ARG, "null argument");
    const size_t M = c->mk.M;
    const float4* v4 = nullptr;
    const float* v1 = nullptr;
    switch (field) {
        case GLSM_MK_LAG: v4 = c->mk.lag; break;
        case GLSM_MK_UL: v4 = c->mk.Ul; break;
        case GLSM_MK_VL: v4 = c->mk.Vl; break;
        case GLSM_MK_FDRAG: v4 = c->mk.Fdrag; break;
        case GLSM_MK_FREP: v4 = c->mk.Frep; break;
        case GLSM_MK_CL: v1 = c->mk.Cl; break;
        case GLSM_MK_DL: v1 = c->mk.Dl; break;
        case GLSM_MK_SL: v1 = c->mk.Sl; break;
        default: return fail(GLSM_ERR_ARG, "unknown marker field %d", field);
    }
    const size_t need = v4 ? 3 * M : M;
    if (count < need) return fail(GLSM_ERR_ARG, "marker field needs %zu floats", need);
    CK(cudaStreamSynchronize(c->stream));
    if (v1) {
        CK(cudaMemcpy(dst, v1, M * sizeof(float), cudaMemcpyDeviceToHost));
    } else {
        std::vector<float4> tmp(M);
        CK(cudaMemcpy(tmp.data(), v4, M * sizeof(float4), cudaMemcpyDeviceToHost));
        for (size_t l = 0; l < M; l++) {
            dst[3 * l] = tmp[l].x;
            dst[3 * l + 1] = tmp[l].y;
            dst[3 * l + 2] = tmp[l].z;
        }
    }
    return GLSM_OK;
}

// ===========================================================================
// Fluid
// ===========================================================================
// Fluid ctor unit conversions in float (src/fluid.cu:167-229)
static void fluid_units(float tau, float h, float& g2l, float& l2g, int& nsub) {
    const float dt = 1e-3f, niu = 1e-6f;
    const float dx_fluid = 40e-6f * h;
    const float dt_fluid = (tau - 0.5f) * dx_fluid * dx_fluid / (3 * niu);
    nsub = std::max(1, (int)llround(dt / dt_fluid));
    g2l = h * dt_fluid / dt;
    l2g = 1.0f / g2l;
}

int glsm_fluid_desc_default(glsm_fluid_desc* d, int nx, int ny, int nz) {
    if (!d) return fail(GLSM_ERR_ARG, "null desc");
    std::memset(d, 0, sizeof(*d));
    d->nx = nx;
    d->ny = ny;
    d->nz = nz;
    d->tau = 0.8f;
    d->h = 0.5f;
    d->beta = 1.0f;
    if (const char* s = getenv("IBM_BETA")) d->beta = (float)atof(s);
    d->ramp_steps = 20000.0f;
    if (const char* s = getenv("IBM_RAMP_STEPS")) d->ramp_steps = std::fmax(0.0f, (float)atof(s));
    float g2l, l2g;
    fluid_units(d->tau, d->h, g2l, l2g, d->nsub);
    d->storage = GLSM_STORE_F32;
    d->fp16_scale = 1048576.0f;  // 2^20
    return GLSM_OK;
}

__global__ void u_rest_kernel(float4* u, long long N);

// last-wave half tiles of the substep launches, in waves of the resident CTAs
constexpr int kTailWaves = 1;

static StepArgs step_args(glsm_fluid f, int k, int iter_arg, bool tail = true) {
    StepArgs a{};
    a.F = f->F;
    a.Mk = f->c->mk;
    a.ctl = f->c->d_ctl;
    a.tickets = f->d_sync;
    a.ibm_done = f->d_sync + f->F.nsub;
    a.n_boxes = (int)f->c->gels.size();
    a.n_ibm = (f->c->mk.M + kMarkersPerTask - 1) / kMarkersPerTask;
    a.iter_arg = iter_arg;
    a.k = k;
    a.last = (k == f->F.nsub - 1);
    a.div_nx = make_fastdiv((unsigned)f->F.nx);
    a.div_nxy = make_fastdiv((unsigned)(f->F.nx * f->F.ny));
    // full tiles, then half tiles for the last kTailWaves waves of resident
    // CTAs (none in a batch, whose launches mix systems)
    const long long N = f->F.N;
    const long long tail_cells = tail ? (long long)kTailWaves * std::max(f->lbm_ctas, 1) * (kTileCells / 2) : 0;
    const long long big = std::max(0LL, (N - tail_cells) / kTileCells);
    a.big_tiles = (int)big;
    a.n_tiles = (int)(big + (N - big * kTileCells + kTileCells / 2 - 1) / (kTileCells / 2));
    if (tail_cells == 0) a.big_tiles = a.n_tiles = (int)((N + kTileCells - 1) / kTileCells);
    a.lbm_ctas = f->lbm_ctas;
    a.lbm_ctas_even = f->lbm_ctas_even;
    a.wait_extra = f->wait_extra;
    a.l2_bytes = f->l2_bytes;
    a.l2_hit = f->l2_hit;
    return a;
}

// L2 residency of the population array (101^3: 78 MB FP32, 39 MB FP16 of the
// 126 MB L2), opt-in per fluid.  The substep launches then carry an
// access-policy window that marks the array persisting, so it stays in L2
// across the substeps of an iteration.  The persisting set-aside is a limit of
// the CUDA context, and L2 it reserves is lost to every access outside a window
// (a batch's launches, other fluids, the caller's own kernels): it is sized to
// the largest window of the fluids that use one and released (set to zero,
// persisting lines reset) when the last of them stops.  The set-aside is kept
// per device: fluids on different devices of one process each size their own.
// Must not run during a capture.
static std::mutex g_l2_mu;
static std::vector<glsm_fluid_s*> g_l2_users;  // fluids with a window, on any device

// Sizes device dev's persisting set-aside to the largest window of the fluids
// on that device (zero, with the persisting lines reset, when none is left) and
// sets their hit ratios.  Runs with dev current and restores the caller's device.
static void l2_setaside_locked(int dev) {
    int prev = dev;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = dev;
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    size_t want = 0;
    for (auto* u : g_l2_users)
        if (u->device == dev) want = std::max(want, (size_t)u->l2_bytes);
    int max_persist = 0;
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev);
    want = std::min(want, (size_t)std::max(max_persist, 0));
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) cudaGetLastError();
    if (want == 0 && cudaCtxResetPersistingL2Cache() != cudaSuccess) cudaGetLastError();
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    for (auto* u : g_l2_users)
        if (u->device == dev) u->l2_hit = cur ? std::min(1.0f, (float)cur / (float)u->l2_bytes) : 0.f;
    if (prev != dev) cudaSetDevice(prev);
}

// enables (on) or disables the window of f and resizes its device's set-aside
static void l2_window(glsm_fluid f, int on) {
    std::lock_guard<std::mutex> lock(g_l2_mu);
    auto it = std::find(g_l2_users.begin(), g_l2_users.end(), f);
    const bool was = it != g_l2_users.end();
    if (was) g_l2_users.erase(it);
    f->l2_on = 0;
    f->l2_bytes = 0;
    f->l2_hit = 0.f;
    const int dev = f->device;
    int max_window = 0, max_persist = 0;
    const size_t esz = (f->F.storage == GLSM_STORE_F32) ? 4 : 2;
    const size_t bytes = (size_t)19 * (size_t)f->F.S * esz;
    // only an array that fits in the set-aside can stay resident; a larger
    // one would reserve L2 without the benefit
    if (on && cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev) == cudaSuccess &&
        bytes <= (size_t)std::max(max_window, 0) && bytes <= (size_t)std::max(max_persist, 0)) {
        f->l2_on = 1;
        f->l2_bytes = bytes;
        g_l2_users.push_back(f);
    }
    cudaGetLastError();
    if (was || f->l2_on) l2_setaside_locked(dev);
    if (f->l2_on && f->l2_hit <= 0.f) {  // no set-aside could be had
        g_l2_users.pop_back();
        f->l2_on = 0;
        f->l2_bytes = 0;
        l2_setaside_locked(dev);
    }
}

int glsm_fluid_create(const glsm_fluid_desc* d, glsm_coupler c, glsm_fluid* out) {
    if (!d || !c || !out) return fail(GLSM_ERR_ARG, "null argument");
    if (c->fluid) return fail(GLSM_ERR_STATE, "coupler already has a fluid");
    if (d->nx < 4 || d->ny < 4 || d->nz < 4) return fail(GLSM_ERR_ARG, "lattice must be >= 4 cells per axis");
    const long long N = (long long)d->nx * d->ny * d->nz;
    // 32-bit cell indices: 19 planes of padded length must stay below 2^32
    if (N > 200000000LL) return fail(GLSM_ERR_ARG, "lattice too large (at most 2e8 cells)");
    if (d->nsub < 1 || d->nsub > 4096) return fail(GLSM_ERR_ARG, "nsub must be in [1, 4096]");
    if (d->storage < 0 || d->storage > 2) return fail(GLSM_ERR_ARG, "unknown storage %d", d->storage);
    if (!(d->tau > 0.5f) || !(d->h > 0.f)) return fail(GLSM_ERR_ARG, "tau must exceed 0.5 and h be positive");
    auto* f = new glsm_fluid_s;
    f->desc = *d;
    FluidDev& F = f->F;
    F.nx = d->nx;
    F.ny = d->ny;
    F.nz = d->nz;
    F.N = N;
    F.S = (long long)align_up((size_t)N, 64);
    F.storage = d->storage;
    F.scale = (d->storage == GLSM_STORE_F16) ? (d->fp16_scale > 0 ? d->fp16_scale : 1048576.0f) : 1.0f;
    F.inv_scale = 1.0f / F.scale;
    F.tau = d->tau;
    F.omega = 1.0f / d->tau;
    F.fpref = 1.0f - 0.5f / d->tau;
    for (int i = 0; i < 3; i++) {
        F.Fc[i] = d->force[i];
        F.per[i] = d->periodic[i] ? 1 : 0;
    }
    F.h = d->h;
    F.dtc = 1e-3f;  // FluidParams dt (fluid.cu:167)
    F.Dc = 1.0f;    // FluidParams D (fluid.cu:193)
    F.inv_dx = 1.0f;  // FluidParams dx = dy = dz = 1 (fluid.cu:190-192)
    F.beta = d->beta;
    F.ramp_steps = d->ramp_steps;
    F.nsub = d->nsub;
    const size_t esz = (d->storage == GLSM_STORE_F32) ? 4 : 2;
    size_t bytes;
    {
        Carver cv{nullptr};
        cv.take<char>(19 * (size_t)F.S * esz);
        cv.take<float4>(N);
        cv.take<float4>(N);
        for (int i = 0; i < 3; i++) cv.take<float>(N);
        cv.take<unsigned>(2 * (size_t)d->nsub);
        cv.take<double>(4 * (size_t)kConsBlocks + 4);
        bytes = align_up(cv.off, 256);
    }
    cudaError_t e = cudaMalloc(&f->arena, bytes);
    if (e != cudaSuccess) {
        delete f;
        return fail(GLSM_ERR_NOMEM, "lattice allocation of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    f->bytes = bytes;
    Carver cv{(char*)f->arena};
    F.pop = cv.take<char>(19 * (size_t)F.S * esz);
    F.u = cv.take<float4>(N);
    F.Fibm = cv.take<float4>(N);
    F.c[0] = cv.take<float>(N);
    F.c[1] = cv.take<float>(N);
    F.source = cv.take<float>(N);
    f->d_sync = cv.take<unsigned>(2 * (size_t)d->nsub);
    f->d_cons = cv.take<double>(4 * (size_t)kConsBlocks + 4);
    // rest state: zero deviations (f = w), u = 0, c = 0 (k_init, fluid_kernels.cu:84-96)
    e = cudaMemsetAsync(f->arena, 0, bytes, c->stream);
    if (e == cudaSuccess) {
        u_rest_kernel<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(F.u, N);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaFree(f->arena);
        delete f;
        return fail(GLSM_ERR_CUDA, "lattice initialisation: %s", cudaGetErrorString(e));
    }
    int nsub_phys;
    fluid_units(d->tau, d->h, c->g2l, c->l2g, nsub_phys);
    f->lbm_ctas = lbm_resident_ctas(d->storage, 1, 0);
    f->lbm_ctas_even = lbm_resident_ctas(d->storage, 0, 0);
    cudaGetDevice(&f->device);
    f->c = c;
    c->fluid = f;
    // the gels' gather now knows the lattice
    *out = f;
    return GLSM_OK;
}

int glsm_fluid_destroy(glsm_fluid f) {
    if (!f) return GLSM_OK;
    if (f->batch) return fail(GLSM_ERR_STATE, "remove the system from its batch first");
    cudaStreamSynchronize(f->c->stream);
    if (f->l2_on) l2_window(f, 0);
    for (auto& row : f->graph)
        for (auto& g : row)
            if (g) cudaGraphExecDestroy(g);
    if (f->scratch) cudaFree(f->scratch);
    snap_release(f->snap);
    cudaFree(f->arena);
    f->c->fluid = nullptr;
    delete f;
    return GLSM_OK;
}

int glsm_fluid_set_deterministic(glsm_fluid f, int on) {
    if (!f) return fail(GLSM_ERR_ARG, "null fluid");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    CK(cudaStreamSynchronize(f->c->stream));
    f->F.det_spread = on ? 1 : 0;
    // the captured iteration graphs hold the old launch arguments
    for (auto& row : f->graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    return GLSM_OK;
}

int glsm_fluid_set_l2_persisting(glsm_fluid f, int on) {
    if (!f) return fail(GLSM_ERR_ARG, "null fluid");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    CK(cudaStreamSynchronize(f->c->stream));
    l2_window(f, on);
    // the captured iteration graphs hold the old launch attributes
    for (auto& row : f->graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    return GLSM_OK;
}

int glsm_l2_reset_persisting(void) {
    CK(cudaCtxResetPersistingL2Cache());
    return GLSM_OK;
}

int glsm_l2_persisting_setaside(size_t* bytes) {
    if (!bytes) return fail(GLSM_ERR_ARG, "null argument");
    CK(cudaDeviceGetLimit(bytes, cudaLimitPersistingL2CacheSize));
    return GLSM_OK;
}

int glsm_fluid_set_f16_rounding(glsm_fluid f, int mode) {
    if (!f) return fail(GLSM_ERR_ARG, "null fluid");
    if (mode < 0 || mode > 2)
        return fail(GLSM_ERR_ARG, "rounding mode %d: 0 nearest, 1 conserving, 2 conserving on odd substeps", mode);
    if (mode && f->F.storage != GLSM_STORE_F16) return fail(GLSM_ERR_ARG, "conserving rounding needs FP16 storage");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    CK(cudaStreamSynchronize(f->c->stream));
    f->F.f16_round = mode;
    f->lbm_ctas = lbm_resident_ctas(f->F.storage, 1, mode);
    f->lbm_ctas_even = lbm_resident_ctas(f->F.storage, 0, mode);
    // the captured iteration graphs hold the old launch arguments
    for (auto& row : f->graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    return GLSM_OK;
}

int glsm_test_ibm_wait_extra(glsm_fluid f, int extra) {
    if (!f || extra < 0) return fail(GLSM_ERR_ARG, "bad argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    CK(cudaStreamSynchronize(f->c->stream));
    f->wait_extra = extra;
    // the captured iteration graphs hold the old launch arguments
    for (auto& row : f->graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    return GLSM_OK;
}

int glsm_f16_conserve_round(const float* in, float* out, size_t n_cells) {
    if (!in || !out) return fail(GLSM_ERR_ARG, "null argument");
    if (n_cells == 0) return GLSM_OK;
    if (n_cells > ((size_t)1 << 26)) return fail(GLSM_ERR_ARG, "at most 2^26 cells per call");
    const size_t bytes = n_cells * 19 * sizeof(float);
    float* d = nullptr;
    CK(cudaMalloc(&d, 2 * bytes));
    cudaError_t e = cudaMemcpy(d, in, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_conserve_round(d, d + n_cells * 19, (long long)n_cells, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d + n_cells * 19, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "conserve_round: %s", cudaGetErrorString(e));
    return GLSM_OK;
}

int glsm_fluid_units(glsm_fluid f, float out[2]) {
    if (!f || !out) return fail(GLSM_ERR_ARG, "null argument");
    out[0] = f->c->g2l;
    out[1] = f->c->l2g;
    return GLSM_OK;
}

int glsm_fluid_info(glsm_fluid f, int64_t out[8]) {
    if (!f || !out) return fail(GLSM_ERR_ARG, "null argument");
    out[0] = f->F.nx;
    out[1] = f->F.ny;
    out[2] = f->F.nz;
    out[3] = f->F.N;
    out[4] = f->F.nsub;
    out[5] = f->F.storage;
    out[6] = (int64_t)f->bytes;
    out[7] = f->substeps;
    return GLSM_OK;
}

// the substeps of one gel step (Fluid::stepVelocity)
static int enqueue_velocity(glsm_fluid f, int iter_arg, cudaStream_t s) {
    const int nsub = f->F.nsub;
    const int p0 = (int)(f->substeps & 1);
    CK(cudaMemsetAsync(f->d_sync, 0, 2 * sizeof(unsigned) * nsub, s));
    for (int k = 0; k < nsub; k++) CK(launch_substep(step_args(f, k, iter_arg), (p0 + k) & 1, s));
    return GLSM_OK;
}

int glsm_fluid_step_velocity(glsm_fluid f, int iter) {
    if (!f || iter < 0) return fail(GLSM_ERR_ARG, "bad argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    int r = enqueue_velocity(f, iter, f->c->stream);
    if (r) return r;
    f->substeps += f->F.nsub;
    return GLSM_OK;
}

// the advection launch's arguments for concentration buffer cur
static ConcArgs conc_args(glsm_fluid f, int cur, int bump_iter) {
    glsm_coupler c = f->c;
    ConcArgs a{f->F, c->mk, c->d_ctl, (int)c->gels.size(), cur, bump_iter, make_fastdiv((unsigned)f->F.nx),
               make_fastdiv((unsigned)(f->F.nx * f->F.ny)), 0, 1};
    conc_layout(a);
    return a;
}

int glsm_fluid_step_concentration(glsm_fluid f, int iter) {
    if (!f || iter < 0) return fail(GLSM_ERR_ARG, "bad argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    glsm_coupler c = f->c;
    MarkerArgs m{c->d_gels, c->mk, f->F.c[f->cur], f->F.source, f->F.nx, f->F.ny, f->F.nz, f->F.h, 0,
                 f->F.det_spread};
    CK(launch_conc_markers(m, c->stream));
    CK(launch_conv_diff(conc_args(f, f->cur, 0), c->stream));
    f->cur ^= 1;
    return GLSM_OK;
}

__global__ void set_iter_kernel(Ctl* ctl, int iter) { ctl->iter = iter; }

// one whole coupled iteration; iter_arg < 0 reads the iteration from the
// control block (graph mode) and advances it at the end
static int enqueue_iteration(glsm_fluid f, int iter_arg, int p0, int cur) {
    glsm_coupler c = f->c;
    cudaStream_t s = c->stream;
    const int nsub = f->F.nsub;
    // the gel kernel zeroes the substeps' ticket counters and gathers the
    // markers only after the nodes moved (or first in a run call)
    const int phases = kPhElastic | kPhChem | kPhRecord | kPhGather | kPhAuto | kPhGatherStale;
    GelArgs ga = coupler_gel_args(c, phases, iter_arg);
    ga.gather_fresh = c->d_fresh;
    ga.zero_words = f->d_sync;
    ga.n_zero_words = 2 * nsub;
    if (c->gels.empty()) CK(cudaMemsetAsync(f->d_sync, 0, 2 * sizeof(unsigned) * nsub, s));
    CK(launch_gel(ga, (int)c->gels.size(), s));
    // markers' concentration exchange and repulsion run beside the substeps
    CK(cudaEventRecord(c->ev_fork, s));
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    MarkerArgs m{c->d_gels, c->mk, f->F.c[cur], f->F.source, f->F.nx, f->F.ny, f->F.nz, f->F.h, 1,
                 f->F.det_spread};
    CK(launch_conc_markers(m, c->side));
    RepulsionArgs r{c->d_gels, c->mk, c->rep_delta, c->rep_gamma, 1, nullptr, (int)c->gels.size(), f->F.h};
    CK(launch_repulsion(r, c->side));
    CK(cudaEventRecord(c->ev_join, c->side));
    for (int k = 0; k < nsub; k++) CK(launch_substep(step_args(f, k, iter_arg), (p0 + k) & 1, s));
    CK(cudaStreamWaitEvent(s, c->ev_join, 0));
    CK(launch_conv_diff(conc_args(f, cur, iter_arg < 0 ? 1 : 0), s));
    return GLSM_OK;
}

static int get_graph(glsm_fluid f, int p0, int cur, cudaGraphExec_t* out) {
    if (f->graph[p0][cur]) {
        *out = f->graph[p0][cur];
        return GLSM_OK;
    }
    cudaStream_t s = f->c->stream;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int r = enqueue_iteration(f, -1, p0, cur);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&f->graph[p0][cur], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    *out = f->graph[p0][cur];
    return GLSM_OK;
}

int glsm_fluid_run(glsm_fluid f, int iter0, int n) {
    if (!f || iter0 < 0 || n < 0) return fail(GLSM_ERR_ARG, "bad argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    if (n == 0) return GLSM_OK;
    glsm_coupler c = f->c;
    // the graphs read the iteration from the control block and advance it; it
    // is set only when it is not already iter0 (a run continuing the last one)
    if (f->dev_iter != iter0) {
        f->dev_iter = -1;
        set_iter_kernel<<<1, 1, 0, c->stream>>>(c->d_ctl, iter0);
        CK(cudaGetLastError());
    }
    // the first iteration gathers the markers afresh when a gel changed since
    // the last run (fields, parameters, per-method steps, checkpoints) or may
    // have (a device pointer is out); otherwise the marker arrays are current
    bool stale = c->markers_stale;
    for (glsm_gel_s* g : c->gels) stale |= g->ptr_out;
    if (stale) {
        CK(cudaMemsetAsync(c->d_fresh, 0, sizeof(int) * c->gels.size(), c->stream));
        c->markers_stale = false;
    }
    f->dev_iter = -1;
    for (int it = 0; it < n; it++) {
        const int p0 = (int)(f->substeps & 1);
        cudaGraphExec_t ge;
        int r = get_graph(f, p0, f->cur, &ge);
        if (r) return r;
        CK(cudaGraphLaunch(ge, c->stream));
        f->substeps += f->F.nsub;
        f->cur ^= 1;
    }
    f->dev_iter = (long long)iter0 + n;
    return GLSM_OK;
}

int glsm_fluid_sync(glsm_fluid f) {
    if (!f) return fail(GLSM_ERR_ARG, "null fluid");
    glsm_coupler c = f->c;
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
    if (c->h_ctl->error) {
        const int err = c->h_ctl->error;
        CK(cudaMemset(&c->d_ctl->error, 0, sizeof(int)));
        return fail(GLSM_ERR_DEVICE, "device error flags 0x%x%s%s%s", err,
                    (err & kErrIbmWait) ? " [IBM wait timed out]" : "",
                    (err & kErrMarkerOut) ? " [marker stencil outside the lattice]" : "",
                    (err & kErrNonFinite) ? " [non-finite gel state]" : "");
    }
    return GLSM_OK;
}

// Fluid::stepVelocity with a CUDA event pair around every substep launch on the
// system stream; ms[k] receives the duration of substep k (for the roofline)
int glsm_fluid_profile_velocity(glsm_fluid f, int iter, float* ms) {
    if (!f || !ms || iter < 0) return fail(GLSM_ERR_ARG, "bad argument");
    cudaStream_t s = f->c->stream;
    const int nsub = f->F.nsub;
    const int p0 = (int)(f->substeps & 1);
    std::vector<cudaEvent_t> ev(2 * (size_t)nsub, nullptr);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    CK(cudaMemsetAsync(f->d_sync, 0, 2 * sizeof(unsigned) * nsub, s));
    int r = GLSM_OK;
    for (int k = 0; k < nsub && r == GLSM_OK; k++) {
        CK(cudaEventRecord(ev[2 * k], s));
        cudaError_t e = launch_substep(step_args(f, k, iter), (p0 + k) & 1, s);
        if (e != cudaSuccess) r = fail(GLSM_ERR_CUDA, "substep launch: %s", cudaGetErrorString(e));
        CK(cudaEventRecord(ev[2 * k + 1], s));
    }
    f->substeps += nsub;
    CK(cudaStreamSynchronize(s));
    for (int k = 0; k < nsub && r == GLSM_OK; k++) CK(cudaEventElapsedTime(&ms[k], ev[2 * k], ev[2 * k + 1]));
    for (auto& e : ev) cudaEventDestroy(e);
    return r;
}

// n_steps calls of Fluid::stepVelocity as one captured graph of their
// n_steps x nsub substep launches, timed with one CUDA event pair around the
// graph on the system stream: the substep kernel back to back as it runs inside
// the fused iteration
int glsm_fluid_profile_substeps_n(glsm_fluid f, int iter, int n_steps, float* total_ms) {
    if (!f || !total_ms || iter < 0 || n_steps < 1 || n_steps > 64) return fail(GLSM_ERR_ARG, "bad argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    cudaStream_t s = f->c->stream;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int r = GLSM_OK;
    for (int j = 0; j < n_steps && r == GLSM_OK; j++) {
        // the AA parity of step j follows from the substeps before it
        r = enqueue_velocity(f, iter + j, s);
        f->substeps += f->F.nsub;
    }
    f->substeps -= (long long)n_steps * f->F.nsub;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) e = cudaGraphLaunch(ge, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaEventElapsedTime(total_ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGraphExecDestroy(ge);
    if (e != cudaSuccess) return fail(GLSM_ERR_CUDA, "profile: %s", cudaGetErrorString(e));
    f->substeps += (long long)n_steps * f->F.nsub;
    return GLSM_OK;
}

int glsm_fluid_profile_substeps(glsm_fluid f, int iter, float* total_ms) {
    return glsm_fluid_profile_substeps_n(f, iter, 1, total_ms);
}

static int ensure_scratch(glsm_fluid f) {
    if (!f->scratch) CK(cudaMalloc(&f->scratch, 19 * sizeof(float) * (size_t)f->F.N));
    return GLSM_OK;
}

// u (to_float3 = 1) or rho (to_float3 = 0) out of the (ux, uy, uz, rho) cells
__global__ void u_pack_kernel(const float4* u, long long N, float* out, int to_float3) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 v = u[i];
    if (to_float3) {
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    } else {
        out[i] = v.w;
    }
}

__global__ void u_rest_kernel(float4* u, long long N) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) u[i] = make_float4(0.f, 0.f, 0.f, 1.0f);
}

__global__ void u_unpack_kernel(const float* in, long long N, float4* u) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    u[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 1.0f);
}

static int batch_wait(glsm_fluid f);

int glsm_fluid_conservation(glsm_fluid f, double out[4]) {
    if (!f || !out) return fail(GLSM_ERR_ARG, "null argument");
    if (int r = batch_wait(f)) return r;
    cudaStream_t s = f->c->stream;
    // after an odd number of substeps the last one was even: populations sit in
    // the opposite slots
    CK(launch_conservation(f->F, (int)(f->substeps & 1), f->d_cons, f->d_cons + 4 * kConsBlocks, s));
    CK(cudaMemcpyAsync(out, f->d_cons + 4 * kConsBlocks, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GLSM_OK;
}

int glsm_fluid_read(glsm_fluid f, int field, float* dst, size_t count) {
    if (!f || !dst) return fail(GLSM_ERR_ARG, "null argument");
    if (int r = batch_wait(f)) return r;
    cudaStream_t s = f->c->stream;
    const long long N = f->F.N;
    const unsigned blocks = (unsigned)((N + 255) / 256);
    int r;
    switch (field) {
        case GLSM_FLUID_POP: {
            const size_t need = 19 * (size_t)N;
            if (count < need) return fail(GLSM_ERR_ARG, "field needs %zu floats", need);
            if ((r = ensure_scratch(f))) return r;
            CK(launch_read_pop(f->F, (f->substeps & 1) == 0, f->scratch, s));
            CK(cudaMemcpyAsync(dst, f->scratch, need * sizeof(float), cudaMemcpyDeviceToHost, s));
            break;
        }
        case GLSM_FLUID_RHO: {
            // d_rho of the reference: the density moment of the last substep's
            // macros (k_macros), kept in u.w
            if (count < (size_t)N) return fail(GLSM_ERR_ARG, "field needs %lld floats", N);
            if ((r = ensure_scratch(f))) return r;
            u_pack_kernel<<<blocks, 256, 0, s>>>(f->F.u, N, f->scratch, 0);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(dst, f->scratch, N * sizeof(float), cudaMemcpyDeviceToHost, s));
            break;
        }
        case GLSM_FLUID_U: {
            if (count < 3 * (size_t)N) return fail(GLSM_ERR_ARG, "field needs %lld floats", 3 * N);
            if ((r = ensure_scratch(f))) return r;
            u_pack_kernel<<<blocks, 256, 0, s>>>(f->F.u, N, f->scratch, 1);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(dst, f->scratch, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, s));
            break;
        }
        case GLSM_FLUID_C1:
            if (count < (size_t)N) return fail(GLSM_ERR_ARG, "field needs %lld floats", N);
            CK(cudaMemcpyAsync(dst, f->F.c[f->cur], N * sizeof(float), cudaMemcpyDeviceToHost, s));
            break;
        default: return fail(GLSM_ERR_ARG, "unknown fluid field %d", field);
    }
    return glsm_fluid_sync(f);
}

int glsm_fluid_snapshot(glsm_fluid f, float* u_dst, float* c_dst) {
    if (!f || !u_dst || !c_dst) return fail(GLSM_ERR_ARG, "null argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    const long long N = f->F.N;
    if (int r = snap_ensure(f->snap, 4 * (size_t)N * sizeof(float))) return r;
    Snapshot& sn = f->snap;
    cudaStream_t s = f->c->stream;
    if (sn.used) CK(cudaStreamWaitEvent(s, sn.done, 0));
    float* dev_u = static_cast<float*>(sn.dev);
    float* dev_c = dev_u + 3 * N;
    u_pack_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(f->F.u, N, dev_u, 1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dev_c, f->F.c[f->cur], N * sizeof(float), cudaMemcpyDeviceToDevice, s));
    CK(cudaEventRecord(sn.taken, s));
    CK(cudaStreamWaitEvent(sn.copy, sn.taken, 0));
    CK(cudaMemcpyAsync(u_dst, dev_u, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, sn.copy));
    CK(cudaMemcpyAsync(c_dst, dev_c, N * sizeof(float), cudaMemcpyDeviceToHost, sn.copy));
    CK(cudaEventRecord(sn.done, sn.copy));
    sn.used = true;
    return GLSM_OK;
}

int glsm_fluid_snapshot_wait(glsm_fluid f) {
    if (!f) return fail(GLSM_ERR_ARG, "null fluid");
    if (f->snap.used) CK(cudaEventSynchronize(f->snap.done));
    return GLSM_OK;
}

int glsm_fluid_write(glsm_fluid f, int field, const float* src, size_t count) {
    if (!f || !src) return fail(GLSM_ERR_ARG, "null argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system is in a batch");
    cudaStream_t s = f->c->stream;
    const long long N = f->F.N;
    const unsigned blocks = (unsigned)((N + 255) / 256);
    int r;
    switch (field) {
        case GLSM_FLUID_POP:
            if (count != 19 * (size_t)N) return fail(GLSM_ERR_ARG, "populations hold %lld floats", 19 * N);
            if ((r = ensure_scratch(f))) return r;
            CK(cudaMemcpyAsync(f->scratch, src, count * sizeof(float), cudaMemcpyHostToDevice, s));
            CK(launch_write_pop(f->F, f->scratch, s));
            f->substeps &= ~1LL;  // natural layout from now on
            break;
        case GLSM_FLUID_U:
            if (count != 3 * (size_t)N) return fail(GLSM_ERR_ARG, "u holds %lld floats", 3 * N);
            if ((r = ensure_scratch(f))) return r;
            CK(cudaMemcpyAsync(f->scratch, src, count * sizeof(float), cudaMemcpyHostToDevice, s));
            u_unpack_kernel<<<blocks, 256, 0, s>>>(f->scratch, N, f->F.u);
            CK(cudaGetLastError());
            break;
        case GLSM_FLUID_C1:
            if (count != (size_t)N) return fail(GLSM_ERR_ARG, "c1 holds %lld floats", N);
            CK(cudaMemcpyAsync(f->F.c[f->cur], src, N * sizeof(float), cudaMemcpyHostToDevice, s));
            break;
        default: return fail(GLSM_ERR_ARG, "field %d is not writable", field);
    }
    CK(cudaStreamSynchronize(s));
    return GLSM_OK;
}


// ===========================================================================
// Batch: several systems advanced together
// ===========================================================================
struct glsm_batch_s {
    std::vector<glsm_fluid_s*> sys;
    std::vector<long long> remaining;  // host mirror of SysDyn::remaining (< 0: no limit)
    int nsub = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    BatchSys* d_sys = nullptr;
    SysDyn* d_dyn = nullptr;
    GelArgs* d_gel = nullptr;
    MarkerArgs* d_mark = nullptr;
    RepulsionArgs* d_rep = nullptr;
    int *d_members = nullptr, *d_ibm_off = nullptr, *d_tile_off = nullptr, *d_conv_off = nullptr,
        *d_warp_off = nullptr, *d_rep_off = nullptr;
    unsigned *d_tickets = nullptr, *d_ibm_done = nullptr;
    int n_gels = 0, warps = 0, rep_warps = 0, conv_blocks = 0;
    bool dirty = true;
    // one iteration graph per parity phase: with an odd nsub every running
    // system's substep parity flips from one iteration to the next
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int phase = 0;
    // streams on which the substep launches of groups 1.. run (group 0 runs
    // on `stream`), and the events that join them back
    std::vector<cudaStream_t> gstreams;
    std::vector<cudaEvent_t> gevents;
};

static int batch_wait(glsm_fluid f) {
    if (f->batch) CK(cudaStreamSynchronize(f->batch->stream));
    return GLSM_OK;
}

static void batch_free_device(glsm_batch_s* b) {
    for (auto& g : b->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    b->phase = 0;
}

// device descriptors of the current members; recapture of the iteration graph
static int batch_rebuild(glsm_batch_s* b) {
    CK(cudaStreamSynchronize(b->stream));
    batch_free_device(b);
    const int n = (int)b->sys.size();
    b->dirty = false;
    if (n == 0) return GLSM_OK;
    std::vector<BatchSys> hs(n);
    std::vector<SysDyn> hd(n);
    std::vector<GelArgs> hg;
    std::vector<MarkerArgs> hm(2 * (size_t)n);
    std::vector<RepulsionArgs> hr(n);
    std::vector<int> conv_off(n + 1, 0), warp_off(n + 1, 0), rep_off(n + 1, 0);
    // Groups: systems that share storage, x periodicity, spread mode and the
    // parity of their substep count share one kernel instantiation for every
    // substep (their parities stay equal).  Each group has its own member
    // list, prefix sums of IBM tasks and tiles, and ticket counters.
    struct Group {
        BatchGroupKey key;
        int p0;
        std::vector<int> members;
    };
    std::vector<Group> groups;
    for (int i = 0; i < n; i++) {
        const glsm_fluid_s* f = b->sys[i];
        const BatchGroupKey key{f->F.storage, f->F.per[0], f->F.det_spread, f->F.f16_round};
        const int p0 = (int)(f->substeps & 1);
        auto it = std::find_if(groups.begin(), groups.end(), [&](const Group& g) {
            return g.key.storage == key.storage && g.key.perx == key.perx && g.key.det == key.det &&
                   g.key.f16_round == key.f16_round && g.p0 == p0;
        });
        if (it == groups.end()) {
            groups.push_back(Group{key, p0, {}});
            it = groups.end() - 1;
        }
        it->members.push_back(i);
    }
    const int G = (int)groups.size();
    std::vector<int> members, gibm_off, gtile_off, g_total(G);
    for (int gi = 0; gi < G; gi++) {
        int io = 0, to = 0;
        gibm_off.push_back(0);
        gtile_off.push_back(0);
        for (int i : groups[gi].members) {
            const StepArgs a = step_args(b->sys[i], 0, -1, false);
            members.push_back(i);
            gibm_off.push_back(io += a.n_ibm);
            gtile_off.push_back(to += a.n_tiles);
        }
        g_total[gi] = io + to;
    }
    for (int i = 0; i < n; i++) {
        glsm_fluid_s* f = b->sys[i];
        glsm_coupler c = f->c;
        StepArgs a = step_args(f, 0, -1, false);
        hs[i].step = a;
        hs[i].conc = conc_args(f, 0, 0);
        hd[i].parity0 = (int)(f->substeps & 1);
        hd[i].cur = f->cur;
        hd[i].remaining = (int)std::min<long long>(b->remaining[i], 1 << 30);
        for (int cb = 0; cb < 2; cb++)
            hm[2 * i + cb] = MarkerArgs{c->d_gels, c->mk, f->F.c[cb], f->F.source, f->F.nx, f->F.ny, f->F.nz, f->F.h, 1,
                                        f->F.det_spread};
        hr[i] = RepulsionArgs{c->d_gels, c->mk, c->rep_delta, c->rep_gamma, 1, nullptr, (int)c->gels.size(), f->F.h};
        // markers packed only when they can have changed, as in glsm_fluid_run
        const int phases = kPhElastic | kPhChem | kPhRecord | kPhGather | kPhAuto | kPhGatherStale;
        for (int g = 0; g < (int)c->gels.size(); g++) {
            GelArgs ga = coupler_gel_args(c, phases, -1);
            ga.first_gel = g;
            ga.gather_fresh = c->d_fresh;
            hg.push_back(ga);
        }
        conv_off[i + 1] = conv_off[i] + conc_blocks(hs[i].conc);
        warp_off[i + 1] = warp_off[i] + c->mk.M;
        rep_off[i + 1] = rep_off[i] + c->mk.M;  // one warp per marker
    }
    b->n_gels = (int)hg.size();
    b->warps = warp_off[n];
    b->rep_warps = rep_off[n];
    b->conv_blocks = conv_off[n];
    size_t bytes;
    {
        Carver cv{nullptr};
        cv.take<BatchSys>(n);
        cv.take<SysDyn>(n);
        cv.take<GelArgs>(std::max<size_t>(1, hg.size()));
        cv.take<MarkerArgs>(2 * (size_t)n);
        cv.take<RepulsionArgs>(n);
        cv.take<int>(n);
        for (int k = 0; k < 2; k++) cv.take<int>(n + G);
        for (int k = 0; k < 3; k++) cv.take<int>(n + 1);
        cv.take<unsigned>((size_t)G * b->nsub);
        cv.take<unsigned>((size_t)n * b->nsub);
        bytes = align_up(cv.off, 256);
    }
    if (bytes > b->arena_bytes) {  // grow only
        if (b->arena) cudaFree(b->arena);
        b->arena = nullptr;
        b->arena_bytes = 0;
        CK(cudaMalloc(&b->arena, bytes * 2));
        b->arena_bytes = bytes * 2;
    }
    Carver cv{(char*)b->arena};
    b->d_sys = cv.take<BatchSys>(n);
    b->d_dyn = cv.take<SysDyn>(n);
    b->d_gel = cv.take<GelArgs>(std::max<size_t>(1, hg.size()));
    b->d_mark = cv.take<MarkerArgs>(2 * (size_t)n);
    b->d_rep = cv.take<RepulsionArgs>(n);
    b->d_members = cv.take<int>(n);
    b->d_ibm_off = cv.take<int>(n + G);
    b->d_tile_off = cv.take<int>(n + G);
    b->d_conv_off = cv.take<int>(n + 1);
    b->d_warp_off = cv.take<int>(n + 1);
    b->d_rep_off = cv.take<int>(n + 1);
    b->d_tickets = cv.take<unsigned>((size_t)G * b->nsub);
    b->d_ibm_done = cv.take<unsigned>((size_t)n * b->nsub);
    for (int i = 0; i < n; i++) {
        hs[i].dyn = b->d_dyn + i;
        hs[i].step.ibm_done = b->d_ibm_done + (size_t)i * b->nsub;
        hs[i].step.tickets = b->d_tickets;
        hr[i].dyn = b->d_dyn + i;
    }
    {
        size_t gi = 0;
        for (int i = 0; i < n; i++)
            for (size_t g = 0; g < b->sys[i]->c->gels.size(); g++) hg[gi++].dyn = b->d_dyn + i;
    }
    CK(cudaMemcpy(b->d_sys, hs.data(), n * sizeof(BatchSys), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_dyn, hd.data(), n * sizeof(SysDyn), cudaMemcpyHostToDevice));
    if (!hg.empty()) CK(cudaMemcpy(b->d_gel, hg.data(), hg.size() * sizeof(GelArgs), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_mark, hm.data(), hm.size() * sizeof(MarkerArgs), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_rep, hr.data(), hr.size() * sizeof(RepulsionArgs), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_members, members.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_ibm_off, gibm_off.data(), (n + G) * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_tile_off, gtile_off.data(), (n + G) * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_conv_off, conv_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_warp_off, warp_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_rep_off, rep_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));

    while ((int)b->gstreams.size() < G - 1) {
        cudaStream_t gs = nullptr;
        cudaEvent_t ge = nullptr;
        CK(cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking));
        b->gstreams.push_back(gs);
        CK(cudaEventCreateWithFlags(&ge, cudaEventDisableTiming));
        b->gevents.push_back(ge);
    }
    std::vector<int> resident(2 * G);
    for (int gi = 0; gi < G; gi++)
        for (int p = 0; p < 2; p++) resident[2 * gi + p] = batch_resident_ctas(groups[gi].key, p);

    // capture one batch iteration per parity phase; the groups' substep
    // chains run on their own streams, side by side on the GPU
    cudaStream_t st = b->stream;
    const int n_phases = (b->nsub & 1) ? 2 : 1;
    for (int ph = 0; ph < n_phases; ph++) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaMemsetAsync(b->d_tickets, 0, (size_t)G * b->nsub * sizeof(unsigned), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_ibm_done, 0, (size_t)n * b->nsub * sizeof(unsigned), st);
        if (e == cudaSuccess) e = launch_gel_batch(b->d_gel, b->n_gels, b->n_gels, st);
        if (e == cudaSuccess) e = cudaEventRecord(b->ev_fork, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side, b->ev_fork, 0);
        if (e == cudaSuccess) e = launch_conc_markers_batch(b->d_mark, b->d_dyn, b->d_warp_off, n, b->warps, b->side);
        if (e == cudaSuccess) e = launch_repulsion_batch(b->d_rep, b->d_rep_off, n, b->rep_warps, b->side);
        if (e == cudaSuccess) e = cudaEventRecord(b->ev_join, b->side);
        int moff = 0;
        for (int gi = 0; gi < G && e == cudaSuccess; gi++) {
            const Group& gr = groups[gi];
            const int ng = (int)gr.members.size();
            cudaStream_t gs = gi == 0 ? st : b->gstreams[gi - 1];
            if (gi > 0) e = cudaStreamWaitEvent(gs, b->ev_fork, 0);
            for (int k = 0; k < b->nsub && e == cudaSuccess; k++) {
                const int parity = (gr.p0 + ph * b->nsub + k) & 1;
                BatchLaunch L{b->d_sys, b->d_members + moff, b->d_ibm_off + moff + gi, b->d_tile_off + moff + gi,
                              b->d_tickets + (size_t)gi * b->nsub, ng, k, k == b->nsub - 1};
                e = launch_substep_batch(L, gr.key, parity, std::min(resident[2 * gi + parity], g_total[gi]), gs);
            }
            if (gi > 0 && e == cudaSuccess) e = cudaEventRecord(b->gevents[gi - 1], gs);
            if (gi > 0 && e == cudaSuccess) e = cudaStreamWaitEvent(st, b->gevents[gi - 1], 0);
            moff += ng;
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->ev_join, 0);
        if (e == cudaSuccess) e = launch_conv_diff_batch(b->d_sys, b->d_conv_off, n, b->conv_blocks, st);
        if (e == cudaSuccess) e = launch_batch_advance(b->d_sys, n, st);
        cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            b->dirty = true;
            return fail(GLSM_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&b->graph[ph], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->dirty = true;
            return fail(GLSM_ERR_CUDA, "batch instantiate: %s", cudaGetErrorString(e));
        }
    }
    return GLSM_OK;
}

int glsm_batch_create(glsm_batch* out) {
    if (!out) return fail(GLSM_ERR_ARG, "null argument");
    auto* b = new glsm_batch_s;
    // non-blocking streams: work on the legacy default stream (the synchronous
    // copies that build new systems) does not wait for a running batch
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete b;
        return fail(GLSM_ERR_CUDA, "batch: %s", cudaGetErrorString(e));
    }
    *out = b;
    return GLSM_OK;
}

int glsm_batch_add(glsm_batch b, glsm_fluid f, int iter0, int n_iters) {
    if (!b || !f || iter0 < 0) return fail(GLSM_ERR_ARG, "bad argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "system already in a batch");
    if (!b->sys.empty() && f->F.nsub != b->nsub) return fail(GLSM_ERR_ARG, "all systems of a batch need the same nsub");
    CK(cudaStreamSynchronize(f->c->stream));
    CK(cudaStreamSynchronize(b->stream));
    // batched launches carry no access-policy window: a joining system gives
    // up its L2 set-aside
    if (f->l2_on) {
        l2_window(f, 0);
        for (auto& row : f->graph)
            for (auto& g : row)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
    }
    if (b->sys.empty()) b->nsub = f->F.nsub;
    set_iter_kernel<<<1, 1, 0, b->stream>>>(f->c->d_ctl, iter0);
    CK(cudaGetLastError());
    f->dev_iter = -1;  // the batch advances the counter
    f->c->markers_stale = true;
    f->batch = b;
    b->sys.push_back(f);
    b->remaining.push_back(n_iters > 0 ? n_iters : -1);
    b->dirty = true;
    return GLSM_OK;
}

int glsm_batch_remove(glsm_batch b, glsm_fluid f) {
    if (!b || !f || f->batch != b) return fail(GLSM_ERR_ARG, "system is not in this batch");
    CK(cudaStreamSynchronize(b->stream));
    const size_t at = std::find(b->sys.begin(), b->sys.end(), f) - b->sys.begin();
    b->sys.erase(b->sys.begin() + at);
    b->remaining.erase(b->remaining.begin() + at);
    f->batch = nullptr;
    f->c->markers_stale = true;
    b->dirty = true;
    return GLSM_OK;
}

int glsm_batch_size(glsm_batch b) { return b ? (int)b->sys.size() : 0; }

int glsm_batch_run(glsm_batch b, int n) {
    if (!b || n < 0) return fail(GLSM_ERR_ARG, "bad argument");
    if (b->dirty) {
        int r = batch_rebuild(b);
        if (r) return r;
    }
    if (b->sys.empty() || n == 0) return GLSM_OK;
    for (glsm_fluid_s* f : b->sys) {
        glsm_coupler c = f->c;
        bool stale = c->markers_stale;
        for (glsm_gel_s* g : c->gels) stale |= g->ptr_out;
        if (stale && !c->gels.empty()) {
            CK(cudaMemsetAsync(c->d_fresh, 0, sizeof(int) * c->gels.size(), b->stream));
            c->markers_stale = false;
        }
    }
    for (int it = 0; it < n; it++) {
        CK(cudaGraphLaunch(b->graph[b->phase], b->stream));
        if (b->graph[1]) b->phase ^= 1;
    }
    for (size_t i = 0; i < b->sys.size(); i++) {
        glsm_fluid_s* f = b->sys[i];
        long long& rem = b->remaining[i];
        const long long ran = rem < 0 ? n : std::min<long long>(n, rem);
        if (rem > 0) rem -= ran;
        f->substeps += ran * f->F.nsub;
        f->cur ^= (int)(ran & 1);
    }
    return GLSM_OK;
}

long long glsm_batch_remaining(glsm_batch b, glsm_fluid f) {
    if (!b || !f || f->batch != b) return -2;
    const size_t at = std::find(b->sys.begin(), b->sys.end(), f) - b->sys.begin();
    return b->remaining[at];
}

int glsm_batch_sync(glsm_batch b) {
    if (!b) return fail(GLSM_ERR_ARG, "null batch");
    CK(cudaStreamSynchronize(b->stream));
    for (auto* f : b->sys) {
        glsm_coupler c = f->c;
        CK(cudaMemcpy(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
        if (c->h_ctl->error) {
            const int err = c->h_ctl->error;
            CK(cudaMemset(&c->d_ctl->error, 0, sizeof(int)));
            return fail(GLSM_ERR_DEVICE, "device error flags 0x%x in a batch member", err);
        }
    }
    return GLSM_OK;
}

int glsm_batch_destroy(glsm_batch b) {
    if (!b) return GLSM_OK;
    cudaStreamSynchronize(b->stream);
    for (auto* f : b->sys) f->batch = nullptr;
    batch_free_device(b);
    if (b->arena) cudaFree(b->arena);
    cudaEventDestroy(b->ev_fork);
    cudaEventDestroy(b->ev_join);
    for (auto ge : b->gevents) cudaEventDestroy(ge);
    for (auto gs : b->gstreams) cudaStreamDestroy(gs);
    cudaStreamDestroy(b->side);
    cudaStreamDestroy(b->stream);
    delete b;
    return GLSM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// exact-restart checkpoint of a coupled system
// ---------------------------------------------------------------------------
// Layout: CkptHeader, one CkptGel per gel, then the raw device bytes in this
// order: the fluid's allocation (populations in their current AA layout, u,
// IBM force, both concentration buffers, source, launch counters), the
// coupler's marker state and control block, and per gel its data arrays and
// its time-series ring.  Every region holds plain data (no device addresses),
// so a checkpoint loads into any system built with the same lattice and gels.
namespace {
constexpr char kCkptMagic[8] = {'G', 'L', 'S', 'M', 'C', 'K', '0', '1'};
struct CkptHeader {
    char magic[8];
    uint32_t n_gels, pad;
    glsm_fluid_desc desc;
    int32_t cur, pad2;
    int64_t substeps;
    uint64_t fluid_bytes, coupler_bytes;
};
// a gel's shape (checked on load) and the settings the API can change after
// creation (restored on load)
struct CkptGel {
    int32_t LX, LY, LZ, type, M, marker_off, series_cap, series_every;
    int32_t tube_mode, use_anchor, active_from, pad;
    float tube_cy, tube_cz, tube_ihy, tube_ihz;
    double anchor_z, f;
    uint64_t plain_bytes, series_doubles;
};

size_t coupler_plain_off(const glsm_coupler_s* c) { return (size_t)((char*)c->mk.lag - (char*)c->arena); }
size_t gel_plain_bytes(const glsm_gel_s* g) { return (size_t)((char*)g->d_self - (char*)g->arena); }

CkptGel gel_record(const glsm_gel_s* g) {
    const GelDev& d = g->d;
    CkptGel r{};
    r.LX = d.LX;
    r.LY = d.LY;
    r.LZ = d.LZ;
    r.type = d.type;
    r.M = d.M;
    r.marker_off = d.marker_off;
    r.series_cap = d.series_cap;
    r.series_every = d.series_every;
    r.tube_mode = d.tube_mode;
    r.use_anchor = d.use_anchor;
    r.active_from = d.active_from;
    r.tube_cy = d.tube_cy;
    r.tube_cz = d.tube_cz;
    r.tube_ihy = d.tube_ihy;
    r.tube_ihz = d.tube_ihz;
    r.anchor_z = d.anchor_z;
    r.f = d.f;
    r.plain_bytes = gel_plain_bytes(g);
    r.series_doubles = 12 * (uint64_t)d.series_cap;
    return r;
}

void apply_gel_settings(GelDev& d, const CkptGel& r) {
    d.tube_mode = r.tube_mode;
    d.tube_cy = r.tube_cy;
    d.tube_cz = r.tube_cz;
    d.tube_ihy = r.tube_ihy;
    d.tube_ihz = r.tube_ihz;
    d.use_anchor = r.use_anchor;
    d.active_from = r.active_from;
    d.anchor_z = r.anchor_z;
    d.f = r.f;
    d.series_every = r.series_every;
}

size_t ckpt_bytes(const glsm_fluid_s* f) {
    size_t n = sizeof(CkptHeader) + f->c->gels.size() * sizeof(CkptGel) + f->bytes +
               (f->c->bytes - coupler_plain_off(f->c));
    for (const glsm_gel_s* g : f->c->gels) n += gel_plain_bytes(g) + 12 * (size_t)g->d.series_cap * sizeof(double);
    return n;
}
}  // namespace

extern "C" {

int glsm_checkpoint_bytes(glsm_fluid f, size_t* bytes) {
    if (!f || !bytes) return fail(GLSM_ERR_ARG, "null argument");
    *bytes = ckpt_bytes(f);
    return GLSM_OK;
}

int glsm_checkpoint_save(glsm_fluid f, void* buf, size_t bytes) {
    if (!f || !buf) return fail(GLSM_ERR_ARG, "null argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "remove the system from its batch before a checkpoint");
    if (bytes < ckpt_bytes(f)) return fail(GLSM_ERR_ARG, "checkpoint needs %zu bytes", ckpt_bytes(f));
    glsm_coupler c = f->c;
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaStreamSynchronize(c->side));
    char* p = (char*)buf;
    CkptHeader h{};
    std::memcpy(h.magic, kCkptMagic, sizeof h.magic);
    h.n_gels = (uint32_t)c->gels.size();
    h.desc = f->desc;
    h.cur = f->cur;
    h.substeps = f->substeps;
    h.fluid_bytes = f->bytes;
    h.coupler_bytes = c->bytes - coupler_plain_off(c);
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    for (const glsm_gel_s* g : c->gels) {
        const CkptGel cg = gel_record(g);
        std::memcpy(p, &cg, sizeof cg);
        p += sizeof cg;
    }
    CK(cudaMemcpy(p, f->arena, f->bytes, cudaMemcpyDeviceToHost));
    p += f->bytes;
    CK(cudaMemcpy(p, (char*)c->arena + coupler_plain_off(c), h.coupler_bytes, cudaMemcpyDeviceToHost));
    p += h.coupler_bytes;
    for (const glsm_gel_s* g : c->gels) {
        CK(cudaMemcpy(p, g->arena, gel_plain_bytes(g), cudaMemcpyDeviceToHost));
        p += gel_plain_bytes(g);
        const size_t sb = 12 * (size_t)g->d.series_cap * sizeof(double);
        CK(cudaMemcpy(p, g->d.series, sb, cudaMemcpyDeviceToHost));
        p += sb;
    }
    return GLSM_OK;
}

int glsm_checkpoint_load(glsm_fluid f, const void* buf, size_t bytes) {
    if (!f || !buf) return fail(GLSM_ERR_ARG, "null argument");
    if (f->batch) return fail(GLSM_ERR_STATE, "remove the system from its batch before loading a checkpoint");
    glsm_coupler c = f->c;
    const char* p = (const char*)buf;
    if (bytes < sizeof(CkptHeader)) return fail(GLSM_ERR_ARG, "checkpoint truncated");
    CkptHeader h;
    std::memcpy(&h, p, sizeof h);
    p += sizeof h;
    if (std::memcmp(h.magic, kCkptMagic, sizeof h.magic) != 0) return fail(GLSM_ERR_ARG, "not a checkpoint");
    if (h.n_gels != c->gels.size()) return fail(GLSM_ERR_ARG, "checkpoint has %u gels, system %zu", h.n_gels,
                                                c->gels.size());
    if (std::memcmp(&h.desc, &f->desc, sizeof h.desc) != 0)
        return fail(GLSM_ERR_ARG, "checkpoint was written by a fluid with other parameters");
    if (h.fluid_bytes != f->bytes || h.coupler_bytes != c->bytes - coupler_plain_off(c))
        return fail(GLSM_ERR_ARG, "checkpoint layout does not match this system");
    if (bytes < ckpt_bytes(f)) return fail(GLSM_ERR_ARG, "checkpoint truncated");
    std::vector<CkptGel> cgs(h.n_gels);
    for (uint32_t i = 0; i < h.n_gels; i++) {
        std::memcpy(&cgs[i], p, sizeof(CkptGel));
        p += sizeof(CkptGel);
        const CkptGel& a = cgs[i];
        const CkptGel b = gel_record(c->gels[i]);
        if (a.LX != b.LX || a.LY != b.LY || a.LZ != b.LZ || a.type != b.type || a.M != b.M ||
            a.marker_off != b.marker_off || a.series_cap != b.series_cap || a.plain_bytes != b.plain_bytes ||
            a.series_doubles != b.series_doubles)
            return fail(GLSM_ERR_ARG, "gel %u of the checkpoint does not match this system", i);
    }
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaStreamSynchronize(c->side));
    CK(cudaMemcpy(f->arena, p, f->bytes, cudaMemcpyHostToDevice));
    p += f->bytes;
    CK(cudaMemcpy((char*)c->arena + coupler_plain_off(c), p, h.coupler_bytes, cudaMemcpyHostToDevice));
    c->markers_stale = true;
    p += h.coupler_bytes;
    for (uint32_t i = 0; i < h.n_gels; i++) {
        glsm_gel_s* g = c->gels[i];
        CK(cudaMemcpy(g->arena, p, gel_plain_bytes(g), cudaMemcpyHostToDevice));
        p += gel_plain_bytes(g);
        const size_t sb = 12 * (size_t)g->d.series_cap * sizeof(double);
        CK(cudaMemcpy(g->d.series, p, sb, cudaMemcpyHostToDevice));
        p += sb;
        apply_gel_settings(g->d, cgs[i]);
        if (int r = upload_gel_desc(g)) return r;
    }
    f->cur = h.cur;
    f->substeps = h.substeps;
    f->dev_iter = -1;  // the control block (iteration counter) came from the checkpoint
    return GLSM_OK;
}

}  // extern "C"

