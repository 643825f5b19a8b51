// dropin.cpp -- the reference's Gel / Coupler / Fluid classes (include/glsm/*.h)
// implemented over the C ABI of libglsm_b200.so, including the .dat writers and
// the text restart of the reference.
//
// Reference members followed (lasite/gLSM_fluid_3D):
//   Gel  src/gel.h:33-165, src/gel.cu:452-553 (recordData/writeFiles),
//        :221-282 (setGoonValue), :555-663 (ctor)
//   Coupler src/coupling.h:14-58, src/coupling.cu:50-80
//   Fluid src/fluid.h:24-84, src/fluid.cu:57-150 (restart, writers), :152-232 (ctor)
// The .dat files keep the reference's format exactly: "%9s" of std::to_string
// (6 decimals) joined by six spaces; vm and wm use the stream's default
// 6-significant-digit format (src/gel.cu:491-492).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/glsm/coupling.h"
#include "../../include/glsm/fluid.h"
#include "../../include/glsm/gel.h"

namespace {

// errors: reported on stderr; thrown when GLSM_THROW is set
void check(int rc, const char* what) {
    if (rc == GLSM_OK) return;
    std::string msg = std::string(what) + ": " + glsm_last_error();
    if (std::getenv("GLSM_THROW")) throw std::runtime_error(msg);
    std::fprintf(stderr, "glsm: %s\n", msg.c_str());
}

std::string fmt_fixed(double v) {  // std::setw(9) << std::to_string(v)
    char b[64], o[80];
    std::snprintf(b, sizeof(b), "%f", v);
    std::snprintf(o, sizeof(o), "%9s", b);
    return o;
}

std::string fmt_default(double v) {  // std::setw(9) << v  (precision 6, %g-like)
    std::ostringstream s;
    s << v;
    char o[80];
    std::snprintf(o, sizeof(o), "%9s", s.str().c_str());
    return o;
}

const char* kSep = "      ";

// format n lines with fn(i, out) on a pool of threads, then write them in order
template <typename Fn>
void write_lines(const std::string& path, size_t n, Fn fn) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t T = n < 20000 ? 1 : hw;
    std::vector<std::string> parts(T);
    std::vector<std::thread> pool;
    for (size_t t = 0; t < T; t++) {
        pool.emplace_back([&, t] {
            const size_t a = n * t / T, b = n * (t + 1) / T;
            std::string& out = parts[t];
            out.reserve((b - a) * 48);
            for (size_t i = a; i < b; i++) fn(i, out);
        });
    }
    for (auto& th : pool) th.join();
    std::ofstream f(path, std::ios::binary);
    for (auto& p : parts) f.write(p.data(), (std::streamsize)p.size());
}

void vec_line(const double3& v, std::string& out) {
    out += fmt_fixed(v.x);
    out += kSep;
    out += fmt_fixed(v.y);
    out += kSep;
    out += fmt_fixed(v.z);
    out += '\n';
}

void read_gel(glsm_gel h, int field, void* dst, size_t count) {
    check(glsm_gel_read(h, field, static_cast<double*>(dst), count), "read gel field");
}

// errors on a writer thread are reported, never thrown
void report(int rc, const char* what) {
    if (rc != GLSM_OK) std::fprintf(stderr, "glsm: %s: %s\n", what, glsm_last_error());
}

// the .dat files of one gel at `time` (Gel::recordData, src/gel.cu:452-541):
// node fields rn, Fn, Veln over the interior nodes and element fields rm, um,
// vm, wm over the interior elements, z slowest; the centre-element records of
// iterations in ((time - 1) df, time df] appended to gel<id>bodycenter.dat
// (columns of src/gel.cu:512-524)
void write_gel_dat(int id, int time, int df, int3 grid, const double3* rn, const double3* Fn, const double3* Veln,
                   const double3* rm, const double* um, const double* vm, const double* wm, const double* series,
                   size_t n_records) {
    const int LX = grid.x, LY = grid.y, LZ = grid.z;
    auto gi = [&](int x, int y, int z, int size) { return x + y * (LX + size) + z * (LY + size) * (LX + size); };
    const std::string sid = std::to_string(id), t = std::to_string(time);
    std::vector<int> nodes, elems;
    for (int zi = 1; zi < LZ + 1; zi++)
        for (int yi = 1; yi < LY + 1; yi++)
            for (int xi = 1; xi < LX + 1; xi++) nodes.push_back(gi(xi, yi, zi, 2));
    for (int zi = 1; zi < LZ; zi++)
        for (int yi = 1; yi < LY; yi++)
            for (int xi = 1; xi < LX; xi++) elems.push_back(gi(xi, yi, zi, 1));
    write_lines("gel" + sid + "rn" + t + ".dat", nodes.size(), [&](size_t i, std::string& o) { vec_line(rn[nodes[i]], o); });
    write_lines("gel" + sid + "Fn" + t + ".dat", nodes.size(), [&](size_t i, std::string& o) { vec_line(Fn[nodes[i]], o); });
    write_lines("gel" + sid + "Veln" + t + ".dat", nodes.size(),
                [&](size_t i, std::string& o) { vec_line(Veln[nodes[i]], o); });
    write_lines("gel" + sid + "rm" + t + ".dat", elems.size(), [&](size_t i, std::string& o) { vec_line(rm[elems[i]], o); });
    write_lines("gel" + sid + "um" + t + ".dat", elems.size(), [&](size_t i, std::string& o) {
        o += fmt_fixed(um[elems[i]]);
        o += '\n';
    });
    write_lines("gel" + sid + "vm" + t + ".dat", elems.size(), [&](size_t i, std::string& o) {
        o += fmt_default(vm[elems[i]]);
        o += '\n';
    });
    write_lines("gel" + sid + "wm" + t + ".dat", elems.size(), [&](size_t i, std::string& o) {
        o += fmt_default(wm[elems[i]]);
        o += '\n';
    });
    std::ofstream bc("gel" + sid + "bodycenter.dat", std::ios::app);
    for (size_t r = 0; r < n_records; r++) {
        const double* rec = series + 12 * r;
        if (rec[0] <= 0.0 || (int)rec[0] > time * df || (int)rec[0] <= (time - 1) * df) continue;
        std::string line = fmt_fixed(rec[0]);
        for (int k = 1; k < 12; k++) {
            line += kSep;
            line += fmt_fixed(rec[k]);
        }
        bc << line << "\n";
    }
}

// Velb<t>.dat and Conc<t>.dat (Fluid::recordData, src/fluid.cu:115-138), x fastest
void write_fluid_dat(int time, size_t N, const float* u, const float* c) {
    const std::string t = std::to_string(time);
    write_lines("Velb" + t + ".dat", N, [&](size_t i, std::string& o) {
        vec_line(make_double3(u[3 * i], u[3 * i + 1], u[3 * i + 2]), o);
    });
    write_lines("Conc" + t + ".dat", N, [&](size_t i, std::string& o) {
        o += fmt_fixed(c[i]);
        o += '\n';
    });
}

}  // namespace

// ===========================================================================
// Gel
// ===========================================================================
Gel::Gel(int3 gelSize, double3 gelPosition, int gelType, int gel_id, int time)
    : m_gelId(gel_id), m_gelType(gelType), m_gelPosition(gelPosition), m_gelSize(gelSize) {
    handle = nullptr;
    check(glsm_gel_create(gelSize.x, gelSize.y, gelSize.z, gelPosition.x, gelPosition.y, gelPosition.z, gelType,
                          gel_id, &handle),
          "Gel");
    if (!handle) throw std::runtime_error(std::string("Gel: ") + glsm_last_error());
    m_dt = 1e-3;
    m_df = int(1 / m_dt);
    m_dx = m_dy = m_dz = 1;
    int64_t info[8];
    glsm_gel_info(handle, info);
    m_gelNodeGrid = make_int3((int)info[0], (int)info[1], (int)info[2]);
    m_numGelElements = (int)info[3];
    m_numGelNodes = (int)info[4];
    m_boundaryCount = (int)info[5];
    m_gel_stream = nullptr;
    m_hgp = new GelParams;
    std::memset(m_hgp, 0, sizeof(GelParams));
    GelParams& p = *m_hgp;
    p.LX = m_gelNodeGrid.x;
    p.LY = m_gelNodeGrid.y;
    p.LZ = m_gelNodeGrid.z;
    p.f = 0.9;
    p.ep = 0.3;
    p.q = 1e-4;
    p.P1 = 0.0124;
    p.P2 = 0.77;
    p.dt = m_dt;
    p.dtx = 5 * m_dt;
    p.dx = p.dy = p.dz = 1;
    p.CH0 = 0.338;
    p.CH1 = 0.518;
    p.CHS = 0.1;
    p.C0 = 1.3e-3;
    p.c0_bis = 5e-4;
    p.b = 0.01;
    p.AZ0 = 100.0;
    p.FA0 = 0.139;
    p.maxFilamentlen = 300;
    p.gelType = gelType;
    double ss[3];
    glsm_gel_steady_state(handle, ss);
    p.uss = ss[0];
    p.vss = ss[1];
    p.wss = ss[2];
    const size_t nE = m_numGelElements, nN = m_numGelNodes;
    m_hum = new double[nE]();
    m_hvm = new double[nE]();
    m_hwm = new double[nE]();
    m_hrm = new double3[nE]();
    m_hrn = new double3[nN]();
    m_hFn = new double3[nN]();
    m_hVeln = new double3[nN]();
    m_hbIndex = new int[m_boundaryCount]();
    m_hseries = new double[12 * 1000]();
    auto dp = [&](int f) { return glsm_gel_device_ptr(handle, f); };
    m_dum = (double*)dp(GLSM_GEL_UM);
    m_dum_norm = (double*)dp(GLSM_GEL_UM_NORM);
    m_dun_norm = (double*)dp(GLSM_GEL_UN_NORM);
    m_dun_robin = (double*)dp(GLSM_GEL_UN_ROBIN);
    m_dvm = (double*)dp(GLSM_GEL_VM);
    m_dvm_norm = (double*)dp(GLSM_GEL_VM_NORM);
    m_dvn_norm = (double*)dp(GLSM_GEL_VN_NORM);
    m_dwm = (double*)dp(GLSM_GEL_WM);
    m_dwmp = (double*)dp(GLSM_GEL_WMP);
    m_dT0m = (double*)dp(GLSM_GEL_T0);
    m_dT1m = (double*)dp(GLSM_GEL_T1);
    m_dT2m = (double*)dp(GLSM_GEL_T2);
    m_drn = (double3*)dp(GLSM_GEL_RN);
    m_drm = (double3*)dp(GLSM_GEL_RM);
    m_dVeln = (double3*)dp(GLSM_GEL_VELN);
    m_dVels = (double3*)dp(GLSM_GEL_VELS);
    m_dFn = (double3*)dp(GLSM_GEL_FN);
    m_dFn_robin = (double3*)dp(GLSM_GEL_FN_ROBIN);
    m_drm_loc = (double3*)dp(GLSM_GEL_RM_LOC);
    m_dnmSm = (double3*)dp(GLSM_GEL_NMSM);
    m_dVolm = (double*)dp(GLSM_GEL_VOLM);
    m_dPrem = (double*)dp(GLSM_GEL_PREM);
    // surface node order of buildBoundaryIndex (src/gel.cu:161-177)
    int c = 0;
    const int LX = p.LX, LY = p.LY, LZ = p.LZ;
    for (int k = 1; k <= LZ; k++)
        for (int j = 1; j <= LY; j++)
            for (int i = 1; i <= LX; i++)
                if (i == 1 || i == LX || j == 1 || j == LY || k == 1 || k == LZ) m_hbIndex[c++] = idx3(i, j, k, LX + 2, LY + 2);
    if (time) setGoonValue(time);
}

Gel::~Gel() {
    if (m_file_writer_thread.joinable()) m_file_writer_thread.join();
    if (m_snap) cudaFreeHost(m_snap);
    check(glsm_gel_destroy(handle), "~Gel");
    delete[] m_hum;
    delete[] m_hvm;
    delete[] m_hwm;
    delete[] m_hrm;
    delete[] m_hrn;
    delete[] m_hFn;
    delete[] m_hVeln;
    delete[] m_hbIndex;
    delete[] m_hseries;
    delete m_hgp;
}

int Gel::get_index(int xi, int yi, int zi, int size) {
    return xi + yi * (m_gelNodeGrid.x + size) + zi * (m_gelNodeGrid.y + size) * (m_gelNodeGrid.x + size);
}

int Gel::idx3(int x, int y, int z, int Nx, int Ny) { return x + y * Nx + z * Nx * Ny; }

void Gel::stepElasticity(int iter) { check(glsm_gel_step_elasticity(handle, iter), "stepElasticity"); }
void Gel::stepChemistry(int iter) { check(glsm_gel_step_chemistry(handle, iter), "stepChemistry"); }
void Gel::recordCenter(int iter) { check(glsm_gel_record_center(handle, iter), "recordCenter"); }

void Gel::resetToQuiescent() {
    check(glsm_gel_reset_quiescent(handle), "resetToQuiescent");
    read_gel(handle, GLSM_GEL_UM, m_hum, m_numGelElements);
    read_gel(handle, GLSM_GEL_VM, m_hvm, m_numGelElements);
    read_gel(handle, GLSM_GEL_WM, m_hwm, m_numGelElements);
}

void Gel::fireExcitationPulse() { check(glsm_gel_fire_pulse(handle), "fireExcitationPulse"); }

void Gel::setAnchorZ(double anchor_z) {
    m_anchor_z = anchor_z;
    m_use_anchor = true;
    check(glsm_gel_set_anchor_z(handle, anchor_z), "setAnchorZ");
}

void Gel::buildTubeMask(int wall_thickness, bool circular) {
    check(glsm_gel_build_tube_mask(handle, wall_thickness, circular ? 1 : 0), "buildTubeMask");
    m_hgp->tube_mode = circular ? 2 : 1;
}

void Gel::copyDataToHost() {
    read_gel(handle, GLSM_GEL_UM, m_hum, m_numGelElements);
    read_gel(handle, GLSM_GEL_VM, m_hvm, m_numGelElements);
    read_gel(handle, GLSM_GEL_WM, m_hwm, m_numGelElements);
    read_gel(handle, GLSM_GEL_RM, m_hrm, 3 * (size_t)m_numGelElements);
    read_gel(handle, GLSM_GEL_RN, m_hrn, 3 * (size_t)m_numGelNodes);
    read_gel(handle, GLSM_GEL_FN, m_hFn, 3 * (size_t)m_numGelNodes);
    read_gel(handle, GLSM_GEL_VELN, m_hVeln, 3 * (size_t)m_numGelNodes);
    check(glsm_gel_series_read(handle, m_hseries, 12 * 1000), "series");
}

void Gel::copyDataToDevice() {
    check(glsm_gel_write(handle, GLSM_GEL_UM, m_hum, m_numGelElements), "write um");
    check(glsm_gel_write(handle, GLSM_GEL_VM, m_hvm, m_numGelElements), "write vm");
    check(glsm_gel_write(handle, GLSM_GEL_WM, m_hwm, m_numGelElements), "write wm");
    check(glsm_gel_write(handle, GLSM_GEL_RN, (double*)m_hrn, 3 * (size_t)m_numGelNodes), "write rn");
}

// Gel::recordData, src/gel.cu:452-541: the .dat files of the host mirrors
// (filled by copyDataToHost)
void Gel::recordData(int time) {
    write_gel_dat(m_gelId, time, m_df, m_gelNodeGrid, m_hrn, m_hFn, m_hVeln, m_hrm, m_hum, m_hvm, m_hwm, m_hseries,
                  1000);
}

// Gel::writeFiles, src/gel.cu:543-553.  Where the reference copies the fields
// to the host synchronously (waiting for every queued kernel) and formats them
// on a writer thread, this takes an output snapshot -- a device-side copy
// behind the queued work, then a transfer on a copy stream into page-locked
// staging -- and returns at once; the writer thread waits for the transfer and
// formats the staging.  The host mirrors are left as they are.
void Gel::writeFiles(int iter) {
    const double time = iter * m_dt;
    if (iter % 1000 == 0) {
        if (m_file_writer_thread.joinable()) m_file_writer_thread.join();
        const size_t nN3 = 3 * (size_t)m_numGelNodes, nE = m_numGelElements;
        const size_t ns = glsm_gel_field_size(handle, GLSM_GEL_SERIES);
        const size_t need = 3 * nN3 + 3 * nE + 3 * nE + ns;
        if (need > m_snap_doubles) {
            if (m_snap) cudaFreeHost(m_snap);
            m_snap = nullptr;
            m_snap_doubles = 0;
            if (cudaMallocHost(&m_snap, need * sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                check(GLSM_ERR_NOMEM, "writeFiles: page-locked staging");
                return;
            }
            m_snap_doubles = need;
        }
        double* const dst[8] = {m_snap, m_snap + nN3, m_snap + 2 * nN3, m_snap + 3 * nN3, m_snap + 3 * nN3 + 3 * nE,
                                m_snap + 3 * nN3 + 4 * nE, m_snap + 3 * nN3 + 5 * nE, m_snap + 3 * nN3 + 6 * nE};
        const int fields[8] = {GLSM_GEL_RN, GLSM_GEL_FN, GLSM_GEL_VELN, GLSM_GEL_RM,
                               GLSM_GEL_UM, GLSM_GEL_VM, GLSM_GEL_WM, GLSM_GEL_SERIES};
        check(glsm_gel_snapshot(handle, 8, fields, dst), "writeFiles: snapshot");
        m_file_writer_thread = std::thread(&Gel::writeSnapshot, this, int(time));
    }
}

// writer thread of writeFiles: waits for the snapshot, formats the staging
void Gel::writeSnapshot(int time) {
    report(glsm_gel_snapshot_wait(handle), "writeFiles: snapshot");
    const size_t nN3 = 3 * (size_t)m_numGelNodes, nE = m_numGelElements;
    const double* p = m_snap;
    write_gel_dat(m_gelId, time, m_df, m_gelNodeGrid, reinterpret_cast<const double3*>(p),
                  reinterpret_cast<const double3*>(p + nN3), reinterpret_cast<const double3*>(p + 2 * nN3),
                  reinterpret_cast<const double3*>(p + 3 * nN3), p + 3 * nN3 + 3 * nE, p + 3 * nN3 + 4 * nE,
                  p + 3 * nN3 + 5 * nE, p + 3 * nN3 + 6 * nE, (m_snap_doubles - 3 * nN3 - 6 * nE) / 12);
}

// Gel::setGoonValue, src/gel.cu:221-282: restart from gel<id>{rn,um,vm,wm}<time>.dat
void Gel::setGoonValue(int time) {
    const int LX = m_gelNodeGrid.x, LY = m_gelNodeGrid.y, LZ = m_gelNodeGrid.z;
    const std::string id = std::to_string(m_gelId), t = std::to_string(time);
    read_gel(handle, GLSM_GEL_UM, m_hum, m_numGelElements);
    read_gel(handle, GLSM_GEL_VM, m_hvm, m_numGelElements);
    read_gel(handle, GLSM_GEL_WM, m_hwm, m_numGelElements);
    read_gel(handle, GLSM_GEL_RN, m_hrn, 3 * (size_t)m_numGelNodes);
    std::ifstream fu("gel" + id + "um" + t + ".dat"), fv("gel" + id + "vm" + t + ".dat"),
        fw("gel" + id + "wm" + t + ".dat"), fr("gel" + id + "rn" + t + ".dat");
    if (!fu || !fv || !fw || !fr) {
        check(GLSM_ERR_ARG, ("restart files gel" + id + "*" + t + ".dat not found").c_str());
        return;
    }
    for (int zi = 1; zi < LZ; zi++)
        for (int yi = 1; yi < LY; yi++)
            for (int xi = 1; xi < LX; xi++) {
                const int gi = get_index(xi, yi, zi, 1);
                fu >> m_hum[gi];
                fv >> m_hvm[gi];
                fw >> m_hwm[gi];
            }
    for (int zi = 1; zi < LZ + 1; zi++)
        for (int yi = 1; yi < LY + 1; yi++)
            for (int xi = 1; xi < LX + 1; xi++) {
                double3& r = m_hrn[get_index(xi, yi, zi, 2)];
                fr >> r.x >> r.y >> r.z;
            }
    copyDataToDevice();
}

// ===========================================================================
// Coupler
// ===========================================================================
Coupler::Coupler(std::vector<Gel*>& gels_) : gels(gels_) {
    numGels = (int)gels.size();
    std::vector<glsm_gel> hs;
    sumGelBoundaryCount = 0;
    for (auto* g : gels) {
        h_offsets.push_back(sumGelBoundaryCount);
        h_gelBoundaryCount.push_back(g->m_boundaryCount);
        for (int l = 0; l < g->m_boundaryCount; l++) h_owner.push_back((int)hs.size());
        sumGelBoundaryCount += g->m_boundaryCount;
        hs.push_back(g->handle);
    }
    handle = nullptr;
    check(glsm_coupler_create(hs.data(), numGels, &handle), "Coupler");
    if (!handle) throw std::runtime_error(std::string("Coupler: ") + glsm_last_error());
    threads = 256;
    blocksM = (sumGelBoundaryCount + threads - 1) / threads;
    h_cp = new CouplerParams;
    h_cp->M = sumGelBoundaryCount;
    h_cp->delta = 1e-4f;
    h_cp->gamma = 1.5f;
    h_cp->gel_to_lbm_vel = 1.0f;
    h_cp->lbm_to_gel_vel = 1.0f;
    coupler_stream = (cudaStream_t)glsm_coupler_stream(handle);
    for (auto* g : gels) g->m_gel_stream = coupler_stream;
}

Coupler::~Coupler() {
    check(glsm_coupler_destroy(handle), "~Coupler");
    delete h_cp;
}

void Coupler::packFromGels() { check(glsm_coupler_pack(handle), "packFromGels"); }
void Coupler::scatterToGels() { check(glsm_coupler_scatter(handle), "scatterToGels"); }
void Coupler::applyGelRepulsion() { check(glsm_coupler_repulsion(handle), "applyGelRepulsion"); }

// ===========================================================================
// Fluid
// ===========================================================================
Fluid::Fluid(int3 fluidSize_, int time, Coupler* coupler_) : coupler(coupler_), fluidSize(fluidSize_) {
    h = 0.5f;
    // 2*s + 1 cells per axis (src/fluid.cu:169-171)
    const int3 dims = make_int3(int(fluidSize.x / h) + 1, int(fluidSize.y / h) + 1, int(fluidSize.z / h) + 1);
    init(dims, 0, GLSM_STORE_F32, time);
}

Fluid::Fluid(int3 latticeDims, int nsub, int storage, Coupler* coupler_) : coupler(coupler_) {
    h = 0.5f;
    fluidSize = make_int3((latticeDims.x - 1) / 2, (latticeDims.y - 1) / 2, (latticeDims.z - 1) / 2);
    init(latticeDims, nsub, storage, 0);
}

void Fluid::init(int3 dims, int nsub, int storage, int time) {
    dt = 1e-3f;
    df = int(1 / dt);
    fluidNodeGrid = dims;
    N = dims.x * dims.y * dims.z;
    Nd = 19 * N;
    glsm_fluid_desc d;
    glsm_fluid_desc_default(&d, dims.x, dims.y, dims.z);
    if (nsub > 0) d.nsub = nsub;
    d.storage = storage;
    handle = nullptr;
    check(glsm_fluid_create(&d, coupler->handle, &handle), "Fluid");
    if (!handle) throw std::runtime_error(std::string("Fluid: ") + glsm_last_error());
    Nsub = d.nsub;
    niu = 1e-6f;
    dx_fluid = 40e-6f * h;
    dt_fluid = (d.tau - 0.5f) * dx_fluid * dx_fluid / (3 * niu);
    h_fp = new FluidParams;
    std::memset(h_fp, 0, sizeof(FluidParams));
    static const int c[19][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                                 {1, 1, 0},  {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}, {1, 0, 1},  {-1, 0, 1}, {-1, 0, -1},
                                 {1, 0, -1}, {0, 1, 1},  {0, 1, -1}, {0, -1, -1}, {0, -1, 1}};
    static const int opp[19] = {0, 2, 1, 4, 3, 6, 5, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16};
    for (int q = 0; q < 19; q++) {
        h_fp->c[q] = make_int3(c[q][0], c[q][1], c[q][2]);
        h_fp->w[q] = q == 0 ? 1.f / 3.f : (q <= 6 ? 1.f / 18.f : 1.f / 36.f);
        h_fp->opp[q] = opp[q];
    }
    h_fp->tau = d.tau;
    h_fp->cs2 = 1.f / 3.f;
    h_fp->nu = h_fp->cs2 * (h_fp->tau - 0.5f);
    h_fp->F_const = make_float3(d.force[0], d.force[1], d.force[2]);
    h_fp->beta = d.beta;
    h_fp->N = N;
    h_fp->M = coupler->sumGelBoundaryCount;
    h_fp->L = dims;
    h_fp->h = h;
    h_fp->dx = h_fp->dy = h_fp->dz = 1;
    h_fp->dt = dt;
    h_fp->D = 1;
    float units[2];
    glsm_fluid_units(handle, units);
    coupler->h_cp->gel_to_lbm_vel = units[0];
    coupler->h_cp->lbm_to_gel_vel = units[1];
    for (auto* g : coupler->gels) g->m_hgp->lbm_to_gel_vel = units[1];
    fluid_stream = coupler->coupler_stream;
    h_u = new float3[N]();
    h_c1 = new float[N]();
    if (time) setGoonValue(time);
}

Fluid::~Fluid() {
    if (file_writer_thread.joinable()) file_writer_thread.join();
    if (m_snap_u) cudaFreeHost(m_snap_u);
    check(glsm_fluid_destroy(handle), "~Fluid");
    delete[] h_u;
    delete[] h_c1;
    delete h_fp;
}

int Fluid::idx3(int x, int y, int z, int Nx, int Ny) { return x + y * Nx + z * Nx * Ny; }

void Fluid::stepVelocity(int iter) { check(glsm_fluid_step_velocity(handle, iter), "stepVelocity"); }
void Fluid::stepConcentration(int iter) { check(glsm_fluid_step_concentration(handle, iter), "stepConcentration"); }
void Fluid::run(int iter0, int n) { check(glsm_fluid_run(handle, iter0, n), "run"); }

void Fluid::copyDataToHost() {
    check(glsm_fluid_read(handle, GLSM_FLUID_U, reinterpret_cast<float*>(h_u), 3 * (size_t)N), "read u");
    check(glsm_fluid_read(handle, GLSM_FLUID_C1, h_c1, (size_t)N), "read c1");
}

// Fluid::recordData, src/fluid.cu:115-138: the .dat files of the host mirrors
// (filled by copyDataToHost)
void Fluid::recordData(int time) { write_fluid_dat(time, (size_t)N, reinterpret_cast<const float*>(h_u), h_c1); }

// Fluid::writeFiles, src/fluid.cu:140-150, with an output snapshot as in
// Gel::writeFiles: returns without waiting for the queued iterations; the
// writer thread waits for the transfer and formats the staging
void Fluid::writeFiles(int iter) {
    const double time = iter * dt;
    if (iter % 2000 == 0) {
        if (file_writer_thread.joinable()) file_writer_thread.join();
        if (!m_snap_u) {
            if (cudaMallocHost(&m_snap_u, 4 * sizeof(float) * (size_t)N) != cudaSuccess) {
                cudaGetLastError();
                m_snap_u = nullptr;
                check(GLSM_ERR_NOMEM, "writeFiles: page-locked staging");
                return;
            }
            m_snap_c = m_snap_u + 3 * (size_t)N;
        }
        check(glsm_fluid_snapshot(handle, m_snap_u, m_snap_c), "writeFiles: snapshot");
        file_writer_thread = std::thread(&Fluid::writeSnapshot, this, int(time));
    }
}

// writer thread of writeFiles: waits for the snapshot, formats the staging
void Fluid::writeSnapshot(int time) {
    report(glsm_fluid_snapshot_wait(handle), "writeFiles: snapshot");
    write_fluid_dat(time, (size_t)N, m_snap_u, m_snap_c);
}

// Fluid::setGoonValue, src/fluid.cu:57-83: u and c1 from Velb<t>.dat / Conc<t>.dat,
// populations at rest
void Fluid::setGoonValue(int time) {
    const std::string t = std::to_string(time);
    std::ifstream fv("Velb" + t + ".dat"), fc("Conc" + t + ".dat");
    if (!fv || !fc) {
        check(GLSM_ERR_ARG, ("restart files Velb/Conc" + t + ".dat not found").c_str());
        return;
    }
    for (int i = 0; i < N; i++) {
        fv >> h_u[i].x >> h_u[i].y >> h_u[i].z;
        fc >> h_c1[i];
    }
    check(glsm_fluid_write(handle, GLSM_FLUID_U, reinterpret_cast<float*>(h_u), 3 * (size_t)N), "write u");
    check(glsm_fluid_write(handle, GLSM_FLUID_C1, h_c1, (size_t)N), "write c1");
}
