// glsm_oracle.cpp -- CPU restatement of the gLSM_fluid_3D coupled step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
// (glsm_fluid_3d_b200) is compared against.  Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline / reference legs load it.  The product never links,
// imports or falls back to it.
//
// It restates, loop by loop, the reference kernels and host code of
// lasite/gLSM_fluid_3D (paths relative to that project):
//   fluid:   src/fluid_kernels.cu:60-459, src/fluid.cu:152-284
//   gel:     src/gel_kernels.cu:95-880, src/gel.cu:161-344, :424-450, :555-713
//   coupler: src/coupling_kernels.cu:8-146, src/coupling.cu:50-123
//   driver:  src/sim.cpp:60-112 (per-iteration call order)
// Differences from the reference that are deliberate:
//   * the fluid real type R is a template parameter: double (the FP64 oracle) or
//     float (a "reference-like" FP32 mode used to size tolerances);
//   * spreads are sequential in marker order (deterministic; the reference uses
//     float atomics);
//   * every call runs in program order (the reference uses unsynchronised streams);
//   * the lattice dims and Nsub are set directly (the reference derives them).
// The gel is always FP64, as in the reference.
//
// Build:  g++ -O3 -fopenmp -shared -fPIC glsm_oracle.cpp -o _build/libglsm_oracle.so
// C API at the bottom (orc_*), used through ctypes.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "orc_noise.h"

namespace orc {

struct V3 {
    double x, y, z;
};
static inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
static inline V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 hadamard(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 hdiv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
// cross() in the component order of src/gel_kernels.cu:80-83
static inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - b.y * a.z, b.x * a.z - a.x * b.z, a.x * b.y - b.x * a.y);
}

// seeded noise: see orc_noise.h
static inline double noise_pm1(uint64_t seed, uint64_t gel_id, uint64_t slot, uint64_t field) {
    return orc_noise_pm1(seed, gel_id, slot, field);
}

// ---------------------------------------------------------------------------
// Gel (FP64), src/gel.h:5-165, src/gel.cu, src/gel_kernels.cu
// ---------------------------------------------------------------------------
struct Gel {
    // geometry
    int LX = 0, LY = 0, LZ = 0;  // nodes per axis (gelSize + 1), gel.cu:605-607
    int nE = 0, nN = 0, M = 0;   // element slots, node slots, boundary markers
    int id = 0, type = 1;
    double px = 0, py = 0, pz = 0;
    // GelParams, gel.cu:628-661
    double f = 0.9, q = 1e-4, ep = 0.3, P1 = 0.0124, P2 = 0.77;
    double dt = 1e-3, dtx = 5e-3, dx = 1, dy = 1, dz = 1;
    double CH0 = 0.338, CH1 = 0.518, CHS = 0.1, C0 = 1.3e-3, AZ0 = 100.0, FA0 = 0.139;
    double c0_bis = 5e-4, b = 0.01;
    double uss = 0, vss = 0, wss = 0;
    int rn_offset[27][3];
    // tube mask (gel.h:26-30), anchor (gel.h:163-164)
    int tube_mode = 0;
    float tube_cy = 0, tube_cz = 0, tube_ihy = 0, tube_ihz = 0;
    bool use_anchor = false;
    double anchor_z = 0;
    // activity control used by the scenario drivers (sim_array.cpp:93-103)
    int active_from = 0;
    // fields
    std::vector<double> um, vm, wm, wmp, um_norm, vm_norm, T0, T1, T2, Volm, Prem;
    std::vector<V3> rm, rm_loc, nmSm;
    std::vector<V3> rn, Veln, Vels, Fn, Fn_robin, Fdrag_robin;
    std::vector<double> un_norm, un_robin, vn_norm;
    std::vector<int> map_node, map_element, bIndex;

    // get_index(...,1) and get_index(...,2), gel_kernels.cu:95-98
    int E(int x, int y, int z) const { return x + y * (LX + 1) + z * (LY + 1) * (LX + 1); }
    int Nd(int x, int y, int z) const { return x + y * (LX + 2) + z * (LY + 2) * (LX + 2); }
    int idx_size(int x, int y, int z, int size) const {
        return x + y * (LX + size) + z * (LY + size) * (LX + size);
    }

    // Gel::fu_h, gel.cu:445-450
    double fu_h(double u, double v, double w, double phi) const {
        double ww = (1.0 - w) * (1.0 - w);
        return ww * u - u * u - (1.0 - w) * (f * v + phi) * (u - q * ww) / (u + q * ww);
    }
    // Gel::steadyStateValue, gel.cu:424-443 (bisection on v with w = FA0)
    void steady_state(double& u, double& v, double& w, double phi) const {
        w = FA0;
        double vsa = 1.0, vsb = 0.0;
        while (std::fabs(vsa - vsb) > 1e-10) {
            double vsm = 0.5 * (vsa + vsb);
            double usm = vsm / (1 - w);
            double usa = vsa / (1 - w);
            if (fu_h(usm, vsm, w, phi) * fu_h(usa, vsa, w, phi) < 0)
                vsb = vsm;
            else
                vsa = vsm;
        }
        u = vsb / (1.0 - w);
        v = vsb;
    }

    // Gel::setType, gel.cu:284-344
    void set_type(std::vector<int>& a, int size) {
        int X = LX + size - 1, Y = LY + size - 1, Z = LZ + size - 1;
        for (int xi = 1; xi < X; xi++)
            for (int yi = 1; yi < Y; yi++)
                for (int zi = 1; zi < Z; zi++) a[idx_size(xi, yi, zi, size)] = 0;
        for (int yi = 1; yi < Y; yi++)
            for (int zi = 1; zi < Z; zi++) {
                a[idx_size(0, yi, zi, size)] = 1;
                a[idx_size(X, yi, zi, size)] = 2;
            }
        for (int xi = 1; xi < X; xi++)
            for (int zi = 1; zi < Z; zi++) {
                a[idx_size(xi, 0, zi, size)] = 3;
                a[idx_size(xi, Y, zi, size)] = 4;
            }
        for (int xi = 1; xi < X; xi++)
            for (int yi = 1; yi < Y; yi++) {
                a[idx_size(xi, yi, 0, size)] = 5;
                a[idx_size(xi, yi, Z, size)] = 6;
            }
        for (int xi = 1; xi < X; xi++) {
            a[idx_size(xi, 0, 0, size)] = 7;
            a[idx_size(xi, 0, Z, size)] = 8;
            a[idx_size(xi, Y, 0, size)] = 9;
            a[idx_size(xi, Y, Z, size)] = 10;
        }
        for (int yi = 1; yi < Y; yi++) {
            a[idx_size(0, yi, 0, size)] = 11;
            a[idx_size(0, yi, Z, size)] = 12;
            a[idx_size(X, yi, 0, size)] = 13;
            a[idx_size(X, yi, Z, size)] = 14;
        }
        for (int zi = 1; zi < Z; zi++) {
            a[idx_size(0, 0, zi, size)] = 15;
            a[idx_size(0, Y, zi, size)] = 16;
            a[idx_size(X, 0, zi, size)] = 17;
            a[idx_size(X, Y, zi, size)] = 18;
        }
        a[idx_size(0, 0, 0, size)] = 19;
        a[idx_size(0, 0, Z, size)] = 20;
        a[idx_size(0, Y, 0, size)] = 21;
        a[idx_size(0, Y, Z, size)] = 22;
        a[idx_size(X, 0, 0, size)] = 23;
        a[idx_size(X, 0, Z, size)] = 24;
        a[idx_size(X, Y, 0, size)] = 25;
        a[idx_size(X, Y, Z, size)] = 26;
    }

    // Gel ctor + setInitValue + buildBoundaryIndex, gel.cu:555-663, :179-219, :161-177
    void init(int sx, int sy, int sz, double x, double y, double z, int gtype, int gid) {
        LX = sx + 1;
        LY = sy + 1;
        LZ = sz + 1;
        nE = (LX + 1) * (LY + 1) * (LZ + 1);
        nN = (LX + 2) * (LY + 2) * (LZ + 2);
        M = LX * LY * LZ - (LX - 2) * (LY - 2) * (LZ - 2);
        px = x;
        py = y;
        pz = z;
        type = gtype;
        id = gid;
        steady_state(uss, vss, wss, 0);
        static const int off[27][3] = {
            {0, 0, 0},   {1, 0, 0},   {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},  {0, 0, 1},   {0, 0, -1},
            {0, 1, 1},   {0, 1, -1},  {0, -1, 1},  {0, -1, -1}, {1, 0, 1},   {1, 0, -1},  {-1, 0, 1},
            {-1, 0, -1}, {1, 1, 0},   {1, -1, 0},  {-1, 1, 0},  {-1, -1, 0}, {1, 1, 1},   {1, 1, -1},
            {1, -1, 1},  {1, -1, -1}, {-1, 1, 1},  {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
        std::memcpy(rn_offset, off, sizeof(off));
        auto zd = [](std::vector<double>& v, int n) { v.assign(n, 0.0); };
        auto z3 = [](std::vector<V3>& v, int n) { v.assign(n, V3{0, 0, 0}); };
        for (auto* v : {&um, &vm, &wm, &wmp, &um_norm, &vm_norm, &T0, &T1, &T2, &Volm, &Prem}) zd(*v, nE);
        z3(rm, nE);
        z3(rm_loc, 8 * nE);
        z3(nmSm, 6 * nE);
        for (auto* v : {&rn, &Veln, &Vels, &Fn, &Fn_robin, &Fdrag_robin}) z3(*v, nN);
        for (auto* v : {&un_norm, &un_robin, &vn_norm}) zd(*v, nN);
        map_node.assign(nN, 0);
        map_element.assign(nE, 0);
        bIndex.assign(M, 0);
        // chemistry: interior elements get the steady state
        for (int zi = 1; zi < LZ; zi++)
            for (int yi = 1; yi < LY; yi++)
                for (int xi = 1; xi < LX; xi++) {
                    int gi = E(xi, yi, zi);
                    um[gi] = uss;
                    vm[gi] = vss;
                    wm[gi] = wss;
                }
        // node lattice scaled by lam (all (LX+2)^3 slots)
        double lam = std::pow(FA0 / wss, 1 / 3.0);
        for (int zi = 0; zi < LZ + 2; zi++)
            for (int yi = 0; yi < LY + 2; yi++)
                for (int xi = 0; xi < LX + 2; xi++) {
                    int hi = Nd(xi, yi, zi);
                    rn[hi].x = px + (2 * double(xi) - double(LX) - 1) * dx * lam / 2;
                    rn[hi].y = py + (2 * double(yi) - double(LY) - 1) * dy * lam / 2;
                    rn[hi].z = pz + (2 * double(zi) - double(LZ) - 1) * dz * lam / 2;
                }
        set_type(map_node, 2);
        set_type(map_element, 1);
        int count = 0;
        for (int k = 1; k < LZ + 1; ++k)
            for (int j = 1; j < LY + 1; ++j)
                for (int i = 1; i < LX + 1; ++i)
                    if (i == 1 || i == LX || j == 1 || j == LY || k == 1 || k == LZ)
                        bIndex[count++] = i + j * (LX + 2) + k * (LX + 2) * (LY + 2);
    }

    // Gel::buildTubeMask, gel.cu:811-867: tube axis along x at the element
    // centre, inner half-extents = half the node extent minus the wall; void
    // elements (the tube's lumen) restart at the steady state.  Float
    // arithmetic as in the reference.
    void build_tube_mask(int wall, bool circular) {
        float cy = (LY + 1) * 0.5f, cz = (LZ + 1) * 0.5f;
        float ihy = (LY * 0.5f) - wall, ihz = (LZ * 0.5f) - wall;
        if (ihy <= 0) ihy = 0;
        if (ihz <= 0) ihz = 0;
        tube_mode = circular ? 2 : 1;
        tube_cy = cy;
        tube_cz = cz;
        tube_ihy = ihy;
        tube_ihz = ihz;
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++) {
                float dyv = (float)yi - cy, dzv = (float)zi - cz;
                bool v;
                if (circular) {
                    float r2 = dyv * dyv / (ihy * ihy + 1e-6f) + dzv * dzv / (ihz * ihz + 1e-6f);
                    v = (ihy > 0 && ihz > 0 && r2 < 1.0f);
                } else {
                    v = (std::fabs(dyv) < ihy && std::fabs(dzv) < ihz);
                }
                if (!v) continue;
                for (int xi = 1; xi <= LX; xi++) {
                    int gi = E(xi, yi, zi);
                    um[gi] = uss;
                    vm[gi] = vss;
                    wm[gi] = wss;
                }
            }
    }

    void add_noise(uint64_t seed, double amp) {
        for (int zi = 1; zi < LZ; zi++)
            for (int yi = 1; yi < LY; yi++)
                for (int xi = 1; xi < LX; xi++) {
                    int gi = E(xi, yi, zi);
                    um[gi] += amp * noise_pm1(seed, (uint64_t)id, (uint64_t)gi, 0);
                    vm[gi] += amp * noise_pm1(seed, (uint64_t)id, (uint64_t)gi, 1);
                }
    }

    // Gel::resetToQuiescent, gel.cu:731-747
    void reset_quiescent() {
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++)
                for (int xi = 1; xi <= LX; xi++) {
                    int gi = E(xi, yi, zi);
                    um[gi] = uss * 0.01;
                    vm[gi] = vss * 0.01;
                    wm[gi] = wss;
                }
    }
    // isVoidElement, gel_kernels.cu:104-117 (float arithmetic kept)
    bool is_void(int yi, int zi) const {
        if (tube_mode == 0) return false;
        float dyv = (float)yi - tube_cy, dzv = (float)zi - tube_cz;
        if (tube_mode == 1) return (std::fabs(dyv) < tube_ihy && std::fabs(dzv) < tube_ihz);
        float rhy = tube_ihy, rhz = tube_ihz;
        if (rhy < 0.5f || rhz < 0.5f) return false;
        float r2 = (dyv * dyv) / (rhy * rhy) + (dzv * dzv) / (rhz * rhz);
        return r2 < 1.0f;
    }
    // Gel::fireExcitationPulse, gel.cu:751-783
    void fire_pulse() {
        int pulse_width = std::max(1, LX / 10);
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++) {
                bool v = false;
                float cy = tube_cy, cz = tube_cz;
                float dyv = (float)yi - cy, dzv = (float)zi - cz;
                if (tube_mode == 1) {
                    v = (std::fabs(dyv) < tube_ihy && std::fabs(dzv) < tube_ihz);
                } else if (tube_mode == 2) {
                    float rhy = tube_ihy, rhz = tube_ihz;
                    if (rhy >= 0.5f && rhz >= 0.5f) v = ((dyv * dyv) / (rhy * rhy) + (dzv * dzv) / (rhz * rhz) < 1.0f);
                }
                if (v) continue;
                for (int xi = 1; xi <= pulse_width; xi++) {
                    int gi = E(xi, yi, zi);
                    um[gi] = uss * 3.0;
                    vm[gi] = vss * 0.1;
                }
            }
    }

    // ---- kernels -----------------------------------------------------------
    // calServiceNodesPositionD, gel_kernels.cu:615-631
    void service_nodes() {
        for (int zi = 0; zi <= LZ + 1; zi++)
            for (int yi = 0; yi <= LY + 1; yi++)
                for (int xi = 0; xi <= LX + 1; xi++) {
                    int gi = Nd(xi, yi, zi);
                    int t = map_node[gi];
                    if (t == 0) continue;
                    const int* o = rn_offset[t];
                    int g1 = Nd(xi + o[0], yi + o[1], zi + o[2]);
                    int g2 = Nd(xi + 2 * o[0], yi + 2 * o[1], zi + 2 * o[2]);
                    rn[gi] = 2 * rn[g1] - rn[g2];
                }
    }

    // calElementPropertiesD, gel_kernels.cu:216-483 (the `if (true)` branch)
    // face f: the 4 corner nodes in the order of coordinate_st, the fixed natural
    // coordinate value of the face, which two natural coordinates vary (a, b) and
    // the sign applied to the summed cross product.
    void element_properties() {
        // corner index = i*4 + j*2 + k for node (xi+i, yi+j, zi+k)
        // natural coordinates: s <-> x (i), n <-> y (j), t <-> z (k)
        for (int zi = 0; zi <= LZ; zi++)
            for (int yi = 0; yi <= LY; yi++)
                for (int xi = 0; xi <= LX; xi++) {
                    int gi = E(xi, yi, zi);
                    V3 node[8];
                    V3 bc = v3(0, 0, 0);
                    int c = 0;
                    for (int i = 0; i < 2; i++)
                        for (int j = 0; j < 2; j++)
                            for (int k = 0; k < 2; k++) {
                                node[c] = rn[Nd(xi + i, yi + j, zi + k)];
                                bc = bc + node[c];
                                c++;
                            }
                    bc = bc / 8;
                    rm[gi] = bc;
                    for (int i = 0; i < 8; i++) {
                        node[i] = node[i] - bc;
                        rm_loc[8 * gi + i] = node[i];
                    }
                    // 2x2 evaluation points at +-0.5 with unit weight, k_s = 4/point^2 = 1
                    const double pts[2] = {-0.5, 0.5};
                    // Each face: corner nodes (coordinate_st order), sign.  The
                    // derivative of the corner shape functions along the two in-face
                    // coordinates (a, b) at (a, b) is ds(corner)*(1 + db*b)/4 for the
                    // first and db(corner)*(1 + da*a)/4 for the second, where (da, db)
                    // are the corner's +-1 natural coordinates in the face.
                    struct Face {
                        int c[4];
                        double sign;
                        int ax;  // which 3D axes play the roles of (a, b): 0 -> (n,t), 1 -> (s,t), 2 -> (s,n)
                    };
                    static const Face faces[6] = {
                        {{0, 1, 3, 2}, -1.0, 0}, {{4, 6, 7, 5}, +1.0, 0}, {{0, 4, 5, 1}, +1.0, 1},
                        {{2, 3, 7, 6}, -1.0, 1}, {{0, 2, 6, 4}, -1.0, 2}, {{1, 5, 7, 3}, +1.0, 2}};
                    for (int fidx = 0; fidx < 6; fidx++) {
                        const Face& F = faces[fidx];
                        V3 acc = v3(0, 0, 0);
                        for (int ia = 0; ia < 2; ia++)
                            for (int ib = 0; ib < 2; ib++) {
                                double a = pts[ia], bq = pts[ib];
                                V3 Ja = v3(0, 0, 0), Jb = v3(0, 0, 0);
                                for (int m = 0; m < 4; m++) {
                                    int cn = F.c[m];
                                    int ci = (cn >> 2) & 1, cj = (cn >> 1) & 1, ck = cn & 1;
                                    double nat[3] = {2.0 * ci - 1, 2.0 * cj - 1, 2.0 * ck - 1};
                                    // the fixed coordinate of this face
                                    int fixed = (F.ax == 0) ? 0 : (F.ax == 1 ? 1 : 2);
                                    int ra = (F.ax == 0) ? 1 : 0;
                                    int rb = (F.ax == 2) ? 1 : 2;
                                    double sf = nat[fixed];
                                    // 3D shape function derivative restricted to the face:
                                    // N = (1+s s_c)(1+n n_c)(1+t t_c)/8 at the fixed coordinate = s_c
                                    double fac = (1 + sf * sf) / 8;  // (1 +- fixed)^... = 2/8
                                    double dNa = nat[ra] * (1 + nat[rb] * bq) * fac;
                                    double dNb = nat[rb] * (1 + nat[ra] * a) * fac;
                                    Ja = Ja + node[cn] * dNa;
                                    Jb = Jb + node[cn] * dNb;
                                }
                                acc = acc + cross(Ja, Jb);
                            }
                        nmSm[6 * gi + fidx] = F.sign * acc;
                    }
                    // volume: 2x2x2 evaluation points at +-0.5, k_v = 8/point^3 = 1
                    double detJv = 0;
                    for (int is = 0; is < 2; is++)
                        for (int in = 0; in < 2; in++)
                            for (int it = 0; it < 2; it++) {
                                double s = pts[is], n = pts[in], t = pts[it];
                                double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                                for (int m = 0; m < 8; m++) {
                                    double sc = 2.0 * ((m >> 2) & 1) - 1;
                                    double nc = 2.0 * ((m >> 1) & 1) - 1;
                                    double tc = 2.0 * (m & 1) - 1;
                                    double d0 = sc * (1 + nc * n) * (1 + tc * t) / 8;
                                    double d1 = nc * (1 + sc * s) * (1 + tc * t) / 8;
                                    double d2 = tc * (1 + sc * s) * (1 + nc * n) / 8;
                                    J[0][0] += d0 * node[m].x;
                                    J[0][1] += d0 * node[m].y;
                                    J[0][2] += d0 * node[m].z;
                                    J[1][0] += d1 * node[m].x;
                                    J[1][1] += d1 * node[m].y;
                                    J[1][2] += d1 * node[m].z;
                                    J[2][0] += d2 * node[m].x;
                                    J[2][1] += d2 * node[m].y;
                                    J[2][2] += d2 * node[m].z;
                                }
                                detJv += J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) -
                                         J[0][1] * (J[1][0] * J[2][2] - J[2][0] * J[1][2]) +
                                         J[0][2] * (J[1][0] * J[2][1] - J[2][0] * J[1][1]);
                            }
                    double vol = detJv;
                    Volm[gi] = vol;
                    wmp[gi] = wm[gi];
                    wm[gi] = dx * dy * dz * FA0 / vol;
                }
    }

    // calChemBoundaryD, gel_kernels.cu:757-778 (no-flux ghost copy)
    void chem_boundary() {
        for (int zi = 0; zi <= LZ; zi++)
            for (int yi = 0; yi <= LY; yi++)
                for (int xi = 0; xi <= LX; xi++) {
                    int gi = E(xi, yi, zi);
                    const int* o = rn_offset[map_element[gi]];
                    int g1 = E(xi + o[0], yi + o[1], zi + o[2]);
                    um[gi] = um[g1];
                    vm[gi] = vm[g1];
                    um_norm[gi] = um[gi] / (1 - wm[gi]);
                    vm_norm[gi] = vm[gi] / (1 - wm[gi]);
                }
    }

    // calUnnormD, gel_kernels.cu:795-821
    void unnorm() {
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++)
                for (int xi = 1; xi <= LX; xi++) {
                    double su = 0, sv = 0;
                    for (int i = 0; i < 2; i++)
                        for (int j = 0; j < 2; j++)
                            for (int k = 0; k < 2; k++) {
                                su += um_norm[E(xi - i, yi - j, zi - k)];
                                sv += vm_norm[E(xi - i, yi - j, zi - k)];
                            }
                    int n = Nd(xi, yi, zi);
                    un_norm[n] = su / 8 + un_robin[n];
                    vn_norm[n] = sv / 8;
                }
    }

    // calPressureD, gel_kernels.cu:496-516
    void pressure() {
        for (int zi = 1; zi <= LZ - 1; zi++)
            for (int yi = 1; yi <= LY - 1; yi++)
                for (int xi = 1; xi <= LX - 1; xi++) {
                    int gi = E(xi, yi, zi);
                    double w = wm[gi];
                    if (type == 1) {
                        Prem[gi] = -(w + std::log(1.0 - w) + (CH0 + CH1 * w) * w * w) + C0 * w / (2.0 * FA0) +
                                   CHS * w * vm[gi];
                    } else if (type == 2) {
                        double c0 = c0_bis + b * vm[gi];
                        Prem[gi] = -(w + std::log(1.0 - w) + (CH0 + CH1 * w) * w * w) + c0 * w / (2.0 * FA0);
                    }
                }
    }

    // calNodesVelocityD, gel_kernels.cu:518-598
    void nodes_velocity() {
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++)
                for (int xi = 1; xi <= LX; xi++) {
                    int gi = Nd(xi, yi, zi);
                    double wn = 0;
                    for (int i = 0; i < 2; i++)
                        for (int j = 0; j < 2; j++)
                            for (int k = 0; k < 2; k++) wn += wm[E(xi - i, yi - j, zi - k)];
                    wn /= 8;
                    double Mn = 8. * AZ0 * std::sqrt(FA0 / wn) * (1 - wn) / (dx * dy * dz);
                    V3 f1n = v3(0, 0, 0), f2n = v3(0, 0, 0);
                    V3 rm_ = rn[gi];
                    // the eight elements around the node, in the reference's order:
                    // direction (a, b, c) in {+1,-1}^3, a outermost, '+' first
                    for (int ia = 0; ia < 2; ia++)
                        for (int ib = 0; ib < 2; ib++)
                            for (int ic = 0; ic < 2; ic++) {
                                int a = ia ? -1 : 1, bb = ib ? -1 : 1, cc = ic ? -1 : 1;
                                bool ok = (a > 0 ? xi < LX : xi > 1) && (bb > 0 ? yi < LY : yi > 1) &&
                                          (cc > 0 ? zi < LZ : zi > 1);
                                if (!ok) continue;
                                int ex = a > 0 ? xi : xi - 1, ey = bb > 0 ? yi : yi - 1, ez = cc > 0 ? zi : zi - 1;
                                int gn = 6 * E(ex, ey, ez);
                                V3 s4 = rn[Nd(xi + a, yi + bb, zi + cc)] + rn[Nd(xi, yi + bb, zi + cc)] +
                                        rn[Nd(xi + a, yi, zi + cc)] + rn[Nd(xi + a, yi + bb, zi)] - 4 * rm_;
                                f1n = f1n + s4;
                                int fx = a > 0 ? 0 : 1, fy = bb > 0 ? 2 : 3, fz = cc > 0 ? 4 : 5;
                                f2n = f2n + Prem[E(ex, ey, ez)] * (nmSm[gn + fx] + nmSm[gn + fy] + nmSm[gn + fz]);
                            }
                    // pow(dx*dy*dz, 1/3) is pow(., 0) == 1 in the reference (integer 1/3)
                    if (type == 1) {
                        f1n = f1n * (1.0 * C0 / 12.);
                    } else if (type == 2) {
                        double c0 = c0_bis + b * vn_norm[gi] * (1 - wn);
                        f1n = f1n * (1.0 * c0 / 12.);
                    }
                    f2n = f2n / 4.;
                    Fn[gi] = f1n + f2n;
                    Veln[gi] = Mn * Fn[gi];
                    Vels[gi] = (-wn * Veln[gi]) / (1 - wn);
                }
    }

    // calInternalNodesPositionD, gel_kernels.cu:600-613
    void advance_nodes() {
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++)
                for (int xi = 1; xi <= LX; xi++) {
                    int gi = Nd(xi, yi, zi);
                    rn[gi] = rn[gi] + dtx * Veln[gi];
                }
    }

    // anchorBottomNodesD, gel_kernels.cu:870-880
    void anchor_bottom() {
        int zi = 1;
        for (int yi = 1; yi <= LY; yi++)
            for (int xi = 1; xi <= LX; xi++) {
                int gi = Nd(xi, yi, zi);
                Veln[gi] = v3(0, 0, 0);
                rn[gi].z = anchor_z;
            }
    }

    // calTermsD, gel_kernels.cu:633-703
    void terms() {
        for (int zi = 1; zi <= LZ - 1; zi++)
            for (int yi = 1; yi <= LY - 1; yi++)
                for (int xi = 1; xi <= LX - 1; xi++) {
                    int gi = E(xi, yi, zi);
                    double wm_m = wm[gi], um_m = um_norm[gi];
                    V3 rm_m = rm[gi];
                    T0[gi] = (1 - wm_m / wmp[gi]) / dtx;
                    V3 vmum = v3(0, 0, 0);
                    int c = 0;
                    for (int i = 0; i < 2; i++)
                        for (int j = 0; j < 2; j++)
                            for (int k = 0; k < 2; k++) {
                                V3 rl = rm_loc[8 * gi + c];
                                c++;
                                int id2 = Nd(xi + i, yi + j, zi + k);
                                double N = 0.125 * (1 + (2 * double(i) - 1) * rl.x) * (1 + (2 * double(j) - 1) * rl.y) *
                                           (1 + (2 * double(k) - 1) * rl.z);
                                vmum = vmum + (N * Veln[id2]) * un_norm[id2];
                            }
                    double dT1 = 0;
                    for (int fi = 0; fi < 6; fi++) dT1 += dot(nmSm[6 * gi + fi], vmum);
                    T1[gi] = dT1 / Volm[gi];
                    int g1 = E(xi + 1, yi, zi), g2 = E(xi - 1, yi, zi), g3 = E(xi, yi + 1, zi);
                    int g4 = E(xi, yi - 1, zi), g5 = E(xi, yi, zi + 1), g6 = E(xi, yi, zi - 1);
                    auto dist = [](V3 p, V3 q2) {
                        double ax = p.x - q2.x, ay = p.y - q2.y, az = p.z - q2.z;
                        return std::sqrt(ax * ax + ay * ay + az * az);
                    };
                    V3 a_add = v3(dist(rm[g1], rm_m), dist(rm[g3], rm_m), dist(rm[g5], rm_m));
                    V3 a_sub = v3(dist(rm[g2], rm_m), dist(rm[g4], rm_m), dist(rm[g6], rm_m));
                    V3 a_add2 = hadamard(a_add, a_add), a_sub2 = hadamard(a_sub, a_sub);
                    V3 a_addsub = hadamard(hadamard(a_add, a_sub), a_add + a_sub);
                    V3 wm_add = v3(wm[g1], wm[g3], wm[g5]), wm_sub = v3(wm[g2], wm[g4], wm[g6]);
                    V3 um_add = v3(um_norm[g1], um_norm[g3], um_norm[g5]);
                    V3 um_sub = v3(um_norm[g2], um_norm[g4], um_norm[g6]);
                    V3 dwm = hdiv(wm_m * (a_add2 - a_sub2) + hadamard(wm_add, a_sub2) - hadamard(wm_sub, a_add2), a_addsub);
                    V3 dum = hdiv(um_m * (a_add2 - a_sub2) + hadamard(um_add, a_sub2) - hadamard(um_sub, a_add2), a_addsub);
                    V3 d2um = hdiv(2 * (hadamard(um_add, a_sub) + hadamard(um_sub, a_add) - um_m * (a_add + a_sub)), a_addsub);
                    T2[gi] = -dot(dwm, dum) + (1 - wm_m) * (d2um.x + d2um.y + d2um.z);
                }
    }

    // fv / fu, gel_kernels.cu:129-145 (I = 0; P1, P2, q fixed in the kernel)
    static double fv_k(double u, double v, double w) {
        return (1.0 - w) * (1.0 - w) * u - (1.0 - w) * v + 0.0 * (0.5 * 0.0124 + 0.77);
    }
    static double fu_k(double u, double v, double w, double fpar) {
        const double qk = 1e-4;
        double ww = (1.0 - w) * (1.0 - w);
        return ww * u - u * u - (1.0 - w) * (fpar * v + 0.0 * 0.0124) * (u - qk * ww) / (u + qk * ww) + 0.0 * 0.77;
    }

    // calChemD, gel_kernels.cu:705-731 (forward Euler)
    void chem() {
        for (int zi = 1; zi <= LZ - 1; zi++)
            for (int yi = 1; yi <= LY - 1; yi++)
                for (int xi = 1; xi <= LX - 1; xi++) {
                    int gi = E(xi, yi, zi);
                    if (is_void(yi, zi)) {
                        vm[gi] = vss;
                        um[gi] = uss;
                        wm[gi] = wss;
                        continue;
                    }
                    double v = vm[gi], u = um[gi], w = wm[gi];
                    vm[gi] += dt * (-v * T0[gi] + ep * fv_k(u, v, w));
                    um[gi] += dt * (-u * T0[gi] + T1[gi] + T2[gi] + fu_k(u, v, w, f));
                }
    }

    // setZero, gel_kernels.cu:780-793 (Fdrag_robin untouched)
    void set_zero() {
        for (int zi = 1; zi <= LZ; zi++)
            for (int yi = 1; yi <= LY; yi++)
                for (int xi = 1; xi <= LX; xi++) {
                    int n = Nd(xi, yi, zi);
                    un_robin[n] = 0;
                    Fn_robin[n] = v3(0, 0, 0);
                }
    }

    // Gel::stepElasticity, gel.cu:682-698
    void step_elasticity(int iter) {
        if (iter % 5 == 0) {
            service_nodes();
            element_properties();
            chem_boundary();
            unnorm();
            pressure();
            nodes_velocity();
            advance_nodes();
            if (use_anchor) anchor_bottom();
            terms();
        }
        set_zero();
    }
    // Gel::stepChemistry, gel.cu:700-704
    void step_chemistry(int) { chem(); }
};

// ---------------------------------------------------------------------------
// Fluid + coupler, templated on the fluid real type R
// ---------------------------------------------------------------------------
static const int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0};
static const int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
static const int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, -1, 1};
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16};

struct SimBase {
    virtual ~SimBase() {}
};

template <typename R>
struct Sim : SimBase {
    int nx, ny, nz;
    long long N;
    int nsub = 25;
    int perX = 0, perY = 0, perZ = 0;
    R tau, cs2, w[19];
    R Fc[3] = {0, 0, 0};
    R h = R(0.5), dtc = R(1e-3), Dc = R(1), dxc = R(1);
    R beta = R(1);
    float ramp_steps = 20000.0f;
    float g2l = 0.f, l2g = 0.f;
    R rep_delta = R(1e-4), rep_gamma = R(1.5);
    std::vector<R> f, fpost, rho, u, Fibm, c1, c2, source;
    std::vector<Gel> gels;
    int M = 0;
    std::vector<int> owner, offsets;
    std::vector<R> lag, Ul, Vl, Fdrag, Frep, Cl, Dl, Sl;
    bool finalized = false;
    int last_iter = -1;

    Sim(int X, int Y, int Z) : nx(X), ny(Y), nz(Z) {
        N = (long long)X * Y * Z;
        tau = R(0.8);
        cs2 = R(1) / R(3);
        w[0] = R(1) / R(3);
        for (int q = 1; q <= 6; q++) w[q] = R(1) / R(18);
        for (int q = 7; q < 19; q++) w[q] = R(1) / R(36);
    }
    long long id3(int x, int y, int z) const { return x + (long long)y * nx + (long long)z * nx * ny; }

    // Fluid ctor unit conversions (float arithmetic as in src/fluid.cu:167-229)
    void units() {
        float hf = 0.5f, dtf = 1e-3f, tauf = 0.8f, niu = 1e-6f;
        float dx_fluid = 40e-6f * hf;
        float dt_fluid = (tauf - 0.5f) * dx_fluid * dx_fluid / (3 * niu);
        g2l = hf * dt_fluid / dtf;
        l2g = 1.0f / g2l;
    }

    void finalize() {
        units();
        f.assign(19 * N, 0);
        fpost.assign(19 * N, 0);
        rho.assign(N, 1);
        u.assign(3 * N, 0);
        Fibm.assign(3 * N, 0);
        c1.assign(N, 0);
        c2.assign(N, 0);
        source.assign(N, 0);
        // k_init, fluid_kernels.cu:84-96
        for (int q = 0; q < 19; q++)
            for (long long i = 0; i < N; i++) f[i + q * N] = w[q];
        M = 0;
        offsets.clear();
        owner.clear();
        for (size_t g = 0; g < gels.size(); g++) {
            offsets.push_back(M);
            for (int l = 0; l < gels[g].M; l++) owner.push_back((int)g);
            M += gels[g].M;
        }
        for (auto* v : {&lag, &Ul, &Vl, &Fdrag, &Frep}) v->assign(3 * (size_t)M, 0);
        for (auto* v : {&Cl, &Dl, &Sl}) v->assign(M, 0);
        finalized = true;
    }

    // delta4, fluid_kernels.cu:60-71
    static R delta4(R r) {
        r = std::fabs(r);
        if (r <= R(1)) return R(0.125) * (R(3) - R(2) * r + std::sqrt(R(1) + R(4) * r - R(4) * r * r));
        if (r <= R(2)) return R(0.125) * (R(5) - R(2) * r - std::sqrt(R(-7) + R(12) * r - R(4) * r * r));
        return R(0);
    }

    // stencil bounds for marker l, clipped at the box (fluid_kernels.cu:251-262)
    struct Stencil {
        R gx, gy, gz;
        int x0, x1, y0, y1, z0, z1;
    };
    Stencil stencil(int l) const {
        Stencil s;
        s.gx = lag[3 * l] / h;
        s.gy = lag[3 * l + 1] / h;
        s.gz = lag[3 * l + 2] / h;
        int ix = (int)std::floor(s.gx), iy = (int)std::floor(s.gy), iz = (int)std::floor(s.gz);
        s.x0 = std::max(0, ix - 1);
        s.x1 = std::min(nx - 1, ix + 2);
        s.y0 = std::max(0, iy - 1);
        s.y1 = std::min(ny - 1, iy + 2);
        s.z0 = std::max(0, iz - 1);
        s.z1 = std::min(nz - 1, iz + 2);
        return s;
    }

    // k_ibm_interpolate_velocity, fluid_kernels.cu:244-281
    void ibm_interp() {
        for (int l = 0; l < M; l++) {
            Stencil s = stencil(l);
            R ux = 0, uy = 0, uz = 0, ws = 0;
            for (int ii = s.x0; ii <= s.x1; ++ii) {
                R phx = delta4(s.gx - (R)ii);
                for (int jj = s.y0; jj <= s.y1; ++jj) {
                    R phy = delta4(s.gy - (R)jj);
                    for (int kk = s.z0; kk <= s.z1; ++kk) {
                        R phz = delta4(s.gz - (R)kk);
                        R wgt = phx * phy * phz;
                        long long id = id3(ii, jj, kk);
                        ux += u[3 * id] * wgt;
                        uy += u[3 * id + 1] * wgt;
                        uz += u[3 * id + 2] * wgt;
                        ws += wgt;
                    }
                }
            }
            if (ws > R(0)) {
                Ul[3 * l] = ux / ws;
                Ul[3 * l + 1] = uy / ws;
                Ul[3 * l + 2] = uz / ws;
            } else {
                Ul[3 * l] = Ul[3 * l + 1] = Ul[3 * l + 2] = 0;
            }
        }
    }

    // generic delta-4 spread of a per-marker value into a field with `nc` components
    // (k_ibm_spread_forces fluid_kernels.cu:300-348, k_ibm_spread_concentration :414-459)
    void ibm_spread(const std::vector<R>& val, int nc, std::vector<R>& field) {
        for (int l = 0; l < M; l++) {
            Stencil s = stencil(l);
            R ws = 0;
            for (int ii = s.x0; ii <= s.x1; ++ii) {
                R phx = delta4(s.gx - (R)ii);
                for (int jj = s.y0; jj <= s.y1; ++jj) {
                    R phy = delta4(s.gy - (R)jj);
                    for (int kk = s.z0; kk <= s.z1; ++kk) {
                        R phz = delta4(s.gz - (R)kk);
                        ws += phx * phy * phz;
                    }
                }
            }
            if (ws == R(0)) continue;
            R inv_h3 = (R)(1.0 / (double)(h * h * h));
            R scale = R(1) * inv_h3 / ws;
            for (int ii = s.x0; ii <= s.x1; ++ii) {
                R phx = delta4(s.gx - (R)ii);
                for (int jj = s.y0; jj <= s.y1; ++jj) {
                    R phy = delta4(s.gy - (R)jj);
                    for (int kk = s.z0; kk <= s.z1; ++kk) {
                        R phz = delta4(s.gz - (R)kk);
                        R wgt = phx * phy * phz * scale;
                        long long id = id3(ii, jj, kk);
                        for (int c = 0; c < nc; c++) field[nc * id + c] += val[nc * l + c] * wgt;
                    }
                }
            }
        }
    }

    // k_ibm_sample_concentration, fluid_kernels.cu:350-387
    void ibm_sample_c(const std::vector<R>& c, std::vector<R>& out) {
        for (int l = 0; l < M; l++) {
            Stencil s = stencil(l);
            R cl = 0, ws = 0;
            for (int ii = s.x0; ii <= s.x1; ++ii) {
                R phx = delta4(s.gx - (R)ii);
                for (int jj = s.y0; jj <= s.y1; ++jj) {
                    R phy = delta4(s.gy - (R)jj);
                    for (int kk = s.z0; kk <= s.z1; ++kk) {
                        R phz = delta4(s.gz - (R)kk);
                        R wgt = phx * phy * phz;
                        cl += c[id3(ii, jj, kk)] * wgt;
                        ws += wgt;
                    }
                }
            }
            out[l] = (ws > R(0)) ? cl / ws : R(0);
        }
    }

    // k_macros + k_collide (fluid_kernels.cu:98-111, :125-142), F_tot = F_const + F_ibm
    void collide() {
        const R inv_tau = R(1) / tau;
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < N; i++) {
            R Ft[3] = {Fc[0] + Fibm[3 * i], Fc[1] + Fibm[3 * i + 1], Fc[2] + Fibm[3 * i + 2]};
            R rh = 0, sx = 0, sy = 0, sz = 0;
            for (int q = 0; q < 19; q++) {
                R fi = f[i + q * N];
                rh += fi;
                sx += fi * (R)CX[q];
                sy += fi * (R)CY[q];
                sz += fi * (R)CZ[q];
            }
            rho[i] = rh;
            R ux = (sx + R(0.5) * Ft[0]) / rh, uy = (sy + R(0.5) * Ft[1]) / rh, uz = (sz + R(0.5) * Ft[2]) / rh;
            u[3 * i] = ux;
            u[3 * i + 1] = uy;
            u[3 * i + 2] = uz;
            R uu = ux * ux + uy * uy + uz * uz;
            R uF = ux * Ft[0] + uy * Ft[1] + uz * Ft[2];
            for (int q = 0; q < 19; q++) {
                R cu = (R)CX[q] * ux + (R)CY[q] * uy + (R)CZ[q] * uz;
                R feq = w[q] * rh * (R(1) + (cu / cs2) + R(0.5) * (cu * cu) / (cs2 * cs2) - R(0.5) * (uu / cs2));
                R ciF = (R)CX[q] * Ft[0] + (R)CY[q] * Ft[1] + (R)CZ[q] * Ft[2];
                R Fterm = w[q] * (R(1) - R(0.5) * inv_tau) * ((ciF / cs2) + (cu * ciF) / (cs2 * cs2) - (uF / cs2));
                R fi = f[i + q * N];
                fpost[i + q * N] = fi - inv_tau * (fi - feq) + Fterm;
            }
        }
    }

    // k_stream_bounce (fluid_kernels.cu:144-165) in pull form: the population that
    // arrives at x in direction q comes from x - c_q, or is the bounced-back
    // opp(q) population of x itself when x - c_q lies outside the box.  Periodic
    // axes (an extension; the reference bounces back on all six faces) wrap.
    void stream() {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; z++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    long long i = id3(x, y, z);
                    for (int q = 0; q < 19; q++) {
                        int sx = x - CX[q], sy = y - CY[q], sz = z - CZ[q];
                        if (perX) sx = (sx + nx) % nx;
                        if (perY) sy = (sy + ny) % ny;
                        if (perZ) sz = (sz + nz) % nz;
                        bool inside = sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz;
                        f[i + q * N] = inside ? fpost[id3(sx, sy, sz) + q * N] : fpost[i + OPP[q] * N];
                    }
                }
    }

    // Fluid::stepVelocity, fluid.cu:263-284
    void step_velocity(int iter) {
        float ramp = (ramp_steps <= 0.0f) ? 1.0f : std::fmin(1.0f, (iter + 1) / ramp_steps);
        R beta_eff = beta * (R)ramp;
        for (int kk = 0; kk < nsub; kk++) {
            ibm_interp();
            for (int l = 0; l < M; l++)
                for (int c = 0; c < 3; c++) Fdrag[3 * l + c] = beta_eff * (Vl[3 * l + c] - Ul[3 * l + c]);
            ibm_spread(Fdrag, 3, Fibm);
            collide();
            stream();
            std::fill(Fibm.begin(), Fibm.end(), R(0));
        }
    }

    // k_convection_diffusion, fluid_kernels.cu:177-242
    void convection_diffusion() {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; z++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    int xp = (x + 1 < nx) ? x + 1 : (perX ? 0 : x);
                    int xm = (x - 1 >= 0) ? x - 1 : (perX ? nx - 1 : x);
                    int yp = (y + 1 < ny) ? y + 1 : (perY ? 0 : y);
                    int ym = (y - 1 >= 0) ? y - 1 : (perY ? ny - 1 : y);
                    int zp = (z + 1 < nz) ? z + 1 : (perZ ? 0 : z);
                    int zm = (z - 1 >= 0) ? z - 1 : (perZ ? nz - 1 : z);
                    long long i = id3(x, y, z);
                    long long ixp = id3(xp, y, z), ixm = id3(xm, y, z), iyp = id3(x, yp, z), iym = id3(x, ym, z);
                    long long izp = id3(x, y, zp), izm = id3(x, y, zm);
                    R ih = R(1) / dxc, ih2 = ih * ih;
                    R c = c1[i], cxp = c1[ixp], cxm = c1[ixm], cyp = c1[iyp], cym = c1[iym], czp = c1[izp],
                      czm = c1[izm];
                    R uL = R(0.5) * (u[3 * ixm] + u[3 * i]), uR = R(0.5) * (u[3 * i] + u[3 * ixp]);
                    R vL = R(0.5) * (u[3 * iym + 1] + u[3 * i + 1]), vR = R(0.5) * (u[3 * i + 1] + u[3 * iyp + 1]);
                    R wL = R(0.5) * (u[3 * izm + 2] + u[3 * i + 2]), wR = R(0.5) * (u[3 * i + 2] + u[3 * izp + 2]);
                    R cLx = (uL >= R(0)) ? cxm : c, cLy = (vL >= R(0)) ? cym : c, cLz = (wL >= R(0)) ? czm : c;
                    R cRx = (uR >= R(0)) ? c : cxp, cRy = (vR >= R(0)) ? c : cyp, cRz = (wR >= R(0)) ? c : czp;
                    R dFx = uR * cRx - uL * cLx, dFy = vR * cRy - vL * cLy, dFz = wR * cRz - wL * cLz;
                    R conv = -(dFx * ih + dFy * ih + dFz * ih);
                    R secx = cxm - R(2) * c + cxp, secy = cym - R(2) * c + cyp, secz = czm - R(2) * c + czp;
                    R diff = Dc * (secx * ih2 + secy * ih2 + secz * ih2);
                    c2[i] = c + dtc * (conv + diff + source[i]);
                }
        std::swap(c1, c2);
    }

    // Fluid::stepConcentration, fluid.cu:251-261
    void step_concentration(int) {
        ibm_sample_c(c1, Dl);
        for (int l = 0; l < M; l++) Sl[l] = R(1) * (Cl[l] - Dl[l]);
        std::fill(source.begin(), source.end(), R(0));
        ibm_spread(Sl, 1, source);
        convection_diffusion();
    }

    // Coupler::packFromGels + k_gather_boundary, coupling.cu:82-98, coupling_kernels.cu:42-56
    void pack() {
        for (size_t g = 0; g < gels.size(); g++) {
            const Gel& G = gels[g];
            int off = offsets[g];
            for (int l = 0; l < G.M; l++) {
                int id = G.bIndex[l];
                lag[3 * (off + l)] = (R)G.rn[id].x;
                lag[3 * (off + l) + 1] = (R)G.rn[id].y;
                lag[3 * (off + l) + 2] = (R)G.rn[id].z;
                Vl[3 * (off + l)] = (R)(G.Vels[id].x * (double)g2l);
                Vl[3 * (off + l) + 1] = (R)(G.Vels[id].y * (double)g2l);
                Vl[3 * (off + l) + 2] = (R)(G.Vels[id].z * (double)g2l);
                Cl[off + l] = (R)G.un_norm[id];
            }
        }
    }

    // Coupler::applyGelRepulsion + k_gel_repulsion, coupling.cu:120-123, coupling_kernels.cu:58-146
    void repulsion() {
        R rcut = R(2.5) * rep_gamma, rc2 = rcut * rcut, sig2 = rep_gamma * rep_gamma;
        for (int a = 0; a < M; a++) {
            R fx = 0, fy = 0, fz = 0;
            for (int bq = 0; bq < M; bq++) {
                if (owner[a] == owner[bq]) continue;
                R dxv = lag[3 * a] - lag[3 * bq], dyv = lag[3 * a + 1] - lag[3 * bq + 1], dzv = lag[3 * a + 2] - lag[3 * bq + 2];
                R d2 = dxv * dxv + dyv * dyv + dzv * dzv;
                if (d2 <= R(0) || d2 >= rc2) continue;
                R inv = R(1) / d2, sr2 = sig2 * inv, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
                R fac = R(24) * rep_delta * (R(2) * sr12 - sr6) * inv;
                fx += fac * dxv;
                fy += fac * dyv;
                fz += fac * dzv;
            }
            Frep[3 * a] = fx;
            Frep[3 * a + 1] = fy;
            Frep[3 * a + 2] = fz;
        }
    }

    // Coupler::scatterToGels + C2/C3, coupling.cu:100-118, coupling_kernels.cu:8-35
    void scatter() {
        for (size_t g = 0; g < gels.size(); g++) {
            Gel& G = gels[g];
            int off = offsets[g];
            for (int l = 0; l < G.M; l++) {
                int id = G.bIndex[l];
                G.Fn_robin[id].x -= (double)Frep[3 * (off + l)];
                G.Fn_robin[id].y -= (double)Frep[3 * (off + l) + 1];
                G.Fn_robin[id].z -= (double)Frep[3 * (off + l) + 2];
                G.un_robin[id] -= (double)Sl[off + l];
                G.Fdrag_robin[id].x -= (double)Fdrag[3 * (off + l)];
                G.Fdrag_robin[id].y -= (double)Fdrag[3 * (off + l) + 1];
                G.Fdrag_robin[id].z -= (double)Fdrag[3 * (off + l) + 2];
            }
        }
    }

    // one coupled iteration in the order of src/sim.cpp:97-112; a gel whose
    // active_from lies in the future is skipped (src/sim_array.cpp:93-103) and
    // fires its excitation pulse at iter == active_from (src/sim_array.cpp:86-90)
    void iterate(int iter) {
        for (auto& G : gels)
            if (G.active_from > 0 && iter == G.active_from) G.fire_pulse();
        for (auto& G : gels) {
            if (G.active_from > 0 && iter < G.active_from) continue;
            G.step_elasticity(iter);
            G.step_chemistry(iter);
        }
        pack();
        step_velocity(iter);
        step_concentration(iter);
        repulsion();
        scatter();
        last_iter = iter;
    }
};

}  // namespace orc

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
using namespace orc;

enum {
    ORC_F_POP = 0,  // 19*N populations, natural (post-stream) layout f[i + q*N]
    ORC_F_RHO = 1,
    ORC_F_U = 2,  // 3*N
    ORC_F_C1 = 3,
    ORC_F_FIBM = 4,
    ORC_M_LAG = 10,
    ORC_M_UL = 11,
    ORC_M_VL = 12,
    ORC_M_FDRAG = 13,
    ORC_M_FREP = 14,
    ORC_M_CL = 15,
    ORC_M_DL = 16,
    ORC_M_SL = 17,
    ORC_G_RN = 20,  // 3*nN
    ORC_G_VELN = 21,
    ORC_G_VELS = 22,
    ORC_G_FN = 23,
    ORC_G_UM = 24,  // nE
    ORC_G_VM = 25,
    ORC_G_WM = 26,
    ORC_G_UN_NORM = 27,  // nN
    ORC_G_VN_NORM = 28,
    ORC_G_T0 = 29,
    ORC_G_T1 = 30,
    ORC_G_T2 = 31,
    ORC_G_RM = 32,  // 3*nE
    ORC_G_NMSM = 33,  // 18*nE
    ORC_G_VOLM = 34,
    ORC_G_PREM = 35,
    ORC_G_UN_ROBIN = 36,
    ORC_G_UM_NORM = 37,
    ORC_G_VM_NORM = 38,
    ORC_G_WMP = 39,
    ORC_G_FN_ROBIN = 40,
};

struct OrcHandle {
    int fp32 = 0;
    std::unique_ptr<Sim<double>> d;
    std::unique_ptr<Sim<float>> s;
};

template <typename R>
static long long field_io(Sim<R>& S, int field, int gel, double* buf, long long n, bool write) {
    auto vec_io = [&](auto& v, long long count) -> long long {
        if (!buf) return count;
        if (n < count) return -2;
        for (long long i = 0; i < count; i++) {
            if (write)
                v[i] = (typename std::remove_reference<decltype(v[0])>::type)buf[i];
            else
                buf[i] = (double)v[i];
        }
        return count;
    };
    auto v3_io = [&](std::vector<V3>& v) -> long long {
        long long count = 3 * (long long)v.size();
        if (!buf) return count;
        if (n < count) return -2;
        for (size_t i = 0; i < v.size(); i++) {
            if (write) {
                v[i].x = buf[3 * i];
                v[i].y = buf[3 * i + 1];
                v[i].z = buf[3 * i + 2];
            } else {
                buf[3 * i] = v[i].x;
                buf[3 * i + 1] = v[i].y;
                buf[3 * i + 2] = v[i].z;
            }
        }
        return count;
    };
    if (field < 10) {
        switch (field) {
            case ORC_F_POP: return vec_io(S.f, 19 * S.N);
            case ORC_F_RHO: return vec_io(S.rho, S.N);
            case ORC_F_U: return vec_io(S.u, 3 * S.N);
            case ORC_F_C1: return vec_io(S.c1, S.N);
            case ORC_F_FIBM: return vec_io(S.Fibm, 3 * S.N);
        }
        return -1;
    }
    if (field < 20) {
        switch (field) {
            case ORC_M_LAG: return vec_io(S.lag, 3LL * S.M);
            case ORC_M_UL: return vec_io(S.Ul, 3LL * S.M);
            case ORC_M_VL: return vec_io(S.Vl, 3LL * S.M);
            case ORC_M_FDRAG: return vec_io(S.Fdrag, 3LL * S.M);
            case ORC_M_FREP: return vec_io(S.Frep, 3LL * S.M);
            case ORC_M_CL: return vec_io(S.Cl, S.M);
            case ORC_M_DL: return vec_io(S.Dl, S.M);
            case ORC_M_SL: return vec_io(S.Sl, S.M);
        }
        return -1;
    }
    if (gel < 0 || gel >= (int)S.gels.size()) return -3;
    Gel& G = S.gels[gel];
    switch (field) {
        case ORC_G_RN: return v3_io(G.rn);
        case ORC_G_VELN: return v3_io(G.Veln);
        case ORC_G_VELS: return v3_io(G.Vels);
        case ORC_G_FN: return v3_io(G.Fn);
        case ORC_G_UM: return vec_io(G.um, G.nE);
        case ORC_G_VM: return vec_io(G.vm, G.nE);
        case ORC_G_WM: return vec_io(G.wm, G.nE);
        case ORC_G_UN_NORM: return vec_io(G.un_norm, G.nN);
        case ORC_G_VN_NORM: return vec_io(G.vn_norm, G.nN);
        case ORC_G_T0: return vec_io(G.T0, G.nE);
        case ORC_G_T1: return vec_io(G.T1, G.nE);
        case ORC_G_T2: return vec_io(G.T2, G.nE);
        case ORC_G_RM: return v3_io(G.rm);
        case ORC_G_NMSM: return v3_io(G.nmSm);
        case ORC_G_VOLM: return vec_io(G.Volm, G.nE);
        case ORC_G_PREM: return vec_io(G.Prem, G.nE);
        case ORC_G_UN_ROBIN: return vec_io(G.un_robin, G.nN);
        case ORC_G_UM_NORM: return vec_io(G.um_norm, G.nE);
        case ORC_G_VM_NORM: return vec_io(G.vm_norm, G.nE);
        case ORC_G_WMP: return vec_io(G.wmp, G.nE);
        case ORC_G_FN_ROBIN: return v3_io(G.Fn_robin);
    }
    return -1;
}

#define DISPATCH(h, expr)                \
    do {                                 \
        if ((h)->fp32) {                 \
            auto& S = *(h)->s;           \
            expr;                        \
        } else {                         \
            auto& S = *(h)->d;           \
            expr;                        \
        }                                \
    } while (0)

extern "C" {

void* orc_create(int nx, int ny, int nz, int nsub, int fp32) {
    if (nx < 4 || ny < 4 || nz < 4 || nsub < 1) return nullptr;
    auto* h = new OrcHandle;
    h->fp32 = fp32;
    if (fp32) {
        h->s.reset(new Sim<float>(nx, ny, nz));
        h->s->nsub = nsub;
    } else {
        h->d.reset(new Sim<double>(nx, ny, nz));
        h->d->nsub = nsub;
    }
    return h;
}

void orc_destroy(void* p) { delete (OrcHandle*)p; }

int orc_set_params(void* p, double beta, double ramp_steps, double fx, double fy, double fz, int perX, int perY,
                   int perZ) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        S.beta = (decltype(S.beta))beta;
        S.ramp_steps = (float)ramp_steps;
        S.Fc[0] = (decltype(S.beta))fx;
        S.Fc[1] = (decltype(S.beta))fy;
        S.Fc[2] = (decltype(S.beta))fz;
        S.perX = perX;
        S.perY = perY;
        S.perZ = perZ;
    });
    return 0;
}

int orc_add_gel(void* p, int sx, int sy, int sz, double px, double py, double pz, int type, int id) {
    auto* h = (OrcHandle*)p;
    int idx = -1;
    DISPATCH(h, {
        if (S.finalized) return -1;
        Gel G;
        G.init(sx, sy, sz, px, py, pz, type, id);
        S.gels.push_back(std::move(G));
        idx = (int)S.gels.size() - 1;
    });
    return idx;
}

int orc_gel_noise(void* p, int gel, unsigned long long seed, double amp) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        if (gel < 0 || gel >= (int)S.gels.size()) return -3;
        S.gels[gel].add_noise(seed, amp);
    });
    return 0;
}

int orc_gel_control(void* p, int gel, int what, double value) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        if (gel < 0 || gel >= (int)S.gels.size()) return -3;
        Gel& G = S.gels[gel];
        switch (what) {
            case 0: G.reset_quiescent(); break;
            case 1: G.fire_pulse(); break;
            case 2:
                G.use_anchor = true;
                G.anchor_z = value;
                break;
            case 3: G.active_from = (int)value; break;
            case 4: G.build_tube_mask((int)value, false); break;  // square tube, wall = value
            case 5: G.build_tube_mask((int)value, true); break;   // cylindrical tube
            default: return -1;
        }
    });
    return 0;
}

int orc_finalize(void* p) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, S.finalize());
    return 0;
}

int orc_info(void* p, long long* out) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        out[0] = S.N;
        out[1] = S.M;
        out[2] = (long long)S.gels.size();
        out[3] = S.nsub;
    });
    return 0;
}

int orc_gel_info(void* p, int gel, long long* out) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        if (gel < 0 || gel >= (int)S.gels.size()) return -3;
        Gel& G = S.gels[gel];
        out[0] = G.LX;
        out[1] = G.LY;
        out[2] = G.LZ;
        out[3] = G.nE;
        out[4] = G.nN;
        out[5] = G.M;
        out[6] = S.offsets.empty() ? 0 : S.offsets[gel];
    });
    return 0;
}

int orc_gel_steady(void* p, int gel, double* out) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        if (gel < 0 || gel >= (int)S.gels.size()) return -3;
        out[0] = S.gels[gel].uss;
        out[1] = S.gels[gel].vss;
        out[2] = S.gels[gel].wss;
    });
    return 0;
}

int orc_units(void* p, double* out) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        S.units();
        out[0] = S.g2l;
        out[1] = S.l2g;
    });
    return 0;
}

// run iterations iter0 .. iter0 + n - 1
int orc_run(void* p, int iter0, int n) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        if (!S.finalized) return -1;
        for (int k = 0; k < n; k++) S.iterate(iter0 + k);
    });
    return 0;
}

// individual phases (for kernel-level tests)
int orc_phase(void* p, int phase, int iter) {
    auto* h = (OrcHandle*)p;
    DISPATCH(h, {
        switch (phase) {
            case 0:
                for (auto& G : S.gels) G.step_elasticity(iter);
                break;
            case 1:
                for (auto& G : S.gels) G.step_chemistry(iter);
                break;
            case 2: S.pack(); break;
            case 3: S.step_velocity(iter); break;
            case 4: S.step_concentration(iter); break;
            case 5: S.repulsion(); break;
            case 6: S.scatter(); break;
            case 7: S.collide(); break;
            case 8: S.stream(); break;
            case 9: S.ibm_interp(); break;
            default: return -1;
        }
    });
    return 0;
}

long long orc_field(void* p, int field, int gel, double* buf, long long n, int write) {
    auto* h = (OrcHandle*)p;
    long long r = 0;
    DISPATCH(h, r = field_io(S, field, gel, buf, n, write != 0));
    return r;
}

int orc_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

double orc_noise(unsigned long long seed, unsigned long long gel_id, unsigned long long slot, unsigned long long field) {
    return noise_pm1(seed, gel_id, slot, field);
}

}  // extern "C"
