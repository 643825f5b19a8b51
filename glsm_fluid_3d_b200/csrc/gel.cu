// gel.cu -- the gel lattice-spring model (FP64) and the marker exchange, sm_100a.
//
//   gel_kernel          one CTA per gel; every phase of Gel::stepElasticity,
//                       Gel::stepChemistry, Gel::recordCenter and the gather of
//                       Coupler::packFromGels, separated by block barriers.
//   conc_markers_kernel one warp per marker: concentration sample, Robin flux,
//                       delta-4 spread into the source field (Fluid::stepConcentration
//                       marker part), optionally the un_robin scatter.
//   repulsion_kernel    LJ repulsion between markers of different gels.
//   scatter_kernel      Coupler::scatterToGels.
//
// Reference semantics followed (lasite/gLSM_fluid_3D):
//   Gel::stepElasticity / stepChemistry / recordCenter  src/gel.cu:682-713
//   calServiceNodesPositionD src/gel_kernels.cu:615   calElementPropertiesD :216
//   calChemBoundaryD :757  calUnnormD :795  calPressureD :496  calNodesVelocityD :518
//   calInternalNodesPositionD :600  anchorBottomNodesD :870  calTermsD :633
//   calChemD :705 (fu/fv :129-145)  setZero :780  recordCenterElementD :823
//   Gel::fireExcitationPulse src/gel.cu:751-783
//   k_gather_boundary src/coupling_kernels.cu:42   k_add_reaction_to_gel :8
//   k_gel_repulsion :90   k_ibm_sample_concentration src/fluid_kernels.cu:350
//   k_robin_boundary :293  k_ibm_spread_concentration :414
#include <atomic>
#include <cuda_runtime.h>

#include "gel.h"

namespace glsm {

// ---------------------------------------------------------------------------
// small double3 helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double3 d3(double x, double y, double z) { return make_double3(x, y, z); }
__device__ __forceinline__ double3 add(double3 a, double3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 sub(double3 a, double3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 mul(double s, double3 a) { return d3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 crs(double3 a, double3 b) {
    return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double len(double3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

// Peskin 4-point kernel (src/fluid_kernels.cu:60-71), float arithmetic
__device__ __forceinline__ float delta4f(float r) {
    r = fabsf(r);
    if (r <= 1.f) return 0.125f * (3.f - 2.f * r + sqrtf(1.f + 4.f * r - 4.f * r * r));
    if (r <= 2.f) return 0.125f * (5.f - 2.f * r - sqrtf(-7.f + 12.f * r - 4.f * r * r));
    return 0.f;
}

// BZ reaction terms of calChemD (src/gel_kernels.cu:129-145) with I = 0 and the
// kernel's fixed q = 1e-4
__device__ __forceinline__ double bz_fv(double u, double v, double w) {
    const double a = 1.0 - w;
    return a * a * u - a * v;
}
__device__ __forceinline__ double bz_fu(double u, double v, double w, double f) {
    const double a = 1.0 - w, aa = a * a, q = 1e-4;
    return aa * u - u * u - a * (f * v) * (u - q * aa) / (u + q * aa);
}

// tube mask of isVoidElement (src/gel_kernels.cu:104-117)
__device__ __forceinline__ bool void_element(const GelDev& G, int yi, int zi) {
    if (G.tube_mode == 0) return false;
    const float dy = (float)yi - G.tube_cy, dz = (float)zi - G.tube_cz;
    if (G.tube_mode == 1) return fabsf(dy) < G.tube_ihy && fabsf(dz) < G.tube_ihz;
    if (G.tube_ihy < 0.5f || G.tube_ihz < 0.5f) return false;
    return (dy * dy) / (G.tube_ihy * G.tube_ihy) + (dz * dz) / (G.tube_ihz * G.tube_ihz) < 1.0f;
}

struct Idx {
    int LX, LY;
    __device__ __forceinline__ int e(int x, int y, int z) const { return x + (LX + 1) * (y + (LY + 1) * z); }
    __device__ __forceinline__ int n(int x, int y, int z) const { return x + (LX + 2) * (y + (LY + 2) * z); }
};

// loop over an inclusive 3-D index range with all threads of the CTA
#define GEL_FOR3(x0, x1, y0, y1, z0, z1, ...)                                           \
    {                                                                                   \
        const int _nx = (x1) - (x0) + 1, _ny = (y1) - (y0) + 1, _nz = (z1) - (z0) + 1;  \
        const int _cnt = _nx * _ny * _nz;                                               \
        for (int _t = threadIdx.x; _t < _cnt; _t += blockDim.x) {                       \
            const int x = (x0) + _t % _nx;                                              \
            const int y = (y0) + (_t / _nx) % _ny;                                      \
            const int z = (z0) + _t / (_nx * _ny);                                      \
            __VA_ARGS__                                                                 \
        }                                                                               \
    }

// inward direction of a slot on the ghost layer of an index range [0, top]
__device__ __forceinline__ int inward(int c, int top) { return c == 0 ? 1 : (c == top ? -1 : 0); }

// ---------------------------------------------------------------------------
// mechanics phases (every 5th iteration)
// ---------------------------------------------------------------------------
// Element slots are processed in passes of blockDim.x (slot t = x + (LX+1)(y +
// (LY+1) z) by thread t - t0).  A pass's rm_loc (8 double3 per element) and
// nmSm (6 double3) are staged in shared memory at odd strides and written out
// as the contiguous byte ranges they are, coalesced: thread-per-element
// stores of 24- and 18-double records would scatter every warp store over
// 32 cache lines.
constexpr int kLocStride = 25;   // doubles per element in the rm_loc stage (24 used)
constexpr int kFaceStride = 19;  // doubles per element in the nmSm stage (18 used)
constexpr size_t kGelStageBytes = (size_t)kGelThreads * (kLocStride + kFaceStride) * sizeof(double);

// rm_loc and nmSm as node_forces and terms read them: from the stage when the
// gel's element slots fit one pass of element_geometry (which then leaves the
// whole arrays there), else from global memory; the same doubles either way
struct GeomStage {
    const double* s;
    bool on;
    __device__ __forceinline__ double3 loc(const GelDev& G, int e, int m) const {
        if (!on) return G.rm_loc[8 * e + m];
        const double* p = s + kLocStride * e + 3 * m;
        return d3(p[0], p[1], p[2]);
    }
    __device__ __forceinline__ double3 face(const GelDev& G, int e, int f) const {
        if (!on) return G.nmSm[6 * e + f];
        const double* p = s + kLocStride * kGelThreads + kFaceStride * e + 3 * f;
        return d3(p[0], p[1], p[2]);
    }
};

__device__ __forceinline__ GeomStage geom_stage(const GelDev& G, const double* stage) {
    return GeomStage{stage, (G.LX + 1) * (G.LY + 1) * (G.LZ + 1) <= (int)blockDim.x && blockDim.x == kGelThreads};
}

__device__ void element_geometry(const GelDev& G, const Idx& I, double* stage) {
    const int ex = G.LX + 1, ey = G.LY + 1;
    const int cnt = ex * ey * (G.LZ + 1);
    for (int t0 = 0; t0 < cnt; t0 += blockDim.x) {
        const int t = t0 + (int)threadIdx.x, n_pass = min((int)blockDim.x, cnt - t0);
        double* st_loc = stage + kLocStride * threadIdx.x;
        double* st_face = stage + kLocStride * blockDim.x + kFaceStride * threadIdx.x;
        if (t < cnt) {
            double3 p[8];
            const int x = t % ex, y = (t / ex) % ey, z = t / (ex * ey);
            const int e = I.e(x, y, z);
            double3 c = d3(0, 0, 0);
_Pragma("unroll")
            for (int m = 0; m < 8; m++) {
                p[m] = G.rn[I.n(x + (m >> 2), y + ((m >> 1) & 1), z + (m & 1))];
                c = add(c, p[m]);
            }
            c = mul(1.0 / 8.0, c);
            G.rm[e] = c;
_Pragma("unroll")
            for (int m = 0; m < 8; m++) {
                p[m] = sub(p[m], c);
                st_loc[3 * m] = p[m].x;
                st_loc[3 * m + 1] = p[m].y;
                st_loc[3 * m + 2] = p[m].z;
            }
            // Outward face area vectors.  The reference integrates cross(dx/da, dx/db)
            // of the bilinear face over 2x2 points at +-0.5 (src/gel_kernels.cu:255-436);
            // for a bilinear face that sum equals (1/4) (sum_m a_m P_m) x (sum_m b_m P_m).
            // corner m = 4i + 2j + k
            const double3 ax0 = sub(add(p[2], p[3]), add(p[0], p[1])), bx0 = sub(add(p[1], p[3]), add(p[0], p[2]));
            const double3 ax1 = sub(add(p[6], p[7]), add(p[4], p[5])), bx1 = sub(add(p[5], p[7]), add(p[4], p[6]));
            const double3 ay0 = sub(add(p[4], p[5]), add(p[0], p[1])), by0 = sub(add(p[1], p[5]), add(p[0], p[4]));
            const double3 ay1 = sub(add(p[6], p[7]), add(p[2], p[3])), by1 = sub(add(p[3], p[7]), add(p[2], p[6]));
            const double3 az0 = sub(add(p[4], p[6]), add(p[0], p[2])), bz0 = sub(add(p[2], p[6]), add(p[0], p[4]));
            const double3 az1 = sub(add(p[5], p[7]), add(p[1], p[3])), bz1 = sub(add(p[3], p[7]), add(p[1], p[5]));
            const double3 face[6] = {mul(-0.25, crs(ax0, bx0)), mul(0.25, crs(ax1, bx1)), mul(0.25, crs(ay0, by0)),
                                     mul(-0.25, crs(ay1, by1)), mul(-0.25, crs(az0, bz0)), mul(0.25, crs(az1, bz1))};
_Pragma("unroll")
            for (int f = 0; f < 6; f++) {
                st_face[3 * f] = face[f].x;
                st_face[3 * f + 1] = face[f].y;
                st_face[3 * f + 2] = face[f].z;
            }
            // Volume: det J of the trilinear map summed over the 2x2x2 points
            // (+-0.5)^3 with unit weights (src/gel_kernels.cu:437-479).  With
            // x = (a0 + a1 s + a2 n + a3 t + a4 sn + a5 st + a6 nt + a7 snt) / 8,
            // where a_k is the sum of the corners signed by the corner's s, n, t
            // factors (a butterfly over the three index bits), J's columns are
            //   js = (a1 + n a4 + t a5 + nt a7) / 8, jn = (a2 + s a4 + t a6 + st a7) / 8,
            //   jt = (a3 + s a5 + n a6 + sn a7) / 8,
            // and the sum over s, n, t = +-h keeps only the terms even in each:
            //   sum det J = (8 / 512) [a1.(a2 x a3) + h^2 (a1.(a4 x a5) + a4.(a2 x a6) + a5.(a6 x a3))].
            double3 q[8];
_Pragma("unroll")
            for (int m = 0; m < 8; m++) q[m] = p[m];
_Pragma("unroll")
            for (int bit = 1; bit < 8; bit <<= 1) {
_Pragma("unroll")
                for (int m = 0; m < 8; m++) {
                    if (m & bit) continue;
                    const double3 lo = q[m], hi = q[m | bit];
                    q[m] = add(lo, hi);
                    q[m | bit] = sub(hi, lo);
                }
            }
            // q[4] = a1 (s), q[2] = a2 (n), q[1] = a3 (t), q[6] = a4 (sn), q[5] = a5 (st), q[3] = a6 (nt)
            const double3 a1 = q[4], a2 = q[2], a3 = q[1], a4 = q[6], a5 = q[5], a6 = q[3];
            const double vol = (8.0 / 512.0) * (dot(a1, crs(a2, a3)) + 0.25 * (dot(a1, crs(a4, a5)) +
                                                                                dot(a4, crs(a2, a6)) +
                                                                                dot(a5, crs(a6, a3))));
            G.vol[e] = vol;
            G.wmp[e] = G.wm[e];
            G.wm[e] = G.dx * G.dy * G.dz * G.FA0 / vol;
        }
        __syncthreads();
        double* rl = reinterpret_cast<double*>(G.rm_loc + 8 * (size_t)t0);
        for (int k = threadIdx.x; k < 24 * n_pass; k += blockDim.x) rl[k] = stage[kLocStride * (k / 24) + k % 24];
        const double* sf = stage + kLocStride * blockDim.x;
        double* nf = reinterpret_cast<double*>(G.nmSm + 6 * (size_t)t0);
        for (int k = threadIdx.x; k < 18 * n_pass; k += blockDim.x) nf[k] = sf[kFaceStride * (k / 18) + k % 18];
        __syncthreads();
    }
}

__device__ void ghost_nodes(const GelDev& G, const Idx& I) {
    GEL_FOR3(0, G.LX + 1, 0, G.LY + 1, 0, G.LZ + 1, {
        const int ox = inward(x, G.LX + 1), oy = inward(y, G.LY + 1), oz = inward(z, G.LZ + 1);
        if (ox | oy | oz) {
            const double3 r1 = G.rn[I.n(x + ox, y + oy, z + oz)];
            const double3 r2 = G.rn[I.n(x + 2 * ox, y + 2 * oy, z + 2 * oz)];
            G.rn[I.n(x, y, z)] = sub(mul(2.0, r1), r2);
        }
    })
}

// no-flux ghost elements + normalised concentrations; and the osmotic pressure
__device__ void chem_boundary_and_pressure(const GelDev& G, const Idx& I) {
    GEL_FOR3(0, G.LX, 0, G.LY, 0, G.LZ, {
        const int e = I.e(x, y, z);
        const int ox = inward(x, G.LX), oy = inward(y, G.LY), oz = inward(z, G.LZ);
        double u = G.um[e], v = G.vm[e];
        if (ox | oy | oz) {
            const int s = I.e(x + ox, y + oy, z + oz);
            u = G.um[s];
            v = G.vm[s];
            G.um[e] = u;
            G.vm[e] = v;
        }
        const double w = G.wm[e];
        G.um_norm[e] = u / (1 - w);
        G.vm_norm[e] = v / (1 - w);
        if (!(ox | oy | oz)) {
            // interior element: osmotic pressure (calPressureD)
            const double flory = -(w + log(1.0 - w) + (G.CH0 + G.CH1 * w) * w * w);
            if (G.type == 1)
                G.pm[e] = flory + G.C0 * w / (2.0 * G.FA0) + G.CHS * w * v;
            else if (G.type == 2)
                G.pm[e] = flory + (G.c0_bis + G.b * v) * w / (2.0 * G.FA0);
        }
    })
}

__device__ void node_averages(const GelDev& G, const Idx& I) {
    GEL_FOR3(1, G.LX, 1, G.LY, 1, G.LZ, {
        double su = 0, sv = 0;
_Pragma("unroll")
        for (int m = 0; m < 8; m++) {
            const int e = I.e(x - (m >> 2), y - ((m >> 1) & 1), z - (m & 1));
            su += G.um_norm[e];
            sv += G.vm_norm[e];
        }
        const int n = I.n(x, y, z);
        G.un_norm[n] = su / 8 + G.un_robin[n];
        G.vn_norm[n] = sv / 8;
    })
}

// nodal elastic + osmotic force, mobility, velocities; then setZero
__device__ void node_forces(const GelDev& G, const Idx& I, const GeomStage& gs) {
    GEL_FOR3(1, G.LX, 1, G.LY, 1, G.LZ, {
        const int n = I.n(x, y, z);
        double wn = 0;
_Pragma("unroll")
        for (int m = 0; m < 8; m++) wn += G.wm[I.e(x - (m >> 2), y - ((m >> 1) & 1), z - (m & 1))];
        wn /= 8;
        const double Mn = 8. * G.AZ0 * sqrt(G.FA0 / wn) * (1 - wn) / (G.dx * G.dy * G.dz);
        const double3 r0 = G.rn[n];
        double3 f1 = d3(0, 0, 0), f2 = d3(0, 0, 0);
        // the eight elements sharing the node: octant (a, b, c) in {+1,-1}^3
_Pragma("unroll")
        for (int o = 0; o < 8; o++) {
            const int a = (o & 4) ? -1 : 1, b = (o & 2) ? -1 : 1, c = (o & 1) ? -1 : 1;
            const bool ok = (a > 0 ? x < G.LX : x > 1) && (b > 0 ? y < G.LY : y > 1) && (c > 0 ? z < G.LZ : z > 1);
            if (!ok) continue;
            // spring term: the element's three face-diagonal and one body-diagonal
            // neighbours of the node, relative to the node
            const double3 s = add(add(G.rn[I.n(x + a, y + b, z + c)], G.rn[I.n(x, y + b, z + c)]),
                                  add(G.rn[I.n(x + a, y, z + c)], G.rn[I.n(x + a, y + b, z)]));
            f1 = add(f1, sub(s, mul(4.0, r0)));
            // osmotic term: pressure times the element's faces that meet at the node
            const int e = I.e(a > 0 ? x : x - 1, b > 0 ? y : y - 1, c > 0 ? z : z - 1);
            const double3 nf = add(add(gs.face(G, e, a > 0 ? 0 : 1), gs.face(G, e, b > 0 ? 2 : 3)),
                                   gs.face(G, e, c > 0 ? 4 : 5));
            f2 = add(f2, mul(G.pm[e], nf));
        }
        // the reference multiplies by pow(dx*dy*dz, 1/3) with an integer 1/3, i.e. by 1
        const double kel = (G.type == 2) ? (G.c0_bis + G.b * G.vn_norm[n] * (1 - wn)) / 12. : G.C0 / 12.;
        const double3 Fn = add(mul(kel, f1), mul(0.25, f2));
        const double3 Ve = mul(Mn, Fn);
        G.Fn[n] = Fn;
        G.Veln[n] = Ve;
        G.Vels[n] = mul(-wn / (1 - wn), Ve);
    })
}

// rn += dtx Veln (+ anchor of the bottom layer)
__device__ void advance(const GelDev& G, const Idx& I) {
    GEL_FOR3(1, G.LX, 1, G.LY, 1, G.LZ, {
        const int n = I.n(x, y, z);
        double3 r = add(G.rn[n], mul(G.dtx, G.Veln[n]));
        if (G.use_anchor && z == 1) {
            G.Veln[n] = d3(0, 0, 0);
            r.z = G.anchor_z;
        }
        G.rn[n] = r;
    })
}

__device__ void terms(const GelDev& G, const Idx& I, const GeomStage& gs) {
    GEL_FOR3(1, G.LX - 1, 1, G.LY - 1, 1, G.LZ - 1, {
        const int e = I.e(x, y, z);
        const double w = G.wm[e], u = G.um_norm[e];
        G.T0[e] = (1 - w / G.wmp[e]) / G.dtx;
        // T1: shape-function-weighted nodal flux dotted with the face vectors.
        // (The faces close the element, so this is round-off sized, as in the
        // reference's calTermsD.)
        double3 vu = d3(0, 0, 0);
_Pragma("unroll")
        for (int m = 0; m < 8; m++) {
            const int i = m >> 2, j = (m >> 1) & 1, k = m & 1;
            const double3 rl = gs.loc(G, e, m);
            const double N = 0.125 * (1 + (2 * i - 1) * rl.x) * (1 + (2 * j - 1) * rl.y) * (1 + (2 * k - 1) * rl.z);
            const int nn = I.n(x + i, y + j, z + k);
            vu = add(vu, mul(N * G.un_norm[nn], G.Veln[nn]));
        }
        double t1 = 0;
_Pragma("unroll")
        for (int f = 0; f < 6; f++) t1 += dot(gs.face(G, e, f), vu);
        G.T1[e] = t1 / G.vol[e];
        // T2: -grad w . grad u + (1 - w) lap u with three-point derivatives on
        // the deformed (non-uniform) element-centre grid
        const double3 rc = G.rm[e];
        double gg = 0, lap = 0;
_Pragma("unroll")
        for (int d = 0; d < 3; d++) {
            const int ep = I.e(x + (d == 0), y + (d == 1), z + (d == 2));
            const int em = I.e(x - (d == 0), y - (d == 1), z - (d == 2));
            const double hp = len(sub(G.rm[ep], rc)), hm = len(sub(G.rm[em], rc));
            const double den = hp * hm * (hp + hm);
            const double dw = (w * (hp * hp - hm * hm) + G.wm[ep] * hm * hm - G.wm[em] * hp * hp) / den;
            const double du = (u * (hp * hp - hm * hm) + G.um_norm[ep] * hm * hm - G.um_norm[em] * hp * hp) / den;
            gg += dw * du;
            lap += 2 * (G.um_norm[ep] * hm + G.um_norm[em] * hp - u * (hp + hm)) / den;
        }
        G.T2[e] = -gg + (1 - w) * lap;
    })
}

// ---------------------------------------------------------------------------
// per-iteration phases
// ---------------------------------------------------------------------------
__device__ void set_zero(const GelDev& G, const Idx& I) {
    GEL_FOR3(1, G.LX, 1, G.LY, 1, G.LZ, {
        const int n = I.n(x, y, z);
        G.un_robin[n] = 0;
        G.Fn_robin[n] = d3(0, 0, 0);
    })
}

__device__ void chemistry(const GelDev& G, const Idx& I) {
    GEL_FOR3(1, G.LX - 1, 1, G.LY - 1, 1, G.LZ - 1, {
        const int e = I.e(x, y, z);
        if (void_element(G, y, z)) {
            G.vm[e] = G.vss;
            G.um[e] = G.uss;
            G.wm[e] = G.wss;
        } else {
            const double v = G.vm[e], u = G.um[e], w = G.wm[e], t0 = G.T0[e];
            G.vm[e] = v + G.dt * (-v * t0 + G.ep * bz_fv(u, v, w));
            G.um[e] = u + G.dt * (-u * t0 + G.T1[e] + G.T2[e] + bz_fu(u, v, w, G.f));
        }
    })
}

// Gel::fireExcitationPulse (src/gel.cu:751-783): u above threshold, v low on
// the first tenth of the gel along x
__device__ void fire_pulse(const GelDev& G, const Idx& I) {
    const int pw = max(1, G.LX / 10);
    GEL_FOR3(1, pw, 1, G.LY, 1, G.LZ, {
        if (!void_element(G, y, z)) {
            const int e = I.e(x, y, z);
            G.um[e] = G.uss * 3.0;
            G.vm[e] = G.vss * 0.1;
        }
    })
}

__device__ void record_center(const GelDev& G, const Idx& I, int iter) {
    if (threadIdx.x != 0 || !G.series || G.series_every <= 0 || iter % G.series_every) return;
    const int slot = (iter / G.series_every) % G.series_cap;
    double* r = G.series + 12 * (long long)slot;
    const int e = I.e(G.LX / 2, G.LY / 2, G.LZ / 2);
    const int n = I.n((G.LX + 1) / 2, (G.LY + 1) / 2, (G.LZ + 1) / 2);
    const double3 rn = G.rn[n], Fn = G.Fn[n], Ve = G.Veln[n];
    r[0] = iter;
    r[1] = rn.x;  // node position (the reference's "rm_center" holds rn)
    r[2] = rn.y;
    r[3] = rn.z;
    r[4] = Fn.x;
    r[5] = Fn.y;
    r[6] = Fn.z;
    r[7] = Ve.x;
    r[8] = Ve.y;
    r[9] = Ve.z;
    r[10] = G.vm[e];
    r[11] = G.wm[e];
}

// k_gather_boundary + the per-iteration stencil cache and the force-region box
__device__ void gather(const GelDev& G, const GelArgs& a, int gel_index, int* s_box) {
    const MarkerDev& Mk = a.Mk;
    if (threadIdx.x < 6) s_box[threadIdx.x] = (threadIdx.x & 1) ? -1 : 0x7fffffff;
    __syncthreads();
    for (int j = threadIdx.x; j < G.M; j += blockDim.x) {
        const int l = G.marker_off + j;
        const int id = G.bIndex[j];
        const double3 r = G.rn[id], v = G.Vels[id];
        const float4 lag = make_float4(__double2float_rn(r.x), __double2float_rn(r.y), __double2float_rn(r.z), 0.f);
        Mk.lag[l] = lag;
        Mk.Vl[l] = make_float4(__double2float_rn(v.x * (double)a.g2l), __double2float_rn(v.y * (double)a.g2l),
                               __double2float_rn(v.z * (double)a.g2l), 0.f);
        Mk.Cl[l] = __double2float_rn(G.un_norm[id]);
        // delta-4 stencil of the marker, clipped at the lattice
        const float g[3] = {lag.x / a.h, lag.y / a.h, lag.z / a.h};
        const int n[3] = {a.nx, a.ny, a.nz};
        int b0[3], valid = 0;
        float ph[3][4];
        const unsigned act = __activemask();
        const bool leader = (threadIdx.x & 31) == __ffs(act) - 1;
_Pragma("unroll")
        for (int d = 0; d < 3; d++) {
            const int ic = (int)floorf(g[d]);
            b0[d] = ic - 1;
            int lo = 0x7fffffff, hi = -1;
_Pragma("unroll")
            for (int k = 0; k < 4; k++) {
                const int cc = ic - 1 + k;
                const bool in = cc >= 0 && cc < n[d];
                ph[d][k] = in ? delta4f(g[d] - (float)cc) : 0.f;
                if (in) {
                    valid |= 1 << (4 * d + k);
                    lo = min(lo, cc);
                    hi = max(hi, cc);
                }
            }
            // the warp's extent first, then one shared atomic per warp
            lo = __reduce_min_sync(act, lo);
            hi = __reduce_max_sync(act, hi);
            if (leader && hi >= 0) {
                atomicMin(&s_box[2 * d], lo);
                atomicMax(&s_box[2 * d + 1], hi);
            }
        }
        float ws = 0.f;
        for (int i = 0; i < 4; i++)
            for (int jj = 0; jj < 4; jj++)
                for (int k = 0; k < 4; k++)
                    if (((valid >> i) & 1) && ((valid >> (4 + jj)) & 1) && ((valid >> (8 + k)) & 1))
                        ws += ph[0][i] * ph[1][jj] * ph[2][k];
        Mk.base[l] = make_int4(b0[0], b0[1], b0[2], valid);
        Mk.phx[l] = make_float4(ph[0][0], ph[0][1], ph[0][2], ph[0][3]);
        Mk.phy[l] = make_float4(ph[1][0], ph[1][1], ph[1][2], ph[1][3]);
        Mk.phz[l] = make_float4(ph[2][0], ph[2][1], ph[2][2], ph[2][3]);
        Mk.wsum[l] = ws;
        if (ws == 0.f) atomicOr(&a.ctl->error, kErrMarkerOut);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Box b;
        b.x0 = s_box[0];
        b.x1 = s_box[1];
        b.y0 = s_box[2];
        b.y1 = s_box[3];
        b.z0 = s_box[4];
        b.z1 = s_box[5];
        if (b.x1 < 0 || b.y1 < 0 || b.z1 < 0) b = Box{1, 0, 1, 0, 1, 0};
        Mk.boxes[gel_index] = b;
    }
}

// every phase of one gel, run by one CTA
__device__ void gel_run(const GelArgs& a, int gel_index, int* s_box, double* stage) {
    const GelDev& G = a.gels[gel_index];
    const Idx I{G.LX, G.LY};
    const int iter = a.iter_arg >= 0 ? a.iter_arg : a.ctl->iter;
    bool active = true, moved = false;
    if ((a.phases & kPhAuto) && G.active_from > 0) {
        if (iter == G.active_from) {
            fire_pulse(G, I);
            __syncthreads();
        }
        active = iter >= G.active_from;
    }
    if ((a.phases & kPhElastic) && active) {
        if (iter % 5 == 0) {
            moved = true;
            ghost_nodes(G, I);
            __syncthreads();
            element_geometry(G, I, stage);
            chem_boundary_and_pressure(G, I);
            __syncthreads();
            node_averages(G, I);
            __syncthreads();
            node_forces(G, I, geom_stage(G, stage));
            __syncthreads();
            advance(G, I);
            __syncthreads();  // the anchor zeroes Veln before calTermsD reads it
            terms(G, I, geom_stage(G, stage));
            __syncthreads();
        }
        // no barrier: nothing after it in this launch reads the Robin fields it
        // clears, and the chemistry's element loads overlap its node stores
        set_zero(G, I);
    }
    if ((a.phases & kPhChem) && active) {
        chemistry(G, I);
        __syncthreads();
    }
    if (a.phases & kPhRecord) {
        record_center(G, I, iter);
        __syncthreads();
    }
    if (a.phases & kPhGather) {
        if (!(a.phases & kPhGatherStale)) {
            gather(G, a, gel_index, s_box);
        } else if (moved || !a.gather_fresh[gel_index]) {
            gather(G, a, gel_index, s_box);  // every thread read the flag before its barriers
            if (threadIdx.x == 0) a.gather_fresh[gel_index] = 1;
        }
    }
}

__global__ void __launch_bounds__(kGelThreads) gel_kernel(GelArgs a) {
    __shared__ int s_box[6];
    extern __shared__ double stage[];  // kGelStageBytes
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < a.n_zero_words; i += blockDim.x) a.zero_words[i] = 0u;
    gel_run(a, blockIdx.x + a.first_gel, s_box, stage);
}

// batched: CTA b runs gel entries[b].first_gel of the system described by entries[b]
__global__ void __launch_bounds__(kGelThreads) gel_batch_kernel(const GelArgs* entries, int n) {
    __shared__ int s_box[6];
    if ((int)blockIdx.x >= n) return;
    const GelArgs& a = entries[blockIdx.x];
    if (a.dyn && a.dyn->remaining == 0) return;
    extern __shared__ double stage[];  // kGelStageBytes
    gel_run(a, a.first_gel, s_box, stage);
}

// ---------------------------------------------------------------------------
// concentration exchange at the markers (one warp per marker)
// ---------------------------------------------------------------------------
// one warp: marker l of the system described by a
__device__ void conc_marker(const MarkerArgs& a, int l) {
    const int lane = threadIdx.x & 31;
    const MarkerDev& Mk = a.Mk;
    if (l >= Mk.M) return;
    const int4 b = Mk.base[l];
    const float4 ph[3] = {Mk.phx[l], Mk.phy[l], Mk.phz[l]};
    const float ws = Mk.wsum[l];
    const long long nx = a.nx, nxy = (long long)a.nx * a.ny;
    float s = 0.f, w[2];
    long long cell[2];
    bool ok[2];
_Pragma("unroll")
    for (int j = 0; j < 2; j++) {
        const int p = lane + 32 * j;
        const int ax = p >> 4, ay = (p >> 2) & 3, az = p & 3;
        ok[j] = ((b.w >> ax) & 1) && ((b.w >> (4 + ay)) & 1) && ((b.w >> (8 + az)) & 1);
        const float px = ax == 0 ? ph[0].x : ax == 1 ? ph[0].y : ax == 2 ? ph[0].z : ph[0].w;
        const float py = ay == 0 ? ph[1].x : ay == 1 ? ph[1].y : ay == 2 ? ph[1].z : ph[1].w;
        const float pz = az == 0 ? ph[2].x : az == 1 ? ph[2].y : az == 2 ? ph[2].z : ph[2].w;
        w[j] = px * py * pz;
        cell[j] = (long long)(b.x + ax) + (long long)(b.y + ay) * nx + (long long)(b.z + az) * nxy;
        if (ok[j]) s += a.c[cell[j]] * w[j];
    }
_Pragma("unroll")
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const float Dl = ws > 0.f ? s / ws : 0.f;
    const float Sl = 1.0f * (Mk.Cl[l] - Dl);
    if (lane == 0) {
        Mk.Dl[l] = Dl;
        Mk.Sl[l] = Sl;
        if (a.scatter) {
            const GelDev& G = a.gels[Mk.owner[l]];
            G.un_robin[G.bIndex[l - G.marker_off]] -= (double)Sl;
        }
    }
    if (ws == 0.f || a.det) return;
    const float inv_h3 = 1.0f / (a.h * a.h * a.h);
    const float scale = inv_h3 / ws;
_Pragma("unroll")
    for (int j = 0; j < 2; j++)
        if (ok[j]) atomicAdd(&a.source[cell[j]], Sl * (w[j] * scale));
}

__global__ void __launch_bounds__(256) conc_markers_kernel(MarkerArgs a) {
    conc_marker(a, blockIdx.x * 8 + (threadIdx.x >> 5));
}

// batched: warp w belongs to the system whose [first, next) warp range holds it;
// pairs[2 s + c] are system s's arguments with concentration buffer c, and
// dyn[s].cur selects the current one
__global__ void __launch_bounds__(256) conc_markers_batch_kernel(const MarkerArgs* pairs, const SysDyn* dyn,
                                                                 const int* warp_offsets, int n) {
    const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (n <= 0 || w >= warp_offsets[n]) return;
    int lo = 0, hi = n;  // last system with warp_offsets[s] <= w
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (warp_offsets[mid] <= w) lo = mid; else hi = mid;
    }
    if (dyn[lo].remaining == 0) return;
    conc_marker(pairs[2 * lo + dyn[lo].cur], w - warp_offsets[lo]);
}

// ---------------------------------------------------------------------------
// repulsion between markers of different gels: one warp per marker, the lanes
// striding over the other markers, then a tree reduction
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// the LJ force of marker j on marker i, added to f when within the cut-off
__device__ __forceinline__ void lj_pair(const RepulsionArgs& a, float4 pi, float4 pj, float rc2, float sig2, float& fx,
                                        float& fy, float& fz) {
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 <= 0.0f || r2 >= rc2) return;
    const float inv = 1.0f / r2, sr2 = sig2 * inv, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
    const float fac = 24.0f * a.delta * (2.0f * sr12 - sr6) * inv;
    fx += fac * dx;
    fy += fac * dy;
    fz += fac * dz;
}

// marker i of the system described by a (k_gel_repulsion, src/coupling_kernels.cu:90-146).
// With the marker boxes known (h > 0), a gel is visited only when marker i lies
// within the cut-off of its box (the union of its markers' stencils, which
// holds every one of its markers): the same pairs, without the far gels' markers.
__device__ void repulsion_marker(const RepulsionArgs& a, int i) {
    const MarkerDev& Mk = a.Mk;
    const int M = Mk.M, lane = threadIdx.x & 31;
    const float rcut = 2.5f * a.gamma, rc2 = rcut * rcut, sig2 = a.gamma * a.gamma;
    const float4 pi = Mk.lag[i];
    const int oi = Mk.owner[i];
    float fx = 0.f, fy = 0.f, fz = 0.f;
    if (a.h > 0.0f) {
        for (int g = 0; g < a.n_gels; g++) {
            if (g == oi) continue;
            const Box b = Mk.boxes[g];
            if (b.x0 > b.x1) continue;
            if (pi.x < b.x0 * a.h - rcut || pi.x > (b.x1 + 1) * a.h + rcut || pi.y < b.y0 * a.h - rcut ||
                pi.y > (b.y1 + 1) * a.h + rcut || pi.z < b.z0 * a.h - rcut || pi.z > (b.z1 + 1) * a.h + rcut)
                continue;
            const int2 r = Mk.gel_range[g];
            for (int j = r.x + lane; j < r.y; j += 32) lj_pair(a, pi, Mk.lag[j], rc2, sig2, fx, fy, fz);
        }
    } else {
        for (int j = lane; j < M; j += 32)
            if (Mk.owner[j] != oi) lj_pair(a, pi, Mk.lag[j], rc2, sig2, fx, fy, fz);
    }
    fx = warp_sum_f(fx);
    fy = warp_sum_f(fy);
    fz = warp_sum_f(fz);
    if (lane == 0) {
        Mk.Frep[i] = make_float4(fx, fy, fz, 0.f);
        if (a.scatter) {
            const GelDev& G = a.gels[oi];
            double3& f = G.Fn_robin[G.bIndex[i - G.marker_off]];
            f.x -= (double)fx;
            f.y -= (double)fy;
            f.z -= (double)fz;
        }
    }
}

__global__ void __launch_bounds__(256) repulsion_kernel(RepulsionArgs a) {
    const int i = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (i < a.Mk.M) repulsion_marker(a, i);
}

// batched: warp w belongs to the system whose [first, next) marker range holds it
__global__ void __launch_bounds__(256) repulsion_batch_kernel(const RepulsionArgs* systems, const int* warp_offsets,
                                                              int n) {
    const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (n <= 0 || w >= warp_offsets[n]) return;
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (warp_offsets[mid] <= w) lo = mid; else hi = mid;
    }
    if (!(systems[lo].dyn && systems[lo].dyn->remaining == 0)) repulsion_marker(systems[lo], w - warp_offsets[lo]);
}

// Coupler::scatterToGels: un_robin -= Sl and Fn_robin -= Frep at each marker's node
__global__ void scatter_kernel(GelDev* gels, MarkerDev Mk) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= Mk.M) return;
    const GelDev& G = gels[Mk.owner[l]];
    const int id = G.bIndex[l - G.marker_off];
    const float4 fr = Mk.Frep[l];
    G.Fn_robin[id].x -= (double)fr.x;
    G.Fn_robin[id].y -= (double)fr.y;
    G.Fn_robin[id].z -= (double)fr.z;
    G.un_robin[id] -= (double)Mk.Sl[l];
}

// ---------------------------------------------------------------------------
// the gel kernels' stage exceeds the default 48 KB of dynamic shared memory:
// raise their limit once per device
static cudaError_t gel_smem_limit() {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load() & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(gel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGelStageBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(gel_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGelStageBytes);
    if (e == cudaSuccess) done.fetch_or(bit);
    return e;
}

cudaError_t launch_gel(const GelArgs& a, int n_gels, cudaStream_t s) {
    if (n_gels <= 0) return cudaSuccess;
    cudaError_t e = gel_smem_limit();
    if (e != cudaSuccess) return e;
    gel_kernel<<<n_gels, kGelThreads, kGelStageBytes, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_conc_markers(const MarkerArgs& a, cudaStream_t s) {
    if (a.Mk.M <= 0) return cudaSuccess;
    conc_markers_kernel<<<(a.Mk.M + 7) / 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_repulsion(const RepulsionArgs& a, cudaStream_t s) {
    if (a.Mk.M <= 0) return cudaSuccess;
    repulsion_kernel<<<(a.Mk.M + 7) / 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_gel_batch(const GelArgs* entries, int n, int grid, cudaStream_t s) {
    if (grid <= 0) return cudaSuccess;
    cudaError_t e = gel_smem_limit();
    if (e != cudaSuccess) return e;
    gel_batch_kernel<<<grid, kGelThreads, kGelStageBytes, s>>>(entries, n);
    return cudaGetLastError();
}

cudaError_t launch_conc_markers_batch(const MarkerArgs* pairs, const SysDyn* dyn, const int* warp_offsets, int n,
                                      int warps, cudaStream_t s) {
    if (warps <= 0) return cudaSuccess;
    conc_markers_batch_kernel<<<(warps + 7) / 8, 256, 0, s>>>(pairs, dyn, warp_offsets, n);
    return cudaGetLastError();
}

cudaError_t launch_repulsion_batch(const RepulsionArgs* systems, const int* warp_offsets, int n, int warps,
                                   cudaStream_t s) {
    if (warps <= 0) return cudaSuccess;
    repulsion_batch_kernel<<<(warps + 7) / 8, 256, 0, s>>>(systems, warp_offsets, n);
    return cudaGetLastError();
}

cudaError_t launch_scatter(GelDev* gels, const MarkerDev& Mk, cudaStream_t s) {
    if (Mk.M <= 0) return cudaSuccess;
    scatter_kernel<<<(Mk.M + 255) / 256, 256, 0, s>>>(gels, Mk);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// filament (iso-line) diagnostic, calFilamentD (src/gel_kernels.cu:837-866)
// ---------------------------------------------------------------------------
// The point (xb, yb) in the unit square where the bilinear interpolants of
// u (corners A B / C D) and of v (E F / G H) both equal viso, if there is one:
// u - viso = a00 + a10 x + a01 y + a11 x y, likewise v; eliminating y leaves
// c2 x^2 + c1 x + c0 = 0 (solveBilinear, src/gel_kernels.cu:165-212, with its
// tolerance 1e-12 and its order of root trials).
__device__ bool iso_crossing(double A, double B, double C, double D, double E, double Fv, double G, double H,
                             double viso, double& xb, double& yb) {
    const double eps = 1e-12;
    const double a00 = A - viso, a10 = B - A, a01 = C - A, a11 = A - B + D - C;
    const double b00 = E - viso, b10 = Fv - E, b01 = G - E, b11 = E - Fv + H - G;
    const double c2 = b10 * a11 - b11 * a10;
    const double c1 = b00 * a11 + b10 * a01 - b01 * a10 - b11 * a00;
    const double c0 = b00 * a01 - b01 * a00;
    double r[2];
    int n = 0;
    if (fabs(c2) < eps) {
        if (fabs(c1) < eps) return false;
        r[n++] = -c0 / c1;
    } else {
        const double disc = c1 * c1 - 4.0 * c2 * c0;
        if (disc < 0.0) return false;
        const double sq = sqrt(disc);
        r[n++] = (-c1 + sq) / (2.0 * c2);
        r[n++] = (-c1 - sq) / (2.0 * c2);
    }
    for (int i = 0; i < n; i++) {
        const double x = r[i];
        if (x < -eps || x > 1.0 + eps) continue;
        const double den = a01 + a11 * x;
        if (fabs(den) < eps) continue;
        const double y = -(a00 + a10 * x) / den;
        if (y < -eps || y > 1.0 + eps) continue;
        xb = fmin(fmax(x, 0.0), 1.0);
        yb = fmin(fmax(y, 0.0), 1.0);
        return true;
    }
    return false;
}

// one thread per node face (xi, yi, zi), xi in [1, LX-1] etc.: out[face] =
// (1, xi + xb, yi + yb, zi) where the u_norm = v_norm = 0.15 crossing lies,
// else (0, 0, 0, 0); faces in x-fastest order
__global__ void filament_kernel(GelDev G, double4* out) {
    const int fx = G.LX - 1, fy = G.LY - 1, fz = G.LZ - 1;
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= (long long)fx * fy * fz) return;
    const int xi = 1 + (int)(f % fx), yi = 1 + (int)((f / fx) % fy), zi = 1 + (int)(f / ((long long)fx * fy));
    const int sx = G.LX + 2, sxy = (G.LX + 2) * (G.LY + 2);
    const int n00 = xi + yi * sx + zi * sxy, n10 = n00 + 1, n01 = n00 + sx, n11 = n01 + 1;
    double xb = 0.0, yb = 0.0;
    const bool ok = iso_crossing(G.un_norm[n00], G.un_norm[n10], G.un_norm[n01], G.un_norm[n11], G.vn_norm[n00],
                                 G.vn_norm[n10], G.vn_norm[n01], G.vn_norm[n11], 0.15, xb, yb);
    out[f] = ok ? make_double4(1.0, xi + xb, yi + yb, (double)zi) : make_double4(0.0, 0.0, 0.0, 0.0);
}

cudaError_t launch_filament(const GelDev& G, double4* out, cudaStream_t s) {
    const long long faces = (long long)(G.LX - 1) * (G.LY - 1) * (G.LZ - 1);
    if (faces <= 0) return cudaSuccess;
    filament_kernel<<<(unsigned)((faces + 255) / 256), 256, 0, s>>>(G, out);
    return cudaGetLastError();
}

}  // namespace glsm
