// lbm.cu -- the fluid side of one coupled iteration on sm_100a:
//   * lbm_substep_kernel: one LBM substep = IBM (interpolate, penalty force,
//     spread) + BGK/Guo collide + stream with half-way bounce-back, in place
//     (AA pattern), populations stored as deviations from the rest weights.
//   * conv_diff_kernel: upwind advection-diffusion of the concentration.
//   * read_pop_kernel: populations back in the reference's natural layout.
//
// Reference semantics followed (lasite/gLSM_fluid_3D):
//   Fluid::stepVelocity           src/fluid.cu:263-284 (substep order, IBM ramp)
//   k_ibm_interpolate_velocity    src/fluid_kernels.cu:244-281
//   k_scale_negbeta               src/fluid_kernels.cu:283-291
//   k_ibm_spread_forces           src/fluid_kernels.cu:300-348
//   k_macros / k_collide          src/fluid_kernels.cu:98-111, :125-142
//   k_stream_bounce               src/fluid_kernels.cu:144-165
//   k_convection_diffusion        src/fluid_kernels.cu:177-242
#include <algorithm>
#include <cuda_bf16.h>
#include <cstdlib>
#include <cuda_fp16.h>

#include "d3q19.cuh"
#include "fastdiv.h"
#include "glsm_internal.h"
#include "lbm.h"

namespace glsm {

// ---------------------------------------------------------------------------
// population storage: FP32 deviations, or FP16 / BF16 deviations (scaled)
// ---------------------------------------------------------------------------
// FP16 storage with the conserving rounding of conserve_round: a template
// value of the substep kernels only (the fluid's storage stays kStoreF16 and
// FluidDev::f16_round selects these instantiations)
constexpr int kStoreF16C = 3;

// whether a substep of this parity rounds conservingly under FP16 rounding
// mode f16_round (0 nearest, 1 every substep, 2 odd substeps only)
__host__ __device__ constexpr bool f16_conserving(int f16_round, int parity) {
    return f16_round == 1 || (f16_round == 2 && parity != 0);
}

// FP32 population loads carry an L2 prefetch-size hint of one 128-byte line
// (PTX ld.global.L2::128B): measured +1.3% coupled MLUPS at 101^3 (on the 16-bit
// storages the hint cost 0.7% (FP16) and 1.9% (BF16), so their loads stay
// plain).  The asm reads memory ("memory" clobber), so no store of the same
// cell's slots is moved across it.
__device__ __forceinline__ float ld_pop(const float* p) {
    float v;
    asm volatile("ld.global.L2::128B.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}

template <int ST>
struct PopIO;
template <>
struct PopIO<kStoreF32> {
    using T = float;
    static constexpr bool kScaled = false;
    static constexpr bool kConserve = false;
    static __device__ __forceinline__ float ld(const T* p, float) { return ld_pop(p); }
    static __device__ __forceinline__ void st(T* p, float v, float) { *p = v; }
    static __device__ __forceinline__ float raw(const T* p) { return ld_pop(p); }
    static __device__ __forceinline__ void st_raw(T* p, float v) { *p = v; }
};
template <>
struct PopIO<kStoreF16> {
    using T = __half;
    static constexpr bool kScaled = true;  // stored value = deviation * scale
    static constexpr bool kConserve = false;
    static __device__ __forceinline__ float ld(const T* p, float inv_scale) { return __half2float(*p) * inv_scale; }
    static __device__ __forceinline__ void st(T* p, float v, float scale) { *p = __float2half_rn(v * scale); }
    static __device__ __forceinline__ float raw(const T* p) { return __half2float(*p); }
    static __device__ __forceinline__ void st_raw(T* p, float v) { *p = __float2half_rn(v); }
};
template <>
struct PopIO<kStoreBF16> {
    using T = __nv_bfloat16;
    static __device__ __forceinline__ float ld(const T* p, float inv_scale) {
        return __bfloat162float(*p) * inv_scale;
    }
    static __device__ __forceinline__ void st(T* p, float v, float scale) { *p = __float2bfloat16_rn(v * scale); }
    static constexpr bool kScaled = false;  // stored unscaled
    static constexpr bool kConserve = false;
    static __device__ __forceinline__ float raw(const T* p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ void st_raw(T* p, float v) { *p = __float2bfloat16_rn(v); }
};

template <>
struct PopIO<kStoreF16C> : PopIO<kStoreF16> {
    static constexpr bool kConserve = true;
};

// Two adjacent cells' populations of one direction as one vector (the even
// cell in the low half); S and the pair's first cell are even, so the vector
// is aligned.
template <int ST>
struct PairIO;
template <>
struct PairIO<kStoreF32> {
    using V = float2;
    static __device__ __forceinline__ float lo(V v) { return v.x; }
    static __device__ __forceinline__ float hi(V v) { return v.y; }
    static __device__ __forceinline__ V set_lo(V v, float f) { return make_float2(f, v.y); }
    static __device__ __forceinline__ V set_hi(V v, float f) { return make_float2(v.x, f); }
};
template <>
struct PairIO<kStoreF16> {
    using V = __half2;
    static __device__ __forceinline__ float lo(V v) { return __low2float(v); }
    static __device__ __forceinline__ float hi(V v) { return __high2float(v); }
    static __device__ __forceinline__ V set_lo(V v, float f) { return __halves2half2(__float2half_rn(f), __high2half(v)); }
    static __device__ __forceinline__ V set_hi(V v, float f) { return __halves2half2(__low2half(v), __float2half_rn(f)); }
    static __device__ __forceinline__ __half lo_raw(V v) { return __low2half(v); }
    static __device__ __forceinline__ __half hi_raw(V v) { return __high2half(v); }
    static __device__ __forceinline__ V make(__half a, __half b) { return __halves2half2(a, b); }
    static __device__ __forceinline__ V set_lo_raw(V v, __half a) { return __halves2half2(a, __high2half(v)); }
    static __device__ __forceinline__ V set_hi_raw(V v, __half b) { return __halves2half2(__low2half(v), b); }
};
template <>
struct PairIO<kStoreBF16> {
    using V = __nv_bfloat162;
    static __device__ __forceinline__ float lo(V v) { return __low2float(v); }
    static __device__ __forceinline__ float hi(V v) { return __high2float(v); }
    static __device__ __forceinline__ V set_lo(V v, float f) {
        return __halves2bfloat162(__float2bfloat16_rn(f), __high2bfloat16(v));
    }
    static __device__ __forceinline__ V set_hi(V v, float f) {
        return __halves2bfloat162(__low2bfloat16(v), __float2bfloat16_rn(f));
    }
    static __device__ __forceinline__ __nv_bfloat16 lo_raw(V v) { return __low2bfloat16(v); }
    static __device__ __forceinline__ __nv_bfloat16 hi_raw(V v) { return __high2bfloat16(v); }
    static __device__ __forceinline__ V make(__nv_bfloat16 a, __nv_bfloat16 b) { return __halves2bfloat162(a, b); }
    static __device__ __forceinline__ V set_lo_raw(V v, __nv_bfloat16 a) { return __halves2bfloat162(a, __high2bfloat16(v)); }
    static __device__ __forceinline__ V set_hi_raw(V v, __nv_bfloat16 b) { return __halves2bfloat162(__low2bfloat16(v), b); }
};
template <>
struct PairIO<kStoreF16C> : PairIO<kStoreF16> {};

__device__ __forceinline__ int current_iter(int iter_arg, const Ctl* ctl) {
    return iter_arg >= 0 ? iter_arg : ctl->iter;
}

// IBM penalty ramp of Fluid::stepVelocity (src/fluid.cu:265-270), float arithmetic
__device__ __forceinline__ float beta_eff(float beta, float ramp_steps, int iter) {
    float ramp = (ramp_steps <= 0.0f) ? 1.0f : fminf(1.0f, (float)(iter + 1) / ramp_steps);
    return beta * ramp;
}

__device__ __forceinline__ float comp4(const float4& v, int a) {
    return a == 0 ? v.x : (a == 1 ? v.y : (a == 2 ? v.z : v.w));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Tile extent (inclusive cell ranges per axis, conservative) of the linear cell
// range [c0, c1].
struct TileExt {
    int x0, x1, y0, y1, z0, z1;
};
__device__ __forceinline__ TileExt tile_extent(unsigned c0, unsigned c1, unsigned nx, unsigned ny,
                                               const FastDiv& dnx, const FastDiv& dnxy) {
    const unsigned nxy = nx * ny;
    TileExt e;
    e.z0 = (int)fdiv(c0, dnxy);
    e.z1 = (int)fdiv(c1, dnxy);
    if (e.z0 != e.z1) {
        e.y0 = 0;
        e.y1 = ny - 1;
        e.x0 = 0;
        e.x1 = nx - 1;
        return e;
    }
    const unsigned r0 = c0 - (unsigned)e.z0 * nxy, r1 = c1 - (unsigned)e.z0 * nxy;
    e.y0 = (int)fdiv(r0, dnx);
    e.y1 = (int)fdiv(r1, dnx);
    if (e.y0 != e.y1) {
        e.x0 = 0;
        e.x1 = nx - 1;
    } else {
        e.x0 = (int)(r0 - (unsigned)e.y0 * nx);
        e.x1 = (int)(r1 - (unsigned)e.y0 * nx);
    }
    return e;
}

__device__ __forceinline__ bool overlaps(const Box& b, const TileExt& e) {
    return b.x0 <= e.x1 && b.x1 >= e.x0 && b.y0 <= e.y1 && b.y1 >= e.y0 && b.z0 <= e.z1 && b.z1 >= e.z0;
}
__device__ __forceinline__ bool inside(const Box& b, int x, int y, int z) {
    return x >= b.x0 && x <= b.x1 && y >= b.y0 && y <= b.y1 && z >= b.z0 && z <= b.z1;
}

// Collect into shared memory, in box (gel) order, the marker boxes that overlap
// this CTA's tile and their gel indices.  Returns the count (all threads).
// Uses one __syncthreads().
__device__ __forceinline__ int tile_boxes(const Box* boxes, int n_boxes, const TileExt& e, Box* s_b, int* s_g,
                                          int* s_nb) {
    if (threadIdx.x < 32) {
        const unsigned lane = threadIdx.x;
        int nb = 0;
        for (int j0 = 0; j0 < n_boxes; j0 += 32) {
            const int j = j0 + (int)lane;
            Box b{1, 0, 1, 0, 1, 0};
            bool hit = false;
            if (j < n_boxes) {
                b = boxes[j];
                hit = b.x0 <= b.x1 && overlaps(b, e);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                const int k = nb + __popc(m & ((1u << lane) - 1u));
                s_b[k] = b;
                s_g[k] = j;
            }
            nb += __popc(m);
        }
        if (lane == 0) *s_nb = nb;
    }
    __syncthreads();
    return *s_nb;
}

// Deterministic form of the spreads: the sum at cell (x, y, z) of the values of
// gel g's markers (in marker order) whose clipped 4x4x4 stencil covers the cell,
// each times its delta-4 weight there and 1/(h^3 sum w) -- what the atomic
// spreads (k_ibm_spread_forces, src/fluid_kernels.cu:300-348, and
// k_ibm_spread_concentration, :414-459) add to the cell, in a fixed order.
// CONC: the concentration source Sl (scalar, in .x); else the IBM force Fdrag.
template <bool CONC>
__device__ __forceinline__ void det_gather(const MarkerDev& Mk, int g, int x, int y, int z, float inv_h3, float4& acc) {
    const int2 r = Mk.gel_range[g];
    for (int l = r.x; l < r.y; l++) {
        const int4 b = __ldg(&Mk.base[l]);
        const unsigned ax = (unsigned)(x - b.x), ay = (unsigned)(y - b.y), az = (unsigned)(z - b.z);
        if (ax > 3u || ay > 3u || az > 3u) continue;
        if (!(((b.w >> ax) & 1) && ((b.w >> (4 + ay)) & 1) && ((b.w >> (8 + az)) & 1))) continue;
        const float ws = __ldg(&Mk.wsum[l]);
        if (ws == 0.0f) continue;
        const float w = comp4(__ldg(&Mk.phx[l]), (int)ax) * comp4(__ldg(&Mk.phy[l]), (int)ay) *
                        comp4(__ldg(&Mk.phz[l]), (int)az);
        const float wg = w * (inv_h3 / ws);
        if (CONC) {
            acc.x += __ldcg(&Mk.Sl[l]) * wg;
        } else {
            const float4 fd = __ldcg(&Mk.Fdrag[l]);
            acc.x += fd.x * wg;
            acc.y += fd.y * wg;
            acc.z += fd.z * wg;
        }
    }
}

// ---------------------------------------------------------------------------
// IBM task: one warp per marker.  Lane j owns stencil points j and j+32 of
// the 4x4x4 stencil (point p = ax*16 + ay*4 + az, x outermost as in the
// reference loops).  Interpolates u of the previous substep, forms the penalty
// force beta_eff (Vl - Ul) and spreads it with vector float atomics.
// ---------------------------------------------------------------------------
// IBM interpolation and spreading of marker l by one warp
__device__ __forceinline__ void ibm_marker(const StepArgs& a, int l) {
    const int lane = threadIdx.x & 31;
    const FluidDev& F = a.F;
    const MarkerDev& Mk = a.Mk;
    {
        const float be = beta_eff(F.beta, F.ramp_steps, current_iter(a.iter_arg, a.ctl));
        const int4 b = Mk.base[l];
        const float4 px = Mk.phx[l], py = Mk.phy[l], pz = Mk.phz[l];
        const float ws = Mk.wsum[l];
        const long long nx = F.nx, nxy = (long long)F.nx * F.ny;
        float sx = 0.f, sy = 0.f, sz = 0.f;
        long long cell[2];
        float w[2];
        bool ok[2];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int p = lane + 32 * j;
            const int ax = p >> 4, ay = (p >> 2) & 3, az = p & 3;
            ok[j] = ((b.w >> ax) & 1) && ((b.w >> (4 + ay)) & 1) && ((b.w >> (8 + az)) & 1);
            w[j] = comp4(px, ax) * comp4(py, ay) * comp4(pz, az);
            cell[j] = (long long)(b.x + ax) + (long long)(b.y + ay) * nx + (long long)(b.z + az) * nxy;
            if (ok[j]) {
                const float4 uu = F.u[cell[j]];
                sx += uu.x * w[j];
                sy += uu.y * w[j];
                sz += uu.z * w[j];
            }
        }
        sx = warp_sum(sx);
        sy = warp_sum(sy);
        sz = warp_sum(sz);
        float4 Ul = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ws > 0.0f) Ul = make_float4(sx / ws, sy / ws, sz / ws, 0.f);
        const float4 Vl = Mk.Vl[l];
        const float4 Fd = make_float4(be * (Vl.x - Ul.x), be * (Vl.y - Ul.y), be * (Vl.z - Ul.z), 0.f);
        if (lane == 0) {
            Mk.Ul[l] = Ul;
            Mk.Fdrag[l] = Fd;
        }
        if (ws != 0.0f && !F.det_spread) {
            const float inv_h3 = (float)(1.0 / (double)(F.h * F.h * F.h));
            const float scale = inv_h3 / ws;
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (!ok[j]) continue;
                const float wg = w[j] * scale;
                atomicAdd(&F.Fibm[cell[j]], make_float4(Fd.x * wg, Fd.y * wg, Fd.z * wg, 0.f));
            }
        }
    }
}

// one IBM task of a CTA: kMarkersPerTask markers, a warp per marker
__device__ void ibm_task(const StepArgs& a, unsigned task) {
    const int warp = threadIdx.x >> 5;
    const int l = (int)task * kMarkersPerTask + warp;
    if (warp < kMarkersPerTask && l < a.Mk.M) ibm_marker(a, l);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&a.ibm_done[a.k], 1u);
    }
}

// Bounded wait of a force-region tile for the IBM tasks of this substep.  On
// time-out the error bit kErrIbmWait is set (the host reports it at the next
// glsm_fluid_sync) and the tile goes on with the forces spread so far, so the
// launch always completes and the context stays usable.
__device__ __forceinline__ void wait_ibm(const StepArgs& a) {
    if (threadIdx.x == 0) {
        const volatile unsigned* flag = a.ibm_done + a.k;
        const volatile int* err = &a.ctl->error;
        const unsigned target = (unsigned)a.n_ibm + (unsigned)a.wait_extra;
        unsigned spins = 0;
        while (*flag < target) {
            // give up after ~0.3 s (or at once when another tile already gave up)
            if (++spins > (1u << 22) || (*err & kErrIbmWait)) {
                atomicOr(&a.ctl->error, kErrIbmWait);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// the substep kernel
// ---------------------------------------------------------------------------
template <int C>
__device__ __forceinline__ float sgn(float v) {
    return C > 0 ? v : -v;
}
// c . v for a D3Q19 direction (at most two non-zero components), without
// adding IEEE zeros that the compiler could not fold away
template <int CX, int CY, int CZ>
__device__ __forceinline__ float cdot(float x, float y, float z) {
    if constexpr (CX != 0 && CY != 0) return sgn<CX>(x) + sgn<CY>(y);
    else if constexpr (CX != 0 && CZ != 0) return sgn<CX>(x) + sgn<CZ>(z);
    else if constexpr (CY != 0 && CZ != 0) return sgn<CY>(y) + sgn<CZ>(z);
    else if constexpr (CX != 0) return sgn<CX>(x);
    else if constexpr (CY != 0) return sgn<CY>(y);
    else return sgn<CZ>(z);
}

// The collision works on v = 3u and G = 3F (so that 3 c.u = c.v and 9 (c.u)(c.F)
// = (c.v)(c.G)) with the weight w of each direction class (faces 1/18,
// diagonals 1/36) and the storage scale folded into per-class constants:
//   deq_q + F_q (even part) = cv (ae cv + h) + K,   odd part = aod cv + h
//   ae = w omega rho / 2, aod = w omega rho, h = w fp cG,
//   K = w (omega (drho - rho uu 3/2) - 3 fp uF)
struct CollideTerms {
    float vx, vy, vz, Gx, Gy, Gz;
    float omc;                    // 1 - omega
    float K[2], ae[2], aod[2], b[2];
};

template <int Q>
__device__ __forceinline__ void collide_pair(float (&d)[19], const CollideTerms& t) {
    constexpr int O = qopp(Q);
    constexpr int C = (Q <= 6) ? 0 : 1;  // direction class
    const float cv = cdot<qcx(Q), qcy(Q), qcz(Q)>(t.vx, t.vy, t.vz);
    const float cG = cdot<qcx(Q), qcy(Q), qcz(Q)>(t.Gx, t.Gy, t.Gz);
    const float h = t.b[C] * cG;
    const float Od = fmaf(t.aod[C], cv, h);
    const float E = fmaf(fmaf(t.ae[C], cv, h), cv, t.K[C]);
    d[Q] = fmaf(t.omc, d[Q], E + Od);
    d[O] = fmaf(t.omc, d[O], E - Od);
}

template <int Q>
__device__ __forceinline__ void moment_pair(const float (&d)[19], float& drho, float& jx, float& jy, float& jz) {
    constexpr int O = qopp(Q);
    const float sum = d[Q] + d[O], dif = d[Q] - d[O];
    drho += sum;
    if constexpr (qcx(Q) != 0) jx += sgn<qcx(Q)>(dif);
    if constexpr (qcy(Q) != 0) jy += sgn<qcy(Q)>(dif);
    if constexpr (qcz(Q) != 0) jz += sgn<qcz(Q)>(dif);
}

// BGK collision with Guo forcing in deviation form:
// d_q <- d_q + omega (deq_q - d_q) + F_q with
//   deq_q = w_q (drho + rho (3 cu + 4.5 cu^2 - 1.5 uu))
//   F_q   = w_q (1 - 1/(2 tau)) (3 cF + 9 cu cF - 3 uF)
// d holds deviations times the storage scale when SCALED (inv = 1/scale); Fh is
// half the body force.  The first members of the nine (q, opp q) pairs:
// 1 3 5 7 8 11 12 15 16.
template <bool SCALED>
__device__ __forceinline__ void collide(float (&d)[19], float Fhx, float Fhy, float Fhz, float omega, float fp,
                                        float inv, float scale, float& ux, float& uy, float& uz, float& rho) {
    float drho = d[0], jx = 0.f, jy = 0.f, jz = 0.f;
    moment_pair<1>(d, drho, jx, jy, jz);
    moment_pair<3>(d, drho, jx, jy, jz);
    moment_pair<5>(d, drho, jx, jy, jz);
    moment_pair<7>(d, drho, jx, jy, jz);
    moment_pair<8>(d, drho, jx, jy, jz);
    moment_pair<11>(d, drho, jx, jy, jz);
    moment_pair<12>(d, drho, jx, jy, jz);
    moment_pair<15>(d, drho, jx, jy, jz);
    moment_pair<16>(d, drho, jx, jy, jz);
    if (SCALED) {
        drho *= inv;
        jx *= inv;
        jy *= inv;
        jz *= inv;
    }
    rho = 1.0f + drho;
    const float ir = __frcp_rn(rho);
    ux = (jx + Fhx) * ir;
    uy = (jy + Fhy) * ir;
    uz = (jz + Fhz) * ir;
    CollideTerms t;
    t.vx = 3.0f * ux;
    t.vy = 3.0f * uy;
    t.vz = 3.0f * uz;
    t.Gx = 6.0f * Fhx;
    t.Gy = 6.0f * Fhy;
    t.Gz = 6.0f * Fhz;
    t.omc = 1.0f - omega;
    const float vv = t.vx * t.vx + t.vy * t.vy + t.vz * t.vz;  // 9 uu
    const float vG = t.vx * t.Gx + t.vy * t.Gy + t.vz * t.Gz;  // 9 uF
    const float wr = SCALED ? omega * rho * scale : omega * rho;
    const float sfp = SCALED ? fp * scale : fp;
    // omega (drho - 1.5 rho uu) - 3 fp uF, times the scale
    const float K1 = fmaf(-(1.0f / 6.0f) * wr, vv, fmaf(-(1.0f / 3.0f) * sfp, vG, (SCALED ? omega * scale : omega) * drho));
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const float w = c == 0 ? qw(1) : qw(7);
        t.K[c] = w * K1;
        t.aod[c] = w * wr;
        t.ae[c] = (0.5f * w) * wr;
        t.b[c] = w * sfp;
    }
    d[0] = fmaf(t.omc, d[0], qw(0) * K1);
    collide_pair<1>(d, t);
    collide_pair<3>(d, t);
    collide_pair<5>(d, t);
    collide_pair<7>(d, t);
    collide_pair<8>(d, t);
    collide_pair<11>(d, t);
    collide_pair<12>(d, t);
    collide_pair<15>(d, t);
    collide_pair<16>(d, t);
}

// Conserving FP16 rounding of one cell's 19 scaled post-collision values.
// With round-to-nearest every cell emits a random mass and momentum error each
// substep; summed over the lattice these errors excite long-wavelength
// acoustic and shear modes that viscosity damps slowly, and over thousands of
// steps that accumulated noise, not the rounding of the current step,
// dominates the velocity error.  Here every value is first rounded to
// nearest; then, direction by direction (1..18), a value moves to its other
// FP16 neighbour (one FP16 spacing towards the exact value) when that lowers
// M^2 + |P|^2, M and P being the cell's summed mass and momentum rounding
// errors so far.  What a cell emits then carries almost no mass or momentum
// error, so the injected noise is a divergence of per-cell errors and sits at
// short wavelengths, which viscosity removes within a few steps.  d[q]
// receives the float value of the chosen FP16 number (exactly representable,
// so the store's round-to-nearest conversion reproduces it).  The arithmetic
// uses explicitly rounded intrinsics, so the result does not depend on FMA
// contraction and a float32 restatement reproduces it bit for bit.
__device__ __forceinline__ void conserve_round(float (&d)[19]) {
    float e[19];
    float M = 0.f, Px = 0.f, Py = 0.f, Pz = 0.f;
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const float h = __half2float(__float2half_rn(d[q]));
        e[q] = __fsub_rn(d[q], h);
        d[q] = h;
        M = __fadd_rn(M, e[q]);
        if (qcx(q)) Px = qcx(q) > 0 ? __fadd_rn(Px, e[q]) : __fsub_rn(Px, e[q]);
        if (qcy(q)) Py = qcy(q) > 0 ? __fadd_rn(Py, e[q]) : __fsub_rn(Py, e[q]);
        if (qcz(q)) Pz = qcz(q) > 0 ? __fadd_rn(Pz, e[q]) : __fsub_rn(Pz, e[q]);
    }
#pragma unroll
    for (int q = 1; q < 19; q++) {
        const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
        // FP16 spacing at d[q]: 2^(exponent - 10), 2^-24 below the normal
        // range.  At a power of two reached from below the step down is twice
        // the spacing there, which still lands on an FP16 number.
        const float ulp = fmaxf(__int_as_float((__float_as_int(d[q]) & 0x7f800000) - (10 << 23)), 0x1p-24f);
        const float de = copysignf(ulp, -e[q]);  // change of e[q] if d[q] moves
        float t = M;
        if (cx) t = cx > 0 ? __fadd_rn(t, Px) : __fsub_rn(t, Px);
        if (cy) t = cy > 0 ? __fadd_rn(t, Py) : __fsub_rn(t, Py);
        if (cz) t = cz > 0 ? __fadd_rn(t, Pz) : __fsub_rn(t, Pz);
        // the move changes M^2 + |P|^2 by de (2 t + (1 + |c|^2) de), which is
        // negative exactly when t has the sign of e[q] and |t| exceeds
        // (1 + |c|^2) / 2 spacings: one for a face, 1.5 for a diagonal
        const float thr = (cx * cx + cy * cy + cz * cz == 2) ? __fmul_rn(1.5f, ulp) : ulp;
        if (fabsf(t) > thr && ((__float_as_int(t) ^ __float_as_int(e[q])) >= 0)) {
            d[q] = __fsub_rn(d[q], de);
            M = __fadd_rn(M, de);
            if (cx) Px = cx > 0 ? __fadd_rn(Px, de) : __fsub_rn(Px, de);
            if (cy) Py = cy > 0 ? __fadd_rn(Py, de) : __fsub_rn(Py, de);
            if (cz) Pz = cz > 0 ? __fadd_rn(Pz, de) : __fsub_rn(Pz, de);
        }
    }
}

// body force (uniform F_const plus, inside the marker boxes, the IBM force,
// which the cell consumes) and collision; returns (ux, uy, uz, rho)
template <int ST>
__device__ __forceinline__ float4 force_collide(const StepArgs& a, unsigned i, bool inb, float (&d)[19]) {
    const FluidDev& F = a.F;
    float Fx = 0.5f * F.Fc[0], Fy = 0.5f * F.Fc[1], Fz = 0.5f * F.Fc[2];  // half the force
    if (inb) {
        const float4 fi = __ldcg(&F.Fibm[i]);
        Fx = fmaf(0.5f, fi.x, Fx);
        Fy = fmaf(0.5f, fi.y, Fy);
        Fz = fmaf(0.5f, fi.z, Fz);
        __stcg(&F.Fibm[i], make_float4(0.f, 0.f, 0.f, 0.f));
    }
    float4 u;
    collide<PopIO<ST>::kScaled>(d, Fx, Fy, Fz, F.omega, F.fpref, F.inv_scale, F.scale, u.x, u.y, u.z, u.w);
    return u;
}

// the velocity moment where the next substep's interpolation (marker boxes) or
// the concentration step (last substep) reads it
__device__ __forceinline__ void store_u(const StepArgs& a, unsigned i, bool inb, float4 u) {
    if (inb || a.last) a.F.u[i] = u;
}

// force, collision and AA-pattern scatter of one cell; TAB: the launch's
// per-direction base pointers (StepArgs::scatter) address the even and the
// wall-free odd scatters
template <int ST, int PARITY, int PERX, bool TAB>
__device__ __forceinline__ void collide_scatter(const StepArgs& a, unsigned i, unsigned x, bool fast, bool xin,
                                                bool inb, float (&d)[19]) {
    using IO = PopIO<ST>;
    using T = typename IO::T;
    const FluidDev& F = a.F;
    const unsigned nx = F.nx, ny = F.ny, nz = F.nz;
    const unsigned S = (unsigned)F.S, nxy = nx * ny;
    T* P = reinterpret_cast<T*>(F.pop);
    const long long LS = S, Lnx = nx, Lnxy = nxy;
    const float4 u = force_collide<ST>(a, i, inb, d);
    if constexpr (IO::kConserve) conserve_round(d);

    T* Pi = P + i;
    if (TAB && (PARITY == 0 || (fast && xin))) {
#pragma unroll
        for (int q = 0; q < 19; q++) IO::st_raw(reinterpret_cast<T*>(a.scatter[q]) + i, d[q]);
    } else if (PARITY == 0) {
#pragma unroll
        for (int q = 0; q < 19; q++) IO::st_raw(Pi + qopp(q) * LS, d[q]);
    } else if (fast && xin) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            // post-collision f_q(x) streams to x + c_q, slot q
            const long long off = qcx(q) + qcy(q) * Lnx + qcz(q) * Lnxy;
            IO::st_raw(Pi + (q * LS + off), d[q]);
        }
    } else if (fast) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            // post-collision f_q(x) streams to x + c_q (slot q), or bounces back
            // into slot opp(q) of x when x + c_q lies beyond a wall
            const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
            const unsigned nbr = i + (unsigned)(cx + cy * (int)nx + cz * (int)nxy);
            if (cx == 0) {
                if (TAB)
                    IO::st_raw(reinterpret_cast<T*>(a.scatter[q]) + i, d[q]);
                else
                    IO::st_raw(P + (q * S + nbr), d[q]);
            } else {
                const bool edge = (cx > 0) ? (x == nx - 1) : (x == 0);
                if (PERX)
                    IO::st_raw(P + (q * S + (edge ? nbr - (unsigned)(cx * (int)nx) : nbr)), d[q]);
                else
                    IO::st_raw(P + (edge ? qopp(q) * S + i : q * S + nbr), d[q]);
            }
        }
    } else {
        const unsigned z = fdiv(i, a.div_nxy);
        const unsigned y = fdiv(i - z * nxy, a.div_nx);
        int mo[3], po[3];
        bool mw[3], pw[3];
        const unsigned c[3] = {x, y, z}, n[3] = {nx, ny, nz}, st[3] = {1u, nx, nxy};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            mw[k] = pw[k] = false;
            mo[k] = -(int)st[k];
            po[k] = (int)st[k];
            if (c[k] == 0) {
                if (F.per[k]) mo[k] = (int)((n[k] - 1) * st[k]);
                else mw[k] = true;
            }
            if (c[k] == n[k] - 1) {
                if (F.per[k]) po[k] = -(int)((n[k] - 1) * st[k]);
                else pw[k] = true;
            }
        }
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
            const bool wall = (cx > 0 && pw[0]) || (cx < 0 && mw[0]) || (cy > 0 && pw[1]) || (cy < 0 && mw[1]) ||
                              (cz > 0 && pw[2]) || (cz < 0 && mw[2]);
            const int off = (cx > 0 ? po[0] : cx < 0 ? mo[0] : 0) + (cy > 0 ? po[1] : cy < 0 ? mo[1] : 0) +
                            (cz > 0 ? po[2] : cz < 0 ? mo[2] : 0);
            IO::st_raw(P + (wall ? qopp(q) * S + i : q * S + i + (unsigned)off), d[q]);
        }
    }
    store_u(a, i, inb, u);
}

// one cell of a substep: gather (AA pattern), collide, scatter.  Addresses are a
// per-thread base pointer (the cell in plane 0) plus per-direction offsets that
// depend only on the lattice, the same for every lane; with TAB the even and
// the wall-free odd accesses use the launch's per-direction base pointers
// (StepArgs::gather / scatter) instead, one add per access.
template <int ST, int PARITY, int PERX, bool TAB>
__device__ __forceinline__ void lbm_cell(const StepArgs& a, unsigned i, bool inb) {
    using IO = PopIO<ST>;
    using T = typename IO::T;
    const FluidDev& F = a.F;
    const unsigned nx = F.nx, ny = F.ny, nz = F.nz;
    const unsigned S = (unsigned)F.S, nxy = nx * ny;
    const unsigned z = fdiv(i, a.div_nxy);
    const unsigned rem = i - z * nxy;
    const unsigned y = fdiv(rem, a.div_nx);
    const unsigned x = rem - y * nx;
    const T* Pi = reinterpret_cast<const T*>(F.pop) + i;
    const long long LS = S, Lnx = nx, Lnxy = nxy;
    float d[19];
    // odd substeps: warps whose cells are all off the y and z boundary planes
    // stream with constant neighbour offsets; among them, warps with no cell on
    // an x wall need no per-lane choice at all
    bool fast = true, xin = true;
    if (PARITY == 1) {
        const unsigned act = __activemask();
        fast = __all_sync(act, (y - 1u < ny - 2u) && (z - 1u < nz - 2u));
        xin = __all_sync(act, x - 1u < nx - 2u);
    }
    if (TAB && (PARITY == 0 || (fast && xin))) {
#pragma unroll
        for (int q = 0; q < 19; q++) d[q] = IO::raw(reinterpret_cast<const T*>(a.gather[q]) + i);
    } else if (PARITY == 0) {
#pragma unroll
        for (int q = 0; q < 19; q++) d[q] = IO::raw(Pi + q * LS);
    } else if (fast && xin) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            // arriving f_q(x) = post-collision f_q(x - c_q), in slot opp(q) at x - c_q
            const long long off = qcx(q) + qcy(q) * Lnx + qcz(q) * Lnxy;
            d[q] = IO::raw(Pi + (qopp(q) * LS - off));
        }
    } else if (fast) {
        const T* P = reinterpret_cast<const T*>(F.pop);
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
            const long long off = cx + cy * Lnx + cz * Lnxy;
            if (cx == 0) {
                // no x wall in the way: the launch's table holds the address
                d[q] = TAB ? IO::raw(reinterpret_cast<const T*>(a.gather[q]) + i) : IO::raw(Pi + (qopp(q) * LS - off));
            } else {
                // across an x wall: the bounced opp(q) population of x, in slot q
                // at x; periodic x: the wrapped neighbour
                const bool edge = (cx > 0) ? (x == 0) : (x == nx - 1);
                const unsigned nbr = i - (unsigned)off;
                if (PERX)
                    d[q] = IO::raw(P + (qopp(q) * S + (edge ? nbr + (unsigned)(cx * (int)nx) : nbr)));
                else
                    d[q] = IO::raw(P + (edge ? q * S + i : qopp(q) * S + nbr));
            }
        }
    } else {
        const T* P = reinterpret_cast<const T*>(F.pop);
        int mo[3], po[3];
        bool mw[3], pw[3];
        const unsigned c[3] = {x, y, z}, n[3] = {nx, ny, nz}, st[3] = {1u, nx, nxy};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            mw[k] = pw[k] = false;
            mo[k] = -(int)st[k];
            po[k] = (int)st[k];
            if (c[k] == 0) {
                if (F.per[k]) mo[k] = (int)((n[k] - 1) * st[k]);
                else mw[k] = true;
            }
            if (c[k] == n[k] - 1) {
                if (F.per[k]) po[k] = -(int)((n[k] - 1) * st[k]);
                else pw[k] = true;
            }
        }
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
            const bool wall = (cx > 0 && mw[0]) || (cx < 0 && pw[0]) || (cy > 0 && mw[1]) || (cy < 0 && pw[1]) ||
                              (cz > 0 && mw[2]) || (cz < 0 && pw[2]);
            const int off = (cx > 0 ? mo[0] : cx < 0 ? po[0] : 0) + (cy > 0 ? mo[1] : cy < 0 ? po[1] : 0) +
                            (cz > 0 ? mo[2] : cz < 0 ? po[2] : 0);
            d[q] = IO::raw(P + (wall ? q * S + i : qopp(q) * S + i + (unsigned)off));
        }
    }
    collide_scatter<ST, PARITY, PERX, TAB>(a, i, x, fast, xin, inb, d);
}

// Per-tile state prepared by warp 0 one tile ahead: the ticket and the marker
// boxes that overlap the tile's cells.
struct TileSlot {
    unsigned t;
    int nb;
    Box b[kMaxBoxes];
    int g[kMaxBoxes];  // gel index of each box
};

// Cell range of lattice tile `tile`: tiles of kTileCells cells, then, for
// the last wave of a launch, tiles of half that size.  A persistent launch
// ends when its slowest CTA finishes its last tile, so finer tiles at the end
// shorten the time the other CTAs wait, while the bulk keeps the per-tile
// overhead of full tiles.  Half tiles start at even cells, as the paired FP16
// even substep needs.
__device__ __forceinline__ void tile_range(const StepArgs& a, unsigned tile, unsigned& c0, unsigned& c1) {
    const unsigned big = (unsigned)a.big_tiles;
    const bool full = tile < big;
    c0 = full ? tile * kTileCells : big * kTileCells + (tile - big) * (kTileCells / 2);
    c1 = min(c0 + (full ? kTileCells : kTileCells / 2) - 1, (unsigned)a.F.N - 1);
}

__device__ __forceinline__ void prepare_slot(const StepArgs& a, unsigned t, TileSlot& sl) {
    const unsigned lane = threadIdx.x & 31;
    int nb = 0;
    if (t >= (unsigned)a.n_ibm && t < (unsigned)(a.n_ibm + a.n_tiles)) {
        const FluidDev& F = a.F;
        unsigned c0, c1;
        tile_range(a, t - a.n_ibm, c0, c1);
        const TileExt ext = tile_extent(c0, c1, F.nx, F.ny, a.div_nx, a.div_nxy);
        for (int j0 = 0; j0 < a.n_boxes; j0 += 32) {
            const int j = j0 + (int)lane;
            Box b{1, 0, 1, 0, 1, 0};
            bool hit = false;
            if (j < a.n_boxes) {
                b = a.Mk.boxes[j];
                hit = b.x0 <= b.x1 && overlaps(b, ext);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                sl.b[nb + __popc(m & ((1u << lane) - 1u))] = b;
                sl.g[nb + __popc(m & ((1u << lane) - 1u))] = j;
            }
            nb += __popc(m);
        }
    }
    if (lane == 0) {
        sl.t = t;
        sl.nb = nb;
    }
}

// even substep of two adjacent cells i0 (even) and i0 + 1: one vector load and
// one vector store per direction, the pair's populations staying packed in
// registers while each cell collides in turn
template <int ST, bool TAB>
__device__ __forceinline__ void lbm_pair_even(const StepArgs& a, unsigned i0, bool inb0, bool inb1) {
    using PIO = PairIO<ST>;
    using V = typename PIO::V;
    const FluidDev& F = a.F;
    const long long LS2 = F.S >> 1;  // vectors per plane
    V* Pv = reinterpret_cast<V*>(F.pop) + (i0 >> 1);
    V r[19];
#pragma unroll
    for (int q = 0; q < 19; q++)
        r[q] = TAB ? reinterpret_cast<const V*>(a.gather[q])[i0 >> 1] : Pv[q * LS2];
    {
        float d[19];
#pragma unroll
        for (int q = 0; q < 19; q++) d[q] = PIO::lo(r[q]);
        store_u(a, i0, inb0, force_collide<ST>(a, i0, inb0, d));
        if constexpr (PopIO<ST>::kConserve) conserve_round(d);
#pragma unroll
        for (int q = 0; q < 19; q++) r[q] = PIO::set_lo(r[q], d[q]);
    }
    {
        float d[19];
#pragma unroll
        for (int q = 0; q < 19; q++) d[q] = PIO::hi(r[q]);
        store_u(a, i0 + 1, inb1, force_collide<ST>(a, i0 + 1, inb1, d));
        if constexpr (PopIO<ST>::kConserve) conserve_round(d);
#pragma unroll
        for (int q = 0; q < 19; q++) r[q] = PIO::set_hi(r[q], d[q]);
    }
    // post-collision f_q goes to the cell's own slot opp(q)
#pragma unroll
    for (int q = 0; q < 19; q++) {
        if (TAB)
            reinterpret_cast<V*>(a.scatter[q])[i0 >> 1] = r[q];
        else
            Pv[qopp(q) * LS2] = r[q];
    }
}

// whether cell i lies in a marker box of the tile; with deterministic spreads a
// box cell also gathers its IBM force from the markers of the boxes that hold
// it (gel order, then marker order) into Fibm[i], where the collision reads it
// as it reads the atomically spread force otherwise
// (DET: the deterministic-spread instantiations of the kernels)
template <bool DET>
__device__ __forceinline__ bool in_boxes(const StepArgs& a, const TileSlot& sl, int nb, unsigned i) {
    const FluidDev& F = a.F;
    const unsigned z = fdiv(i, a.div_nxy);
    const unsigned rem = i - z * (F.nx * F.ny);
    const unsigned y = fdiv(rem, a.div_nx);
    const unsigned x = rem - y * F.nx;
    bool inb = false;
    for (int j = 0; j < nb; j++) inb |= inside(sl.b[j], (int)x, (int)y, (int)z);
    if (DET && inb) {
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
        const float inv_h3 = (float)(1.0 / (double)(F.h * F.h * F.h));
        for (int j = 0; j < nb; j++)
            if (inside(sl.b[j], (int)x, (int)y, (int)z)) det_gather<false>(a.Mk, sl.g[j], (int)x, (int)y, (int)z, inv_h3, f);
        __stcg(&F.Fibm[i], f);
    }
    return inb;
}

// a lattice tile of consecutive cells (tile_range), up to kCellsPerThread per
// thread: adjacent pairs on even substeps of FP16 storage, else cells kTile apart
template <int ST, int PARITY, int PERX, bool PAIR = false, bool DET = false, bool TAB = false>
__device__ __forceinline__ void lbm_tile(const StepArgs& a, unsigned tile, const TileSlot& sl) {
    unsigned c0, c1;
    tile_range(a, tile, c0, c1);
    const int nb = sl.nb;
    if (nb > 0) wait_ibm(a);
    if constexpr (PAIR && PARITY == 0 && (ST == kStoreF16 || ST == kStoreF16C) && kCellsPerThread == 2) {
        const unsigned i0 = c0 + 2 * threadIdx.x;
        const bool inb0 = nb > 0 && i0 <= c1 && in_boxes<DET>(a, sl, nb, i0);
        const bool inb1 = nb > 0 && i0 + 1 <= c1 && in_boxes<DET>(a, sl, nb, i0 + 1);
        if (i0 + 1 <= c1) {
            lbm_pair_even<ST, TAB>(a, i0, inb0, inb1);
        } else if (i0 <= c1) {
            lbm_cell<ST, PARITY, PERX, TAB>(a, i0, inb0);
        }
    } else {
#pragma unroll 1
        for (int r = 0; r < kCellsPerThread; r++) {
            const unsigned i = c0 + r * kTile + threadIdx.x;
            if (i <= c1) lbm_cell<ST, PARITY, PERX, TAB>(a, i, nb > 0 && in_boxes<DET>(a, sl, nb, i));
        }
    }
}

// Persistent substep kernel: each CTA takes tickets until none are left.
// Tickets [0, n_ibm) are IBM tasks, the rest lattice tiles in cell order.  A
// tile that meets a marker box waits for all IBM tasks of this substep; every
// IBM ticket is held by a CTA that runs it before taking another ticket, so
// the wait always ends (it is also bounded).  Warp 0 fetches the next ticket
// and prepares its tile while the CTA works on the current one, so each tile
// costs one block barrier.
template <int ST, int PARITY>
constexpr int lbm_ctas_per_sm() {
    // 64 registers (4 CTAs of 256 threads per SM); 80 (3 CTAs) for the paired
    // even substeps of FP16 storage, whose threads hold two cells
    return (PARITY == 0 && (ST == kStoreF16 || ST == kStoreF16C)) ? 768 / kTile : 1024 / kTile;
}

template <int ST, int PARITY, int PERX, bool DET>
__global__ void __launch_bounds__(kTile, (lbm_ctas_per_sm<ST, PARITY>())) lbm_substep_kernel(StepArgs a) {
    __shared__ TileSlot s_slot[2];
    // programmatic dependent launch: the next substep's CTAs may start on the
    // SMs this launch frees and run their prologue (ticket, marker boxes) while
    // this launch's last tiles finish; they wait below for all of it
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned total = (unsigned)a.n_ibm + (unsigned)a.n_tiles;
    const bool warp0 = threadIdx.x < 32;
    if (warp0) {
        unsigned t0 = 0;
        if (threadIdx.x == 0) t0 = atomicAdd(&a.tickets[a.k], 1u);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        prepare_slot(a, t0, s_slot[0]);
    }
    // every access to the previous substep's results (u, Fibm, populations)
    // comes after the previous launch has completed and its writes are visible
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __syncthreads();
    for (int j = 0;; j ^= 1) {
        const unsigned t = s_slot[j].t;
        if (t >= total) break;
        unsigned tn = 0;
        if (threadIdx.x == 0) tn = atomicAdd(&a.tickets[a.k], 1u);
        if (t < (unsigned)a.n_ibm)
            ibm_task(a, t);
        else
            lbm_tile<ST, PARITY, PERX, true, DET, true>(a, t - a.n_ibm, s_slot[j]);
        if (warp0) {
            tn = __shfl_sync(0xffffffffu, tn, 0);
            prepare_slot(a, tn, s_slot[j ^ 1]);
        }
        __syncthreads();
    }
}


// ---------------------------------------------------------------------------
// batched substep: several systems in one persistent launch
// ---------------------------------------------------------------------------
// The systems of a batch are launched in groups that share storage, x
// periodicity, spread mode and substep parity, so each group launch is the
// single-system kernel's instantiation with a different ticket resolver.
struct BatchSlot {
    TileSlot ts;     // group ticket and the tile's marker boxes
    unsigned local;  // IBM task or tile index within the system
    int is_ibm;
    int idle;        // the ticket belongs to a system that has finished
    StepArgs a;      // the system's arguments for this substep
};

__device__ __forceinline__ int find_sys(const int* offsets, int n, unsigned t) {
    int lo = 0, hi = n;  // the last s with offsets[s] <= t
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if ((unsigned)offsets[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// warp 0: resolve group ticket t to (system, local work) and prepare the slot
__device__ void prepare_batch_slot(const BatchLaunch& L, unsigned t, BatchSlot& sl) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned n_ibm_all = (unsigned)L.ibm_offsets[L.n];
    const unsigned total = n_ibm_all + (unsigned)L.tile_offsets[L.n];
    int nb = 0;
    if (t < total) {
        const bool ibm = t < n_ibm_all;
        const int g = ibm ? find_sys(L.ibm_offsets, L.n, t) : find_sys(L.tile_offsets, L.n, t - n_ibm_all);
        const BatchSys& sys = L.sys[L.members[g]];
        if (sys.dyn->remaining == 0) {  // an idle system: nothing to do for this ticket
            if (lane == 0) {
                sl.ts.t = t;
                sl.ts.nb = 0;
                sl.idle = 1;
            }
            return;
        }
        const unsigned local = ibm ? t - L.ibm_offsets[g] : (t - n_ibm_all) - L.tile_offsets[g];
        const int* src = reinterpret_cast<const int*>(&sys.step);
        int* dst = reinterpret_cast<int*>(&sl.a);
        for (int w = lane; w < (int)(sizeof(StepArgs) / 4); w += 32) dst[w] = src[w];
        __syncwarp();  // the whole copy lands before lane 0 sets the per-launch fields
        if (lane == 0) {
            sl.idle = 0;
            sl.a.k = L.k;
            sl.a.last = L.last;
            sl.local = local;
            sl.is_ibm = ibm;
        }
        if (!ibm) {
            const StepArgs& a = sys.step;
            unsigned c0, c1;
            tile_range(a, local, c0, c1);
            const TileExt ext = tile_extent(c0, c1, a.F.nx, a.F.ny, a.div_nx, a.div_nxy);
            for (int j0 = 0; j0 < a.n_boxes; j0 += 32) {
                const int j = j0 + (int)lane;
                Box b{1, 0, 1, 0, 1, 0};
                bool hit = false;
                if (j < a.n_boxes) {
                    b = a.Mk.boxes[j];
                    hit = b.x0 <= b.x1 && overlaps(b, ext);
                }
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (hit) {
                    sl.ts.b[nb + __popc(m & ((1u << lane) - 1u))] = b;
                    sl.ts.g[nb + __popc(m & ((1u << lane) - 1u))] = j;
                }
                nb += __popc(m);
            }
        }
    }
    if (lane == 0) {
        sl.ts.t = t;
        sl.ts.nb = nb;
    }
}

// The batched tiles read the system's parameters from the shared-memory slot
// rather than from the constant bank; on even substeps that costs registers
// (at 64 a thread spills about 170 bytes), so the batched even substeps take
// 80 registers (3 CTAs of 256 threads per SM) and the odd ones the
// single-system budget.
template <int ST, int PARITY>
constexpr int batch_ctas_per_sm() {
    return PARITY == 0 ? 768 / kTile : lbm_ctas_per_sm<ST, PARITY>();
}

// Tickets: first the group's IBM tasks, then its tiles, so the
// forward-progress argument of lbm_substep_kernel carries over (a tile waits
// only for IBM tasks of its own system, all of which have lower tickets).
template <int ST, int PARITY, int PERX, bool DET>
__global__ void __launch_bounds__(kTile, (batch_ctas_per_sm<ST, PARITY>())) lbm_substep_batch_kernel(BatchLaunch L) {
    __shared__ BatchSlot s_slot[2];
    // programmatic dependent launch as in lbm_substep_kernel (from the second
    // substep of an iteration on)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned total = (unsigned)(L.ibm_offsets[L.n] + L.tile_offsets[L.n]);
    const bool warp0 = threadIdx.x < 32;
    if (warp0) {
        unsigned t0 = 0;
        if (threadIdx.x == 0) t0 = atomicAdd(&L.tickets[L.k], 1u);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        prepare_batch_slot(L, t0, s_slot[0]);
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __syncthreads();
    for (int j = 0;; j ^= 1) {
        const BatchSlot& sl = s_slot[j];
        if (sl.ts.t >= total) break;
        unsigned tn = 0;
        if (threadIdx.x == 0) tn = atomicAdd(&L.tickets[L.k], 1u);
        if (sl.idle) {
            // nothing: the system has run all its requested iterations
        } else if (sl.is_ibm) {
            ibm_task(sl.a, sl.local);
        } else {
            lbm_tile<ST, PARITY, PERX, true, DET>(sl.a, sl.local, sl.ts);
        }
        if (warp0) {
            tn = __shfl_sync(0xffffffffu, tn, 0);
            prepare_batch_slot(L, tn, s_slot[j ^ 1]);
        }
        __syncthreads();
    }
}

using BatchKernel = void (*)(BatchLaunch);

// the group instantiation; even substeps move no population across a cell
// boundary, so they have no x-periodic form
template <int ST>
BatchKernel batch_kernel_of(int parity, int perx, int det) {
    if (!parity) return det ? lbm_substep_batch_kernel<ST, 0, 0, true> : lbm_substep_batch_kernel<ST, 0, 0, false>;
    if (perx) return det ? lbm_substep_batch_kernel<ST, 1, 1, true> : lbm_substep_batch_kernel<ST, 1, 1, false>;
    return det ? lbm_substep_batch_kernel<ST, 1, 0, true> : lbm_substep_batch_kernel<ST, 1, 0, false>;
}

BatchKernel batch_kernel(int storage, int parity, int perx, int det, int f16_round) {
    switch (storage) {
        case kStoreF32: return batch_kernel_of<kStoreF32>(parity, perx, det);
        case kStoreF16:
            return f16_conserving(f16_round, parity) ? batch_kernel_of<kStoreF16C>(parity, perx, det)
                                                     : batch_kernel_of<kStoreF16>(parity, perx, det);
        case kStoreBF16: return batch_kernel_of<kStoreBF16>(parity, perx, det);
        default: return nullptr;
    }
}

// ---------------------------------------------------------------------------
// upwind advection + diffusion of the concentration (once per iteration)
// ---------------------------------------------------------------------------
// One CTA: kTile consecutive cells of an xy plane (x fastest), each thread
// marching its column through a.zc planes from z0 = bz * a.zc.  The column's
// x and y neighbours are fixed, and the z neighbours' concentration and
// vertical velocity pass from one plane to the next in registers, so a cell
// costs five concentration and five velocity loads (the centre as one
// float4).  The arithmetic is k_convection_diffusion's, term for term.
template <bool DET>
__device__ void conv_diff_cols(const ConcArgs& a, unsigned bx, unsigned bz, Box* s_b, int* s_g, int* s_nb_p) {
    if (threadIdx.x == 0 && a.bump_iter && bx == 0 && bz == 0) a.ctl->iter += 1;  // nothing in this kernel reads it
    const FluidDev& F = a.F;
    const unsigned nx = F.nx, ny = F.ny, nz = F.nz, nxy = nx * ny;
    const unsigned p0 = bx * kTile, p1 = min(p0 + kTile - 1, nxy - 1);
    const unsigned z0 = bz * (unsigned)a.zc, z1 = min(z0 + (unsigned)a.zc - 1, nz - 1);
    TileExt ext = tile_extent(p0, p1, nx, ny, a.div_nx, a.div_nxy);  // one plane: z0 = z1 = 0
    ext.z0 = (int)z0;
    ext.z1 = (int)z1;
    const int nb = tile_boxes(a.Mk.boxes, a.n_boxes, ext, s_b, s_g, s_nb_p);
    const unsigned p = p0 + threadIdx.x;
    if (p > p1) return;
    const unsigned y = fdiv(p, a.div_nx);
    const unsigned x = p - y * nx;
    const unsigned xp = (x + 1 < nx) ? x + 1 : (F.per[0] ? 0 : x);
    const unsigned xm = (x >= 1) ? x - 1 : (F.per[0] ? nx - 1 : x);
    const unsigned yp = (y + 1 < ny) ? y + 1 : (F.per[1] ? 0 : y);
    const unsigned ym = (y >= 1) ? y - 1 : (F.per[1] ? ny - 1 : y);
    const unsigned pxp = y * nx + xp, pxm = y * nx + xm, pyp = yp * nx + x, pym = ym * nx + x;

    const float* c1p = F.c[a.cur];
    float* c2p = F.c[a.cur ^ 1];
    const float* U = reinterpret_cast<const float*>(F.u);
    const float ih = F.inv_dx, ih2 = ih * ih;
    const unsigned zm0 = (z0 >= 1) ? z0 - 1 : (F.per[2] ? nz - 1 : z0);
    float czm = c1p[zm0 * nxy + p], uzm = U[4 * (zm0 * nxy + p) + 2];
    float c = c1p[z0 * nxy + p];
    float4 u = F.u[z0 * nxy + p];
    for (unsigned z = z0; z <= z1; z++) {
        const unsigned zp = (z + 1 < nz) ? z + 1 : (F.per[2] ? 0 : z);
        const unsigned b = z * nxy, i = b + p;
        const float czp = c1p[zp * nxy + p];
        const float4 up = F.u[zp * nxy + p];
        const float cxp = c1p[b + pxp], cxm = c1p[b + pxm], cyp = c1p[b + pyp], cym = c1p[b + pym];
        const float ux = u.x, uy = u.y, uz = u.z;
        const float uL = 0.5f * (U[4 * (b + pxm)] + ux), uR = 0.5f * (ux + U[4 * (b + pxp)]);
        const float vL = 0.5f * (U[4 * (b + pym) + 1] + uy), vR = 0.5f * (uy + U[4 * (b + pyp) + 1]);
        const float wL = 0.5f * (uzm + uz), wR = 0.5f * (uz + up.z);
        const float cLx = (uL >= 0.0f) ? cxm : c, cLy = (vL >= 0.0f) ? cym : c, cLz = (wL >= 0.0f) ? czm : c;
        const float cRx = (uR >= 0.0f) ? c : cxp, cRy = (vR >= 0.0f) ? c : cyp, cRz = (wR >= 0.0f) ? c : czp;
        const float conv = -((uR * cRx - uL * cLx) * ih + (vR * cRy - vL * cLy) * ih + (wR * cRz - wL * cLz) * ih);
        const float diff =
            F.Dc * ((cxm - 2.0f * c + cxp) * ih2 + (cym - 2.0f * c + cyp) * ih2 + (czm - 2.0f * c + czp) * ih2);
        bool inb = false;
        for (int j = 0; j < nb; j++) inb |= inside(s_b[j], (int)x, (int)y, (int)z);
        float src = 0.f;
        if (DET && inb) {
            // deterministic spreads: the markers' concentration source, gathered
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            const float inv_h3 = 1.0f / (F.h * F.h * F.h);
            for (int j = 0; j < nb; j++)
                if (inside(s_b[j], (int)x, (int)y, (int)z)) det_gather<true>(a.Mk, s_g[j], (int)x, (int)y, (int)z, inv_h3, acc);
            src = acc.x;
        } else if (inb) {
            src = __ldcg(&F.source[i]);
            __stcg(&F.source[i], 0.f);
        }
        c2p[i] = c + F.dtc * (conv + diff + src);
        czm = c;
        uzm = uz;
        c = czp;
        u = up;
    }
}

template <bool DET>
__global__ void __launch_bounds__(kTile) conv_diff_kernel(ConcArgs a) {
    __shared__ int s_nb;
    __shared__ Box s_b[kMaxBoxes];
    __shared__ int s_g[kMaxBoxes];
    conv_diff_cols<DET>(a, blockIdx.x, blockIdx.y, s_b, s_g, &s_nb);
}

__device__ __forceinline__ int find_system(const int* offsets, int n, unsigned t) {
    int lo = 0, hi = n;  // the last s with offsets[s] <= t
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if ((unsigned)offsets[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// batched: block b belongs to the system whose [first, next) block range holds
// it; the system's current concentration buffer comes from its SysDyn
__global__ void __launch_bounds__(kTile) conv_diff_batch_kernel(const BatchSys* sys, const int* block_offsets, int n) {
    __shared__ int s_nb;
    __shared__ Box s_b[kMaxBoxes];
    __shared__ int s_g[kMaxBoxes];
    const unsigned b = blockIdx.x;
    if (n == 0 || b >= (unsigned)block_offsets[n]) return;
    const int s = find_system(block_offsets, n, b);
    if (sys[s].dyn->remaining == 0) return;
    ConcArgs a = sys[s].conc;
    a.cur = sys[s].dyn->cur;
    const unsigned lb = b - block_offsets[s];
    if (a.F.det_spread)
        conv_diff_cols<true>(a, lb % a.plane_blocks, lb / a.plane_blocks, s_b, s_g, &s_nb);
    else
        conv_diff_cols<false>(a, lb % a.plane_blocks, lb / a.plane_blocks, s_b, s_g, &s_nb);
}

// end of a batch iteration: advance every system's iteration, AA parity and
// concentration buffer
__global__ void batch_advance_kernel(const BatchSys* sys, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    SysDyn* d = sys[i].dyn;
    if (d->remaining == 0) return;
    if (d->remaining > 0) d->remaining -= 1;
    sys[i].step.ctl->iter += 1;
    d->parity0 ^= (sys[i].step.F.nsub & 1);
    d->cur ^= 1;
}

// ---------------------------------------------------------------------------
// populations in the reference's layout f[i + q*N] (absolute values)
// ---------------------------------------------------------------------------
template <int ST>
__global__ void read_pop_kernel(FluidDev F, int natural, float* out) {
    using IO = PopIO<ST>;
    using T = typename IO::T;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.N) return;
    const int nx = F.nx, ny = F.ny, nz = F.nz;
    const long long nxy = (long long)nx * ny, S = F.S;
    const int z = (int)(i / nxy);
    const long long rem = i - (long long)z * nxy;
    const int y = (int)(rem / nx);
    const int x = (int)(rem - (long long)y * nx);
    const T* P = reinterpret_cast<const T*>(F.pop);
#pragma unroll
    for (int q = 0; q < 19; q++) {
        long long src = (long long)q * S + i;
        if (!natural) {
            const int sx = x - qcx(q), sy = y - qcy(q), sz = z - qcz(q);
            int wx = F.per[0] ? (sx + nx) % nx : sx;
            int wy = F.per[1] ? (sy + ny) % ny : sy;
            int wz = F.per[2] ? (sz + nz) % nz : sz;
            const bool in = wx >= 0 && wx < nx && wy >= 0 && wy < ny && wz >= 0 && wz < nz;
            src = in ? (long long)qopp(q) * S + wx + (long long)wy * nx + (long long)wz * nxy : (long long)q * S + i;
        }
        out[(long long)q * F.N + i] = IO::ld(P + src, F.inv_scale) + qw(q);
    }
}

// write absolute populations given in the reference layout; leaves the array
// in natural layout (the caller resets its parity bookkeeping)
template <int ST>
__global__ void write_pop_kernel(FluidDev F, const float* in) {
    using IO = PopIO<ST>;
    using T = typename IO::T;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.N) return;
    T* P = reinterpret_cast<T*>(F.pop);
#pragma unroll
    for (int q = 0; q < 19; q++) IO::st(P + (long long)q * F.S + i, in[(long long)q * F.N + i] - qw(q), F.scale);
}

// ---------------------------------------------------------------------------
// global mass and momentum, reduced in FP64
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums over every cell of the stored deviations (mass: sum rho = N + sum d)
// and of c_q d_q (momentum: the rest weights carry none), each value widened
// to FP64 before it is added.  Every block covers a fixed set of cells and
// writes its four partial sums; conservation_final adds them in block order,
// so the result does not depend on scheduling.
template <int ST>
__global__ void __launch_bounds__(256) conservation_kernel(FluidDev F, double* partial) {
    using IO = PopIO<ST>;
    const typename IO::T* P = reinterpret_cast<const typename IO::T*>(F.pop);
    double m = 0.0, px = 0.0, py = 0.0, pz = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < F.N;
         i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const double v = (double)IO::raw(P + (long long)q * F.S + i);
            m += v;
            if (qcx(q)) px += qcx(q) * v;
            if (qcy(q)) py += qcy(q) * v;
            if (qcz(q)) pz += qcz(q) * v;
        }
    }
    __shared__ double s[4][8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    m = warp_sum_d(m);
    px = warp_sum_d(px);
    py = warp_sum_d(py);
    pz = warp_sum_d(pz);
    if (lane == 0) {
        s[0][w] = m;
        s[1][w] = px;
        s[2][w] = py;
        s[3][w] = pz;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += s[threadIdx.x][k];
        partial[4 * blockIdx.x + threadIdx.x] = t;
    }
}

// out = (N + inv sum d, sign inv sum c d): sign = -1 when the populations sit
// in the opposite slots (after an even AA substep)
__global__ void conservation_final(const double* partial, int n, double inv, double cells, double sign,
                                   double* out) {
    const int k = threadIdx.x;
    if (k >= 4) return;
    double t = 0.0;
    for (int b = 0; b < n; b++) t += partial[4 * b + k];
    out[k] = (k == 0) ? cells + inv * t : sign * inv * t;
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
int lbm_grid(const StepArgs& a, int parity) {
    const int total = a.n_ibm + a.n_tiles;
    const int ctas = parity ? a.lbm_ctas : a.lbm_ctas_even;
    return ctas > 0 ? min(total, ctas) : total;
}

int lbm_resident_ctas(int storage, int parity, int f16_round) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (storage == kStoreF16 && f16_conserving(f16_round, parity) && parity == 0)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_substep_kernel<kStoreF16C, 0, 0, false>, kTile, 0);
    else if (storage == kStoreF16 && f16_conserving(f16_round, parity))
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_substep_kernel<kStoreF16C, 1, 0, false>, kTile, 0);
    else if (storage == kStoreF16 && parity == 0)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_substep_kernel<kStoreF16, 0, 0, false>, kTile, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_substep_kernel<kStoreF32, 1, 0, false>, kTile, 0);
    return max(1, sms * max(1, per_sm));
}

cudaError_t launch_substep(const StepArgs& a_in, int parity, cudaStream_t s) {
    StepArgs a = a_in;
    {
        // the per-direction base pointers of this parity (element offsets from
        // the population array; odd: shifted by the neighbour offset)
        const size_t esz = a.F.storage == kStoreF32 ? 4 : 2;
        char* P = static_cast<char*>(a.F.pop);
        const long long S = a.F.S, nx = a.F.nx, nxy = (long long)a.F.nx * a.F.ny;
        for (int q = 0; q < 19; q++) {
            const long long off = qcx(q) + qcy(q) * nx + qcz(q) * nxy;
            const long long g = parity ? qopp(q) * S - off : q * S;
            const long long w = parity ? q * S + off : qopp(q) * S;
            a.gather[q] = P + g * (long long)esz;
            a.scatter[q] = P + w * (long long)esz;
        }
    }
    dim3 grid(lbm_grid(a, parity)), block(kTile);
    // substeps after the first are launched with programmatic stream
    // serialization (the kernel waits for its predecessor itself,
    // griddepcontrol.wait); the first follows the kernels that rewrite the
    // marker boxes its prologue reads, so it is launched plainly.  GLSM_NO_PDL=1
    // launches every substep plainly.
    static const bool no_pdl = getenv("GLSM_NO_PDL") != nullptr;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = (no_pdl || a.k == 0) ? 0 : 1;
    int n_attr = 1;
    if (a.l2_bytes > 0) {
        // the population array stays in the persisting part of L2 across the
        // substeps of an iteration
        attr[1].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[1].val.accessPolicyWindow.base_ptr = a.F.pop;
        attr[1].val.accessPolicyWindow.num_bytes = (size_t)a.l2_bytes;
        attr[1].val.accessPolicyWindow.hitRatio = a.l2_hit;
        attr[1].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[1].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        n_attr = 2;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = n_attr;
#define GLSM_SUB2(ST, DET)                                                     \
    if (parity && a.F.per[0])                                                  \
        return cudaLaunchKernelEx(&cfg, lbm_substep_kernel<ST, 1, 1, DET>, a); \
    else if (parity)                                                           \
        return cudaLaunchKernelEx(&cfg, lbm_substep_kernel<ST, 1, 0, DET>, a); \
    else                                                                       \
        return cudaLaunchKernelEx(&cfg, lbm_substep_kernel<ST, 0, 0, DET>, a);
#define GLSM_SUB(ST)            \
    if (a.F.det_spread) {       \
        GLSM_SUB2(ST, true)     \
    } else {                    \
        GLSM_SUB2(ST, false)    \
    }
    switch (a.F.storage) {
        case kStoreF32: GLSM_SUB(kStoreF32); break;
        case kStoreF16:
            if (f16_conserving(a.F.f16_round, parity)) {
                GLSM_SUB(kStoreF16C);
            } else {
                GLSM_SUB(kStoreF16);
            }
            break;
        case kStoreBF16: GLSM_SUB(kStoreBF16); break;
        default: return cudaErrorInvalidValue;
    }
#undef GLSM_SUB
#undef GLSM_SUB2
    return cudaGetLastError();
}

cudaError_t launch_substep_batch(const BatchLaunch& L, const BatchGroupKey& g, int parity, int grid, cudaStream_t s) {
    static const bool no_pdl = getenv("GLSM_NO_PDL") != nullptr;
    const BatchKernel k = batch_kernel(g.storage, parity, g.perx, g.det, g.f16_round);
    if (!k) return cudaErrorInvalidValue;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = (no_pdl || L.k == 0) ? 0 : 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kTile);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, L);
}

cudaError_t launch_conv_diff_batch(const BatchSys* sys, const int* block_offsets, int n, int blocks, cudaStream_t s) {
    if (blocks <= 0) return cudaSuccess;
    conv_diff_batch_kernel<<<blocks, kTile, 0, s>>>(sys, block_offsets, n);
    return cudaGetLastError();
}

cudaError_t launch_batch_advance(const BatchSys* sys, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    batch_advance_kernel<<<(n + 127) / 128, 128, 0, s>>>(sys, n);
    return cudaGetLastError();
}

int batch_resident_ctas(const BatchGroupKey& g, int parity) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const BatchKernel k = batch_kernel(g.storage, parity, g.perx, g.det, g.f16_round);
    if (k) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTile, 0);
    return max(1, sms * max(1, per_sm));
}

void conc_layout(ConcArgs& a) {
    const long long nxy = (long long)a.F.nx * a.F.ny;
    a.plane_blocks = (int)((nxy + kTile - 1) / kTile);
    // a few planes per thread where the lattice gives enough CTAs without
    a.zc = (int)std::min<long long>(8, std::max<long long>(1, (long long)a.F.nz * a.plane_blocks / 1024));
}

int conc_blocks(const ConcArgs& a) { return a.plane_blocks * ((a.F.nz + a.zc - 1) / a.zc); }

cudaError_t launch_conv_diff(const ConcArgs& a, cudaStream_t s) {
    dim3 grid((unsigned)a.plane_blocks, (unsigned)((a.F.nz + a.zc - 1) / a.zc)), block(kTile);
    if (a.F.det_spread)
        conv_diff_kernel<true><<<grid, block, 0, s>>>(a);
    else
        conv_diff_kernel<false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_read_pop(const FluidDev& F, int natural, float* out, cudaStream_t s) {
    dim3 grid((unsigned)((F.N + 255) / 256)), block(256);
    switch (F.storage) {
        case kStoreF32: read_pop_kernel<kStoreF32><<<grid, block, 0, s>>>(F, natural, out); break;
        case kStoreF16: read_pop_kernel<kStoreF16><<<grid, block, 0, s>>>(F, natural, out); break;
        case kStoreBF16: read_pop_kernel<kStoreBF16><<<grid, block, 0, s>>>(F, natural, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_conservation(const FluidDev& F, int reversed, double* partial, double* out, cudaStream_t s) {
    switch (F.storage) {
        case kStoreF32: conservation_kernel<kStoreF32><<<kConsBlocks, 256, 0, s>>>(F, partial); break;
        case kStoreF16: conservation_kernel<kStoreF16><<<kConsBlocks, 256, 0, s>>>(F, partial); break;
        case kStoreBF16: conservation_kernel<kStoreBF16><<<kConsBlocks, 256, 0, s>>>(F, partial); break;
        default: return cudaErrorInvalidValue;
    }
    const double inv = PopIO<kStoreF16>::kScaled && F.storage == kStoreF16 ? (double)F.inv_scale : 1.0;
    conservation_final<<<1, 32, 0, s>>>(partial, kConsBlocks, inv, (double)F.N, reversed ? -1.0 : 1.0, out);
    return cudaGetLastError();
}

cudaError_t launch_write_pop(const FluidDev& F, const float* in, cudaStream_t s) {
    dim3 grid((unsigned)((F.N + 255) / 256)), block(256);
    switch (F.storage) {
        case kStoreF32: write_pop_kernel<kStoreF32><<<grid, block, 0, s>>>(F, in); break;
        case kStoreF16: write_pop_kernel<kStoreF16><<<grid, block, 0, s>>>(F, in); break;
        case kStoreBF16: write_pop_kernel<kStoreBF16><<<grid, block, 0, s>>>(F, in); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// conserve_round over n cells of 19 values each ([cell][direction]), for the
// bit-for-bit check against its float32 restatement
__global__ void conserve_round_kernel(const float* in, float* out, long long n) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float d[19];
#pragma unroll
    for (int q = 0; q < 19; q++) d[q] = in[c * 19 + q];
    conserve_round(d);
#pragma unroll
    for (int q = 0; q < 19; q++) out[c * 19 + q] = d[q];
}

cudaError_t launch_conserve_round(const float* in, float* out, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    conserve_round_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}

}  // namespace glsm
