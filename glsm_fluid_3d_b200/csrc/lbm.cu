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
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "d3q19.cuh"
#include "fastdiv.h"
#include "glsm_internal.h"
#include "lbm.h"

namespace glsm {

// ---------------------------------------------------------------------------
// population storage: FP32 deviations, or FP16 / BF16 deviations (scaled)
// ---------------------------------------------------------------------------
template <int ST>
struct PopIO;
template <>
struct PopIO<kStoreF32> {
    using T = float;
    static __device__ __forceinline__ float ld(const T* p, float) { return *p; }
    static __device__ __forceinline__ void st(T* p, float v, float) { *p = v; }
};
template <>
struct PopIO<kStoreF16> {
    using T = __half;
    static __device__ __forceinline__ float ld(const T* p, float inv_scale) { return __half2float(*p) * inv_scale; }
    static __device__ __forceinline__ void st(T* p, float v, float scale) { *p = __float2half_rn(v * scale); }
};
template <>
struct PopIO<kStoreBF16> {
    using T = __nv_bfloat16;
    static __device__ __forceinline__ float ld(const T* p, float inv_scale) {
        return __bfloat162float(*p) * inv_scale;
    }
    static __device__ __forceinline__ void st(T* p, float v, float scale) { *p = __float2bfloat16_rn(v * scale); }
};

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

// Collect into shared memory the marker boxes that overlap this CTA's tile.
// Returns the count (all threads).  Uses one __syncthreads().
__device__ __forceinline__ int tile_boxes(const Box* boxes, int n_boxes, const TileExt& e, Box* s_b, int* s_nb) {
    if (threadIdx.x < n_boxes) {
        Box b = boxes[threadIdx.x];
        if (b.x0 <= b.x1 && overlaps(b, e)) {
            int s = atomicAdd(s_nb, 1);
            s_b[s] = b;
        }
    }
    __syncthreads();
    return *s_nb;
}

// ---------------------------------------------------------------------------
// IBM task: one warp per marker.  Lane j owns stencil points j and j+32 of
// the 4x4x4 stencil (point p = ax*16 + ay*4 + az, x outermost as in the
// reference loops).  Interpolates u of the previous substep, forms the penalty
// force beta_eff (Vl - Ul) and spreads it with vector float atomics.
// ---------------------------------------------------------------------------
__device__ void ibm_task(const StepArgs& a, unsigned task) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const FluidDev& F = a.F;
    const MarkerDev& Mk = a.Mk;
    const int l = (int)task * kMarkersPerTask + warp;
    if (warp < kMarkersPerTask && l < Mk.M) {
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
        if (ws != 0.0f) {
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
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&a.ibm_done[a.k], 1u);
    }
}

// bounded wait of a force-region tile for the IBM tasks of this substep
__device__ __forceinline__ void wait_ibm(const StepArgs& a) {
    if (threadIdx.x == 0) {
        const volatile unsigned* flag = a.ibm_done + a.k;
        const volatile int* err = &a.ctl->error;
        unsigned spins = 0;
        while (*flag < (unsigned)a.n_ibm) {
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

struct CollideTerms {
    float ux, uy, uz, Fx, Fy, Fz, even0, force0, rho45, rho3, fp9, fp3, omega;
};

// relaxation of the pair (Q, opp(Q)): equilibrium and forcing split into the
// parts even and odd in c_Q, shared by the pair
template <int Q>
__device__ __forceinline__ void collide_pair(float (&d)[19], const CollideTerms& t) {
    constexpr int O = qopp(Q);
    constexpr float w = qw(Q);
    const float cu = cdot<qcx(Q), qcy(Q), qcz(Q)>(t.ux, t.uy, t.uz);
    const float cF = cdot<qcx(Q), qcy(Q), qcz(Q)>(t.Fx, t.Fy, t.Fz);
    const float ev = fmaf(t.rho45 * cu, cu, t.even0), od = t.rho3 * cu;
    const float fe = fmaf(t.fp9 * cu, cF, t.force0), fo = t.fp3 * cF;
    d[Q] = fmaf(t.omega, fmaf(w, ev + od, -d[Q]), fmaf(w, fe + fo, d[Q]));
    d[O] = fmaf(t.omega, fmaf(w, ev - od, -d[O]), fmaf(w, fe - fo, d[O]));
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
// The first members of the nine (q, opp q) pairs: 1 3 5 7 8 11 12 15 16.
__device__ __forceinline__ void collide(float (&d)[19], float Fx, float Fy, float Fz, float omega, float fp,
                                        float& ux, float& uy, float& uz, float& rho) {
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
    rho = 1.0f + drho;
    const float inv = __frcp_rn(rho);
    ux = (jx + 0.5f * Fx) * inv;
    uy = (jy + 0.5f * Fy) * inv;
    uz = (jz + 0.5f * Fz) * inv;
    const float uu = ux * ux + uy * uy + uz * uz;
    const float uF = ux * Fx + uy * Fy + uz * Fz;
    CollideTerms t;
    t.ux = ux;
    t.uy = uy;
    t.uz = uz;
    t.Fx = Fx;
    t.Fy = Fy;
    t.Fz = Fz;
    t.even0 = drho - 1.5f * rho * uu;  // deq / w without the c terms
    t.force0 = -3.0f * fp * uF;         // F / w without the c terms
    t.rho45 = 4.5f * rho;
    t.rho3 = 3.0f * rho;
    t.fp9 = 9.0f * fp;
    t.fp3 = 3.0f * fp;
    t.omega = omega;
    d[0] = fmaf(omega, fmaf(qw(0), t.even0, -d[0]), fmaf(qw(0), t.force0, d[0]));
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

// one cell of a substep: gather (AA pattern), collide, scatter
template <int ST, int PARITY, int PERX>
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
    T* P = reinterpret_cast<T*>(F.pop);
    const float isc = F.inv_scale;
    float d[19];
    // odd substeps: a warp whose cells are all off the y and z boundary planes
    // streams with constant neighbour offsets (x walls or wraps per lane);
    // other warps take the general path
    bool fast = true;
    if (PARITY == 1) fast = __all_sync(__activemask(), (y - 1u < ny - 2u) && (z - 1u < nz - 2u));
    if (PARITY == 0) {
#pragma unroll
        for (int q = 0; q < 19; q++) d[q] = IO::ld(P + (q * S + i), isc);
    } else if (fast) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            // arriving f_q(x) = post-collision f_q(x - c_q), in slot opp(q) at x - c_q;
            // across a wall it is the bounced opp(q) population of x, in slot q at x
            const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
            const unsigned nbr = i - (unsigned)(cx + cy * (int)nx + cz * (int)nxy);
            if (cx == 0) {
                d[q] = IO::ld(P + (qopp(q) * S + nbr), isc);
            } else {
                const bool edge = (cx > 0) ? (x == 0) : (x == nx - 1);
                if (PERX)
                    d[q] = IO::ld(P + (qopp(q) * S + (edge ? nbr + (unsigned)(cx * (int)nx) : nbr)), isc);
                else
                    d[q] = IO::ld(P + (edge ? q * S + i : qopp(q) * S + nbr), isc);
            }
        }
    } else {
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
            d[q] = IO::ld(P + (wall ? q * S + i : qopp(q) * S + i + (unsigned)off), isc);
        }
    }

    // body force: uniform F_const plus the IBM force inside the marker boxes
    float Fx = F.Fc[0], Fy = F.Fc[1], Fz = F.Fc[2];
    if (inb) {
        const float4 fi = __ldcg(&F.Fibm[i]);
        Fx += fi.x;
        Fy += fi.y;
        Fz += fi.z;
        __stcg(&F.Fibm[i], make_float4(0.f, 0.f, 0.f, 0.f));
    }
    float ux, uy, uz, rho;
    collide(d, Fx, Fy, Fz, F.omega, F.fpref, ux, uy, uz, rho);
    // recompute store addresses from an opaque copy of the base pointer instead
    // of keeping the 19 load addresses alive across the collision
    asm volatile("mov.b64 %0, %0;" : "+l"(P));

    const float sc = F.scale;
    if (PARITY == 0) {
#pragma unroll
        for (int q = 0; q < 19; q++) IO::st(P + (qopp(q) * S + i), d[q], sc);
    } else if (fast) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            // post-collision f_q(x) streams to x + c_q (slot q), or bounces back
            // into slot opp(q) of x when x + c_q lies beyond a wall
            const int cx = qcx(q), cy = qcy(q), cz = qcz(q);
            const unsigned nbr = i + (unsigned)(cx + cy * (int)nx + cz * (int)nxy);
            if (cx == 0) {
                IO::st(P + (q * S + nbr), d[q], sc);
            } else {
                const bool edge = (cx > 0) ? (x == nx - 1) : (x == 0);
                if (PERX)
                    IO::st(P + (q * S + (edge ? nbr - (unsigned)(cx * (int)nx) : nbr)), d[q], sc);
                else
                    IO::st(P + (edge ? qopp(q) * S + i : q * S + nbr), d[q], sc);
            }
        }
    } else {
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
            IO::st(P + (wall ? qopp(q) * S + i : q * S + i + (unsigned)off), d[q], sc);
        }
    }
    if (inb || a.last) F.u[i] = make_float4(ux, uy, uz, rho);
}

// Per-tile state prepared by warp 0 one tile ahead: the ticket and the marker
// boxes that overlap the tile's cells.
struct TileSlot {
    unsigned t;
    int nb;
    Box b[kMaxBoxes];
};

__device__ __forceinline__ void prepare_slot(const StepArgs& a, unsigned t, TileSlot& sl) {
    const unsigned lane = threadIdx.x & 31;
    int nb = 0;
    if (t >= (unsigned)a.n_ibm && t < (unsigned)(a.n_ibm + a.n_tiles)) {
        const FluidDev& F = a.F;
        const unsigned c0 = (t - a.n_ibm) * kTileCells;
        const unsigned c1 = min(c0 + kTileCells - 1, (unsigned)F.N - 1);
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
            if (hit) sl.b[nb + __popc(m & ((1u << lane) - 1u))] = b;
            nb += __popc(m);
        }
    }
    if (lane == 0) {
        sl.t = t;
        sl.nb = nb;
    }
}

// a lattice tile of kTileCells consecutive cells, kCellsPerThread per thread
template <int ST, int PARITY, int PERX>
__device__ __forceinline__ void lbm_tile(const StepArgs& a, unsigned tile, const TileSlot& sl) {
    const FluidDev& F = a.F;
    const unsigned c0 = tile * kTileCells;
    const unsigned c1 = min(c0 + kTileCells - 1, (unsigned)F.N - 1);
    const int nb = sl.nb;
    if (nb > 0) wait_ibm(a);
#pragma unroll 1
    for (int r = 0; r < kCellsPerThread; r++) {
        const unsigned i = c0 + r * kTile + threadIdx.x;
        if (i <= c1) {
            bool inb = false;
            if (nb > 0) {
                const unsigned z = fdiv(i, a.div_nxy);
                const unsigned rem = i - z * (F.nx * F.ny);
                const unsigned y = fdiv(rem, a.div_nx);
                const unsigned x = rem - y * F.nx;
                for (int j = 0; j < nb; j++) inb |= inside(sl.b[j], (int)x, (int)y, (int)z);
            }
            lbm_cell<ST, PARITY, PERX>(a, i, inb);
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
template <int ST, int PARITY, int PERX>
__global__ void __launch_bounds__(kTile, 4) lbm_substep_kernel(StepArgs a) {
    __shared__ TileSlot s_slot[2];
    const unsigned total = (unsigned)a.n_ibm + (unsigned)a.n_tiles;
    const bool warp0 = threadIdx.x < 32;
    if (warp0) {
        unsigned t0 = 0;
        if (threadIdx.x == 0) t0 = atomicAdd(&a.tickets[a.k], 1u);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        prepare_slot(a, t0, s_slot[0]);
    }
    __syncthreads();
    for (int j = 0;; j ^= 1) {
        const unsigned t = s_slot[j].t;
        if (t >= total) break;
        unsigned tn = 0;
        if (threadIdx.x == 0) tn = atomicAdd(&a.tickets[a.k], 1u);
        if (t < (unsigned)a.n_ibm)
            ibm_task(a, t);
        else
            lbm_tile<ST, PARITY, PERX>(a, t - a.n_ibm, s_slot[j]);
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
struct BatchSlot {
    TileSlot ts;     // global ticket and the tile's marker boxes
    int sys;         // system index
    unsigned local;  // IBM task or tile index within the system
    int is_ibm;
    int parity;
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

// warp 0: resolve global ticket t to (system, local work) and prepare the slot
__device__ void prepare_batch_slot(const BatchLaunch& L, unsigned t, BatchSlot& sl) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned n_ibm_all = (unsigned)L.ibm_offsets[L.n];
    const unsigned total = n_ibm_all + (unsigned)L.tile_offsets[L.n];
    int nb = 0;
    if (t < total) {
        const bool ibm = t < n_ibm_all;
        const int s = ibm ? find_sys(L.ibm_offsets, L.n, t) : find_sys(L.tile_offsets, L.n, t - n_ibm_all);
        if (L.sys[s].dyn->remaining == 0) {  // an idle system: nothing to do for this ticket
            if (lane == 0) {
                sl.ts.t = t;
                sl.ts.nb = 0;
                sl.idle = 1;
            }
            return;
        }
        const unsigned local = ibm ? t - L.ibm_offsets[s] : (t - n_ibm_all) - L.tile_offsets[s];
        const int* src = reinterpret_cast<const int*>(&L.sys[s].step);
        int* dst = reinterpret_cast<int*>(&sl.a);
        for (int w = lane; w < (int)(sizeof(StepArgs) / 4); w += 32) dst[w] = src[w];
        __syncwarp();  // the whole copy lands before lane 0 sets the per-launch fields
        if (lane == 0) {
            sl.idle = 0;
            sl.a.k = L.k;
            sl.a.last = L.last;
            sl.sys = s;
            sl.local = local;
            sl.is_ibm = ibm;
            sl.parity = (L.sys[s].dyn->parity0 + L.k) & 1;
        }
        if (!ibm) {
            const StepArgs& a = L.sys[s].step;
            const unsigned c0 = local * kTileCells;
            const unsigned c1 = min(c0 + kTileCells - 1, (unsigned)a.F.N - 1);
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
                if (hit) sl.ts.b[nb + __popc(m & ((1u << lane) - 1u))] = b;
                nb += __popc(m);
            }
        }
    }
    if (lane == 0) {
        sl.ts.t = t;
        sl.ts.nb = nb;
    }
}

template <int ST>
__device__ __forceinline__ void batch_tile(const BatchSlot& sl) {
    if (!sl.parity)
        lbm_tile<ST, 0, 0>(sl.a, sl.local, sl.ts);
    else if (sl.a.F.per[0])
        lbm_tile<ST, 1, 1>(sl.a, sl.local, sl.ts);
    else
        lbm_tile<ST, 1, 0>(sl.a, sl.local, sl.ts);
}

// Tickets: first every system's IBM tasks, then every system's tiles, so the
// forward-progress argument of lbm_substep_kernel carries over (a tile waits
// only for IBM tasks of its own system, all of which have lower tickets).
__global__ void __launch_bounds__(kTile, 3) lbm_substep_batch_kernel(BatchLaunch L) {
    __shared__ BatchSlot s_slot[2];
    const unsigned total = (unsigned)(L.ibm_offsets[L.n] + L.tile_offsets[L.n]);
    const bool warp0 = threadIdx.x < 32;
    if (warp0) {
        unsigned t0 = 0;
        if (threadIdx.x == 0) t0 = atomicAdd(&L.tickets[L.k], 1u);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        prepare_batch_slot(L, t0, s_slot[0]);
    }
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
            const int st = sl.a.F.storage;
            if (st == kStoreF32)
                batch_tile<kStoreF32>(sl);
            else if (st == kStoreF16)
                batch_tile<kStoreF16>(sl);
            else
                batch_tile<kStoreBF16>(sl);
        }
        if (warp0) {
            tn = __shfl_sync(0xffffffffu, tn, 0);
            prepare_batch_slot(L, tn, s_slot[j ^ 1]);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// upwind advection + diffusion of the concentration (once per iteration)
// ---------------------------------------------------------------------------
// one 256-cell tile of the upwind advection + diffusion
__device__ void conv_diff_tile(const ConcArgs& a, unsigned block, Box* s_b, int* s_nb_p) {
    int& s_nb = *s_nb_p;
    if (threadIdx.x == 0) {
        s_nb = 0;
        if (a.bump_iter && block == 0) a.ctl->iter += 1;  // nothing in this kernel reads it
    }
    __syncthreads();
    const FluidDev& F = a.F;
    const unsigned nx = F.nx, ny = F.ny, nz = F.nz;
    const unsigned N = (unsigned)F.N, nxy = nx * ny;
    const unsigned c0 = block * kTile;
    const unsigned c1 = min(c0 + kTile - 1, N - 1);
    const TileExt ext = tile_extent(c0, c1, nx, ny, a.div_nx, a.div_nxy);
    const int nb = tile_boxes(a.Mk.boxes, a.n_boxes, ext, s_b, &s_nb);
    const unsigned i = c0 + threadIdx.x;
    if (i > c1) return;
    const unsigned z = fdiv(i, a.div_nxy);
    const unsigned rem = i - z * nxy;
    const unsigned y = fdiv(rem, a.div_nx);
    const unsigned x = rem - y * nx;
    bool inb = false;
    for (int j = 0; j < nb; j++) inb |= inside(s_b[j], (int)x, (int)y, (int)z);

    const unsigned xp = (x + 1 < nx) ? x + 1 : (F.per[0] ? 0 : x);
    const unsigned xm = (x >= 1) ? x - 1 : (F.per[0] ? nx - 1 : x);
    const unsigned yp = (y + 1 < ny) ? y + 1 : (F.per[1] ? 0 : y);
    const unsigned ym = (y >= 1) ? y - 1 : (F.per[1] ? ny - 1 : y);
    const unsigned zp = (z + 1 < nz) ? z + 1 : (F.per[2] ? 0 : z);
    const unsigned zm = (z >= 1) ? z - 1 : (F.per[2] ? nz - 1 : z);
    const unsigned base = z * nxy + y * nx;
    const unsigned ixp = base + xp, ixm = base + xm;
    const unsigned iyp = z * nxy + yp * nx + x, iym = z * nxy + ym * nx + x;
    const unsigned izp = zp * nxy + y * nx + x, izm = zm * nxy + y * nx + x;

    const float* c1p = F.c[a.cur];
    float* c2p = F.c[a.cur ^ 1];
    const float* U = reinterpret_cast<const float*>(F.u);
    const float c = c1p[i], cxp = c1p[ixp], cxm = c1p[ixm], cyp = c1p[iyp], cym = c1p[iym], czp = c1p[izp],
                czm = c1p[izm];
    const float ux = U[4 * i], uy = U[4 * i + 1], uz = U[4 * i + 2];
    const float uL = 0.5f * (U[4 * ixm] + ux), uR = 0.5f * (ux + U[4 * ixp]);
    const float vL = 0.5f * (U[4 * iym + 1] + uy), vR = 0.5f * (uy + U[4 * iyp + 1]);
    const float wL = 0.5f * (U[4 * izm + 2] + uz), wR = 0.5f * (uz + U[4 * izp + 2]);
    const float cLx = (uL >= 0.0f) ? cxm : c, cLy = (vL >= 0.0f) ? cym : c, cLz = (wL >= 0.0f) ? czm : c;
    const float cRx = (uR >= 0.0f) ? c : cxp, cRy = (vR >= 0.0f) ? c : cyp, cRz = (wR >= 0.0f) ? c : czp;
    const float ih = F.inv_dx, ih2 = ih * ih;
    const float conv = -((uR * cRx - uL * cLx) * ih + (vR * cRy - vL * cLy) * ih + (wR * cRz - wL * cLz) * ih);
    const float diff = F.Dc * ((cxm - 2.0f * c + cxp) * ih2 + (cym - 2.0f * c + cyp) * ih2 + (czm - 2.0f * c + czp) * ih2);
    float src = 0.f;
    if (inb) {
        src = __ldcg(&F.source[i]);
        __stcg(&F.source[i], 0.f);
    }
    c2p[i] = c + F.dtc * (conv + diff + src);
}

__global__ void __launch_bounds__(kTile) conv_diff_kernel(ConcArgs a) {
    __shared__ int s_nb;
    __shared__ Box s_b[kMaxBoxes];
    conv_diff_tile(a, blockIdx.x, s_b, &s_nb);
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
    const unsigned b = blockIdx.x;
    if (n == 0 || b >= (unsigned)block_offsets[n]) return;
    const int s = find_system(block_offsets, n, b);
    if (sys[s].dyn->remaining == 0) return;
    ConcArgs a = sys[s].conc;
    a.cur = sys[s].dyn->cur;
    conv_diff_tile(a, b - block_offsets[s], s_b, &s_nb);
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
// host-side launchers
// ---------------------------------------------------------------------------
int lbm_grid(const StepArgs& a) {
    const int total = a.n_ibm + a.n_tiles;
    return a.lbm_ctas > 0 ? min(total, a.lbm_ctas) : total;
}

int lbm_resident_ctas() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_substep_kernel<kStoreF32, 1, 0>, kTile, 0);
    return max(1, sms * max(1, per_sm));
}

cudaError_t launch_substep(const StepArgs& a, int parity, cudaStream_t s) {
    dim3 grid(lbm_grid(a)), block(kTile);
#define GLSM_SUB(ST)                                                           \
    if (parity && a.F.per[0])                                                  \
        lbm_substep_kernel<ST, 1, 1><<<grid, block, 0, s>>>(a);                \
    else if (parity)                                                           \
        lbm_substep_kernel<ST, 1, 0><<<grid, block, 0, s>>>(a);                \
    else                                                                       \
        lbm_substep_kernel<ST, 0, 0><<<grid, block, 0, s>>>(a);
    switch (a.F.storage) {
        case kStoreF32: GLSM_SUB(kStoreF32); break;
        case kStoreF16: GLSM_SUB(kStoreF16); break;
        case kStoreBF16: GLSM_SUB(kStoreBF16); break;
        default: return cudaErrorInvalidValue;
    }
#undef GLSM_SUB
    return cudaGetLastError();
}

cudaError_t launch_substep_batch(const BatchLaunch& L, int grid, cudaStream_t s) {
    lbm_substep_batch_kernel<<<grid, kTile, 0, s>>>(L);
    return cudaGetLastError();
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

int batch_resident_ctas() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_substep_batch_kernel, kTile, 0);
    return max(1, sms * max(1, per_sm));
}

cudaError_t launch_conv_diff(const ConcArgs& a, cudaStream_t s) {
    dim3 grid((unsigned)((a.F.N + kTile - 1) / kTile)), block(kTile);
    conv_diff_kernel<<<grid, block, 0, s>>>(a);
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

}  // namespace glsm
