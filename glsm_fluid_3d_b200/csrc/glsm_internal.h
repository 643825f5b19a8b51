// glsm_internal.h -- device-side data layout of one coupled gel-fluid system.
//
// One system = one D3Q19 lattice (FluidDev) + its markers (MarkerDev) + n gels
// (GelDev).  Everything lives in HBM and is advanced on one CUDA stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace glsm {

#ifndef GLSM_LBM_THREADS
#define GLSM_LBM_THREADS 256
#endif
#ifndef GLSM_LBM_CELLS_PER_THREAD
#define GLSM_LBM_CELLS_PER_THREAD 2
#endif
constexpr int kTile = GLSM_LBM_THREADS;  // threads of an LBM CTA
constexpr int kCellsPerThread = GLSM_LBM_CELLS_PER_THREAD;
constexpr int kTileCells = kTile * kCellsPerThread;  // lattice cells per LBM ticket
constexpr int kMarkersPerTask = kTile / 32;  // IBM task CTA: one warp per marker
constexpr int kMaxBoxes = 64;     // force-region boxes (one per gel) seen by one LBM launch
constexpr int kGelThreads = 512;  // threads of the one-CTA-per-gel kernel

enum Storage : int { kStoreF32 = 0, kStoreF16 = 1, kStoreBF16 = 2 };

// error bits accumulated in Ctl::error (sticky until read by the host)
enum : int {
    kErrIbmWait = 1,     // a force-region tile gave up waiting for the IBM tasks
    kErrMarkerOut = 2,   // a marker's 4^3 stencil left the lattice entirely
    kErrNonFinite = 4,   // a non-finite value was met in the gel state
};

// inclusive lattice-cell box; empty when x0 > x1
struct Box {
    int x0, x1, y0, y1, z0, z1;
};

// Per-launch control block in device memory.
struct Ctl {
    int iter;       // iteration counter advanced on the device in graph mode
    int error;      // sticky error bits
    int pad[2];
};

// Per-system state of a batch that changes every iteration, kept on the device
// so that a captured batch iteration replays without host work.
struct SysDyn {
    int parity0;    // AA parity at the start of the current iteration
    int cur;        // current concentration buffer
    int remaining;  // iterations still to run (< 0: no limit); 0: the system idles
    int pad;
};

// One gel: FP64 state in the reference's layout (src/gel.cu:66-114):
// elements over (LX+1)(LY+1)(LZ+1) slots, nodes over (LX+2)(LY+2)(LZ+2) slots,
// node vectors as double3 AoS.
struct GelDev {
    int LX, LY, LZ;  // interior nodes per axis = elements per axis + 1
    int nE, nN, M;   // element slots, node slots, surface markers
    int marker_off;  // first marker of this gel in the system's marker arrays
    int gel_id;
    int type;        // 1: Flory-Huggins + CHS*w*v; 2: c0 = c0_bis + b*v
    int tube_mode;   // 0 solid, 1 square tube, 2 cylinder (element mask)
    float tube_cy, tube_cz, tube_ihy, tube_ihz;
    int use_anchor;
    int active_from;  // > 0: skipped until this iteration, then excited
    double anchor_z;
    double f, ep, dt, dtx, dx, dy, dz;
    double CH0, CH1, CHS, C0, AZ0, FA0, c0_bis, b;
    double uss, vss, wss;
    // element arrays
    double *um, *vm, *wm, *wmp, *um_norm, *vm_norm, *T0, *T1, *T2, *vol, *pm;
    double3 *rm, *rm_loc, *nmSm;
    // node arrays
    double3 *rn, *Veln, *Vels, *Fn, *Fn_robin;
    double *un_norm, *un_robin, *vn_norm;
    int* bIndex;
    // centre-element time series: records of 12 doubles
    double* series;
    int series_cap;
    int series_every;
};

// Markers of all gels of a system, concatenated in gel order.
struct MarkerDev {
    int M;
    float4 *lag, *Vl, *Ul, *Fdrag, *Frep;  // .w unused
    float *Cl, *Dl, *Sl;
    int* owner;
    // per-iteration stencil cache (positions are fixed during the substeps)
    int4* base;      // first stencil cell (x,y,z) and a validity word
    float4* phx;     // delta-4 weights along x for the 4 stencil columns (0 if clipped)
    float4* phy;
    float4* phz;
    float* wsum;     // sum of the clipped stencil's weights (0 when empty)
    Box* boxes;      // per gel: union of its markers' clipped stencils
    int2* gel_range; // per gel: its markers [x, y) in these arrays
};

// The lattice.  Populations are stored as deviations d_q = f_q - w_q (times
// `scale` for FP16) in SoA planes of stride S cells, updated in place with the
// AA pattern: after an even substep the array holds post-collision values in
// reversed direction slots, after an odd substep it holds post-stream values
// in natural slots.
struct FluidDev {
    int nx, ny, nz;
    long long N, S;
    int storage;
    float scale, inv_scale;
    void* pop;
    float4* u;     // (ux, uy, uz, rho) in lattice units
    float4* Fibm;  // IBM force, non-zero only inside the marker boxes
    float* c[2];   // concentration ping-pong
    float* source;
    float tau, omega, fpref;  // fpref = 1 - 1/(2 tau)
    float Fc[3];
    int per[3];
    float h;       // physical length of one lattice cell
    float dtc, Dc, inv_dx;
    float beta, ramp_steps;
    int nsub;
    int det_spread;  // spreads as fixed-order gathers instead of float atomics
    int f16_round;   // FP16 storage: 0 round to nearest, 1 conserving rounding, 2 conserving on odd substeps
    long long substeps_done;  // host-side bookkeeping of the AA parity
};

}  // namespace glsm
