// lbm.h -- launch arguments and launchers of the fluid kernels (lbm.cu)
#pragma once
#include "fastdiv.h"
#include "glsm_internal.h"

namespace glsm {

struct StepArgs {
    FluidDev F;
    MarkerDev Mk;
    Ctl* ctl;
    unsigned* tickets;   // [nsub] CTA tickets of this iteration's substeps
    unsigned* ibm_done;  // [nsub] finished IBM task CTAs per substep
    int n_boxes;
    int n_ibm;           // IBM task CTAs at the head of each substep launch
    int iter_arg;        // >= 0: iteration number; < 0: read Ctl::iter
    int k;               // substep index within the iteration
    int last;            // k == nsub - 1: write u for every cell
    FastDiv div_nx, div_nxy;
    int n_tiles;         // lattice tiles
    int big_tiles;       // tiles [0, big_tiles) hold kTileCells cells, the rest kTileCells / 2
    int lbm_ctas;        // persistent CTAs per odd-substep launch (0: one per ticket)
    int lbm_ctas_even;   // persistent CTAs per even-substep launch (0: one per ticket)
    int wait_extra;      // test aid: IBM tasks a force-region tile waits for beyond n_ibm (> 0 makes the
                         // bounded wait run out; 0 in every normal launch)
    // Per-direction base pointers of this launch's substep parity, set by
    // launch_substep: the cell i's value of direction q is read at gather[q] + i
    // and written at scatter[q] + i (even: slots q and opp(q) of the cell; odd,
    // away from walls: slot opp(q) of the upstream neighbour, slot q of the
    // downstream one).  Unused (null) in batched launches.
    const void* gather[19];
    void* scatter[19];
    float l2_hit;        // > 0: substep launches mark the first l2_bytes of the population
    unsigned long long l2_bytes;  // array L2-persisting with this hit ratio
};

struct ConcArgs {
    FluidDev F;
    MarkerDev Mk;
    Ctl* ctl;
    int n_boxes;
    int cur;        // index of the current concentration buffer
    int bump_iter;  // advance Ctl::iter (graph mode)
    FastDiv div_nx, div_nxy;
    int plane_blocks;  // CTAs across an xy plane (kTile cells each)
    int zc;            // planes each thread marches through
};

// plane_blocks and zc of a fluid's advection launch (conc_layout), and the
// launch's CTA count
void conc_layout(ConcArgs& a);
int conc_blocks(const ConcArgs& a);

// one system of a batch (device array, written when the batch changes)
struct BatchSys {
    StepArgs step;  // iter_arg < 0: the iteration comes from step.ctl
    ConcArgs conc;  // cur is replaced by dyn->cur
    SysDyn* dyn;
};

// one batched substep launch: the n systems of one group
struct BatchLaunch {
    const BatchSys* sys;      // every system of the batch
    const int* members;       // [n] index into sys of each system of the group
    const int* ibm_offsets;   // [n + 1] prefix sums of IBM tasks per group system
    const int* tile_offsets;  // [n + 1] prefix sums of lattice tiles per group system
    unsigned* tickets;        // [nsub] the group's ticket counters
    int n;
    int k;
    int last;
};

// what a group's systems share: one kernel instantiation serves them all
// (their substep parity is shared too and chosen per launch)
struct BatchGroupKey {
    int storage;
    int perx;  // periodic in x
    int det;   // deterministic spreads
    int f16_round;  // FP16 rounding mode (0 nearest, 1 conserving, 2 conserving on odd substeps)
};

int lbm_grid(const StepArgs& a, int parity);
cudaError_t launch_substep_batch(const BatchLaunch& L, const BatchGroupKey& g, int parity, int grid, cudaStream_t s);
cudaError_t launch_conv_diff_batch(const BatchSys* sys, const int* block_offsets, int n, int blocks, cudaStream_t s);
cudaError_t launch_batch_advance(const BatchSys* sys, int n, cudaStream_t s);
int batch_resident_ctas(const BatchGroupKey& g, int parity);
int lbm_resident_ctas(int storage, int parity, int f16_round);
cudaError_t launch_substep(const StepArgs& a, int parity, cudaStream_t s);
cudaError_t launch_conv_diff(const ConcArgs& a, cudaStream_t s);
cudaError_t launch_read_pop(const FluidDev& F, int natural, float* out, cudaStream_t s);
cudaError_t launch_write_pop(const FluidDev& F, const float* in, cudaStream_t s);
// global mass and momentum in FP64 (deterministic two-pass reduction); `partial`
// holds kConsBlocks x 4 doubles, `out` receives sum(rho), sum(c f) x, y, z
constexpr int kConsBlocks = 296;
// the conserving FP16 rounding of n cells ([cell][19] device arrays)
cudaError_t launch_conserve_round(const float* in, float* out, long long n, cudaStream_t s);
cudaError_t launch_conservation(const FluidDev& F, int reversed, double* partial, double* out, cudaStream_t s);

}  // namespace glsm
