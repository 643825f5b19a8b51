// gel.h -- launch arguments and launchers of the gel/marker kernels (gel.cu)
#pragma once
#include "glsm_internal.h"

namespace glsm {

// phases of the one-CTA-per-gel kernel
enum : int {
    kPhElastic = 1,   // Gel::stepElasticity: mechanics when iter % 5 == 0, then setZero
    kPhChem = 2,      // Gel::stepChemistry
    kPhGather = 4,    // Coupler::packFromGels for this gel + stencil cache + box
    kPhRecord = 8,    // Gel::recordCenter (time series)
    kPhAuto = 16,     // honour active_from: skip before it, fire the pulse at it
    kPhGatherStale = 32,  // with kPhGather: only when the mechanics moved the nodes in
                          // this launch or gather_fresh[gel] is 0 (the marker arrays are
                          // a function of the nodes, which nothing else changes in a run)
};

struct GelArgs {
    GelDev* gels;      // device array
    int first_gel;     // blockIdx.x + first_gel is the gel handled by a CTA
    MarkerDev Mk;
    Ctl* ctl;
    int phases;
    int iter_arg;      // >= 0: iteration number; < 0: read Ctl::iter
    int nx, ny, nz;    // lattice (for the stencil cache)
    float h;
    float g2l;         // gel -> lattice velocity factor
    const SysDyn* dyn; // batched systems: skip the gel when dyn->remaining == 0
    int* gather_fresh; // kPhGatherStale: per gel, 1 while its marker arrays are current
    unsigned* zero_words;  // zeroed by the first CTA before any phase (the substeps'
    int n_zero_words;      // ticket counters of the iteration), or null
};

struct MarkerArgs {
    GelDev* gels;
    MarkerDev Mk;
    const float* c;    // current concentration
    float* source;
    int nx, ny, nz;
    float h;
    int scatter;       // also do un_robin -= Sl (Coupler::scatterToGels, C2 part)
    int det;           // leave the source spread to the advection kernel's gather
};

struct RepulsionArgs {
    GelDev* gels;
    MarkerDev Mk;
    float delta, gamma;
    int scatter;       // also do Fn_robin -= Frep
    const SysDyn* dyn; // batched systems: skip when dyn->remaining == 0
    int n_gels;        // with h > 0: skip gels whose marker box is out of reach
    float h;           // lattice cell width (0: no marker boxes yet, every pair)
};

cudaError_t launch_gel(const GelArgs& a, int n_gels, cudaStream_t s);
cudaError_t launch_conc_markers(const MarkerArgs& a, cudaStream_t s);
cudaError_t launch_repulsion(const RepulsionArgs& a, cudaStream_t s);
cudaError_t launch_scatter(GelDev* gels, const MarkerDev& Mk, cudaStream_t s);
// per node face (x fastest): (1, x, y, z) of the u_norm = v_norm = 0.15 crossing, or zeros
cudaError_t launch_filament(const GelDev& G, double4* out, cudaStream_t s);
// batched forms over several systems (device arrays of per-system arguments)
cudaError_t launch_gel_batch(const GelArgs* entries, int n, int grid, cudaStream_t s);
cudaError_t launch_conc_markers_batch(const MarkerArgs* pairs, const SysDyn* dyn, const int* warp_offsets, int n,
                                      int warps, cudaStream_t s);
cudaError_t launch_repulsion_batch(const RepulsionArgs* systems, const int* warp_offsets, int n, int warps,
                                   cudaStream_t s);

}  // namespace glsm
