// A driver built against the drop-in headers (include/glsm) for the .dat tests:
// one 6x6x6 gel at (4.75, 5.0, 5.25) in a 21x21x21 lattice (fluidSize 10),
// seeded chemistry noise, the reference's per-iteration call order
// (src/sim.cpp:60-111).
//
//   dat_case write <dir> <iterations> <seed>
//       runs the iterations, then writeFiles(2000) of the gel and the fluid:
//       gel1{rn,Fn,Veln,rm,um,vm,wm}2.dat, Velb2.dat, Conc2.dat in <dir>
//   dat_case restart <dir>
//       Gel(..., time = 2) and Fluid(fluidSize, 2, coupler) restart from those
//       files (setGoonValue), then writeFiles(4000) writes the restored state as
//       gel1*4.dat, Velb4.dat, Conc4.dat
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <vector>

#include "coupling.h"
#include "fluid.h"
#include "gel.h"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: dat_case write <dir> <iterations> <seed> | dat_case restart <dir>\n");
        return 2;
    }
    const bool restart = std::strcmp(argv[1], "restart") == 0;
    const int iters = (!restart && argc > 3) ? std::atoi(argv[3]) : 0;
    const unsigned long long seed = (!restart && argc > 4) ? std::strtoull(argv[4], nullptr, 10) : 12345ULL;
    cudaSetDevice(0);
    std::filesystem::create_directories(argv[2]);
    std::filesystem::current_path(argv[2]);
    const int start = restart ? 2 : 0;
    Gel* g = new Gel(make_int3(6, 6, 6), make_double3(4.75, 5.0, 5.25), 1, 1, start);
    if (!restart && glsm_gel_add_noise(g->handle, seed, 1e-3) != GLSM_OK) {
        std::fprintf(stderr, "noise: %s\n", glsm_last_error());
        return 1;
    }
    std::vector<Gel*> gels{g};
    Coupler* coupler = new Coupler(gels);
    Fluid* fluid = new Fluid(make_int3(10, 10, 10), start, coupler);
    for (int iter = 0; iter < iters; ++iter) {
        for (auto gg : gels) {
            gg->stepElasticity(iter);
            gg->stepChemistry(iter);
        }
        coupler->packFromGels();
        fluid->stepVelocity(iter);
        fluid->stepConcentration(iter);
        coupler->applyGelRepulsion();
        coupler->scatterToGels();
    }
    cudaDeviceSynchronize();
    std::printf("Nsub=%d N=%d\n", fluid->Nsub, fluid->N);
    const int out_iter = restart ? 4000 : 2000;
    for (auto gg : gels) gg->writeFiles(out_iter);
    fluid->writeFiles(out_iter);
    delete fluid;  // joins the writer threads
    for (auto gg : gels) delete gg;
    delete coupler;
    return 0;
}
