// A driver in the style of the reference's src/sim.cpp, built against the
// drop-in headers (include/glsm): two 6x6x6 gels 2 apart in a 41x21x21 lattice (fluidSize
// 20x10x10), the reference's per-iteration call order, .dat output every 1000
// iterations.  Usage: sim_twogels <iterations> <output dir> [ramp]
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <vector>

#include "coupling.h"
#include "fluid.h"
#include "gel.h"

int main(int argc, char** argv) {
    const int runstep = argc > 1 ? atoi(argv[1]) : 20;
    const char* out = argc > 2 ? argv[2] : "data";
    cudaSetDevice(0);
    std::filesystem::create_directories(out);
    std::filesystem::current_path(out);
    Gel* g1 = new Gel(make_int3(6, 6, 6), make_double3(6.0, 5.0, 5.0), 1, 1, 0);
    Gel* g2 = new Gel(make_int3(6, 6, 6), make_double3(14.0, 5.0, 5.0), 1, 2, 0);
    std::vector<Gel*> gels{g1, g2};
    Coupler* coupler = new Coupler(gels);
    Fluid* fluid = new Fluid(make_int3(20, 10, 10), 0, coupler);
    for (int iter = 0; iter <= runstep; ++iter) {
        for (auto g : gels) {
            g->stepElasticity(iter);
            g->stepChemistry(iter);
            g->recordCenter(iter);
        }
        coupler->packFromGels();
        fluid->stepVelocity(iter);
        fluid->stepConcentration(iter);
        coupler->applyGelRepulsion();
        coupler->scatterToGels();
        if (iter % 10 == 0 || iter == runstep) {
            cudaDeviceSynchronize();
            double vmax = 0;
            for (auto g : gels) {
                cudaMemcpy(g->m_hVeln, g->m_dVeln, g->m_numGelNodes * sizeof(double3), cudaMemcpyDeviceToHost);
                for (int n = 0; n < g->m_numGelNodes; n++) {
                    const double3 v = g->m_hVeln[n];
                    vmax = std::fmax(vmax, std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z));
                }
            }
            printf("iter=%d Vg_max=%.12e Nsub=%d h=%g\n", iter, vmax, fluid->Nsub, fluid->h_fp->h);
        }
        for (auto g : gels) g->writeFiles(iter);
        fluid->writeFiles(iter);
    }
    for (auto g : gels) delete g;
    delete fluid;
    delete coupler;
    return 0;
}
