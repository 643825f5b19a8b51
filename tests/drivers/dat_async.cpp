// Output without stalling the device, built against the drop-in headers
// (include/glsm): the benchmark's lattice (101^3, fluidSize 50) with two
// 6x6x6 gels placed as in src/sim.cpp.  After a warm-up (which also allocates
// the writers' staging), 300 iterations are enqueued as graph launches and
// writeFiles(2000) of both gels and the fluid is timed on the host while the
// device still works through them; once the device has drained, the same
// state is written again through the synchronous copyDataToHost + recordData
// (time 3) for comparison.  Usage: dat_async <output dir>
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <filesystem>
#include <vector>

#include "coupling.h"
#include "fluid.h"
#include "gel.h"

int main(int argc, char** argv) {
    const char* out = argc > 1 ? argv[1] : "data";
    cudaSetDevice(0);
    std::filesystem::create_directories(out);
    std::filesystem::current_path(out);
    Gel* g1 = new Gel(make_int3(6, 6, 6), make_double3(16.67, 25.0, 25.0), 1, 1, 0);
    Gel* g2 = new Gel(make_int3(6, 6, 6), make_double3(33.33, 25.0, 25.0), 1, 2, 0);
    std::vector<Gel*> gels{g1, g2};
    for (auto g : gels) glsm_gel_add_noise(g->handle, 12345, 1e-3);
    Coupler* coupler = new Coupler(gels);
    Fluid* fluid = new Fluid(make_int3(50, 50, 50), 0, coupler);
    using clk = std::chrono::steady_clock;
    auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };

    fluid->run(0, 5);  // warm-up: graph capture
    for (auto g : gels) g->writeFiles(0);  // first output: the staging is allocated
    fluid->writeFiles(0);
    cudaDeviceSynchronize();
    for (auto g : gels) g->m_file_writer_thread.join();
    fluid->file_writer_thread.join();

    const auto t0 = clk::now();
    fluid->run(5, 300);
    const auto t1 = clk::now();
    for (auto g : gels) g->writeFiles(2000);
    fluid->writeFiles(2000);
    const auto t2 = clk::now();
    cudaDeviceSynchronize();
    const auto t3 = clk::now();
    for (auto g : gels) g->m_file_writer_thread.join();
    fluid->file_writer_thread.join();
    const auto t4 = clk::now();

    for (auto g : gels) {
        g->copyDataToHost();
        g->recordData(3);
    }
    fluid->copyDataToHost();
    fluid->recordData(3);
    std::printf("enqueue_ms=%.3f writefiles_ms=%.3f drain_ms=%.3f writers_ms=%.3f N=%d Nsub=%d\n", ms(t0, t1),
                ms(t1, t2), ms(t2, t3), ms(t3, t4), fluid->N, fluid->Nsub);
    for (auto g : gels) delete g;
    delete fluid;
    delete coupler;
    return 0;
}
