// fluid.h -- drop-in replacement of the reference's Fluid class
// (src/fluid.h:7-84) on top of libglsm_b200.so.  The lattice has 2*s+1 cells per
// axis for fluidSize s (h = 0.5), as in the reference; a second constructor takes
// the lattice dims and Nsub directly.  The populations and velocity live in the
// library's own layout, so the reference's d_f / d_u pointers are not exposed;
// use the read methods below.
#pragma once
#include <cuda_runtime.h>

#include <thread>

#include "coupling.h"

struct FluidParams {
    int3 c[19];
    float w[19];
    int opp[19];
    float tau, cs2, nu;
    float3 F_const;
    float beta;
    int N;
    int M;
    int3 L;
    float h;
    float dx, dy, dz;
    float dt;
    float D;
    int perX, perY, perZ;
};

class Fluid {
public:
    Fluid(int3 fluidSize, int time, Coupler* coupler);
    // lattice cells given directly; nsub <= 0 keeps the reference's derived value
    Fluid(int3 latticeDims, int nsub, int storage, Coupler* coupler);
    ~Fluid();
    void stepVelocity(int iter);
    void stepConcentration(int iter);
    void writeFiles(int iter);
    void copyDataToHost();
    void recordData(int time);
    void setGoonValue(int time);
    int idx3(int x, int y, int z, int Nx, int Ny);
    // whole coupled iterations (gels, pack, velocity, concentration, repulsion,
    // scatter) as CUDA graph launches
    void run(int iter0, int n);

    float3* h_u;
    float* h_c1;
    FluidParams* h_fp;
    Coupler* coupler;
    int3 fluidSize;
    int3 fluidNodeGrid;
    int df;
    float dt;
    float h;
    int N;
    int Nd;
    float dt_fluid;
    int Nsub;
    float niu;
    float dx_fluid;
    std::thread file_writer_thread;
    cudaStream_t fluid_stream;

    glsm_fluid handle;  // the library object

private:
    void init(int3 dims, int nsub, int storage, int time);
    // page-locked staging of the output snapshot (u, c1) that writeFiles'
    // writer thread formats
    float* m_snap_u = nullptr;
    float* m_snap_c = nullptr;
    void writeSnapshot(int time);
};
