// coupling.h -- drop-in replacement of the reference's Coupler class
// (src/coupling.h:6-58) on top of libglsm_b200.so.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../glsm_b200.h"

class Gel;

struct CouplerParams {
    int M;
    float delta;
    float gamma;
    float gel_to_lbm_vel;
    float lbm_to_gel_vel;
};

class Coupler {
public:
    Coupler(std::vector<Gel*>& gels);
    ~Coupler();
    void packFromGels();
    void scatterToGels();
    void applyGelRepulsion();

    CouplerParams* h_cp;
    std::vector<int> h_offsets;
    std::vector<int> h_gelBoundaryCount;
    std::vector<int> h_owner;
    double dt = 1e-3;
    int numGels;
    int sumGelBoundaryCount;
    cudaStream_t coupler_stream;
    int threads;
    int blocksM;
    std::vector<Gel*>& gels;

    glsm_coupler handle;  // the library object
};
