// gel.h -- drop-in replacement of the reference's Gel class (src/gel.h:5-165)
// on top of libglsm_b200.so.  Same constructor, methods and public members that
// the reference's drivers use; device pointers (m_d*) are live device buffers in
// the reference's layout.  Compile a driver with -I<repo>/include/glsm and link
// -lglsm_b200.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <thread>

#include "../glsm_b200.h"

// GelParams, src/gel.h:5-31 (host copy of the parameters in use)
struct GelParams {
    int LX, LY, LZ;
    double f, q, ep, P1, P2;
    double dt, dtx;
    double dx, dy, dz;
    double CH0, CH1, CHS, C0, AZ0, FA0;
    double c0_bis, b;
    double uss, vss, wss, I;
    int gelType;
    int maxFilamentlen;
    float lbm_to_gel_vel;
    int tube_mode;
    float tube_cy, tube_cz, tube_inner_hy, tube_inner_hz;
};

class Gel {
public:
    Gel(int3 gelSize, double3 gelPosition, int gelType, int gel_id, int time);
    ~Gel();
    void stepChemistry(int iter);
    void stepElasticity(int iter);
    void recordCenter(int iter);
    void writeFiles(int iter);
    void resetToQuiescent();
    void fireExcitationPulse();
    void setAnchorZ(double anchor_z);
    void buildTubeMask(int wall_thickness, bool circular = false);
    int get_index(int xi, int yi, int zi, int size);
    int idx3(int x, int y, int z, int Nx, int Ny);
    void copyDataToHost();
    void copyDataToDevice();
    void recordData(int time);
    void setGoonValue(int time);

    // parameters
    GelParams* m_hgp;
    // host mirrors (filled by copyDataToHost / writeFiles)
    double* m_hum;
    double* m_hvm;
    double* m_hwm;
    double3* m_hrn;
    double3* m_hrm;
    double3* m_hFn;
    double3* m_hVeln;
    int* m_hbIndex;
    double* m_hseries;
    // device buffers, reference layout
    double* m_dum;
    double* m_dum_norm;
    double* m_dun_norm;
    double* m_dun_robin;
    double* m_dvm;
    double* m_dvm_norm;
    double* m_dvn_norm;
    double* m_dwm;
    double* m_dwmp;
    double* m_dT0m;
    double* m_dT1m;
    double* m_dT2m;
    double3* m_drn;
    double3* m_drm;
    double3* m_dVeln;
    double3* m_dVels;
    double3* m_dFn;
    double3* m_dFn_robin;
    double3* m_drm_loc;
    double3* m_dnmSm;
    double* m_dVolm;
    double* m_dPrem;

    int m_gelId;
    int m_gelType;
    double3 m_gelPosition;
    int3 m_gelSize;
    double m_dx, m_dy, m_dz;
    int3 m_gelNodeGrid;
    double m_dt;
    int m_df;
    int m_numGelElements;
    int m_numGelNodes;
    int m_boundaryCount;
    cudaStream_t m_gel_stream;
    std::thread m_file_writer_thread;
    double m_anchor_z = 0.0;
    bool m_use_anchor = false;
    bool flag = false;

    glsm_gel handle;  // the library object

private:
    // page-locked staging of the output snapshot that writeFiles' writer
    // thread formats (rn, Fn, Veln, rm, um, vm, wm, the time series)
    double* m_snap = nullptr;
    size_t m_snap_doubles = 0;
    void writeSnapshot(int time);
};
