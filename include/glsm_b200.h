/*
 * glsm_b200.h -- C ABI of libglsm_b200.so, the B200 (sm_100a) implementation of
 * the coupled gel-fluid step of lasite/gLSM_fluid_3D.
 *
 * The three opaque handle types stand for the reference's three classes
 * (src/gel.h:33-165 Gel, src/coupling.h:14-58 Coupler, src/fluid.h:24-84 Fluid).
 * Each entry point names the reference member it replaces.  Conventions:
 *   - every function returns an int status: GLSM_OK (0) or a negative code;
 *     glsm_last_error() gives a one-line message (thread-local);
 *   - host buffers are owned by the caller, device memory by the library;
 *   - objects are created in the reference's order Gel -> Coupler -> Fluid
 *     (src/fluid.cu:221-229 writes the unit conversions into the coupler and
 *     every gel, so the fluid comes last);
 *   - once coupled, all work of a system runs in program order on one CUDA
 *     stream owned by the coupler (glsm_coupler_stream).
 * Field layouts follow the reference: lattice cell index x + y*nx + z*nx*ny,
 * populations f[i + q*N] in the D3Q19 order of src/fluid.cu:202-215, gel node
 * vectors as xyz triples over (LX+2)(LY+2)(LZ+2) slots, element scalars over
 * (LX+1)(LY+1)(LZ+1) slots (src/gel.cu:116-119).
 */
#ifndef GLSM_B200_H
#define GLSM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GLSM_OK 0
#define GLSM_ERR_ARG (-1)    /* invalid argument or size */
#define GLSM_ERR_CUDA (-2)   /* a CUDA runtime call failed */
#define GLSM_ERR_STATE (-3)  /* call not valid in the object's current state */
#define GLSM_ERR_DEVICE (-4) /* a kernel raised an error flag (see message) */
#define GLSM_ERR_NOMEM (-5)  /* device allocation failed */

/* population storage of the lattice */
#define GLSM_STORE_F32 0  /* FP32 deviations f_q - w_q */
#define GLSM_STORE_F16 1  /* FP16 deviations, scaled by fp16_scale */
#define GLSM_STORE_BF16 2 /* BF16 deviations */

typedef struct glsm_gel_s* glsm_gel;
typedef struct glsm_coupler_s* glsm_coupler;
typedef struct glsm_fluid_s* glsm_fluid;

/* gel fields (FP64, reference layout) for glsm_gel_read / _write / _device_ptr */
enum glsm_gel_field {
    GLSM_GEL_RN = 0,       /* m_drn      node positions (3 per node slot)     */
    GLSM_GEL_VELN = 1,     /* m_dVeln    node (polymer) velocities            */
    GLSM_GEL_VELS = 2,     /* m_dVels    solvent velocities                   */
    GLSM_GEL_FN = 3,       /* m_dFn      nodal forces                         */
    GLSM_GEL_UM = 4,       /* m_dum      activator per element slot           */
    GLSM_GEL_VM = 5,       /* m_dvm      catalyst per element slot            */
    GLSM_GEL_WM = 6,       /* m_dwm      polymer volume fraction              */
    GLSM_GEL_UN_NORM = 7,  /* m_dun_norm nodal normalised activator           */
    GLSM_GEL_VN_NORM = 8,  /* m_dvn_norm                                      */
    GLSM_GEL_T0 = 9,       /* m_dT0m                                          */
    GLSM_GEL_T1 = 10,      /* m_dT1m                                          */
    GLSM_GEL_T2 = 11,      /* m_dT2m                                          */
    GLSM_GEL_RM = 12,      /* m_drm      element centres (3 per element slot) */
    GLSM_GEL_NMSM = 13,    /* m_dnmSm    face area vectors (18 per element)   */
    GLSM_GEL_VOLM = 14,    /* m_dVolm                                         */
    GLSM_GEL_PREM = 15,    /* m_dPrem                                         */
    GLSM_GEL_UN_ROBIN = 16,/* m_dun_robin                                     */
    GLSM_GEL_UM_NORM = 17, /* m_dum_norm                                      */
    GLSM_GEL_VM_NORM = 18, /* m_dvm_norm                                      */
    GLSM_GEL_WMP = 19,     /* m_dwmp                                          */
    GLSM_GEL_FN_ROBIN = 20,/* m_dFn_robin                                     */
    GLSM_GEL_RM_LOC = 21,  /* m_drm_loc  (24 per element)                     */
    GLSM_GEL_NFIELDS = 22,
    /* the centre-element time series (glsm_gel_series_config): 12 doubles per
     * record x capacity, for glsm_gel_read / glsm_gel_field_size / snapshots */
    GLSM_GEL_SERIES = 64
};

/* lattice fields for glsm_fluid_read / _write (FP32, reference layout) */
enum glsm_fluid_field {
    GLSM_FLUID_POP = 0, /* d_f after the last substep: 19*N absolute populations */
    GLSM_FLUID_RHO = 1, /* d_rho: N, density moment of the last substep's macros  */
    GLSM_FLUID_U = 2,   /* d_u: 3*N, velocity of the last substep's macros       */
    GLSM_FLUID_C1 = 3   /* d_c1: N, concentration                                */
};

/* marker fields of a coupler for glsm_coupler_read (FP32) */
enum glsm_marker_field {
    GLSM_MK_LAG = 0,   /* d_lag_all_   3*M */
    GLSM_MK_UL = 1,    /* d_Ul_all_    3*M */
    GLSM_MK_VL = 2,    /* d_Vl_all_    3*M */
    GLSM_MK_FDRAG = 3, /* d_Fdrag_all_ 3*M */
    GLSM_MK_FREP = 4,  /* d_Frep_all_  3*M */
    GLSM_MK_CL = 5,    /* d_Cl_all_    M   */
    GLSM_MK_DL = 6,    /* d_Dl_all_    M   */
    GLSM_MK_SL = 7     /* d_Sl_all_    M   */
};

/* lattice description; glsm_fluid_desc_default fills the reference's values */
typedef struct glsm_fluid_desc {
    int nx, ny, nz;      /* lattice cells per axis (any size >= 4)                   */
    int nsub;            /* LBM substeps per gel step (reference: 25, fluid.cu:194-197) */
    int storage;         /* GLSM_STORE_*                                             */
    float tau;           /* BGK relaxation time (0.8, fluid.cu:184)                  */
    float beta;          /* IBM penalty (1.0 or $IBM_BETA, fluid.cu:198-201)          */
    float ramp_steps;    /* IBM ramp length (20000 or $IBM_RAMP_STEPS, fluid.cu:265)  */
    float force[3];      /* uniform body force F_const (0, fluid.cu:219)              */
    int periodic[3];     /* periodic axes (the reference walls all six faces)         */
    float fp16_scale;    /* power-of-two scale of FP16 deviations (default 2^20)       */
    float h;             /* physical length of a lattice cell (0.5, fluid.cu:168)     */
} glsm_fluid_desc;

const char* glsm_last_error(void);
int glsm_version(void);

/* ---- Gel ---------------------------------------------------------------- */
/* Gel::Gel(int3 gelSize, double3 gelPosition, int gelType, int gel_id, int time)
 * src/gel.h:35, src/gel.cu:555-663 (time = 0; steady state by bisection,
 * gel.cu:424-450; node lattice, gel.cu:179-219; surface order, gel.cu:161-177) */
int glsm_gel_create(int sx, int sy, int sz, double px, double py, double pz, int gel_type, int gel_id,
                    glsm_gel* out);
/* Gel::~Gel, src/gel.cu:665-668.  A gel that still belongs to a coupler is
 * released together with that coupler (it must not be used in between). */
int glsm_gel_destroy(glsm_gel g);
/* sizes: LX, LY, LZ, element slots, node slots, markers, gel id, gel type */
int glsm_gel_info(glsm_gel g, int64_t out[8]);
/* GelParams uss, vss, wss (src/gel.h:12) */
int glsm_gel_steady_state(glsm_gel g, double out[3]);
/* Gel::stepElasticity(int iter), src/gel.cu:682-698 */
int glsm_gel_step_elasticity(glsm_gel g, int iter);
/* Gel::stepChemistry(int iter), src/gel.cu:700-704 */
int glsm_gel_step_chemistry(glsm_gel g, int iter);
/* Gel::recordCenter(int iter), src/gel.cu:706-713: one record every `every`
 * iterations into a ring of `capacity` records (set by glsm_gel_series_config) */
int glsm_gel_record_center(glsm_gel g, int iter);
/* records of 12 doubles: iter, rn(3), Fn(3), Veln(3) of the centre node, vm, wm
 * of the centre element (the columns of gel<id>bodycenter.dat, gel.cu:505-537) */
int glsm_gel_series_config(glsm_gel g, int every, int capacity);
int glsm_gel_series_read(glsm_gel g, double* dst, size_t count);
/* Output snapshot of gel fields (extension; Gel::copyDataToHost,
 * src/gel.cu:355-373, is synchronous): fields[k] (GLSM_GEL_* fields, the
 * time-series ring included) are copied on the device behind the queued work,
 * then transferred into dst[k] on a copy stream; returns at once (as
 * glsm_fluid_snapshot; dst page-locked and untouched until
 * glsm_gel_snapshot_wait returns).  At most 32 fields. */
int glsm_gel_snapshot(glsm_gel g, int n_fields, const int* fields, double* const* dst);
int glsm_gel_snapshot_wait(glsm_gel g);
/* Gel::resetToQuiescent(), src/gel.cu:731-747 */
int glsm_gel_reset_quiescent(glsm_gel g);
/* Gel::fireExcitationPulse(), src/gel.cu:751-783 */
int glsm_gel_fire_pulse(glsm_gel g);
/* Gel::setAnchorZ(double), src/gel.cu:788-795 */
int glsm_gel_set_anchor_z(glsm_gel g, double anchor_z);
/* Gel::buildTubeMask(int, bool), src/gel.cu:811-867 */
int glsm_gel_build_tube_mask(glsm_gel g, int wall_thickness, int circular);
/* the drivers' delayed start (src/sim_array.cpp:86-103) for glsm_fluid_run:
 * the gel is skipped before `iter` and fires its pulse at `iter` (0: always on) */
int glsm_gel_set_active_from(glsm_gel g, int iter);
/* GelParams::f (the BZ stoichiometric factor, src/gel.cu:634): sets f, recomputes
 * the steady state by bisection and restarts the interior chemistry from it, as
 * the reference's constructor does for its fixed f.  Call before stepping. */
int glsm_gel_set_bz_f(glsm_gel g, double f);
/* seeded uniform noise in [-amplitude, amplitude) added to um and vm of the
 * interior elements (splitmix64 keyed by seed, gel id, slot, field) */
int glsm_gel_add_noise(glsm_gel g, uint64_t seed, double amplitude);
/* host copies of a field (count = number of doubles); the write replaces the
 * field (restart, src/gel.cu:221-282) */
int glsm_gel_read(glsm_gel g, int field, double* dst, size_t count);
int glsm_gel_write(glsm_gel g, int field, const double* src, size_t count);
size_t glsm_gel_field_size(glsm_gel g, int field);
/* device pointer of a field: the reference's public m_d* members.  From then on
 * glsm_fluid_run packs this gel's markers afresh at the start of every call, so
 * writes through the pointer between calls reach the markers. */
void* glsm_gel_device_ptr(glsm_gel g, int field);
/* calFilamentD (src/gel_kernels.cu:837-866, run by Gel::recordCenter,
 * src/gel.cu:706-713): the points where the nodal u_norm and v_norm fields both
 * equal 0.15 on the node faces of each z layer -- (xi + xb, yi + yb, zi) in node
 * units, one per face that holds a crossing, in x-fastest face order (the
 * reference appends them in atomic order into a 300-slot buffer it never
 * writes out).  As in the reference, y is solved from the u contour, so a face
 * where u_norm does not vary along y reports no crossing.  Writes up to
 * max_points points (3 doubles each) into xyz and the total count into
 * *n_points. */
int glsm_gel_filament(glsm_gel g, double* xyz, size_t max_points, size_t* n_points);

/* ---- Coupler ------------------------------------------------------------ */
/* Coupler::Coupler(std::vector<Gel*>&), src/coupling.h:16, src/coupling.cu:50-80 */
int glsm_coupler_create(const glsm_gel* gels, int n_gels, glsm_coupler* out);
/* Coupler::~Coupler, src/coupling.cu:158-161 (gels stay alive) */
int glsm_coupler_destroy(glsm_coupler c);
/* Coupler::packFromGels(), src/coupling.cu:82-98 */
int glsm_coupler_pack(glsm_coupler c);
/* Coupler::scatterToGels(), src/coupling.cu:100-118 */
int glsm_coupler_scatter(glsm_coupler c);
/* Coupler::applyGelRepulsion(), src/coupling.cu:120-123 */
int glsm_coupler_repulsion(glsm_coupler c);
/* marker count M (sumGelBoundaryCount, src/coupling.h:47) */
int glsm_coupler_markers(glsm_coupler c);
int glsm_coupler_read(glsm_coupler c, int field, float* dst, size_t count);
/* the system stream (a cudaStream_t) */
void* glsm_coupler_stream(glsm_coupler c);

/* ---- Fluid -------------------------------------------------------------- */
int glsm_fluid_desc_default(glsm_fluid_desc* d, int nx, int ny, int nz);
/* Fluid::Fluid(int3 fluidSize, int time, Coupler*), src/fluid.h:26,
 * src/fluid.cu:152-232; lattice dims and nsub are given directly */
int glsm_fluid_create(const glsm_fluid_desc* d, glsm_coupler c, glsm_fluid* out);
/* Fluid::~Fluid, src/fluid.cu:234-237 */
int glsm_fluid_destroy(glsm_fluid f);
/* Fluid::stepVelocity(int iter), src/fluid.cu:263-284 */
int glsm_fluid_step_velocity(glsm_fluid f, int iter);
/* Fluid::stepConcentration(int iter), src/fluid.cu:251-261 */
int glsm_fluid_step_concentration(glsm_fluid f, int iter);
/* n whole coupled iterations iter0 .. iter0+n-1 in the order of src/sim.cpp:97-112
 * (gels, pack, stepVelocity, stepConcentration, repulsion, scatter), each one a
 * CUDA graph launch; asynchronous on the system stream.  The pack runs when the
 * markers can have changed: after a gel's mechanics moved its nodes, and first in
 * a call after a gel was changed through this interface or has a device pointer
 * out (glsm_gel_device_ptr); it gives the same markers as packing every time. */
int glsm_fluid_run(glsm_fluid f, int iter0, int n);
/* wait for the system stream and report device-side error flags */
int glsm_fluid_sync(glsm_fluid f);

/* ---- Exact-restart checkpoint (extension) -------------------------------
 * The whole coupled system reachable from f (the fluid, its coupler and its
 * gels): populations in their current layout, u, IBM force, both
 * concentration buffers, marker state, every gel array, the time-series ring,
 * the iteration counter and the mutable gel settings (BZ f, anchor, activation,
 * tube mask).  Loading it restores that state byte for byte; the run then
 * continues as an uninterrupted one would, up to the ordering of the
 * floating-point atomics in the spreads (which also separates two runs).
 * The reference restarts from its .dat text files through Gel::setGoonValue
 * (src/gel.cu:221-282) and Fluid::setGoonValue, which re-initialises the
 * populations at rest (src/fluid.cu:57-59) and reads only u and c back.
 * A checkpoint loads into any system built with the same fluid descriptor and
 * the same gels (sizes, types, order); the system must not be in a batch. */
int glsm_checkpoint_bytes(glsm_fluid f, size_t* bytes);
int glsm_checkpoint_save(glsm_fluid f, void* buf, size_t bytes);
int glsm_checkpoint_load(glsm_fluid f, const void* buf, size_t bytes);
/* host copies of lattice fields (FP32, reference layout) */
int glsm_fluid_read(glsm_fluid f, int field, float* dst, size_t count);
/* Output snapshot (extension; Fluid::copyDataToHost, src/fluid.cu:85-90, is
 * synchronous): enqueues behind the work already queued on the system stream a
 * device-side copy of u (3 N floats, xyz) and of the current c1 (N floats),
 * then their transfer into u_dst and c_dst on a copy stream, and returns at
 * once.  Iterations enqueued afterwards run on without waiting for the transfer.
 * For the transfer to overlap, u_dst and c_dst must be page-locked host memory
 * (cudaMallocHost); they must stay untouched until glsm_fluid_snapshot_wait
 * returns.  A later snapshot waits on the device for the earlier transfer. */
int glsm_fluid_snapshot(glsm_fluid f, float* u_dst, float* c_dst);
int glsm_fluid_snapshot_wait(glsm_fluid f);
/* replace populations (GLSM_FLUID_POP, absolute values), u (GLSM_FLUID_U) or c1 */
int glsm_fluid_write(glsm_fluid f, int field, const float* src, size_t count);
/* Global mass and momentum of the lattice (extension; the reference computes
 * neither): out[0] = sum over cells of rho, out[1..3] = sum over cells and
 * directions of c_q f_q (the population momentum, before the half-force shift
 * of u).  Each stored population is widened to FP64 and the sums are reduced
 * on the device in a fixed order, so the result is deterministic.  Bounce-back
 * walls and Guo forcing conserve the mass; with all axes periodic the momentum
 * grows by N F_const per substep. */
int glsm_fluid_conservation(glsm_fluid f, double out[4]);
/* Deterministic spreads (extension; the reference spreads with float atomics,
 * src/fluid_kernels.cu:300-348, :414-459): on = 1 makes every cell inside a
 * marker box gather its IBM force and its concentration source from the
 * markers whose stencils cover it -- gels in order, markers in order -- instead
 * of the markers adding them with atomics, so that a run repeats bit for bit.
 * Results differ from the atomic form only by round-off.  Cost: one pass over
 * the box's markers per box cell and substep. */
int glsm_fluid_set_deterministic(glsm_fluid f, int on);
/* Rounding of FP16 population storage (extension; the reference stores FP32).
 * mode 0 (default): each post-collision value rounds to nearest.  mode 1,
 * conserving: each cell's 19 values are rounded so that the cell's summed mass
 * and momentum rounding errors nearly cancel (round to nearest, then one
 * greedy pass in which a value may take its other FP16 neighbour when that
 * lowers the squared mass and momentum error).  mode 2: conserving on odd
 * substeps, to nearest on even ones.  Round-to-nearest noise accumulates in
 * long-wavelength modes that viscosity damps slowly; the conserving forms keep
 * the long-horizon velocity error near that of a single rounding (mode 1) or
 * halve the accumulation (mode 2), for about 390 more instructions per cell
 * and conserving substep.  Needs FP16 storage; not while the system is in a
 * batch. */
int glsm_fluid_set_f16_rounding(glsm_fluid f, int mode);
/* L2 residency of the population array (extension; the reference leaves L2 to
 * the hardware).  on = 1 (off by default): the substep launches carry an
 * access-policy window that marks the array persisting, so a 101^3 array
 * (78 MB FP32) stays in the 126 MB L2 across the substeps of an iteration.
 * The persisting set-aside is a limit of the process's CUDA context, and the
 * L2 it reserves is lost to every access outside a window (other fluids, a
 * batch, the caller's kernels): it is sized to the largest window in use and
 * released when the last fluid using one turns it off, is destroyed or joins a
 * batch (which turns it off).  For one system alone on the GPU whose array
 * fits in the device's largest set-aside (82.9 MB on a B200: FP32 up to ~103^3
 * cells, FP16 up to ~130^3); for a larger array the call leaves the window off.
 * Not while the system is in a batch. */
int glsm_fluid_set_l2_persisting(glsm_fluid f, int on);
/* Turns every persisting L2 line of the context back into a normal one
 * (cudaCtxResetPersistingL2Cache): a benchmark calls it, with the stream idle,
 * before it flushes L2 between timed steps. */
int glsm_l2_reset_persisting(void);
/* The context's current persisting L2 set-aside in bytes (0 when no fluid keeps
 * its populations L2-persisting). */
int glsm_l2_persisting_setaside(size_t* bytes);
/* The conserving FP16 rounding on its own (verification aid, no counterpart in
 * the reference): in and out hold n_cells x 19 scaled values ([cell][q], q in
 * the D3Q19 order above) in host memory; out receives the float values of the
 * chosen FP16 numbers.  At most 2^26 cells per call. */
int glsm_f16_conserve_round(const float* in, float* out, size_t n_cells);
/* nx, ny, nz, N, nsub, storage, device bytes, substeps done */
int glsm_fluid_info(glsm_fluid f, int64_t out[8]);
/* Fluid::stepVelocity(iter) with a CUDA event pair around each substep launch on
 * the system stream; ms[k] (nsub floats) receives the duration of substep k.
 * Used to report the substep kernel's achieved bandwidth. */
int glsm_fluid_profile_velocity(glsm_fluid f, int iter, float* ms);
/* Fluid::stepVelocity(iter) as one captured graph of its nsub substep launches,
 * with a single CUDA event pair around it: *total_ms is the time of the nsub
 * launches back to back, as they run inside the fused iteration graph. */
int glsm_fluid_profile_substeps(glsm_fluid f, int iter, float* total_ms);
/* n_steps (1..64) calls of Fluid::stepVelocity(iter + j) as one captured graph
 * of n_steps x nsub substep launches with one CUDA event pair around it.  The
 * difference between two n_steps values, divided by the substeps between them,
 * is the substep launch time without the graph's launch overhead (one 2 x nsub
 * word ticket reset per velocity step is included). */
int glsm_fluid_profile_substeps_n(glsm_fluid f, int iter, int n_steps, float* total_ms);
/* Test aid for the bounded device waits (no counterpart in the reference):
 * extra > 0 makes every force-region tile of the following substep launches
 * wait for `extra` IBM tasks that do not exist, so the wait gives up after its
 * limit (a fraction of a second), the launch completes with the forces spread
 * so far, and the next glsm_fluid_sync reports GLSM_ERR_DEVICE with
 * "IBM wait timed out".  extra = 0 (the default) restores normal launches. */
int glsm_test_ibm_wait_extra(glsm_fluid f, int extra);
/* gel_to_lbm_vel and lbm_to_gel_vel (src/fluid.cu:221-222) */
int glsm_fluid_units(glsm_fluid f, float out[2]);

/* Copy-bandwidth probe (extension: a measurement aid with no counterpart in
 * the reference).  Copies a `bytes`-sized buffer back and forth `reps` times in
 * one launch through L2 only (L1 bypassed) and stores read + write bytes per
 * second in *gbs (GB/s).  With 2 x bytes well below the L2 size this is the
 * L2 copy bandwidth the substep kernel is compared with when the population
 * array fits in L2; with 2 x bytes well above it, the HBM copy bandwidth.
 * Allocates and frees its two buffers; bytes a multiple of 16 in [16, 8 GiB],
 * reps in [1, 100000].  glsm_copy_bandwidth_error() explains a failure. */
int glsm_copy_bandwidth(size_t bytes, int reps, double* gbs);
const char* glsm_copy_bandwidth_error(void);
/* Access-pattern probe (extension, a measurement aid with no counterpart in the
 * reference): on an nx x ny x nz lattice in the substep kernel's layout and
 * element size (storage GLSM_STORE_*), every cell reads its 19 populations and
 * writes them back with no collision in between -- in the even AA form (own
 * slots) and in the odd form (the 18 neighbours' slots, for the cells whose
 * neighbours all lie in the array) -- `reps` launches each after a warm-up.
 * *gbs_even / *gbs_odd receive 2 x 19 x element bytes per cell and launch
 * over the time: the bandwidth a collision-free substep could reach with this
 * pattern on this device, the roofline the substep kernel is set against
 * beside the copy probes.  Allocates and frees its array; error text from
 * glsm_copy_bandwidth_error(). */
int glsm_pattern_bandwidth(int nx, int ny, int nz, int storage, int reps, double* gbs_even, double* gbs_odd);

/* ---- Batch: several systems advanced together -----------------------------
 * No single counterpart in the reference (which runs one system per process);
 * this is the serving form of Fluid::stepVelocity & co.  Systems (fluid handles
 * with their coupler and gels) of any lattice size and gel count join a batch;
 * glsm_batch_run advances every member by n whole coupled iterations, each one
 * a CUDA graph of batched launches (one persistent launch per substep for all
 * members).  All members need the same nsub.  While in a batch a system cannot
 * be stepped on its own; reads wait for the batch.  Membership changes
 * re-capture the graph at the next run. */
typedef struct glsm_batch_s* glsm_batch;
int glsm_batch_create(glsm_batch* out);
int glsm_batch_destroy(glsm_batch b);
/* f enters the batch; its next iteration number is iter0; it runs n_iters more
 * iterations (then idles until removed), or without limit when n_iters <= 0 */
int glsm_batch_add(glsm_batch b, glsm_fluid f, int iter0, int n_iters);
/* iterations f still has to run in the batch (-1: no limit, -2: not a member) */
long long glsm_batch_remaining(glsm_batch b, glsm_fluid f);
int glsm_batch_remove(glsm_batch b, glsm_fluid f);
int glsm_batch_size(glsm_batch b);
int glsm_batch_run(glsm_batch b, int n);
int glsm_batch_sync(glsm_batch b);

/* ---- Substep without device allocation ------------------------------------
 * No counterpart in the reference: an extra entry point for callers that cannot
 * call cudaMalloc (a host framework that owns all device memory through its own
 * pool, a plug-in whose host process must account for every device byte, a
 * real-time loop where an allocation may synchronise the device).  Such callers
 * cannot create the handles above, which own their buffers.
 *
 * One LBM substep with immersed-boundary forcing on caller-owned device
 * buffers, enqueued on `stream` (a cudaStream_t, NULL for the default stream):
 *   pop      19 planes of `plane_stride` floats: population deviations f_q - w_q
 *            in the D3Q19 order of the reference, updated in place with the AA
 *            pattern (parity 0 turns natural-layout post-stream values into
 *            post-collision values in reversed slots; parity 1 turns those back
 *            into natural post-stream values, so two calls make one full step)
 *   u4       per cell (ux, uy, uz, rho): read as the previous substep's velocity
 *            for the interpolation, overwritten with this substep's
 *   lag4     per marker (x, y, z, -) positions in physical units (lattice
 *            coordinate = position / h); vel4 per marker target velocity (lattice)
 *   Ul4, Fdrag4  per marker outputs: interpolated velocity, penalty force
 * Walls bounce back on all six faces; tau, the uniform force (fx, fy, fz) and
 * beta_eff are the BGK relaxation time, F_const and the ramped IBM penalty.
 * Limits: at most 262,144 lattice cells and 16,384 markers per call.  The
 * scratch lives in one file-scope device array of 5,308,416 bytes that every
 * GPU loading the library holds until the process exits; the first call on a
 * device looks up its address, so make that first call before any stream
 * capture.  All calls on a device share the scratch (it is cleared at the
 * start of each call): calls that overlap on the GPU race on it.
 * Returns GLSM_OK or a negative status; glsm_noalloc_last_error() explains. */
int glsm_substep_noalloc(float* pop, int64_t plane_stride, float* u4, int nx, int ny, int nz, int parity, float tau,
                         float fx, float fy, float fz, const float* lag4, const float* vel4, int n_markers, float h,
                         float beta_eff, float* Ul4, float* Fdrag4, void* stream);
const char* glsm_noalloc_last_error(void);
size_t glsm_noalloc_scratch_bytes(void);

#ifdef __cplusplus
}
#endif
#endif /* GLSM_B200_H */
