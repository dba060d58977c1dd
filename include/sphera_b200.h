/*
 * sphera_b200.h -- C ABI of the B200 (sm_100a) implementation of SPHERA's
 * per-step particle hot path (SA-SPH, leapfrog, linear barotropic EoS).
 *
 * Every entry point is extern "C", takes plain pointers, sizes and POD
 * structs with fixed-width members, and returns an int status (SPH_OK = 0),
 * so a Fortran `bind(C)` interface can map it one to one.
 *
 * The reference (SPHERA v10.0.0, Fortran 90 + OpenMP) implements the same
 * path as argument-less subroutines that read and write module globals
 * (pg(:), Icont, NPartOrd, PartIntorno, PartKernel, rag,
 * BoundaryDataPointer, BoundaryDataTab).  Each fine-grained entry point below
 * replaces one call site of src/Main_algorithm/time_step_loop.f90; the cited
 * file:line is the reference unit it stands in for.
 *
 * Ownership: the library owns device memory and the handle.  Host buffers
 * passed in are caller-owned and only read or written during the call.  The
 * library keeps particles in its own cell-sorted order on the device and
 * reads/writes host arrays in the caller's particle order (index npi-1 of
 * pg(npi)), keeping the permutation itself.
 *
 * Threading: a handle is not re-entrant (the reference calls these units
 * from the master thread).  Separate handles may be driven from separate
 * host threads; each handle owns its CUDA stream.
 */
#ifndef SPHERA_B200_H
#define SPHERA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Status codes.  Codes >= 100 mirror the reference's fatal                */
/* diagnostic(arg1,arg2) pairs as 100*arg1 + arg2                          */
/* (src/Memory_I_O/diagnostic.f90); the library never aborts or traps.     */
/* ---------------------------------------------------------------------- */
#define SPH_OK                       0
#define SPH_ERR_INVALID_ARGUMENT     1   /* bad pointer, size or parameter          */
#define SPH_ERR_UNSUPPORTED          2   /* feature outside the implemented path    */
#define SPH_ERR_CUDA                 3   /* a CUDA runtime call failed              */
#define SPH_ERR_NO_DEVICE            5   /* no sm_100 device visible                */
#define SPH_ERR_TIMEOUT              6   /* a bounded device wait gave up           */
#define SPH_CANCELLED                7   /* the host cancelled the simulation       */
#define SPH_ERR_ALLOC              400   /* diagnostic(4): allocation failure       */
#define SPH_ERR_BDT_OVERFLOW       802   /* diagnostic(8,2): BoundaryDataTab full   */
#define SPH_ERR_CLOSE_FACES        807   /* diagnostic(8,7): > MAXCLOSEBOUNDFACES   */
#define SPH_ERR_CLOSE_SIDES        808   /* diagnostic(8,8): > MAXCLOSEBOUNDSIDES   */
#define SPH_ERR_NCBF_MAX           904   /* diagnostic(9,4): Ncbf_Max too large     */

/* Warning bits (non-fatal; the reference writes a message and continues). */
#define SPH_WARN_NEIGHBOURS_TRUNCATED  0x1  /* CalcVarLength.f90:197-205 list cap  */
#define SPH_WARN_PARTICLES_REMOVED     0x2  /* OrdGrid1.f90:71-82 out of grid     */

/* Precision forms. */
#define SPH_PREC_FP64   0   /* plain FP64, the reference's arithmetic           */
#define SPH_PREC_FP32C  1   /* FP32 pair sums with compensated accumulation,
                               FP64 positions/integration                        */

/* Boundary zone types (Tratto%tipo).  Only solid walls are on this path.  */
#define SPH_ZONE_FIXE   1   /* "fixe": fixed wall                                */
#define SPH_ZONE_TAPI   2   /* "tapi": wall translating at constant velocity     */

/* ---------------------------------------------------------------------- */
/* Parameters: the subset of Domain, Med(1) and input_any_t the hot path    */
/* reads (src/Modules/Hybrid_allocation_module.f90, ReadInput*.f90).        */
/* ---------------------------------------------------------------------- */
typedef struct SphParams {
    int32_t dim;                    /* 2 (SPACE_2D, x-z plane) or 3 (SPACE_3D)        */
    int32_t precision;              /* SPH_PREC_FP64 or SPH_PREC_FP32C                */
    double  dx;                     /* Domain%dx                                      */
    double  trunc;                  /* Domain%trunc = h/dx                            */
    double  coef_nmaxpartj;         /* input_any_t%COEFNMAXPARTJ                      */
    int32_t max_close_bound_faces;  /* input_any_t%MAXCLOSEBOUNDFACES (3D)            */
    int32_t dt_alfa_mon;            /* logical dt_alfa_Mon                            */
    double  domain_lo[3];           /* Domain%coord(:,1)                              */
    double  domain_hi[3];           /* Domain%coord(:,2)                              */
    double  den0;                   /* Med%den0                                       */
    double  eps;                    /* Med%eps, bulk modulus K                        */
    double  alfa_mon;               /* Med%alfaMon                                    */
    double  kin_visc;               /* Med%kin_visc = mu/den0                         */
    double  p_ref;                  /* Domain%prif                                    */
    double  grav[3];                /* Domain%grav                                    */
    double  cfl;                    /* input_any_t%CFL                                */
    double  vsc_coeff;              /* input_any_t%vsc_coeff                          */
    double  pesodt;                 /* pesodt                                         */
    int32_t density_thresholds;     /* input_any_t%density_thresholds (0/1)           */
    int32_t bdt_capacity;           /* BoundaryDataTab entries to reserve,            */
                                    /* 0 = 3 n (3D) or 2 n (2D)                       */
    double  teta_p;                 /* input_any_t%TetaP, partial pressure smoothing  */
    double  teta_v;                 /* input_any_t%TetaV, partial velocity smoothing  */
    /* Lateral tank forcing, no reference counterpart: the tank moves as
     * x = A sin(2 pi t / T) and the fluid, computed in the tank frame, feels
     * the body force grav + A (2 pi / T)^2 sin(2 pi t / T) along x, with
     * t the end time of the step being computed (the simulation time when
     * time_step_loop.f90 calls RHS_momentum_equation).  amplitude 0
     * disables it.                                                        */
    double  forcing_amplitude;      /* A [m]                                          */
    double  forcing_period;         /* T [s]                                          */
    /* 1st-order consistency (input_any_t%C1_BE, %C1_divu, %invB_det_thresh):
     * the pressure-gradient terms of the momentum equation are renormalised
     * with B_ren_gradp and, with c1_divu as well, the velocity gradients of
     * the continuity equation with B_ren_divu.  Both precision forms (the
     * matrices, their inversion and the renormalisation in FP64; in the
     * FP32c form the renormalised pair sums are compensated FP32 sums).  A
     * matrix whose |det| is below invb_det_thresh is replaced by -I
     * (B_ren_gradp_inversion.f90:62-73).  In 2D the matrices have a zero y
     * row and column, so they always take that -I (which renormalises
     * nothing) and invb_det_thresh must be > 0 (the reference would divide
     * by the zero determinant).  0 disables.                                */
    int32_t c1_be;
    int32_t c1_divu;
    double  invb_det_thresh;        /* >= 0                                           */
} SphParams;

/* One boundary zone (Tratto). */
typedef struct SphZone {
    int32_t type;                   /* SPH_ZONE_FIXE / SPH_ZONE_TAPI                  */
    int32_t slip_coefficient_mode;  /* Partz%slip_coefficient_mode (1 only)           */
    double  velocity[3];            /* Tratto%velocity (tapi)                         */
    double  bc_shear_stress_input;  /* Partz%BC_shear_stress_input: slip coefficient  */
    int32_t laminar_no_slip_check;  /* Tratto%laminar_no_slip_check (logical)         */
    int32_t reserved;
} SphZone;

/* Boundary geometry.  Indices are 1-based, as in the input deck.          */
typedef struct SphGeometry {
    int32_t        n_vertices;
    const double*  vertices;        /* [n_vertices][3]                                */
    int32_t        n_zones;
    const SphZone* zones;           /* [n_zones]                                      */
    /* 3D: quadrilateral or triangular faces (BoundaryFace) */
    int32_t        n_faces;
    const int32_t* face_nodes;      /* [n_faces][4] vertex ids, 0 pads a triangle     */
    const int32_t* face_zone;       /* [n_faces] zone id                              */
    /* 2D: boundary sides (BoundarySide), vertex 1 -> vertex 2 */
    int32_t        n_sides;
    const int32_t* side_vertices;   /* [n_sides][2] vertex ids                        */
    const int32_t* side_zone;       /* [n_sides] zone id                              */
} SphGeometry;

/* Particle state in the caller's order (pg(1:n)).  The arrays may be host
 * memory or device memory of the handle's device (as may the laminar-flag
 * arrays of sph_replace_particles, sph_set_clock and sph_dump_laminar):
 * copies take their direction from the pointers.                         */
typedef struct SphState {
    int32_t n;
    double* x;                      /* [n][3] pg%coord                                */
    double* v;                      /* [n][3] pg%vel (pg%var equals it, TetaV = 0)    */
    double* rho;                    /* [n]    pg%dens                                 */
    double* p;                      /* [n]    pg%pres                                 */
    double* m;                      /* [n]    pg%mass                                 */
} SphState;

typedef struct SphStepInfo {
    double  time;                   /* simulation_time after the steps                */
    double  dt;                     /* dt of the last completed step                  */
    int32_t step;                   /* on_going_time_step                             */
    int32_t n;                      /* nag (particles still in the grid)              */
    int32_t warnings;               /* SPH_WARN_* bits accumulated                    */
    int32_t max_neighbours;         /* largest neighbour count seen (incl. self)      */
} SphStepInfo;

typedef struct SphDiagnostics {
    int32_t warnings;               /* SPH_WARN_* bits                                */
    int32_t status;                 /* first fatal device status, SPH_OK if none      */
    int32_t removed_out_of_grid;    /* EpOrdGrid                                      */
    int32_t ncbf_max;               /* Ncbf_Max of the last boundary pass             */
    int32_t bdt_entries;            /* BoundaryDataTab entries in use                 */
    int32_t nmaxpartj;              /* NMAXPARTJ                                      */
    int32_t grid_ncd[3];            /* Grid%ncd                                       */
    int32_t n_cells;                /* Grid%nmax                                      */
} SphDiagnostics;

/* The simulation's clock between steps (a checkpoint of time_step_loop's
 * own variables): what Memo_Results.f90 writes before pg(1:nag) in a
 * restart record (it, simulation_time, dt) plus what the next step needs
 * to continue bit for bit.                                                 */
typedef struct SphClock {
    double  time;                   /* simulation_time                                */
    double  dt;                     /* dt of the next step                            */
    double  dt_prev;                /* dt of the last completed step (dtvel's other half) */
    double  dt_average;             /* time_step_duration's running mean (pesodt)     */
    int32_t step;                   /* on_going_time_step (completed steps)           */
    int32_t reserved;
} SphClock;

typedef struct SphHandle SphHandle;

/* ---------------------------------------------------------------------- */
/* Life cycle                                                              */
/* ---------------------------------------------------------------------- */

/* The device (0-based) the calling thread's next sph_create,
 * sph_batch_create or sph_create_slab builds its handle on.  A handle keeps
 * its device: every call on it runs there and gives the caller's current
 * device back on return, so one host thread may drive handles on several
 * GPUs.                                                                    */
int  sph_select_device(int32_t device);

/* Builds the grid (CreaGrid.f90:51-74), the boundary geometry
 * (DefineLocalSystemVersors.f90, GridCellBoundaryFacesIntersections3D.f90 /
 * DefineBoundarySideGeometry2D.f90) and the IC integral tables
 * (ComputeKernelTable.f90, ComputeBoundaryIntegralTab.f90) and reserves
 * device memory for up to n_capacity particles.                           */
int  sph_create(const SphParams* params, const SphGeometry* geometry,
                int32_t n_capacity, SphHandle** out);
void sph_destroy(SphHandle* h);

/* Uploads pg(1:n) and performs the IC part of time_step_loop.f90:82-173:
 * OrdGrid1, neighbour search, ComputeBoundaryDataTab and the IC
 * time_step_duration.  v doubles as pg%var.  x and m are copied first; the
 * sort, the neighbour search and the boundary data run on them while v,
 * rho and p are still being copied (with page-locked buffers; pageable ones
 * give the same results without the overlap).                            */
int  sph_upload(SphHandle* h, const SphState* state);
/* Copies pg(1:n) back in the caller's order (after removals, the
 * reference's swap-with-last order).  Any of x, v, rho, p, m may be NULL.  */
int  sph_download(SphHandle* h, SphState* state);

/* One or more whole leapfrog steps: time_step_loop.f90:175-405 with
 * time_split = 1, Domain%tipo = "semi", TetaP = TetaV = 0.                 */
int  sph_step(SphHandle* h, int32_t nsteps, SphStepInfo* info);

int  sph_get_diagnostics(SphHandle* h, SphDiagnostics* diag);

/* Enqueue nsteps whole steps on the handle's stream without waiting, and
 * wait for them (and read back the device status).  The step is replayed
 * from a CUDA graph built on the first call.                              */
int  sph_step_async(SphHandle* h, int32_t nsteps);
int  sph_sync(SphHandle* h);
/* sph_step(h, nsteps) followed by sph_download(h, state), for a host that
 * keeps the state in its own memory between steps (time_step_loop.f90 with
 * pg(:) on the CPU).  The positions, velocities and masses of the last
 * step are copied to the host while that step's neighbour search, boundary
 * data and continuity pass still run (copied again after the step when a
 * particle left the grid in it, which renumbers the rest).  The buffers must hold the particle
 * count before the call, as the host last saw it (sph_upload, or the last
 * call that returned a count); state->n returns the count after it (lower
 * after out-of-grid removals; rows from there on are unspecified).  The
 * overlap needs page-locked buffers (cudaHostAlloc / cudaHostRegister):
 * pageable ones give the same results without it.  Single simulations
 * only.                                                                    */
int  sph_step_download(SphHandle* h, int32_t nsteps, SphState* state);
/* The handle's cudaStream_t, for callers that order their own work after
 * the library's.                                                          */
void* sph_stream(SphHandle* h);

/* ---------------------------------------------------------------------- */
/* Batches: several independent simulations advanced by the same launches  */
/* (no reference counterpart; the reference runs one case per process).    */
/* All simulations of a batch share dim and precision.                     */
/* ---------------------------------------------------------------------- */
int  sph_batch_create(int32_t nsims, const SphParams* params, const SphGeometry* geometries,
                      const int32_t* n_capacity, SphHandle** out);
int  sph_batch_upload(SphHandle* h, int32_t nsims, const SphState* states);
/* One member's state (as sph_download).  The result is that member's own
 * status: another member's failure does not affect it, and a failed or
 * cancelled member's state is still copied while its code is returned.   */
int  sph_batch_download(SphHandle* h, int32_t sim, SphState* state);
/* A simulation whose time reaches t_end (> 0) stops advancing; its state
 * stays on the device for download while the others continue.             */
int  sph_batch_set_end_time(SphHandle* h, int32_t sim, double t_end);
int  sph_batch_info(SphHandle* h, int32_t sim, SphStepInfo* info, int32_t* frozen);
/* Every simulation's frozen flag, time, completed steps and status
 * ([nsims] each, any may be NULL) from one read-back of the device state.
 * A simulation that meets a fatal condition (status != SPH_OK, e.g.
 * SPH_ERR_BDT_OVERFLOW from its own share of the boundary-data pool)
 * freezes at the end of that step while the others advance unchanged;
 * this call reports it in status[] and itself fails only on CUDA errors
 * (sph_step / sph_sync return the first member's fatal status).           */
int  sph_batch_status(SphHandle* h, int32_t* frozen, double* time, int32_t* steps, int32_t* status);
/* Cancels simulation `sim` of a batch: from the next launch enqueued on the
 * handle's stream it is frozen with status SPH_CANCELLED, its state kept
 * (no wait; the counterpart of the reference's kill file,
 * time_step_loop.f90:485-487, for one member).                            */
int  sph_batch_cancel(SphHandle* h, int32_t sim);

/* Device memory, in bytes, that sph_batch_create would allocate for these
 * arguments (sph_create: nsims = 1), computed on the host without touching
 * the device; the admission test of a server that packs simulations into
 * an HBM budget (no reference counterpart).                               */
int  sph_memory_required(int32_t nsims, const SphParams* params, const SphGeometry* geometries,
                         const int32_t* n_capacity, uint64_t* bytes);
/* *idle = 1 when all work enqueued on the handle's stream has finished,
 * 0 while some is still running; never waits.                             */
int  sph_idle(SphHandle* h, int32_t* idle);

/* Autotuner (no reference counterpart): sizes the persistent grid of the
 * neighbour-list, momentum, continuity and boundary kernels on the live
 * state by timing `reps` launches of each candidate (1 to 32 blocks per
 * SM) of variants that leave the state unchanged, and for the momentum
 * and continuity pair loops also picks their shape (0: lean, one pair's
 * records at a time; 1: several list entries' records loaded together --
 * a list chunk's in the FP32c form, two entries' in the FP64 form; 2, FP32c
 * form only: 1 with two entries' terms computed on paired FP32
 * instructions, the same bits), then rebuilds the step graph.  Without C1
 * in both forms.
 * grid_out (may be NULL; 7 entries) receives in [0..4] the chosen blocks
 * of lists, momentum, continuity, boundary find and integrals, in [5] and
 * [6] the momentum and continuity shapes.                                 */
int  sph_autotune(SphHandle* h, int32_t reps, int32_t* grid_out);
/* Applies a launch configuration in sph_autotune's 7-entry layout (blocks
 * per kernel class, 0 = the default, then the two loop shapes), e.g. one
 * tuned earlier on a similar state; the next step rebuilds its graph.
 * Launch shapes change no result.                                          */
int  sph_set_launch_shape(SphHandle* h, const int32_t* shape);

/* ---------------------------------------------------------------------- */
/* Fine-grained calls, one per replaced Fortran call site                  */
/* ---------------------------------------------------------------------- */

/* time_step_duration.f90:59-123 (time_step_loop.f90:185). */
int  sph_time_step_duration(SphHandle* h, double* dt_out);
/* RHS_momentum_equation.f90:87-179 with inter_EqMoto.f90:108-263,
 * viscomon.f90:54-73, viscomorris.f90:60-71,
 * AddBoundaryContributions_to_ME3D.f90:105-336 / ..._ME2D.f90:96-402 and
 * AddElasticBoundaryReaction_3D.f90:67-154 / ..._2D.f90:63-97
 * (time_step_loop.f90:222).  acc_out ([n][3], caller order) may be NULL.  */
int  sph_rhs_momentum(SphHandle* h, double* acc_out);
/* Leapfrog_momentum.f90:66-99 (time_step_loop.f90:241) using the
 * accelerations of the last sph_rhs_momentum, then (TetaV > 1e-9)
 * velocity_smoothing.f90:85-132 with velocity_smoothing_SA_SPH_3D/2D and
 * velocity_smoothing_2.f90:68-102 (time_step_loop.f90:249-259); with
 * TetaV = 0, var = vel.                                                   */
int  sph_leapfrog_momentum(SphHandle* h);
/* Leapfrog_trajectories.f90:52-66 (time_step_loop.f90:262). */
int  sph_leapfrog_trajectories(SphHandle* h);
/* OrdGrid1.f90:50-105 followed by the neighbour-list replacement of
 * CalcVarLength.f90:133-269 (time_step_loop.f90:286,292).                 */
int  sph_ord_grid(SphHandle* h);
/* ComputeBoundaryDataTab_3D.f90:67-105 / _2D.f90:70-157
 * (time_step_loop.f90:322/324).                                           */
int  sph_boundary_data_tab(SphHandle* h);
/* The OMP block time_step_loop.f90:338-360: dden = 0, SASPH_continuity
 * (SASPH_continuity.f90:89-169 with AddBoundaryContribution_to_CE3D/2D)
 * and Continuity_Equation.f90:90-249.  dden_out ([n]) may be NULL.        */
int  sph_continuity(SphHandle* h, double* dden_out);
/* Leapfrog_continuity.f90:54-68 (time_step_loop.f90:382). */
int  sph_leapfrog_continuity(SphHandle* h);
/* EoS_fluid_loop.f90:59-69 with EoS_barotropic_linear.f90:49-55
 * (time_step_loop.f90:386), then (TetaP > 0) PressureSmoothing_3D.f90:88-160
 * / _2D.f90:102-235 (time_step_loop.f90:397-404); closes the step.        */
int  sph_eos(SphHandle* h);

/* ---------------------------------------------------------------------- */
/* One simulation split into slabs along x (no reference counterpart: the  */
/* reference runs one shared-memory process).  Each slab is a handle that  */
/* holds the particles of its x cells plus one layer of ghost cells on     */
/* each side, copies of the neighbouring slabs' particles; a host          */
/* orchestrator exchanges them (sphera_b200/slab.py).  With every slab's   */
/* particles uploaded in increasing order of their index in the whole      */
/* simulation, each owned particle sees the neighbours, order and          */
/* arithmetic it has in the undivided run, bit for bit.                    */
/* ---------------------------------------------------------------------- */

/* A slab: the whole simulation's grid (CreaGrid.f90:51-74 on
 * params->domain) restricted to x cells cell_lo..cell_hi (1-based,
 * inclusive), its origin and cell size kept, so a particle lies in the cell
 * it has in the whole grid.  Partial smoothing, C1 and pesodt != 0 return
 * SPH_ERR_UNSUPPORTED.                                                     */
int  sph_create_slab(const SphParams* params, const SphGeometry* geometry, int32_t n_capacity,
                     int32_t cell_lo, int32_t cell_hi, SphHandle** out);
/* Replaces the particle set (caller order, as sph_upload) keeping the
 * simulation's time, step and dt, and runs the search on it: OrdGrid1, the
 * neighbour lists and ComputeBoundaryDataTab (time_step_loop.f90:286-324).
 * laminar ([n], caller order, or NULL for all 0) carries pg%laminar_flag,
 * which the next momentum pass's wall terms read.  Every particle must lie
 * inside the slab's grid (nothing is removed in a slab's particle order).
 * Single simulations without C1.                                           */
int  sph_replace_particles(SphHandle* h, const SphState* state, const int32_t* laminar);
/* Sets the next step's dt (e.g. the minimum over the slabs of the dt each
 * closed its step with, which is the whole simulation's dt when pesodt = 0;
 * before the first step the IC's dt too), with dtvel and the body force
 * that follow from it.  pesodt != 0 returns SPH_ERR_UNSUPPORTED.            */
int  sph_set_time_step(SphHandle* h, double dt);

/* ---------------------------------------------------------------------- */
/* Checkpoint and resume (the state part of a restart: Memo_Results.f90    */
/* writes it, pg(1:nag) and the clock; ReadRestartFile.f90 reads it back).  */
/* ---------------------------------------------------------------------- */

/* The clock of a single simulation.                                       */
int  sph_get_clock(SphHandle* h, SphClock* clock);
/* Resume: after sph_upload of a checkpointed state (sph_download), set the
 * clock it was saved with and pg%laminar_flag ([n], caller order, as
 * sph_dump_laminar gave it; NULL for all 0, the IC's value).  The next
 * step then continues as the uninterrupted run would, bit for bit.  dtvel
 * and the next step's body force follow from the clock.  Single
 * simulations; C1 returns SPH_ERR_UNSUPPORTED (its inverted matrices are
 * not part of the state).                                                 */
int  sph_set_clock(SphHandle* h, const SphClock* clock, const int32_t* laminar);

/* ---------------------------------------------------------------------- */
/* Post-processing                                                         */
/* ---------------------------------------------------------------------- */

/* fluid_global_quantities.f90:59-72 (called by time_step_post_processing.f90:81
 * every Domain%icpoi_fr steps): FP64 sums over pg(1:nag) of the mass, the
 * linear momentum m v, the angular momentum m (coord x vel) about the origin
 * (Vector_Product.f90) and the volume m / rho, computed on the device.
 * out[0] mass, out[1..3] linear momentum, out[4..6] angular momentum,
 * out[7] volume.  sim selects one simulation of a batch (0 for sph_create);
 * sim = -1 fills out[nsims][8] for all of them.  The sums are compensated
 * and reduced in a fixed order, so they are the exact sums to within a few
 * ulps whatever the particle order.                                       */
int  sph_global_quantities(SphHandle* h, int32_t sim, double* out);

/* ---------------------------------------------------------------------- */
/* Verification                                                            */
/* ---------------------------------------------------------------------- */

/* The reference's grid arrays for the current positions: pg%cella ([n],
 * caller order), Icont ([n_cells+1], 1-based starts) and NPartOrd ([n],
 * 1-based caller indices), exactly as OrdGrid1.f90:58-105 builds them.
 * Any pointer may be NULL.                                                */
int  sph_dump_grid(SphHandle* h, int32_t* cella, int32_t* icont, int32_t* npartord);
/* The neighbour lists the pair passes read, in the form
 * CalcVarLength.f90:173-269 builds them: counts ([n], nPartIntorno) and
 * lists ([n][nmaxj], PartIntorno, 1-based caller indices in the
 * reference's visiting order, the particle itself included).              */
int  sph_dump_neighbours(SphHandle* h, int32_t nmaxj, int32_t* counts, int32_t* lists);
/* BoundaryDataTab in caller order: ncb ([n], BoundaryDataPointer(1,:) in
 * 3D, IntNcbs in 2D), and for each particle up to max_per entries of
 * clobonum ([n][max_per]) and the 20 doubles LocXYZ(3), BoundaryIntegral(8),
 * IntGiWrRdV(3,3) column-major ([n][max_per][20]).                        */
int  sph_dump_boundary(SphHandle* h, int32_t max_per, int32_t* ncb,
                       int32_t* clobonum, double* values);
/* pg%laminar_flag ([n], caller order) as the last momentum pass set it
 * (inter_EqMoto.f90:269-283).                                             */
int  sph_dump_laminar(SphHandle* h, int32_t* flags);
/* With c1_be: pg%B_ren_gradp and (with c1_divu) pg%B_ren_divu in caller
 * order, 9 doubles per particle, B(i,j) at [9 k + 3 (i-1) + (j-1)].  After
 * a search they hold the fluid sums of CalcVarLength.f90:285-324; after a
 * continuity pass the inverses of the completed matrices.  Either pointer
 * may be NULL.                                                            */
int  sph_dump_renormalisation(SphHandle* h, double* b_gradp, double* b_divu);

/* ---------------------------------------------------------------------- */
/* Allocation-free entry point                                             */
/* ---------------------------------------------------------------------- */

/* No counterpart in the reference.  The OrdGrid1 binning and counting sort
 * (pg%cella, Icont, NPartOrd) for callers that cannot let a library
 * allocate device memory -- a Fortran host whose device arrays come from its
 * own pool (CUDA Fortran / OpenACC data regions), or a time loop that must
 * not meet the implicit synchronisation of cudaMalloc/cudaFree.  It calls
 * no cudaMalloc, cudaFree or allocating library routine: its working memory
 * is a fixed device array of about 20 MB inside the library, held by every
 * GPU that loads the library until the process exits.
 *   d_x        [n][3] positions (device memory, caller order)
 *   d_cella    [n]    out: 1-based cell of each particle, 0 outside the grid
 *   d_icont    [n_cells+1] out: 1-based first NPartOrd slot of each cell
 *   d_npartord [n]    out: 1-based particle indices sorted by cell, then index;
 *                     particles outside the grid are not listed
 *   stream     a cudaStream_t (NULL: the default stream); the call only
 *              enqueues work on it.
 * Limits: n <= 1048576 and Grid%nmax <= 1048576, else
 * SPH_ERR_INVALID_ARGUMENT.  The first call on a device looks up the address
 * of the device array (with that device current) and must come before any
 * stream capture on that device; the address is kept per device context,
 * so after a cudaDeviceReset the next call looks it up again (and must
 * again come before any capture).  Every call shares the one array: calls
 * whose work overlaps on the GPU race and must be serialised.  Particles
 * outside the grid get cella 0 and are left out of NPartOrd (its last
 * n - Icont(nmax+1) + 1 rows are then unspecified); unlike sph_ord_grid,
 * nothing is removed or reordered.                                        */
int  sph_ord_grid_static(const SphParams* params, int32_t n, const double* d_x, int32_t* d_cella,
                         int32_t* d_icont, int32_t* d_npartord, void* stream);

/* ---------------------------------------------------------------------- */
/* Profiling (the counterpart of the reference's start_and_stop phase      */
/* timers, src/Post_processing/elapsed_time/start_and_stop.f90:65-152)      */
/* ---------------------------------------------------------------------- */

/* Runs nsteps whole steps without the graph, timing each phase with CUDA
 * events on the handle's stream; ms[0..5] receive the summed milliseconds of
 * momentum (+leapfrog, trajectories), OrdGrid1, ComputeBoundaryDataTab,
 * the neighbour lists (CalcVarLength), continuity (+Leapfrog_continuity,
 * EoS) and the time-step closing.                                         */
int  sph_profile_phases(SphHandle* h, int32_t nsteps, double* ms);
/* Neighbour candidates tested (c[0]) and pairs accepted incl. the particle
 * itself (c[1]) by the neighbour-list pass; c[2..3] reserved.  reset != 0
 * zeroes them.                                                            */
int  sph_get_counters(SphHandle* h, uint64_t* c, int32_t reset);
/* Measured dense FMA throughput of the current device in TFLOP/s: FP64,
 * or FP32 when fp32 != 0.                                                 */
int  sph_measure_fp64_peak(double* tflops);
int  sph_measure_fma_peak(int32_t fp32, double* tflops);
/* Self-check of the kernels' exact FP64 division: the FP64 passes divide by
 * a shared or constant divisor b through its correctly rounded reciprocal
 * and two remainder corrections (Markstein's method), which must give the
 * IEEE quotient a / b bit for bit.  Compares it with a / b on count
 * generated operand pairs (seeded; random, near-all-ones divisors, quotients
 * next to rounding midpoints, zero dividends, the kernels' own ranges) on
 * the current device; *mismatches receives the number that differ and
 * first_bad (may be NULL) the operands a, b of one of them.               */
int  sph_check_division(uint64_t count, uint64_t seed, uint64_t* mismatches, double* first_bad);

#ifdef __cplusplus
}
#endif

#endif /* SPHERA_B200_H */
