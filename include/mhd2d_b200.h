/*
 * mhd2d_b200 — C ABI of the B200 (sm_100a) implementation of the mhd2d-solver
 * time-step hot path: ENO-Roe / ENO-LF characteristic fluxes, RK3-TVD and
 * Euler stages with boundary fills, the CFL wave-speed reduction and the
 * div-B diagnostics / SOR correction.  Arithmetic is IEEE binary64.
 *
 * Data model (shared with the reference, vector_utilities.cpp:81-98): a
 * state is ONE contiguous block of 8 x NX x NY doubles, NX = nx+4,
 * NY = ny+4, element (k, i, j) at (k*NX + i)*NY + j, k = rho, mx, my, mz,
 * Bx, By, Bz, E; two ghost cells per side; j (y) fastest.  The host pointer
 * a caller passes is exactly the reference's U[0][0].
 *
 * Boundary codes (enums.hpp: BoundaryCondition): 1 periodic, 2 Dirichlet,
 * 3 Neumann, 4 open; bc[] is ordered left, right, bottom, top.
 * Scheme codes (IntegrationMethod): 2 ENO-Roe, 3 ENO-LF.
 * Time codes (TimeStepMethod): 1 Euler, 2 RK3-TVD.
 * Every entry point returns an int holding the reference's ReturnStatus
 * value (enums.hpp); the t_status::isError half comes from
 * mhd_last_error().  No exception crosses this boundary.
 *
 * Threading: a context is single-threaded, like the reference objects it
 * replaces.  All device work of a context runs on the context's own CUDA
 * stream; calls return after that work completed.
 */
#ifndef MHD2D_B200_H
#define MHD2D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ReturnStatus (enums.hpp) plus one code for CUDA runtime failures. */
enum {
   MHD_OK = 0, MHD_NO_CHANGE = 1, MHD_UPDATED = 2,
   MHD_ERR_NOT_IMPLEMENTED = 3, MHD_ERR_TIME_UNDERFLOW = 4, MHD_ERR_NOT_CONVERGED = 5,
   MHD_ERR_NEGATIVE_DENSITY = 6, MHD_ERR_NEGATIVE_PRESSURE = 7,
   MHD_ERR_FILE_NOT_FOUND = 8, MHD_ERR_FAILED_TO_PARSE = 9, MHD_ERR_WRONG_PARAMETER = 10,
   MHD_ERR_CUDA = 100
};

/* mhd_ctx_create flags */
#define MHD_FLAG_CHARACTERISTICS 0x1  /* keep cx, cy, LUx, LUy of the last integrate */
#define MHD_FLAG_FAST_MATH       0x2  /* FMA-contracted kernels (not bit-identical) */

typedef struct mhd_ctx mhd_ctx;

/* [divb corrector] parameters (file_access.cpp:273-299). */
typedef struct {
   int    divb_skip_steps;   /* stepping rate */
   int    sor_steps;         /* outer cleaning passes; <= 0 disables */
   double sor_rsteps;        /* maximum sweeps per solve */
   double sor_rmax;          /* sweep tolerance on max|update| / max|phi| */
   double sor_divbmax;       /* target max|div B| */
   int    omega_use_static;
   double omega;
} mhd_sor_params;

/* Context = the reference's method + stepper pair on one GPU.
   Replaces: SpatialMethodCentralFD2 / SpatialMethodEnoRoe /
   SpatialMethodEnoLF constructors (spatialmethodcentralfd2.cpp:6-24,
   spatialmethodenoroe.cpp:5-20, spatialmethodenolf.cpp:5-20) and
   TimeIntegrationRK3 / TimeIntegrationEuler constructors
   (timeintegrationrk3.cpp:4-27, timeintegrationeuler.cpp:4-15).
   halo must be 2 (bufferWidth = NXFIRST, main.cpp:117); a smaller halo is
   the reference's std::domain_error (spatialmethodeno.cpp:17-20) and
   returns MHD_ERR_WRONG_PARAMETER.  scheme: 1 central FD2, 2 ENO-Roe,
   3 ENO-LF (IntegrationMethod, enums.hpp:54-59).  Central FD2 statuses are
   the reference's: a non-positive density (first cell in loop order) or
   pressure (last cell) is fatal, the message names the cell. */
int mhd_ctx_create( int nx, int ny, int halo, double dx, double dy, double gamma,
                    const int bc[4], int scheme, int time_method,
                    double dt_min, double dt_max, double cfl, int flags, int device,
                    mhd_ctx** out );
int mhd_ctx_destroy( mhd_ctx* ctx );

/* Re-binds the stepper half of a context (time method, dt_min, dt_max,
   CFL number; cfl = 0 is the constant time mode), as constructing a
   TimeIntegrationRK3 / TimeIntegrationEuler around an existing method does
   (main.cpp:141-151).  Stage buffers are allocated on first use. */
int mhd_set_stepper( mhd_ctx* ctx, int time_method, double dt_min, double dt_max, double cfl );

/* Last status message and t_status::isError of this context. */
int mhd_last_error( const mhd_ctx* ctx, char* msg, size_t len, int* is_error );

/* Host <-> device copies of the state block U[0][0] (8*NX*NY doubles). */
int mhd_upload( mhd_ctx* ctx, const double* U );
int mhd_download( mhd_ctx* ctx, double* U );
/* UL (dU/dt) of the last integrate: same block shape, interior valid. */
int mhd_download_ul( mhd_ctx* ctx, double* UL );

/* Replaces SpatialIntegrationMethod::initializeDirichletBoundaries
   (spatialintegrationmethod.cpp:39-59): snapshot of the edge cells of the
   state currently on the device. */
int mhd_init_dirichlet( mhd_ctx* ctx );

/* The same snapshot handed over from the host, as the reference keeps it in
   SpatialIntegrationMethod::dirichletBoundaryLeft/Right/Bottom/Top
   (spatialintegrationmethod.hpp:55-58): left / right are [8][NY], bottom /
   top [8][NX] blocks (only the interior entries are read). */
int mhd_set_dirichlet( mhd_ctx* ctx, const double* left, const double* right,
                       const double* bottom, const double* top );

/* Replaces SpatialMethodEnoRoe::integrate (spatialmethodenoroe.cpp:33-179)
   and SpatialMethodEnoLF::integrate (spatialmethodenolf.cpp:33-230) on the
   device state: boundary fill (in place), fluxes, dtIdeal, UL. */
int mhd_integrate( mhd_ctx* ctx, double* dtIdeal );

/* Host-buffer form of the same call, as the plugin subclass uses it:
   U is uploaded, boundaries filled, UL computed; U (with its ghost cells)
   and UL are copied back. */
int mhd_integrate_host( mhd_ctx* ctx, double* U, double* UL, double* dtIdeal );

/* Replaces TimeIntegrationRK3::step (timeintegrationrk3.cpp:48-156) /
   TimeIntegrationEuler::step (timeintegrationeuler.cpp:26-64) on the device
   state; *dt_inout is the reference's dtCurrent. */
int mhd_step( mhd_ctx* ctx, double* dt_inout );

/* Host-buffer form: upload U, one step, download U. */
int mhd_step_host( mhd_ctx* ctx, double* U, double* dt_inout );

/* Several steps in a row (the loop of TimeIntegrationRK3::step /
   TimeIntegrationEuler::step calls, timeintegrationrk3.cpp:48-156);
   dts (optional, length nsteps) receives each step's dt.  It stops at the
   first failing step and returns its status (dt_inout then holds the last
   completed step's dt).  By default the whole loop is one CUDA graph
   launch: a while node over the steps with the RK3 retry loop as a nested
   while node that the device-side controller drives, so the host waits once
   per call instead of once per step; results are bit-identical to the
   step-by-step loop.  The graph allows 4096 RK3 passes per step (a valid
   run needs far fewer: every retry halves dt at least once); past that the
   call returns MHD_ERR_NOT_CONVERGED. */
int mhd_steps( mhd_ctx* ctx, int nsteps, double* dt_inout, double* dts );

/* 1 (the default): mhd_steps runs as one CUDA graph launch; 0: one host
   round trip per step (mhd_step in a loop).  Same results either way. */
int mhd_set_step_graph( mhd_ctx* ctx, int enable );

/* Replaces SpatialMethodEno::getCharacteristicsX/Y (spatialmethodeno.cpp:55-86)
   as called at timeintegrationrk3.cpp:151-152; requires
   MHD_FLAG_CHARACTERISTICS.  Any pointer may be NULL.  Central FD2 keeps
   no characteristics: MHD_NO_CHANGE, the arrays untouched (the base
   class's getCharacteristicsX/Y return false, spatialintegrationmethod.cpp:69-82). */
int mhd_get_characteristics( mhd_ctx* ctx, double* cx, double* cy, double* LUx, double* LUy );

/* Replaces divBCalculation (div_b_fix.cpp:4-126) on the device state. */
int mhd_divb_calc( mhd_ctx* ctx, double* maxdivb, double* totdivb );

/* The numbers of the reference's non-grid output record (outputNonGridData,
   file_access.cpp:1680-1736) for the context's state: out[0] u_max, out[1]
   |div B|_max, out[2] sum |div B| dx dy, out[3] total mass, out[4] total
   momentum (rho |u|), out[5] total energy, out[6] total entropy
   (log(p rho^-gamma)), each sum times dx dy.  Computed on the device; like the
   reference it fills periodic B ghosts on the way (divBCalculation). */
int mhd_nongrid_data( mhd_ctx* ctx, double out[7] );

/* Replaces divBCorrectionSOR (div_b_fix.cpp:129-403): one solve with the
   sublattice red-black ordering, warm-started from the context's
   potential, followed by the B correction.  *sweeps gets the sweep count. */
int mhd_divb_sor( mhd_ctx* ctx, const mhd_sor_params* p, int* sweeps );

/* enable 1 (the default), on grids of at least 32 tile rows: mhd_step_host
   copies the host state in row bands on a second stream and the first
   spatial operator (ENO-Roe) starts on the bands already copied; with RK3
   (ENO-Roe, ENO-LF) the last spatial operator runs in row bands whose
   results are copied back while the next bands run (copied again after an
   RK3 retry).  0: one copy in, the step, one copy out.  Bit-identical
   either way. */
int mhd_set_step_host_banded( mhd_ctx* ctx, int enable );

/* enable 1 (the default): the sweep loop of an SOR solve runs as one CUDA
   graph launch (a device-side while loop over passes of 16 sweeps, ended by
   the solve's own stop rule); 0: passes issued from the host, which reads the
   stop flag after each.  The same sweeps and values either way. */
int mhd_set_sor_graph( mhd_ctx* ctx, int enable );

/* The cleaning loop of main.cpp:207-242 (up to sor_steps solves until
   max|div B| < sor_divbmax), final max|div B| in *maxdivb. */
int mhd_divb_clean( mhd_ctx* ctx, const mhd_sor_params* p, double* maxdivb, int* total_sweeps );

/* The reference main loop (main.cpp:174-344) on the device, without files:
   step (mhd_step rules), the [divb corrector] cleaning loop every
   divb_skip_steps steps, t += dt, stop at `steps` (time_mode 1, constant) or
   at t >= t_max (time_mode 2, variable), on ErrorTimeUnderflow, on a fatal
   status or on a NaN at U[0][2][2].  The non-grid output records
   (mhd_nongrid_data) are taken at step 0 and then every nongrid_steps steps
   (nongrid_mode 1) or every nongrid_t of simulated time (nongrid_mode 2),
   as main.cpp:284-310 schedules them; up to max_records are stored. */
typedef struct {
   int    time_mode;        /* 1 constant (`steps` steps), 2 variable (until t_max) */
   int    steps;
   double t_max;
   double dt0;              /* initial time step */
   mhd_sor_params sor;      /* sor.sor_steps <= 0: no cleaning */
   int    nongrid_mode;     /* 0 none, 1 by steps, 2 by simulated time */
   int    nongrid_steps;
   double nongrid_t;
} mhd_run_params;

typedef struct {
   int    step;
   double t, dt;
   double values[7];        /* as mhd_nongrid_data */
} mhd_nongrid_record;

typedef struct {
   int    steps;            /* completed steps */
   double t, dt;            /* simulated time and the current dt at the end */
   int    status, is_error; /* of the last step */
   int    nan_stop;         /* stopped on a NaN */
   int    records;          /* records taken (may exceed max_records) */
   long long sor_sweeps;
} mhd_run_result;

int mhd_run( mhd_ctx* ctx, const mhd_run_params* p, mhd_nongrid_record* records,
             int max_records, mhd_run_result* result );

/* The reference's binary grid dump of the context's current state, packed
   on the device: the records outputGridDataBinary writes
   (file_access.cpp:1193-1325) after toNaturalData (conversions.cpp:37-57),
   with outputGridData's div B rules (file_access.cpp:1530-1677: Neumann and
   open sides leave their edge cells at 0, periodic sides read periodic B
   ghosts).  nx*ny records in i-major order of x, y, rho, [u, v, w, p if
   natural], Bx, By, Bz, |div B|, [mx, my, mz, e if conservation], as
   doubles or (single = 1) floats: the bytes the reference fwrites.  out:
   host or device memory of out_bytes; *bytes (optional) gets the size, and
   out = NULL only asks for it.  The state is not changed. */
typedef struct {
   int    natural;          /* [output] natural */
   int    conservation;     /* [output] conservation */
   int    single;           /* 1: binary floats, 0: binary doubles */
   double start_x, start_y; /* grid origin (t_params start_x, start_y) */
} mhd_grid_pack_params;

int mhd_grid_pack( mhd_ctx* ctx, const mhd_grid_pack_params* p, void* out, size_t out_bytes,
                   size_t* bytes );

/* Counters of the last integrate / step: clamped midpoint pressures
   (the reference's "negative pressure" warning count) and kernel launches. */
int mhd_get_counters( mhd_ctx* ctx, long long* neg_pressure, long long* launches );

/* Device row layout of a state block: element (k, i, j) of the device copy
   sits at k*NX*pitch + i*pitch + row_offset + j doubles from its base. */
int mhd_layout( const mhd_ctx* ctx, int* pitch, int* row_offset );

/* Process-wide: stage the flux kernels' state tiles with TMA box copies (1,
   the default where the driver offers tensor maps) or with per-element
   asynchronous copies (0); -1 leaves the setting.  *tma_launches (optional)
   gets the number of flux launches so far whose tiles were staged by TMA.
   Results are bit-identical either way. */
int mhd_set_tile_tma( int enable, long long* tma_launches );

/* SOR sweeps of this context (divBCorrectionSOR, div_b_fix.cpp:129-403):
   1 (the default) runs a sweep as two launches, one per colour, where the
   grid allows it (every periodic side's extent a multiple of 4): periodic
   ghosts are read at their source points and the convergence test runs in
   the second launch; 0 always refreshes the ghosts after each colour and
   tests in a launch of its own (five launches).  Results are identical. */
int mhd_set_sor_fused( mhd_ctx* ctx, int enable );

/* How a thread of an SOR half sweep (div_b_fix.cpp:262-280, red-black)
   walks its rows: 0 (the default) by grid size; 1 one row at a time,
   reusing the loads its previous row made (faster on grids below ~2 M
   cells); 2 two rows' loads in flight at a time (faster above).  A half
   sweep's rows are independent, so the results are identical. */
int mhd_set_sor_rows( mhd_ctx* ctx, int mode );

/* The context's CUDA stream (a cudaStream_t), for callers that record
   events or order their own work against the context's kernels. */
int mhd_stream( const mhd_ctx* ctx, void** stream );

/* Launches `n` back-to-back spatial operators (boundary fill + fused flux
   kernel, no host synchronisation in between) on the device state and
   returns their average device time in ms, measured with CUDA events on the
   context's stream.  For profiling and roofline accounting. */
int mhd_time_integrate( mhd_ctx* ctx, int n, double* avg_ms );

/* Measured FP64 FMA throughput of `device` (TFLOP/s, 2 flops per FMA):
   a grid of independent fused multiply-add chains timed with CUDA events.
   The denominator of the FP64 roofline of the flux kernels. */
int mhd_fp64_peak( int device, double* tflops );

/* No counterpart in the reference.  The div B diagnostic of mhd_divb_calc
   for callers that cannot allocate device memory (plug-ins inside an
   application that owns all device memory through its own pool, runtimes
   that forbid allocation once running, since cudaMalloc can synchronise
   the device and stall every other stream).  It allocates
   nothing: its scratch (one partial max and sum per grid row) is a fixed
   file-scope device array of 2 x 16384 doubles that every GPU loading the
   library keeps until exit, so nx may not exceed 16384
   (MHD_ERR_WRONG_PARAMETER otherwise).
     U       device state block, element (k,i,j) at
             k*(nx+4)*pitch + i*pitch + row_offset + j (pitch = ny+4,
             row_offset = 0 is the reference's own layout); the periodic Bx,
             By ghost layers are written, as divBCalculation does;
     result  device pointer to 2 doubles: max|div B|, integral of |div B|;
     stream  a cudaStream_t (NULL: the default stream).
   The work is enqueued on `stream` and the call returns without waiting.
   The first call on a device looks up the scratch array's device address
   (cudaGetSymbolAddress, with that device current); make that first call
   before any stream capture.  All calls share the scratch array: calls
   whose work overlaps on the GPU race, so serialise them. */
int mhd_divb_calc_noalloc( double* U, int nx, int ny, int pitch, int row_offset,
                           double dx, double dy, const int bc[4], double* result,
                           void* stream );

/* ------------------------------------------------------------------------
 * Batched runs.  The reference runs one problem per process; its
 * "batching" is starting several copies with different INI files.  A batch
 * holds many independent runs of uneven grid sizes, schemes, boundary
 * conditions and end times on one GPU and advances all of them together:
 * each stage is one boundary fill, one ENO-LF dissipation pass, ONE
 * persistent flux launch over the tiles of every active run, one
 * controller pass (a per-run CFL reduction and dt control, the retry logic
 * of TimeIntegrationRK3::step included) and one stage update, replayed
 * from a CUDA graph.  Every run follows the reference main loop
 * (main.cpp:174-344) without file output and SOR: step, t += dt, stop when
 * t >= t_end, on a NaN at U[0][2][2], on a fatal status, or after
 * max_steps steps when max_steps > 0.  Each run's arithmetic is the same as
 * a context's (bit-identical results). */
typedef struct mhd_batch mhd_batch;

typedef struct {
   int    nx, ny;
   double dx, dy, gamma;
   int    bc[4];          /* left, right, bottom, top */
   int    scheme;         /* 2 ENO-Roe, 3 ENO-LF */
   int    time_method;    /* 1 Euler, 2 RK3-TVD */
   double dt_min, dt_max, cfl;
   double dt0;            /* dt entering the first step */
   double t_end;          /* simulated end time ([time] t_max) */
   int    max_steps;      /* 0: no step limit */
} mhd_batch_desc;

typedef struct {
   double    t, dt;
   int       steps;
   int       active;       /* 1 while the run continues */
   int       status;       /* ReturnStatus that stopped it (0: reached its end) */
   int       phase;        /* RK3 stage the next spatial operator belongs to */
   long long retries;      /* RK3 stage-loop restarts (dt reductions) */
   long long neg_pressure; /* midpoint pressures clamped to zero */
} mhd_batch_state;

/* Tile shapes of the persistent flux launch the autotuner chooses from. */
enum { MHD_BATCH_TILE_7x32 = 0, MHD_BATCH_TILE_3x32 = 1, MHD_BATCH_TILE_COUNT = 2 };

int mhd_batch_create( int n, const mhd_batch_desc* runs, int device, mhd_batch** out );
int mhd_batch_destroy( mhd_batch* b );
int mhd_batch_last_error( mhd_batch* b, char* buf, size_t len, int* is_error );

/* Load run `idx` from a host [8][NX][NY] block (ghosts ignored) and re-arm it:
   t = 0, dt = dt0, no steps; Dirichlet sides take their edge snapshot
   (initializeDirichletBoundaries) from this state. */
int mhd_batch_upload( mhd_batch* b, int idx, const double* U );
int mhd_batch_download( mhd_batch* b, int idx, double* U );

/* Advance every active run by up to `stages` spatial-operator stages (an
   RK3 step is 3 stages, an Euler step 1; a dt retry adds stages).  The
   host looks at the active count every `check_every` stages (<= 0: only at
   the end) and returns early when no run is active. */
int mhd_batch_advance( mhd_batch* b, int stages, int check_every, int* n_active );

/* Per-run progress, read back after the last advance. */
int mhd_batch_get_state( mhd_batch* b, int idx, mhd_batch_state* out );

/* Autotuner: times the persistent flux launch of every tile shape (and two
   persistent grid sizes) on the batch's current states, keeps the fastest
   and returns its MHD_BATCH_TILE_* code and CTAs per SM.  The states are
   left exactly as they were. */
int mhd_batch_tune( mhd_batch* b, int reps, int* tile, int* ctas_per_sm, double* best_ms );
/* Use a given tile shape / persistent grid (ctas_per_sm <= 0: the occupancy limit). */
int mhd_batch_set_tile( mhd_batch* b, int tile, int ctas_per_sm );

/* Device-side initial states (problem setups of file_access.cpp), written
   straight into run idx and re-arming it like mhd_batch_upload.
   kind MHD_PROBLEM_EXPLOSION, p[0..8]: x0, y0 (lower-left corner), r,
     rho_in, p_in, rho_out, p_out, Bx, By  (Bz = 0, velocity 0; "jump" transition)
   kind MHD_PROBLEM_WAVE, p[0..15]: x0, y0, Lx, Ly, rho, u, v, w, Bx, By, Bz, p,
     epsilon, wave (0..6 = right eigenvector index), kx, ky  (readProblemWaveTest)
   kind MHD_PROBLEM_ORSZAG_TANG: no parameters (gamma from the run)
   kind MHD_PROBLEM_PLASMA_SHEET, p[0..3+K]: x0, y0, delta, K, a_1..a_K
   kind MHD_PROBLEM_SHOCK_TUBE, p[0..18]: Lx, Ly, interface angle (degrees),
     left state rho, u, v, w, Bx, By, Bz, p, right state (same order)
     (readProblemShockTube, file_access.cpp:300-395; dx = Lx/nx, dy = Ly/ny)
   kind MHD_PROBLEM_SHEET_LOBES, p[0..41]: Lx, Ly, start_x, start_y, sheet
     start, sheet start foot, sheet thickness, profile (0 constant, 1 tanh),
     transition (0 jump, 1 linear), transition points, then the left, right,
     up and down states (rho, u, v, w, Bx, By, Bz, p each)
     (readProblemPlasmaSheet, file_access.cpp:614-919; dx = Lx/nx, dy = Ly/ny) */
enum { MHD_PROBLEM_EXPLOSION = 1, MHD_PROBLEM_WAVE = 2, MHD_PROBLEM_ORSZAG_TANG = 3,
       MHD_PROBLEM_PLASMA_SHEET = 4, MHD_PROBLEM_SHOCK_TUBE = 5, MHD_PROBLEM_SHEET_LOBES = 6 };
int mhd_batch_init_problem( mhd_batch* b, int idx, int kind, const double* p, int np );

int mhd_batch_stream( mhd_batch* b, void** stream );
/* Kernel launches issued so far (graph nodes counted per replay). */
int mhd_batch_launches( mhd_batch* b, long long* launches );

/* ------------------------------------------------------------------------
 * Discrete adjoint of the ENO-Roe time step.  The reference has no
 * differentiation; this is the gradient of its discrete forward map.
 * J = sum over the final interior of |m|^2 / (2 rho) dx dy (kinetic energy).
 *
 * mhd_adj_forward advances the initial state nsteps steps exactly as a
 * context does (TimeIntegrationRK3::step / TimeIntegrationEuler::step with
 * updateDt and the RK3 retry rule, ENO-Roe fluxes; bit-identical results),
 * recording every executed stage (input buffer, stage update, dt), the ENO
 * stencil and upwind choices of every interface and characteristic (4-bit
 * codes), and a checkpoint of U every `checkpoint_every` steps.
 * mhd_adj_backward computes dJ/dU0 of that discrete map with the recorded
 * choices and dt frozen: per checkpoint segment, last first, the segment is
 * replayed from its checkpoint and its stages are differentiated in reverse.
 * Segments whose stage inputs the recording kept in device memory (the
 * stage store, mhd_adj_set_store) are not replayed.
 * mhd_adj_replay runs the same frozen map from another initial state (the
 * frozen-stencil, frozen-dt forward that central finite differences of J
 * need). */
typedef struct mhd_adj mhd_adj;

typedef struct {
   int       steps, stages, checkpoints, retries;
   double    t, dt;              /* simulated time and last dt of the recording */
   double    ms_forward;         /* device time of the recording forward */
   double    ms_backward;        /* device time of the last backward (replays included) */
   double    ms_replay;          /* device time of the last full replay */
   long long launches;
   int       stored_stages;      /* stage inputs the recording kept (stage store) */
   int       replayed_segments;  /* segments the last backward replayed */
} mhd_adj_stats;

int mhd_adj_create( int nx, int ny, double dx, double dy, double gamma, const int bc[4],
                    int time_method, double dt_min, double dt_max, double cfl,
                    int checkpoint_every, int device, mhd_adj** out );
int mhd_adj_destroy( mhd_adj* a );
int mhd_adj_last_error( mhd_adj* a, char* buf, size_t len, int* is_error );
/* Device memory the recording may fill with stage inputs, in bytes: the last
   checkpoint segments that fit are kept whole and the backward uses them
   instead of replaying.  -1 (the default): all free memory but a reserve for
   the backward; 0: none, every segment is replayed from its checkpoint.
   Results are bit-identical either way. */
int mhd_adj_set_store( mhd_adj* a, long long max_bytes );
/* keep_all 1 (the default): the recording keeps the ENO codes of every stage
   (mhd_adj_replay needs them).  0: only those of stored stages; the backward
   records the others again while it replays their segments, so a recording
   needs mask memory for its stored stages only.  Changing it discards the
   recording. */
int mhd_adj_set_masks( mhd_adj* a, int keep_all );
/* enable 1 (the default): the reverse sweep (interface adjoint, gather,
   boundary transpose) is compiled with FMA contraction; the midpoint states
   it recomputes keep the recording's rounding, so it differentiates the
   recorded branches.  0: the parity build's rounding throughout, which is
   the rounding of a plain FP64 tangent-linear model of the same map.  The
   two gradients differ by rounding amplified by the eigen-system's
   conditioning (1e-8 relative near B_perp = 0).  The recording is kept. */
int mhd_adj_set_contract( mhd_adj* a, int enable );
/* Initial state from the host (Dirichlet sides take their edges from it). */
int mhd_adj_upload( mhd_adj* a, const double* U0 );
/* Initial state generated on the device (kinds of mhd_batch_init_problem). */
int mhd_adj_init_problem( mhd_adj* a, int kind, const double* p, int np );
/* Recording forward run; *J (optional) = J of the final state. */
int mhd_adj_forward( mhd_adj* a, int nsteps, double dt0, double* J );
/* Frozen replay from a host initial state (NULL: the recorded one); Dirichlet
   sides take their edges from that state, so dJ/dU0 includes the edge
   snapshot's dependence on U0. */
int mhd_adj_replay( mhd_adj* a, const double* U0, double* J );
/* Frozen replay from a device-generated initial state. */
int mhd_adj_replay_problem( mhd_adj* a, int kind, const double* p, int np, double* J );
int mhd_adj_backward( mhd_adj* a );
/* dJ/dU0 as a host [8][NX][NY] block (ghost entries 0). */
int mhd_adj_gradient( mhd_adj* a, double* dJdU0 );
/* dJ/da_k, k = 1..K, of the plasma-sheet initial state (MHD_PROBLEM_PLASMA_SHEET
   with corner x0, y0): contraction of dJ/dU0 with dU0/da_k. */
int mhd_adj_sheet_gradient( mhd_adj* a, double x0, double y0, int K, double* dJda );
/* which: 0 initial state, 1 final state of the recording, 2 working state. */
int mhd_adj_download( mhd_adj* a, int which, double* U );
int mhd_adj_info( mhd_adj* a, mhd_adj_stats* out );
/* Several recordings or reverse sweeps at once on one device (batched
   gradients): each object keeps its own stream; the host issues their steps
   in lockstep (forward) and their stages round robin (backward), so small
   grids share the GPU.  The stage stores share the free memory in proportion
   to each recording's stage inputs.  Results are bit-identical to separate
   mhd_adj_forward / mhd_adj_backward calls.  J (n values) and ms (device
   time of the whole group) may be NULL; the first failing member's status
   is returned and its message is in its own mhd_adj_last_error. */
int mhd_adj_forward_group( int n, mhd_adj* const* a, const int* nsteps, const double* dt0,
                           double* J, double* ms );
int mhd_adj_backward_group( int n, mhd_adj* const* a, double* ms );

#ifdef __cplusplus
}
#endif
#endif
