/*
 * ORACLE — TEST INFRASTRUCTURE ONLY.  A CPU restatement (plain C) of the
 * time-step hot path of piccolo255/mhd2d-solver.  Only tests/, the smoke
 * check and bench.py's cpu_baseline leg may load it, and only as the
 * checker; the product (libmhd2d_b200.so) never links or calls it.
 *
 * Parity status: pinned.  tests/test_oracle_golden.py checks every entry
 * point below bit for bit against golden vectors produced by the unmodified
 * reference (tests/golden/make_golden.py) and, where oracle/_ref is built,
 * against the reference library directly.
 *
 * Layout: every state array is the reference's contiguous [k][i][j] block
 * (vector_utilities.cpp:81-98): 8 fields x NX x NY doubles with NX = nx+4,
 * NY = ny+4 (2 ghost cells per side, j fastest).  Boundary codes follow the
 * reference enum BoundaryCondition (enums.hpp): 1 periodic, 2 Dirichlet,
 * 3 Neumann, 4 open; bc[] order is left, right, bottom, top.  Return values
 * are the reference's ReturnStatus values (enums.hpp).
 */
#ifndef MHD_ORACLE_H
#define MHD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
   ORC_OK = 0, ORC_NO_CHANGE = 1, ORC_UPDATED = 2, ORC_ERR_NOT_IMPLEMENTED = 3,
   ORC_ERR_TIME_UNDERFLOW = 4, ORC_ERR_NOT_CONVERGED = 5, ORC_ERR_NEGATIVE_DENSITY = 6,
   ORC_ERR_NEGATIVE_PRESSURE = 7, ORC_ERR_WRONG_PARAMETER = 10
};

typedef struct orc_ctx orc_ctx;

typedef struct {
   int    divb_skip_steps;
   int    sor_steps;
   double sor_rsteps;
   double sor_rmax;
   double sor_divbmax;
   int    omega_use_static;
   double omega;
} orc_sor_params;

/* scheme: 1 central FD2, 2 ENO-Roe, 3 ENO-LF.  time_method: 1 Euler, 2 RK3-TVD. */
orc_ctx* orc_create( int scheme, int time_method, int nx, int ny, double dx, double dy,
                     double gamma, const int* bc, double dt_min, double dt_max, double cfl );
void     orc_destroy( orc_ctx* c );

/* Dirichlet edge snapshot (initializeDirichletBoundaries). */
void orc_init_dirichlet( orc_ctx* c, const double* U );

/* Boundary fill in place (applyBoundaryConditions). */
int  orc_apply_bc( orc_ctx* c, double* U, int* is_error );

/* One spatial integration: BCs on U, numerical fluxes, UL, dtIdeal.  The
   characteristic velocities / variables land in the context (see below). */
int  orc_integrate( orc_ctx* c, double* U, double* UL, double* dtIdeal, int* is_error );
void orc_get_characteristics( const orc_ctx* c, double* cx, double* cy, double* LUx, double* LUy );

/* Test hooks for windows of large ENO-LF grids: the dissipation
   coefficients aF [8][ny+4], aG [8][nx+4] of a whole grid (ghosts already
   filled; spatialmethodenolf.cpp:66-125), and fixing them for the next
   integrations of a context (NULL, NULL: computed again). */
int  orc_lf_alpha_grid( double gamma, int nx, int ny, const double* U, double* aF, double* aG );
void orc_set_lf_alpha( orc_ctx* c, const double* aF, const double* aG );

/* Power-of-two CFL step control (updateDt). */
int  orc_update_dt( double dt_min, double dt_max, double cfl, double* dt_inout, double dtIdeal,
                    int* is_error );

/* One time step (RK3-TVD with the reference's retry semantics, or Euler). */
int  orc_step( orc_ctx* c, double* U, double* dt_inout, int* is_error );

/* div B diagnostics (fills periodic B ghosts of U as a side effect). */
void orc_divb_calc( orc_ctx* c, double* U, double* maxdivb, double* totdivb );

/* One SOR solve + B correction.  red_black = 0 reproduces the reference's
   lexicographic sweep; red_black = 1 is the sublattice red-black ordering
   that the CUDA path runs.  The potential lives in the context and
   warm-starts the next call, like the reference's function-static buffer. */
int  orc_divb_sor( orc_ctx* c, const orc_sor_params* sp, double* U, int red_black,
                   int* sweeps, int* is_error );

/* The reference main loop without file output (see ref_harness.cpp). */
int  orc_run( orc_ctx* c, int nsteps, double t_max, const orc_sor_params* sor, int red_black,
              double* U, double* dt_inout, double* t_inout, int* steps_done,
              double* dt_hist, double* divb_hist, int hist_len, int* is_error );

/* Number of RK3 stage restarts (dt retries) this context has taken. */
long long orc_retries( const orc_ctx* c );

/* Single-interface and single-cell kernels, exposed for unit tests. */
int  orc_eigens_f( double gamma, const double* U1, const double* U2, double* lambda,
                   double* lv, double* rv, int* neg_pressure );
int  orc_eigenvalues_at( double gamma, const double* U, double* lambda, int* neg_pressure );

#ifdef __cplusplus
}
#endif
#endif
