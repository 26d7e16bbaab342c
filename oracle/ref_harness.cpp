/*
 * ORACLE TEST INFRASTRUCTURE — not part of the product.
 *
 * A C ABI around the reference solver's own hot-path classes, so that the
 * tests and the CPU baseline can drive the UNMODIFIED reference code
 * (piccolo255/mhd2d-solver) on arbitrary states.  This file is linked with
 * the reference's sources compiled in place (see oracle/Makefile); nothing
 * of the reference is copied here.  Only the test suite, the golden-vector
 * generator and bench.py's CPU baseline load the resulting library.
 *
 * Reference interfaces driven from here:
 *   SpatialIntegrationMethod::initializeDirichletBoundaries
 *                                   spatialintegrationmethod.cpp:39-59
 *   SpatialMethodEnoRoe::integrate   spatialmethodenoroe.cpp:33-179
 *   SpatialMethodEnoLF::integrate    spatialmethodenolf.cpp:33-230
 *   SpatialMethodCentralFD2::integrate  spatialmethodcentralfd2.cpp:44-160
 *   SpatialMethodEno::getCharacteristicsX/Y  spatialmethodeno.cpp:55-86
 *   TimeIntegrationMethod::updateDt  timeintegrationmethod.cpp:35-90
 *   TimeIntegrationRK3::step         timeintegrationrk3.cpp:48-156
 *   TimeIntegrationEuler::step       timeintegrationeuler.cpp:26-64
 *   divBCalculation                  div_b_fix.cpp:4-126
 *   divBCorrectionSOR                div_b_fix.cpp:129-403
 *   main loop (step, div-B cleaning, time update, NaN stop)  main.cpp:174-344
 */
#include "mhd2d.hpp"
#include "spatialmethodenoroe.hpp"
#include "spatialmethodenolf.hpp"
#include "spatialmethodcentralfd2.hpp"
#include "timeintegrationrk3.hpp"
#include "timeintegrationeuler.hpp"

#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

namespace {

/* Pointer tables that view one contiguous [k][i][j] block as t_matrices. */
struct MatView {
   std::vector<double*> rows;
   std::vector<double**> planes;
   MatView( double* base, int n, int sx, int sy ) : rows( size_t(n)*sx ), planes( n ) {
      for( int k = 0; k < n; k++ ){
         planes[k] = &rows[size_t(k)*sx];
         for( int i = 0; i < sx; i++ )
            rows[size_t(k)*sx+i] = base + (size_t(k)*sx+i)*sy;
      }
   }
   t_matrices m() { return planes.data(); }
};

struct VecView {
   std::vector<double*> rows;
   VecView( double* base, int n, int s ) : rows( n ) {
      for( int k = 0; k < n; k++ ) rows[k] = base + size_t(k)*s;
   }
   t_vectors v() { return rows.data(); }
};

BoundaryCondition toBc( int v ){
   switch( v ){
   case 1: return BoundaryCondition::Periodic;
   case 2: return BoundaryCondition::Dirichlet;
   case 3: return BoundaryCondition::Neumann;
   case 4: return BoundaryCondition::Open;
   default: return BoundaryCondition::Undefined;
   }
}

/* bc[] order used across this project's ABI: left, right, bottom, top. */
t_boundary toBoundary( const int* bc ){
   return t_boundary{ toBc( bc[1] ), toBc( bc[3] ), toBc( bc[0] ), toBc( bc[2] ) };
}

void fillParams( t_params& p, int nx, int ny, double dx, double dy, const int* bc ){
   p.nx = nx; p.ny = ny; p.dx = dx; p.dy = dy;
   p.boundary[p.b_left]   = toBc( bc[0] );
   p.boundary[p.b_right]  = toBc( bc[1] );
   p.boundary[p.b_bottom] = toBc( bc[2] );
   p.boundary[p.b_top]    = toBc( bc[3] );
}

void copyMsg( const std::string& s, char* msg, int msglen ){
   if( msg && msglen > 0 ){
      std::strncpy( msg, s.c_str(), size_t(msglen-1) );
      msg[msglen-1] = '\0';
   }
}

std::unique_ptr<SpatialIntegrationMethod> makeMethod( int scheme, int nx, int ny, double dx,
                                                      double dy, double gamma, const int* bc ){
   auto b = toBoundary( bc );
   if( scheme == 1 )
      return std::unique_ptr<SpatialIntegrationMethod>{ new SpatialMethodCentralFD2( nx, ny, 2, dx, dy, b, gamma ) };
   if( scheme == 3 )
      return std::unique_ptr<SpatialIntegrationMethod>{ new SpatialMethodEnoLF( nx, ny, 2, dx, dy, b, gamma ) };
   return std::unique_ptr<SpatialIntegrationMethod>{ new SpatialMethodEnoRoe( nx, ny, 2, dx, dy, b, gamma ) };
}

/* Exposes the protected updateDt of the reference's time-integration base. */
struct DtProbe : public TimeIntegrationMethod {
   DtProbe( double dtMin, double dtMax, double cfl )
      : TimeIntegrationMethod( 1, 1, 2, dtMin, dtMax, cfl, nullptr ) {}
   t_status step( t_matrices, t_matrices, t_matrices, t_matrices, t_matrices,
                  borderVectors, double& ) override { return {}; }
   t_status probe( double& dt, double ideal ){ return updateDt( dt, ideal ); }
};

} // namespace

extern "C" {

typedef struct {
   int    divb_skip_steps;   /* [divb corrector] stepping rate */
   int    sor_steps;         /* sor steps (outer loop); <= 0 disables cleaning */
   double sor_rsteps;        /* sor rsteps (max sweeps per solve) */
   double sor_rmax;          /* sor rmax */
   double sor_divbmax;       /* sor divbmax */
   int    omega_use_static;
   double omega;
} ref_sor_params;

/* One SpatialIntegrationMethod::integrate call on a fresh method object.
   Returns the ReturnStatus value; *is_error carries t_status::isError. */
int ref_integrate( int scheme, int nx, int ny, double dx, double dy, double gamma,
                   const int* bc, double* U_dirichlet, double* U, double* UL, double* dtIdeal,
                   double* cx, double* cy, double* LUx, double* LUy,
                   int* is_error, char* msg, int msglen )
{
   const int NXt = nx+4, NYt = ny+4;
   auto method = makeMethod( scheme, nx, ny, dx, dy, gamma, bc );
   MatView vU( U, PRB_DIM, NXt, NYt ), vUL( UL, PRB_DIM, NXt, NYt );
   if( U_dirichlet ){
      MatView vD( U_dirichlet, PRB_DIM, NXt, NYt );
      method->initializeDirichletBoundaries( vD.m() );
   }
   borderVectors bf{};
   double ideal = 0.0;
   t_status st = method->integrate( vU.m(), vUL.m(), bf, ideal );
   *dtIdeal = ideal;
   if( cx && LUx ){
      MatView a( cx, PRB_DIM, NXt, NYt ), b( LUx, PRB_DIM, NXt, NYt );
      method->getCharacteristicsX( a.m(), b.m() );
   }
   if( cy && LUy ){
      MatView a( cy, PRB_DIM, NXt, NYt ), b( LUy, PRB_DIM, NXt, NYt );
      method->getCharacteristicsY( a.m(), b.m() );
   }
   *is_error = st.isError ? 1 : 0;
   copyMsg( st.message, msg, msglen );
   return int( st.status );
}

/* TimeIntegrationMethod::updateDt on one (dtCurrent, dtIdeal) pair. */
int ref_update_dt( double dt_min, double dt_max, double cfl, double* dt_inout, double dtIdeal,
                   int* is_error )
{
   DtProbe p( dt_min, dt_max, cfl );
   t_status st = p.probe( *dt_inout, dtIdeal );
   *is_error = st.isError ? 1 : 0;
   return int( st.status );
}

/* divBCalculation (fills periodic B ghosts in U as a side effect). */
void ref_divb_calc( int nx, int ny, double dx, double dy, const int* bc, double* U,
                    double* maxdivb, double* totdivb )
{
   t_params p; fillParams( p, nx, ny, dx, dy, bc );
   MatView vU( U, PRB_DIM, nx+4, ny+4 );
   divBCalculation( vU.m(), p, *maxdivb, *totdivb );
}

/* The numbers of one non-grid output record for state U: the reference's
   own toNaturalData (conversions.cpp:37-57) and divBCalculation
   (div_b_fix.cpp:4-126), and the sums of outputNonGridData
   (file_access.cpp:1680-1716; that file needs the INI parser and is not
   compiled here, so its loop is restated).  out: u_max, |div B|_max,
   sum |div B|, total mass, momentum, energy, entropy. */
void ref_nongrid_data( int nx, int ny, double dx, double dy, double gamma, const int* bc,
                       double* U, double* out )
{
   t_params params; fillParams( params, nx, ny, dx, dy, bc );
   params.gamma = gamma;
   const int NXt = nx+4, NYt = ny+4;
   std::vector<double> ubuf( size_t(VEL_DIM)*NXt*NYt ), pbuf( size_t(NXt)*NYt );
   MatView vU( U, PRB_DIM, NXt, NYt ), vu( ubuf.data(), VEL_DIM, NXt, NYt ),
           vp( pbuf.data(), 1, NXt, NYt );
   t_data data{};
   data.U = vU.m();
   data.u = vu.m();
   data.p = vp.m()[0];
   toNaturalData( params, data );
   double totenergy = 0.0, entropy, totentropy = 0.0, totmass = 0.0, totmomentum = 0.0;
   double uu, uumax = 0.0;
   for( int i = NXFIRST; i < NXLAST; i++ ){
      for( int j = NYFIRST; j < NYLAST; j++ ){
         uu = data.u[0][i][j]*data.u[0][i][j] + data.u[1][i][j]*data.u[1][i][j]
            + data.u[2][i][j]*data.u[2][i][j];
         if( uu > uumax ) uumax = uu;
         entropy = log( data.p[i][j]*pow( data.U[0][i][j], -params.gamma ) );
         totentropy  += entropy;
         totenergy   += data.U[7][i][j];
         totmass     += data.U[0][i][j];
         totmomentum += data.U[0][i][j]*sqrt(uu);
      }
   }
   double maxdivb = 0.0, totdivb = 0.0;
   divBCalculation( data.U, params, maxdivb, totdivb );
   const double dxdy = params.dx*params.dy;
   out[0] = sqrt( uumax );
   out[1] = maxdivb;
   out[2] = totdivb;
   out[3] = totmass*dxdy;
   out[4] = totmomentum*dxdy;
   out[5] = totenergy*dxdy;
   out[6] = totentropy*dxdy;
}

/* One divBCorrectionSOR call.  The potential is a function-static buffer of
   the reference, kept across calls within one loaded copy of this library. */
int ref_divb_sor( int nx, int ny, double dx, double dy, const int* bc,
                  const ref_sor_params* sp, double* U, int* is_error )
{
   t_params p; fillParams( p, nx, ny, dx, dy, bc );
   p.divb_sor_rsteps = sp->sor_rsteps;
   p.divb_sor_rmax = sp->sor_rmax;
   p.divb_sor_max = sp->sor_divbmax;
   p.divb_sor_steps = sp->sor_steps;
   p.divb_sor_omega_use_static = sp->omega_use_static != 0;
   p.divb_sor_omega = sp->omega;
   p.log_params = t_log_params{ false, false, false, false };
   MatView vU( U, PRB_DIM, nx+4, ny+4 );
   t_status st = divBCorrectionSOR( vU.m(), p );
   *is_error = st.isError ? 1 : 0;
   return int( st.status );
}

/* The reference main loop (main.cpp:174-344) without file output:
   step -> error check -> div-B cleaning every `divb_skip_steps` steps ->
   t += dt -> stop on step count (nsteps > 0) or t >= t_max (t_max > 0) ->
   stop on NaN in U[0][2][2].  Per-step dt and post-cleaning max|div B| are
   recorded when the history pointers are non-null. */
int ref_run( int scheme, int time_method, int nx, int ny, double dx, double dy, double gamma,
             const int* bc, double dt_min, double dt_max, double cfl,
             int nsteps, double t_max, const ref_sor_params* sor,
             double* U, double* dt_inout, double* t_inout, int* steps_done,
             double* dt_hist, double* divb_hist, int hist_len,
             double* cx, double* cy, double* LUx, double* LUy,
             int* is_error, char* msg, int msglen )
{
   const int NXt = nx+4, NYt = ny+4;
   auto method = makeMethod( scheme, nx, ny, dx, dy, gamma, bc );
   MatView vU( U, PRB_DIM, NXt, NYt );
   method->initializeDirichletBoundaries( vU.m() );
   std::unique_ptr<TimeIntegrationMethod> stepper;
   if( time_method == 1 )
      stepper.reset( new TimeIntegrationEuler( nx, ny, 2, dt_min, dt_max, cfl, std::move( method ) ) );
   else
      stepper.reset( new TimeIntegrationRK3( nx, ny, 2, dt_min, dt_max, cfl, std::move( method ) ) );

   std::vector<double> scx, scy, sLx, sLy;
   const size_t tot = size_t(PRB_DIM)*NXt*NYt;
   if( !cx ){ scx.assign( tot, 0.0 ); cx = scx.data(); }
   if( !cy ){ scy.assign( tot, 0.0 ); cy = scy.data(); }
   if( !LUx ){ sLx.assign( tot, 0.0 ); LUx = sLx.data(); }
   if( !LUy ){ sLy.assign( tot, 0.0 ); LUy = sLy.data(); }
   MatView vcx( cx, PRB_DIM, NXt, NYt ), vcy( cy, PRB_DIM, NXt, NYt );
   MatView vLx( LUx, PRB_DIM, NXt, NYt ), vLy( LUy, PRB_DIM, NXt, NYt );
   std::vector<double> bfl( size_t(PRB_DIM)*NYt ), bfr( size_t(PRB_DIM)*NYt );
   std::vector<double> bfu( size_t(PRB_DIM)*NXt ), bfd( size_t(PRB_DIM)*NXt );
   VecView l( bfl.data(), PRB_DIM, NYt ), r( bfr.data(), PRB_DIM, NYt );
   VecView u( bfu.data(), PRB_DIM, NXt ), d( bfd.data(), PRB_DIM, NXt );
   borderVectors bf{ l.v(), r.v(), u.v(), d.v() };

   t_params p; fillParams( p, nx, ny, dx, dy, bc );
   if( sor ){
      p.divb_skip_steps = sor->divb_skip_steps;
      p.divb_sor_rsteps = sor->sor_rsteps;
      p.divb_sor_rmax = sor->sor_rmax;
      p.divb_sor_max = sor->sor_divbmax;
      p.divb_sor_steps = sor->sor_steps;
      p.divb_sor_omega_use_static = sor->omega_use_static != 0;
      p.divb_sor_omega = sor->omega;
   }
   p.log_params = t_log_params{ false, false, false, false };

   t_status st{ false, ReturnStatus::OK, "" };
   int step = 1;
   bool done = false;
   double dt = *dt_inout, t = *t_inout;
   while( !done ){
      st = stepper->step( vU.m(), vcx.m(), vcy.m(), vLx.m(), vLy.m(), bf, dt );
      if( st.status == ReturnStatus::ErrorTimeUnderflow || st.isError ) break;
      double divbmax = -1.0, divbsum = 0.0;
      if( sor && sor->sor_steps > 0 && step % p.divb_skip_steps == 0 ){
         for( int it = 0; it < p.divb_sor_steps; it++ ){
            divBCalculation( vU.m(), p, divbmax, divbsum );
            if( divbmax < p.divb_sor_max ) break;
            t_status s2 = divBCorrectionSOR( vU.m(), p );
            if( s2.status == ReturnStatus::ErrorNotConverged ) break;
         }
         divBCalculation( vU.m(), p, divbmax, divbsum );
      }
      t += dt;
      if( dt_hist && step <= hist_len ) dt_hist[step-1] = dt;
      if( divb_hist && step <= hist_len ) divb_hist[step-1] = divbmax;
      if( nsteps > 0 && step == nsteps ) done = true;
      if( t_max > 0.0 && t >= t_max ) done = true;
      if( std::isnan( U[(size_t(0)*NXt+2)*NYt+2] ) ) done = true;
      step++;
   }
   *dt_inout = dt;
   *t_inout = t;
   *steps_done = step-1;
   *is_error = st.isError ? 1 : 0;
   copyMsg( st.message, msg, msglen );
   return int( st.status );
}

} // extern "C"

#ifdef MHDREF_BENCH_MAIN
/* CPU baseline driver: the reference TimeIntegrationRK3 + SpatialMethodEnoRoe
   / EnoLF on the Orszag-Tang vortex (initial state as in
   file_access.cpp:578-613, gamma = 5/3), periodic on all sides, CFL-controlled
   dt (cfl 0.4, dt_max 0.03125), for `steps` steps.  Prints one line per step:
   "step <k> <seconds> <dt>", then "cells <n*n>". */
#include <cstdlib>
int main( int argc, char** argv ){
   if( argc < 4 ){
      std::fprintf( stderr, "usage: %s n steps scheme(2=roe,3=lf)\n", argv[0] );
      return 2;
   }
   const int n = std::atoi( argv[1] ), steps = std::atoi( argv[2] ), scheme = std::atoi( argv[3] );
   const int NXt = n+4, NYt = n+4;
   const double gam = 5.0/3.0, L = 2.0*M_PI, dx = L/n, dy = L/n;
   std::vector<double> U( size_t(PRB_DIM)*NXt*NYt, 0.0 );
   auto at = [&]( int k, int i, int j ) -> double& { return U[(size_t(k)*NXt+i)*NYt+j]; };
   for( int i = 2; i < n+2; i++ ) for( int j = 2; j < n+2; j++ ){
      double x = (i-2)*dx, y = (j-2)*dy;
      double r = gam*gam, u = -std::sin( y ), v = std::sin( x ), w = 0.0;
      double bx = -std::sin( y ), by = std::sin( 2*x ), bz = 0.0, p = gam;
      at(0,i,j) = r; at(1,i,j) = u*r; at(2,i,j) = v*r; at(3,i,j) = w*r;
      at(4,i,j) = bx; at(5,i,j) = by; at(6,i,j) = bz;
      at(7,i,j) = p/(gam-1.0) + 0.5*r*(u*u+v*v+w*w) + 0.5*(bx*bx+by*by+bz*bz);
   }
   const int bc[4] = { 1, 1, 1, 1 };
   auto method = makeMethod( scheme, n, n, dx, dy, gam, bc );
   MatView vU( U.data(), PRB_DIM, NXt, NYt );
   method->initializeDirichletBoundaries( vU.m() );
   TimeIntegrationRK3 stepper( n, n, 2, 1e-9, 0.03125, 0.4, std::move( method ) );
   const size_t tot = size_t(PRB_DIM)*NXt*NYt;
   std::vector<double> cx( tot ), cy( tot ), lx( tot ), ly( tot );
   MatView vcx( cx.data(), PRB_DIM, NXt, NYt ), vcy( cy.data(), PRB_DIM, NXt, NYt );
   MatView vlx( lx.data(), PRB_DIM, NXt, NYt ), vly( ly.data(), PRB_DIM, NXt, NYt );
   // the stepper blends these (timeintegrationrk3.cpp:136-145) although nothing reads them
   std::vector<double> bfl( size_t(PRB_DIM)*NYt ), bfr( size_t(PRB_DIM)*NYt );
   std::vector<double> bfu( size_t(PRB_DIM)*NXt ), bfd( size_t(PRB_DIM)*NXt );
   VecView l( bfl.data(), PRB_DIM, NYt ), r( bfr.data(), PRB_DIM, NYt );
   VecView u( bfu.data(), PRB_DIM, NXt ), d( bfd.data(), PRB_DIM, NXt );
   borderVectors bf{ l.v(), r.v(), u.v(), d.v() };
   double dt = 0.03125;
   for( int s = 0; s < steps; s++ ){
      auto t0 = std::chrono::steady_clock::now();
      t_status st = stepper.step( vU.m(), vcx.m(), vcy.m(), vlx.m(), vly.m(), bf, dt );
      std::chrono::duration<double> el = std::chrono::steady_clock::now() - t0;
      if( st.isError ){ std::fprintf( stderr, "step failed: %s\n", st.message.c_str() ); return 1; }
      std::printf( "step %d %.6f %.10g\n", s, el.count(), dt );
      std::fflush( stdout );
   }
   std::printf( "cells %lld\n", (long long)n*n );
   return 0;
}
#endif
